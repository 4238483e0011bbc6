// Register-resident small DFTs and the two-step line transform used by the
// sticks/planes 3D FFT.
//
// Convention (FFTW's, which the reference uses through fft_grid_serial.hpp):
//   DIR = -1 : forward,  X_k = sum_j x_j exp(-2 pi i jk/n)
//   DIR = +1 : backward, X_k = sum_j x_j exp(+2 pi i jk/n)      (both unnormalised)
//
// A line of length n = na * nb is transformed by the threads of a block in
// two in-place passes (Cooley-Tukey); the backward transform leaves the line
// in a digit-reversed order that the forward transform takes as its input, so
// neither needs a reordering pass (see "The line transforms as passes").
//
// The twiddle table holds w_n^m = exp(-2 pi i m / n), m < n, in shared memory;
// the backward direction uses its conjugate.
#pragma once

#include "common.cuh"

namespace q3b {
namespace fft {

// sin/cos constants of the radix-3 and radix-5 butterflies (plain trigonometry)
constexpr double kS3 = 0.86602540378443864676;   // sin(2 pi / 3)
constexpr double kC51 = 0.30901699437494742410;  // cos(2 pi / 5)
constexpr double kC52 = -0.80901699437494742410; // cos(4 pi / 5)
constexpr double kS51 = 0.95105651629515357212;  // sin(2 pi / 5)
constexpr double kS52 = 0.58778525229247312917;  // sin(4 pi / 5)

template <typename T> struct RealOf;
template <> struct RealOf<double2> { using R = double; };
template <> struct RealOf<float2> { using R = float; };

template <int DIR, typename T> __device__ __forceinline__ T twiddle(const T* tw, int m) {
    T w = tw[m];
    if (DIR > 0) w.y = -w.y;
    return w;
}

// ----------------------------------------------------------- radix kernels
template <int DIR, typename T> __device__ __forceinline__ void dft2(T* x) {
    T a = x[0], b = x[1];
    x[0] = a + b;
    x[1] = a - b;
}

template <int DIR, typename T> __device__ __forceinline__ void dft3(T* x) {
    using R = typename RealOf<T>::R;
    T a = x[0], b = x[1], c = x[2];
    T t1 = b + c, t2 = b - c;
    T m1 = a - R(0.5) * t1;
    T n1 = R(DIR * kS3) * mul_i(t2);
    x[0] = a + t1;
    x[1] = m1 + n1;
    x[2] = m1 - n1;
}

template <int DIR, typename T> __device__ __forceinline__ void dft4(T* x) {
    using R = typename RealOf<T>::R;
    T a = x[0], b = x[1], c = x[2], d = x[3];
    T s0 = a + c, d0 = a - c, s1 = b + d, d1 = b - d;
    T wd1 = R(DIR) * mul_i(d1);
    x[0] = s0 + s1;
    x[1] = d0 + wd1;
    x[2] = s0 - s1;
    x[3] = d0 - wd1;
}

template <int DIR, typename T> __device__ __forceinline__ void dft5(T* x) {
    using R = typename RealOf<T>::R;
    T a = x[0], b = x[1], c = x[2], d = x[3], e = x[4];
    T t1 = b + e, t2 = c + d, t3 = b - e, t4 = c - d;
    T m1 = a + R(kC51) * t1 + R(kC52) * t2;
    T m2 = a + R(kC52) * t1 + R(kC51) * t2;
    T n1 = R(DIR) * mul_i(R(kS51) * t3 + R(kS52) * t4);
    T n2 = R(DIR) * mul_i(R(kS52) * t3 - R(kS51) * t4);
    x[0] = a + t1 + t2;
    x[1] = m1 + n1;
    x[4] = m1 - n1;
    x[2] = m2 + n2;
    x[3] = m2 - n2;
}

// N = A * B for the composite small sizes (A is the first-level DFT size)
template <int N> struct Split;
template <> struct Split<6> { static constexpr int A = 3, B = 2; };
template <> struct Split<8> { static constexpr int A = 4, B = 2; };
template <> struct Split<9> { static constexpr int A = 3, B = 3; };
template <> struct Split<10> { static constexpr int A = 5, B = 2; };
template <> struct Split<12> { static constexpr int A = 4, B = 3; };
template <> struct Split<15> { static constexpr int A = 5, B = 3; };
template <> struct Split<16> { static constexpr int A = 4, B = 4; };

// Larger composites, for the register-resident line transforms of the plane
// kernel (planes_reg.cu): a line of up to 108 points held by one to four lanes.
template <> struct Split<18> { static constexpr int A = 6, B = 3; };
template <> struct Split<20> { static constexpr int A = 5, B = 4; };
template <> struct Split<24> { static constexpr int A = 8, B = 3; };
template <> struct Split<25> { static constexpr int A = 5, B = 5; };
template <> struct Split<27> { static constexpr int A = 9, B = 3; };
template <> struct Split<30> { static constexpr int A = 10, B = 3; };
template <> struct Split<32> { static constexpr int A = 8, B = 4; };
template <> struct Split<36> { static constexpr int A = 9, B = 4; };
template <> struct Split<40> { static constexpr int A = 8, B = 5; };
template <> struct Split<45> { static constexpr int A = 9, B = 5; };
template <> struct Split<48> { static constexpr int A = 16, B = 3; };
template <> struct Split<50> { static constexpr int A = 10, B = 5; };
template <> struct Split<54> { static constexpr int A = 9, B = 6; };
template <> struct Split<60> { static constexpr int A = 15, B = 4; };
template <> struct Split<64> { static constexpr int A = 16, B = 4; };
template <> struct Split<72> { static constexpr int A = 9, B = 8; };
template <> struct Split<80> { static constexpr int A = 16, B = 5; };
template <> struct Split<108> { static constexpr int A = 12, B = 9; };

// cos and sin of 2 pi m / N, m < N, as a table built at compile time: the
// angle is reduced to a quadrant exactly in integers, and cos/sin of the
// remainder (below pi/2) are summed from their Taylor series in double (27
// terms; the first omitted term is below 1e-24).  Indexed with the constants
// of unrolled loops, the table folds into literal operands.
struct UnitTerms {
    static constexpr double kHalfPi = 1.57079632679489661923;
    static constexpr double cos_q(double x) {
        double term = 1.0, sum = 1.0;
        for (int k = 1; k < 14; ++k) {
            term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
            sum += term;
        }
        return sum;
    }
    static constexpr double sin_q(double x) {
        double term = x, sum = x;
        for (int k = 1; k < 14; ++k) {
            term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
            sum += term;
        }
        return sum;
    }
};

template <int N> struct UnitTable {
    double c[N];
    double s[N];
    constexpr UnitTable() : c(), s() {
        for (int m = 0; m < N; ++m) {
            const int q = (4 * m) / N;             // quadrant
            const int r = 4 * m - q * N;           // remainder, in units of (pi/2)/N
            const double x = UnitTerms::kHalfPi * static_cast<double>(r) / static_cast<double>(N);
            const double cx = r == 0 ? 1.0 : UnitTerms::cos_q(x);
            const double sx = r == 0 ? 0.0 : UnitTerms::sin_q(x);
            c[m] = q == 0 ? cx : q == 1 ? -sx : q == 2 ? -cx : sx;
            s[m] = q == 0 ? sx : q == 1 ? cx : q == 2 ? -sx : -cx;
        }
    }
};

// cos(2 pi m / N) and sin(2 pi m / N) for m < N, the internal twiddles of the
// composite small DFTs (plain trigonometry, evaluated in extended precision and
// rounded to double; the sizes without a literal table below use UnitTable)
template <int N> __host__ __device__ constexpr double unit_cos(int m) {
    constexpr UnitTable<N> t{};
    return t.c[m];
}
template <int N> __host__ __device__ constexpr double unit_sin(int m) {
    constexpr UnitTable<N> t{};
    return t.s[m];
}
template <> __host__ __device__ constexpr double unit_cos<6>(int m) {
    constexpr double t[6] = {1.0, 0.5, -0.5, -1.0, -0.5, 0.5};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_sin<6>(int m) {
    constexpr double t[6] = {0.0, 0.8660254037844386, 0.8660254037844386, 0.0, -0.8660254037844386, -0.8660254037844386};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_cos<8>(int m) {
    constexpr double t[8] = {1.0, 0.7071067811865476, 0.0, -0.7071067811865476, -1.0, -0.7071067811865476, 0.0, 0.7071067811865476};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_sin<8>(int m) {
    constexpr double t[8] = {0.0, 0.7071067811865476, 1.0, 0.7071067811865476, 0.0, -0.7071067811865476, -1.0, -0.7071067811865476};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_cos<9>(int m) {
    constexpr double t[9] = {1.0, 0.766044443118978, 0.17364817766693036, -0.5, -0.9396926207859084, -0.9396926207859084, -0.5, 0.17364817766693036, 0.766044443118978};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_sin<9>(int m) {
    constexpr double t[9] = {0.0, 0.6427876096865394, 0.984807753012208, 0.8660254037844386, 0.3420201433256687, -0.3420201433256687, -0.8660254037844386, -0.984807753012208, -0.6427876096865394};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_cos<10>(int m) {
    constexpr double t[10] = {1.0, 0.8090169943749475, 0.30901699437494745, -0.30901699437494745, -0.8090169943749475, -1.0, -0.8090169943749475, -0.30901699437494745, 0.30901699437494745, 0.8090169943749475};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_sin<10>(int m) {
    constexpr double t[10] = {0.0, 0.5877852522924731, 0.9510565162951535, 0.9510565162951535, 0.5877852522924731, 0.0, -0.5877852522924731, -0.9510565162951535, -0.9510565162951535, -0.5877852522924731};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_cos<12>(int m) {
    constexpr double t[12] = {1.0, 0.8660254037844386, 0.5, 0.0, -0.5, -0.8660254037844386, -1.0, -0.8660254037844386, -0.5, 0.0, 0.5, 0.8660254037844386};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_sin<12>(int m) {
    constexpr double t[12] = {0.0, 0.5, 0.8660254037844386, 1.0, 0.8660254037844386, 0.5, 0.0, -0.5, -0.8660254037844386, -1.0, -0.8660254037844386, -0.5};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_cos<15>(int m) {
    constexpr double t[15] = {1.0, 0.9135454576426009, 0.6691306063588582, 0.30901699437494745, -0.10452846326765347, -0.5, -0.8090169943749475, -0.9781476007338057, -0.9781476007338057, -0.8090169943749475, -0.5, -0.10452846326765347, 0.30901699437494745, 0.6691306063588582, 0.9135454576426009};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_sin<15>(int m) {
    constexpr double t[15] = {0.0, 0.4067366430758002, 0.7431448254773942, 0.9510565162951535, 0.9945218953682733, 0.8660254037844386, 0.5877852522924731, 0.20791169081775934, -0.20791169081775934, -0.5877852522924731, -0.8660254037844386, -0.9945218953682733, -0.9510565162951535, -0.7431448254773942, -0.4067366430758002};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_cos<16>(int m) {
    constexpr double t[16] = {1.0, 0.9238795325112867, 0.7071067811865476, 0.3826834323650898, 0.0, -0.3826834323650898, -0.7071067811865476, -0.9238795325112867, -1.0, -0.9238795325112867, -0.7071067811865476, -0.3826834323650898, 0.0, 0.3826834323650898, 0.7071067811865476, 0.9238795325112867};
    return t[m];
}
template <> __host__ __device__ constexpr double unit_sin<16>(int m) {
    constexpr double t[16] = {0.0, 0.3826834323650898, 0.7071067811865476, 0.9238795325112867, 1.0, 0.9238795325112867, 0.7071067811865476, 0.3826834323650898, 0.0, -0.3826834323650898, -0.7071067811865476, -0.9238795325112867, -1.0, -0.9238795325112867, -0.7071067811865476, -0.3826834323650898};
    return t[m];
}

// x times w_N^m = exp(-2 pi i DIR' m / N) (conjugate for DIR = +1), m a constant
// after unrolling: quarter turns are sign swaps, the rest a complex product
// with literal constants.
template <int N, int DIR, typename T> __device__ __forceinline__ T rotate_const(T x, int m) {
    using R = typename RealOf<T>::R;
    if (m == 0) return x;
    if (4 * m == N) return DIR > 0 ? mul_i(x) : mk(x.y, -x.x);
    if (2 * m == N) return mk(-x.x, -x.y);
    if (4 * m == 3 * N) return DIR > 0 ? mk(x.y, -x.x) : mul_i(x);
    return cmul(x, mk(R(unit_cos<N>(m)), R(DIR * unit_sin<N>(m))));
}

// In-register DFT of size N.  The internal twiddles of a composite N are
// literal constants; tw/tws (the line's table and n/N) are not read.
template <int N, int DIR, typename T>
__device__ __forceinline__ void dft(T* x, const T* tw, int tws) {
    if constexpr (N == 1) {
        return;
    } else if constexpr (N == 2) {
        dft2<DIR>(x);
    } else if constexpr (N == 3) {
        dft3<DIR>(x);
    } else if constexpr (N == 4) {
        dft4<DIR>(x);
    } else if constexpr (N == 5) {
        dft5<DIR>(x);
    } else {
        constexpr int A = Split<N>::A, B = Split<N>::B;
        T y[N];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) {
            T t[A];
#pragma unroll
            for (int n1 = 0; n1 < A; ++n1) t[n1] = x[n2 + B * n1];
            dft<A, DIR>(t, tw, tws * B);
#pragma unroll
            for (int k1 = 0; k1 < A; ++k1) y[n2 + B * k1] = rotate_const<N, DIR>(t[k1], (n2 * k1) % N);
        }
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            T t[B];
#pragma unroll
            for (int n2 = 0; n2 < B; ++n2) t[n2] = y[n2 + B * k1];
            dft<B, DIR>(t, tw, tws * A);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) x[k1 + A * k2] = t[k2];
        }
    }
}

// Where element j of line l lives: base(l) + j * es
struct LineGeom {
    int n;        // line length
    int na, nb;   // n = na * nb
    int lines;    // number of lines
    int ls;       // line stride (used when bases == nullptr)
    int es;       // element stride
    const int* bases;  // optional per-line base offsets (shared memory)
    __device__ __forceinline__ int base(int l) const { return bases ? bases[l] : l * ls; }
};

// Position -> index map of the digit-reversed order the backward transform
// leaves a line in: position nb*k1 + k2 holds element k1 + na*k2.
__device__ __forceinline__ int digit_reversed(int pos, int na, int nb) { return pos / nb + na * (pos % nb); }

// One in-place pass over every line.  Item (l, q) owns the R values of line l
// at positions q*qs + r*rs, r < R:
//   CONTIG = false: q < nb, positions q + nb*r      (R = na, stride nb)
//   CONTIG = true : q < na, positions nb*q + r      (R = nb, contiguous)
// Either way the items of a line partition it, so a pass is one read and one
// write of every element with no hazard between items, and passes are
// separated by one barrier.  Lines run fastest across lanes: the callers lay
// lines out at an odd pitch, so a warp's accesses fall in distinct banks.
// Which values of an item a pass reads and writes.  AllPositions: every
// one.  ItemMask (stride-nb passes, CONTIG = false): bits[q] has bit r set
// when position q + nb*r of the line holds data; a clear bit reads as zero on
// load, or is not stored.  One shared-memory word per item, then register
// bit tests.
struct AllPositions {
    static constexpr bool kAll = true;
    __device__ __forceinline__ unsigned word(int) const { return ~0u; }
};
struct ItemMask {
    static constexpr bool kAll = false;
    const unsigned* bits;
    __device__ __forceinline__ unsigned word(int q) const { return bits[q]; }
};

template <int R, bool CONTIG, typename T, typename Body, typename LoadSel = AllPositions,
          typename StoreSel = AllPositions>
__device__ __forceinline__ void line_pass(T* buf, const LineGeom& g, const Body& body, const LoadSel& lsel = {},
                                          const StoreSel& ssel = {}) {
    const int Q = CONTIG ? g.na : g.nb;
    const int qs = (CONTIG ? g.nb : 1) * g.es;
    const int rs = (CONTIG ? 1 : g.nb) * g.es;
    const int items = g.lines * Q;
    const int bq = static_cast<int>(blockDim.x) / g.lines, br = static_cast<int>(blockDim.x) % g.lines;
    int l = static_cast<int>(threadIdx.x) % g.lines, q = static_cast<int>(threadIdx.x) / g.lines;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        T* p = buf + g.base(l) + q * qs;
        T x[R];
        const unsigned lw = lsel.word(q), sw = ssel.word(q);
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (LoadSel::kAll || ((lw >> r) & 1u)) x[r] = p[r * rs];
            else x[r] = czero<T>();
        }
        body(x, l, q);
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (StoreSel::kAll || ((sw >> r) & 1u)) p[r * rs] = x[r];
        l += br;
        q += bq;
        if (l >= g.lines) {
            l -= g.lines;
            ++q;
        }
    }
}

// The line transforms as passes (Cooley-Tukey, n = na*nb, DIR +1 backward,
// -1 forward, both unnormalised):
//   backward, natural order in, digit-reversed order out:
//     A+ : DFT_na over x[n2 + nb*n1] (n1 < na) for each n2 < nb, times
//          w^{+n2*k1}, in place;
//     B+ : DFT_nb over the contiguous block nb*k1 + n2 (n2 < nb) for each
//          k1 < na, in place: position nb*k1 + k2 now holds X[k1 + na*k2].
//   forward, digit-reversed order in, natural order out (the factorisation
//   with the roles of na and nb swapped, j = n2 + na*n1, k = k1 + nb*k2):
//     B- : DFT_nb over the contiguous block nb*n2 + n1 (n1 < nb), the
//          elements y[n2 + na*n1], times w^{-n2*k1}, in place;
//     A- : DFT_na over positions nb*n2 + k1 (n2 < na) for each k1 < nb,
//          in place: position k1 + nb*k2 now holds Y[k1 + nb*k2].
// A backward-then-forward round trip fuses B+ and B- in registers, with an
// epilogue applied to each value at its natural index between them.

template <int NA, int DIR, typename T, typename LoadSel = AllPositions, typename StoreSel = AllPositions>
__device__ __forceinline__ void pass_a(T* buf, const LineGeom& g, const T* tw, const LoadSel& lsel = {},
                                       const StoreSel& ssel = {}) {
    const int tws = g.n / NA;
    line_pass<NA, false>(buf, g, [&](T* x, int, int q) {
        dft<NA, DIR>(x, tw, tws);
        if (DIR > 0) {
#pragma unroll
            for (int k = 1; k < NA; ++k)
                if (q != 0) x[k] = cmul(x[k], twiddle<DIR>(tw, q * k));  // q*k < n
        }
    }, lsel, ssel);
}

template <int NB, int DIR, typename T>
__device__ __forceinline__ void pass_b(T* buf, const LineGeom& g, const T* tw) {
    const int tws = g.n / NB;
    line_pass<NB, true>(buf, g, [&](T* x, int, int q) {
        dft<NB, DIR>(x, tw, tws);
        if (DIR < 0) {
#pragma unroll
            for (int k = 1; k < NB; ++k)
                if (q != 0) x[k] = cmul(x[k], twiddle<DIR>(tw, q * k));  // q*k < n
        }
    });
}

template <int NB, typename T, typename Epi>
__device__ __forceinline__ void pass_mid(T* buf, const LineGeom& g, const T* tw, const Epi& epi) {
    const int tws = g.n / NB;
    const int na = g.na;
    line_pass<NB, true>(buf, g, [&](T* x, int l, int q) {
        dft<NB, +1>(x, tw, tws);
#pragma unroll
        for (int r = 0; r < NB; ++r) x[r] = epi(l, q + na * r, x[r]);
        dft<NB, -1>(x, tw, tws);
#pragma unroll
        for (int k = 1; k < NB; ++k)
            if (q != 0) x[k] = cmul(x[k], twiddle<-1>(tw, q * k));
    });
}

#define Q3B_FFT_SIZES(X) X(1) X(2) X(3) X(4) X(5) X(6) X(8) X(9) X(10) X(12) X(15) X(16)

// MAXR: the largest factor a caller instantiates (lengths with a larger
// factor are not transformed); a smaller bound keeps registers down.
template <int DIR, int MAXR, typename T, typename LoadSel = AllPositions, typename StoreSel = AllPositions>
__device__ __forceinline__ void run_a(T* buf, const LineGeom& g, const T* tw, const LoadSel& lsel = {},
                                      const StoreSel& ssel = {}) {
    switch (g.na) {
#define Q3B_A(N) \
    case N:                                                             \
        if constexpr (N <= MAXR) pass_a<N, DIR>(buf, g, tw, lsel, ssel); \
        break;
        Q3B_FFT_SIZES(Q3B_A)
#undef Q3B_A
        default: break;
    }
}

template <int DIR, int MAXR, typename T>
__device__ __forceinline__ void run_b(T* buf, const LineGeom& g, const T* tw) {
    switch (g.nb) {
#define Q3B_B(N) \
    case N:                                                 \
        if constexpr (N <= MAXR) pass_b<N, DIR>(buf, g, tw); \
        break;
        Q3B_FFT_SIZES(Q3B_B)
#undef Q3B_B
        default: break;
    }
}

// Backward transform of every line: natural order in, digit-reversed out.
// Ends with a barrier.
template <int MAXR, typename T>
__device__ __forceinline__ void backward(T* buf, const LineGeom& g, const T* tw) {
    run_a<+1, MAXR>(buf, g, tw);
    __syncthreads();
    run_b<+1, MAXR>(buf, g, tw);
    __syncthreads();
}

// Forward transform of every line: digit-reversed order in, natural out.
// Ends with a barrier.
template <int MAXR, typename T>
__device__ __forceinline__ void forward(T* buf, const LineGeom& g, const T* tw) {
    run_b<-1, MAXR>(buf, g, tw);
    __syncthreads();
    run_a<-1, MAXR>(buf, g, tw);
    __syncthreads();
}

// Backward transform, epi(line, natural index, value) on every value, forward
// transform; natural order in and out.  Three passes, ends with a barrier.
// `sel` marks the positions that hold data on input and are wanted on output
// (the others are read as zero and not written back), for the stride-nb
// passes (see ItemMask).
template <int MAXR, typename T, typename Epi, typename Sel = AllPositions>
__device__ __forceinline__ void roundtrip(T* buf, const LineGeom& g, const T* tw, const Epi& epi,
                                          const Sel& sel = {}) {
    run_a<+1, MAXR>(buf, g, tw, sel, AllPositions{});
    __syncthreads();
    switch (g.nb) {
#define Q3B_M(N) \
    case N:                                                   \
        if constexpr (N <= MAXR) pass_mid<N>(buf, g, tw, epi); \
        break;
        Q3B_FFT_SIZES(Q3B_M)
#undef Q3B_M
        default: break;
    }
    __syncthreads();
    run_a<-1, MAXR>(buf, g, tw, AllPositions{}, sel);
    __syncthreads();
}

}  // namespace fft
}  // namespace q3b
