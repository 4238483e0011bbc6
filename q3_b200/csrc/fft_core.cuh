// Register-resident small DFTs and the two-step line transform used by the
// sticks/planes 3D FFT.
//
// Convention (FFTW's, which the reference uses through fft_grid_serial.hpp):
//   DIR = -1 : forward,  X_k = sum_j x_j exp(-2 pi i jk/n)
//   DIR = +1 : backward, X_k = sum_j x_j exp(+2 pi i jk/n)      (both unnormalised)
//
// A line of length n = NA * NB is transformed by threads in two steps
// (Cooley-Tukey with j = n2 + NB*n1, k = k1 + NA*k2):
//   step 1: item (line, n2): DFT_NA over x[n2 + NB*n1], times w_n^{n2*k1},
//           written back in place to x[n2 + NB*k1];
//   step 2: item (line, k1): DFT_NB over x[n2 + NB*k1], written to x[k1 + NA*k2].
// Step 2 writes where other items read, so every item of step 2 is loaded into
// registers before a barrier and stored after it.  Lines are spread across
// lanes (line index fastest) so that shared-memory accesses of a warp fall on
// consecutive lines, which the callers lay out at an odd pitch.
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

// In-register DFT of size N.  tw/tws: the line's table and n/N, so that
// w_N^m = tw[m * tws].
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
            for (int k1 = 0; k1 < A; ++k1) {
                const int m = (n2 * k1) % N;
                y[n2 + B * k1] = (m == 0) ? t[k1] : cmul(t[k1], twiddle<DIR>(tw, m * tws));
            }
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

struct NoEpilogue {
    template <typename T> __device__ __forceinline__ T operator()(int, int, T v) const { return v; }
};

// step 1: in place, no hazard between items.  Item it = l + lines*n2; the
// (l, n2) pair is stepped by blockDim without dividing in the loop.
template <int NA, int DIR, typename T>
__device__ __forceinline__ void line_step1(T* buf, const LineGeom& g, const T* tw) {
    const int items = g.lines * g.nb;
    const int tws = g.n / NA;
    const int bq = static_cast<int>(blockDim.x) / g.lines, br = static_cast<int>(blockDim.x) % g.lines;
    int l = static_cast<int>(threadIdx.x) % g.lines, n2 = static_cast<int>(threadIdx.x) / g.lines;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        T* p = buf + g.base(l) + n2 * g.es;
        T x[NA];
#pragma unroll
        for (int n1 = 0; n1 < NA; ++n1) x[n1] = p[n1 * g.nb * g.es];
        dft<NA, DIR>(x, tw, tws);
#pragma unroll
        for (int k1 = 0; k1 < NA; ++k1) {
            const int m = n2 * k1;  // < n
            T v = (k1 == 0 || n2 == 0) ? x[k1] : cmul(x[k1], twiddle<DIR>(tw, m));
            p[k1 * g.nb * g.es] = v;
        }
        l += br;
        n2 += bq;
        if (l >= g.lines) {
            l -= g.lines;
            ++n2;
        }
    }
}

// step 2: an item's stores land in other items' inputs, but only within its
// own line.  Lines are therefore taken in rounds of whole lines: every item of
// a round is loaded into registers before a barrier and stored after it.
// MAXIT bounds the items one thread holds per round.
template <int NB, int DIR, int MAXIT, typename T, typename Epi>
__device__ __forceinline__ void line_step2(T* buf, const LineGeom& g, const T* tw, const Epi& epi) {
    const int tws = g.n / NB;
    int per_round = (static_cast<int>(blockDim.x) * MAXIT) / g.na;
    if (per_round < 1) per_round = 1;
    for (int l0 = 0; l0 < g.lines; l0 += per_round) {
        const int lr = min(per_round, g.lines - l0);
        const int items = lr * g.na;
        const int bq = static_cast<int>(blockDim.x) / lr, br = static_cast<int>(blockDim.x) % lr;
        const int lt = static_cast<int>(threadIdx.x) % lr, kt = static_cast<int>(threadIdx.x) / lr;
        T x[MAXIT][NB];
        int ls[MAXIT], ks[MAXIT];
        {
            int l = lt, k1 = kt;
#pragma unroll
            for (int r = 0; r < MAXIT; ++r) {
                ls[r] = l0 + l;
                ks[r] = k1;
                l += br;
                k1 += bq;
                if (l >= lr) {
                    l -= lr;
                    ++k1;
                }
            }
        }
#pragma unroll
        for (int r = 0; r < MAXIT; ++r) {
            const int it = threadIdx.x + r * blockDim.x;
            if (it < items) {
                const T* p = buf + g.base(ls[r]) + ks[r] * g.nb * g.es;
#pragma unroll
                for (int n2 = 0; n2 < NB; ++n2) x[r][n2] = p[n2 * g.es];
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < MAXIT; ++r) {
            const int it = threadIdx.x + r * blockDim.x;
            if (it < items) {
                const int l = ls[r];
                const int k1 = ks[r];
                dft<NB, DIR>(x[r], tw, tws);
                T* p = buf + g.base(l);
#pragma unroll
                for (int k2 = 0; k2 < NB; ++k2) {
                    const int j = k1 + g.na * k2;
                    p[j * g.es] = epi(l, j, x[r][k2]);
                }
            }
        }
        __syncthreads();
    }
}

#define Q3B_FFT_SIZES(X) X(1) X(2) X(3) X(4) X(5) X(6) X(8) X(9) X(10) X(12) X(15) X(16)

template <int DIR, typename T>
__device__ __forceinline__ void run_step1(T* buf, const LineGeom& g, const T* tw) {
    switch (g.na) {
#define Q3B_S1(N) \
    case N: line_step1<N, DIR>(buf, g, tw); break;
        Q3B_FFT_SIZES(Q3B_S1)
#undef Q3B_S1
        default: break;
    }
}

template <int DIR, int MAXIT, typename T, typename Epi>
__device__ __forceinline__ void run_step2(T* buf, const LineGeom& g, const T* tw, const Epi& epi) {
    switch (g.nb) {
#define Q3B_S2(N) \
    case N: line_step2<N, DIR, MAXIT>(buf, g, tw, epi); break;
        Q3B_FFT_SIZES(Q3B_S2)
#undef Q3B_S2
        default: break;
    }
}

// Transform all lines.  Ends with a barrier.  When nb == 1 the first step is
// the whole transform and the second only applies the epilogue.
template <int DIR, int MAXIT, typename T, typename Epi>
__device__ __forceinline__ void lines(T* buf, const LineGeom& g, const T* tw, const Epi& epi) {
    run_step1<DIR>(buf, g, tw);
    __syncthreads();
    run_step2<DIR, MAXIT>(buf, g, tw, epi);
}

}  // namespace fft
}  // namespace q3b
