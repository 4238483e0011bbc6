// The generalized Hermitian eigensolver for small orders in one thread block,
// and many such problems in one launch (dense.cuh, BlockProblem).
//
// The multi-kernel solver of dense.cu spreads each step of an order-n problem
// over the whole device; for the subspaces of small cells (n up to about 100)
// its cost is the launch and barrier latency of a few dozen kernels, not
// arithmetic.  Here one block of 512 threads holds the problem in shared
// memory and runs every step with block barriers only:
//   1. S = U^H U, the upper Cholesky factor in place (right-looking, one
//      pivot row per step, a warp per column of the trailing update);
//   2. U^{-1} by back substitution, one thread per column (kept in the
//      factor's free lower triangle), to global scratch;
//   3. C = U^{-H} H U^{-1} as two register-tiled products (H U^{-1} from the
//      shared copy of H, then U^{-H} T), kept Hermitian from its upper triangle;
//   4. C = Q T Q^H, Householder reflectors H_k = I - tau_k v_k v_k^H chosen so
//      that the subdiagonal comes out real (LAPACK's zlarfg convention), one
//      column per step: p = tau C v by warp-column partial sums, the rank-2
//      update C -= v w^H + w v^H a warp per column, and the next reflector by
//      warp 0 from the first updated column while the others finish;
//   5. the lowest nvec eigenvalues of the real tridiagonal by multisection on
//      Sturm counts, eight lanes per eigenvalue;
//   6. their eigenvectors by inverse iteration, one thread per cluster of close
//      eigenvalues with Gram-Schmidt inside the cluster (as dense.cu);
//   7. z = U^{-1} Q y: the reflectors applied to three vectors at a time by one
//      warp (the vectors in registers), then the triangular product.
// Only __syncthreads / __syncwarp synchronise; nothing waits on another block.
#include <algorithm>
#include <mutex>

#include "context.cuh"
#include "dense.cuh"
#include "tridiag.cuh"
#include "q3b.h"

namespace q3b {
namespace dense {
namespace {

constexpr int kBT = 512;            // threads per problem
constexpr int kBW = kBT / 32;       // warps per problem
constexpr int kTile = 4;            // outputs per thread along each axis of the products
constexpr int kMaxRowsPerLane = 4;  // the back-transform keeps a vector in registers: n <= 128
constexpr size_t kSmemLimit = 232448;

__host__ __device__ inline int pitch_of(int n) { return n | 1; }
__host__ __device__ inline size_t align16(size_t b) { return (b + 15) & ~size_t(15); }

// shared memory: region A (the n x P matrix and a column per warp, or the
// inverse iteration's arrays), then the vectors
__host__ __device__ inline size_t region_a(int n, int nvec) {
    const size_t mat = (size_t)n * pitch_of(n) * 16 + (size_t)kBW * n * 16;
    const size_t inv = 5 * align16((size_t)n * nvec * 8) + align16((size_t)n * nvec);
    return align16(mat > inv ? mat : inv);
}
__host__ __device__ inline size_t vec_bytes(int n) {
    return 4 * align16((size_t)n * 16) + 4 * align16((size_t)n * 8) + 64;
}

__device__ __forceinline__ double2 wsum2(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}
__device__ __forceinline__ double wsum1(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// S = U^H U in place in A (upper triangle, pitch P) from the upper triangle of
// S (ld ld); rdiag[r] = 1 / U[r][r].  Returns false (in every thread) when the
// leading minor of order k+1 is not positive definite, with k+1 in *fail.
__device__ __forceinline__ bool cholesky_in_smem(int n, int P, const double2* S, int ld, double2* A, double* rdiag,
                                                 int* fail) {
    const int tid = threadIdx.x;
    for (int idx = tid; idx < n * n; idx += kBT) {
        const int i = idx % n, j = idx / n;
        if (i <= j) A[i + (size_t)j * P] = S[i + (size_t)j * ld];
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const double piv = A[k + (size_t)k * P].x;
        if (!(piv > 0.0)) {  // the same value in every thread: all leave together
            if (tid == 0) *fail = k + 1;
            return false;
        }
        const double rs = 1.0 / sqrt(piv);
        for (int j = k + 1 + tid; j < n; j += kBT) A[k + (size_t)j * P] = rs * A[k + (size_t)j * P];
        __syncthreads();
        // trailing update of the upper triangle: a warp per column j, lanes along rows i <= j
        for (int j = k + 1 + (tid >> 5); j < n; j += kBW) {
            const double2 ukj = A[k + (size_t)j * P];
            double2* col = A + (size_t)j * P;
            for (int i = k + 1 + (tid & 31); i <= j; i += 32) col[i] = col[i] - cmulc(A[k + (size_t)i * P], ukj);
        }
        if (tid == 0) A[k + (size_t)k * P] = mk(sqrt(piv), 0.0);
        __syncthreads();
    }
    for (int r = tid; r < n; r += kBT) rdiag[r] = 1.0 / A[r + (size_t)r * P].x;
    __syncthreads();
    return true;
}

// U^{-1} (n x n, ld n, zero below the diagonal) into Uinv from the factor in A.
// Thread c solves U x = e_c by back substitution; x is kept transposed in row c
// of A's lower triangle (x_r at A[c][r], r <= c), which no other column reads,
// while every thread reads the strictly upper U.  Four accumulators shorten the
// dependent FMA chain of each dot product.
__device__ __forceinline__ void inverse_to_global(int n, int P, double2* A, const double* rdiag, double2* Uinv) {
    const int c = threadIdx.x;
    if (c < n) {
        double2* xr = A + c;  // x_r at xr[r * P]
        for (int r = c; r >= 0; --r) {
            double2 s0 = mk(0.0, 0.0), s1 = mk(0.0, 0.0), s2 = mk(0.0, 0.0), s3 = mk(0.0, 0.0);
            int k = r + 1;
            for (; k + 3 <= c; k += 4) {
                cfma(s0, A[r + (size_t)k * P], xr[(size_t)k * P]);
                cfma(s1, A[r + (size_t)(k + 1) * P], xr[(size_t)(k + 1) * P]);
                cfma(s2, A[r + (size_t)(k + 2) * P], xr[(size_t)(k + 2) * P]);
                cfma(s3, A[r + (size_t)(k + 3) * P], xr[(size_t)(k + 3) * P]);
            }
            for (; k <= c; ++k) cfma(s0, A[r + (size_t)k * P], xr[(size_t)k * P]);
            const double2 sum = (s0 + s1) + (s2 + s3);
            xr[(size_t)r * P] = rdiag[r] * mk(((r == c) ? 1.0 : 0.0) - sum.x, -sum.y);
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < n * n; idx += kBT) {
        const int r = idx % n, col = idx / n;
        Uinv[idx] = r <= col ? A[col + (size_t)r * P] : mk(0.0, 0.0);
    }
}

__device__ __forceinline__ void hegv_block_body(const BlockProblem& pr) {
    const int n = pr.n, nvec = pr.nvec, ld = pr.ld, P = pitch_of(n);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    extern __shared__ __align__(16) unsigned char sm[];
    double2* A = reinterpret_cast<double2*>(sm);
    double2* xw = A + (size_t)n * P + (size_t)warp * n;  // this warp's column
    double2* part = A + (size_t)n * P;                     // the columns' area as one array
    unsigned char* vb = sm + region_a(n, nvec);
    double2* v = reinterpret_cast<double2*>(vb);
    vb += align16((size_t)n * 16);
    double2* pv = reinterpret_cast<double2*>(vb);
    vb += align16((size_t)n * 16);
    double2* tau = reinterpret_cast<double2*>(vb);
    vb += align16((size_t)n * 16);
    double2* v2 = reinterpret_cast<double2*>(vb);  // the other reflector buffer
    vb += align16((size_t)n * 16);
    double* d = reinterpret_cast<double*>(vb);
    vb += align16((size_t)n * 8);
    double* e = reinterpret_cast<double*>(vb);
    vb += align16((size_t)n * 8);
    double* e2 = reinterpret_cast<double*>(vb);
    vb += align16((size_t)n * 8);
    double* wv = reinterpret_cast<double*>(vb);
    vb += align16((size_t)n * 8);
    double* bounds = reinterpret_cast<double*>(vb);
    double2* Uinv = pr.work;                 // n x n, ld n
    double2* W2 = pr.work + (size_t)n * n;   // T, then C, then the reflectors (column k: rows k+1..)
    double2* Z = pr.Z;                       // n x nvec, ld n

    // ---- 1. S = U^H U (upper triangle, in place); 2. U^{-1} to global scratch
    int* fail = reinterpret_cast<int*>(bounds + 3);
    if (!cholesky_in_smem(n, P, pr.S, ld, A, wv, fail)) {
        if (tid == 0) *pr.info = n + *fail;
        return;
    }
    inverse_to_global(n, P, A, wv, Uinv);
    __syncthreads();

    // ---- 3. C = U^{-H} H U^{-1}
    for (int idx = tid; idx < n * n; idx += kBT) {
        const int i = idx % n, j = idx / n;
        A[i + (size_t)j * P] = i <= j ? pr.H[i + (size_t)j * ld] : conj2(pr.H[j + (size_t)i * ld]);
    }
    __syncthreads();
    const int nt = (n + kTile - 1) / kTile;
    // T = H U^{-1}: rows ib + nt*ii (consecutive threads, consecutive rows), columns j0..j0+3;
    // U^{-1} is upper triangular, so k runs to the tile's last column
    for (int t = tid; t < nt * nt; t += kBT) {
        const int ib = t % nt, j0 = (t / nt) * kTile;
        double2 acc[kTile][kTile];
#pragma unroll
        for (int a = 0; a < kTile; ++a)
#pragma unroll
            for (int c = 0; c < kTile; ++c) acc[a][c] = mk(0.0, 0.0);
        const int kmax = min(n, j0 + kTile);
        for (int k = 0; k < kmax; ++k) {
            double2 x[kTile], y[kTile];
#pragma unroll
            for (int a = 0; a < kTile; ++a) {
                const int i = ib + nt * a;
                x[a] = i < n ? A[i + (size_t)k * P] : mk(0.0, 0.0);
            }
#pragma unroll
            for (int c = 0; c < kTile; ++c) {
                const int j = j0 + c;
                y[c] = j < n ? Uinv[k + (size_t)j * n] : mk(0.0, 0.0);
            }
#pragma unroll
            for (int a = 0; a < kTile; ++a)
#pragma unroll
                for (int c = 0; c < kTile; ++c) cfma(acc[a][c], x[a], y[c]);
        }
#pragma unroll
        for (int a = 0; a < kTile; ++a)
#pragma unroll
            for (int c = 0; c < kTile; ++c) {
                const int i = ib + nt * a, j = j0 + c;
                if (i < n && j < n) W2[i + (size_t)j * n] = acc[a][c];
            }
    }
    __syncthreads();
    for (int idx = tid; idx < n * n; idx += kBT) {
        const int i = idx % n, j = idx / n;
        A[i + (size_t)j * P] = W2[i + (size_t)j * n];
    }
    __syncthreads();
    // C = U^{-H} T, upper triangle: rows i0..i0+3 (k runs to the tile's last row),
    // columns jb + nt*c (consecutive threads, consecutive columns)
    for (int t = tid; t < nt * nt; t += kBT) {
        const int jb = t % nt, i0 = (t / nt) * kTile;
        if (i0 > jb + nt * (kTile - 1)) continue;  // the whole tile is below the diagonal
        double2 acc[kTile][kTile];
#pragma unroll
        for (int a = 0; a < kTile; ++a)
#pragma unroll
            for (int c = 0; c < kTile; ++c) acc[a][c] = mk(0.0, 0.0);
        const int kmax = min(n, i0 + kTile);
        for (int k = 0; k < kmax; ++k) {
            double2 x[kTile], y[kTile];
#pragma unroll
            for (int a = 0; a < kTile; ++a) {
                const int i = i0 + a;
                x[a] = i < n ? conj2(Uinv[k + (size_t)i * n]) : mk(0.0, 0.0);
            }
#pragma unroll
            for (int c = 0; c < kTile; ++c) {
                const int j = jb + nt * c;
                y[c] = j < n ? A[k + (size_t)j * P] : mk(0.0, 0.0);
            }
#pragma unroll
            for (int a = 0; a < kTile; ++a)
#pragma unroll
                for (int c = 0; c < kTile; ++c) cfma(acc[a][c], x[a], y[c]);
        }
#pragma unroll
        for (int a = 0; a < kTile; ++a)
#pragma unroll
            for (int c = 0; c < kTile; ++c) {
                const int i = i0 + a, j = jb + nt * c;
                if (i < n && j < n && i <= j) W2[i + (size_t)j * n] = acc[a][c];
            }
    }
    __syncthreads();
    for (int idx = tid; idx < n * n; idx += kBT) {
        const int i = idx % n, j = idx / n;
        A[i + (size_t)j * P] = i < j ? W2[i + (size_t)j * n]
                                     : (i == j ? mk(W2[i + (size_t)i * n].x, 0.0) : conj2(W2[j + (size_t)i * n]));
    }
    __syncthreads();

    // ---- 4. Householder tridiagonalisation, reflectors to W2
    // Warp 0 forms the reflector of column k (x = C[k+1:n, k]) into vk, with tau[k],
    // d[k] and e[k].  From the second column on it does so inside the previous step:
    // column k is the first column of that step's trailing update, which warp 0
    // updates alone and then turns into the next reflector while the other warps
    // update the rest (one phase and one barrier fewer per step).  v alternates
    // between two buffers, as the other warps still read step k's.
    auto reflector = [&](int k, double2* vk) {
        const int m = n - k - 1;
        double ss = 0.0;
        for (int r = 1 + lane; r < m; r += 32) {
            const double2 xr = A[(k + 1 + r) + (size_t)k * P];
            ss += xr.x * xr.x + xr.y * xr.y;
        }
        ss = wsum1(ss);
        const double2 al = A[(k + 1) + (size_t)k * P];
        double2 tk, scal;
        double beta;
        if (ss == 0.0 && al.y == 0.0) {
            tk = mk(0.0, 0.0);
            scal = mk(0.0, 0.0);
            beta = al.x;
        } else {
            const double nrm = sqrt(al.x * al.x + al.y * al.y + ss);
            beta = al.x >= 0.0 ? -nrm : nrm;
            tk = mk((beta - al.x) / beta, -al.y / beta);
            // 1 / (alpha - beta)
            const double2 den = mk(al.x - beta, al.y);
            const double dd = 1.0 / (den.x * den.x + den.y * den.y);
            scal = mk(den.x * dd, -den.y * dd);
        }
        for (int r = lane; r < m; r += 32)
            vk[r] = r == 0 ? mk(1.0, 0.0) : cmul(A[(k + 1 + r) + (size_t)k * P], scal);
        if (lane == 0) {
            d[k] = A[k + (size_t)k * P].x;
            e[k] = beta;
            tau[k] = tk;
        }
    };
    double2* vbuf[2] = {v, v2};
    if (warp == 0 && n > 1) reflector(0, vbuf[0]);
    __syncthreads();
    for (int k = 0; k + 1 < n; ++k) {
        const int m = n - k - 1;  // x = C[k+1:n, k]
        const double2* vk = vbuf[k & 1];
        const double2 tk = tau[k];
        for (int r = tid; r < m; r += kBT) W2[(k + 1 + r) + (size_t)k * n] = vk[r];
        // p = tau C22 v: warp q sums columns q, q + kBW, ... of rows lane, lane + 32,
        // ... into part[q][row] (the per-warp column area, unused here: kBW n >= kBW m);
        // then one thread per row adds the kBW partial sums
        for (int r = lane; r < m; r += 32) {
            double2 s0 = mk(0.0, 0.0), s1 = mk(0.0, 0.0);
            const double2* row = A + (k + 1 + r) + (size_t)(k + 1) * P;
            int c = warp;
            for (; c + kBW < m; c += 2 * kBW) {
                cfma(s0, row[(size_t)c * P], vk[c]);
                cfma(s1, row[(size_t)(c + kBW) * P], vk[c + kBW]);
            }
            if (c < m) cfma(s0, row[(size_t)c * P], vk[c]);
            part[warp * m + r] = s0 + s1;
        }
        __syncthreads();
        if (tid < m) {
            double2 s = mk(0.0, 0.0);
#pragma unroll
            for (int q = 0; q < kBW; ++q) s = s + part[q * m + tid];
            pv[tid] = cmul(tk, s);
        }
        __syncthreads();
        // alpha = -1/2 tau (p^H v), in every warp; w = p + alpha v; C22 -= v w^H + w v^H:
        // a warp per column, lanes along it, each lane's v and w in registers; warp 0
        // takes the first column and then forms the next reflector from it
        double2 dot = mk(0.0, 0.0);
        for (int c = lane; c < m; c += 32) dot = dot + cmulc(pv[c], vk[c]);
        dot = wsum2(dot);
        const double2 a2 = -0.5 * cmul(tk, dot);
        {
            double2 vr[kMaxRowsPerLane], wr[kMaxRowsPerLane];
#pragma unroll
            for (int q = 0; q < kMaxRowsPerLane; ++q) {
                const int r = lane + 32 * q;
                vr[q] = r < m ? vk[r] : mk(0.0, 0.0);
                wr[q] = r < m ? pv[r] + cmul(a2, vr[q]) : mk(0.0, 0.0);
            }
            const int c0 = warp == 0 ? 0 : warp, cstep = warp == 0 ? m : kBW - 1;
            for (int c = c0; c < m; c += cstep) {
                const double2 vc = conj2(vk[c]), wc = conj2(pv[c] + cmul(a2, vk[c]));
                double2* col = A + (k + 1) + (size_t)(k + 1 + c) * P;
#pragma unroll
                for (int q = 0; q < kMaxRowsPerLane; ++q) {
                    const int r = lane + 32 * q;
                    if (r < m) col[r] = col[r] - cmul(vr[q], wc) - cmul(wr[q], vc);
                }
            }
        }
        if (warp == 0 && k + 2 < n) {
            __syncwarp();  // the lanes' updates of column k+1 are visible to the whole warp
            reflector(k + 1, vbuf[(k + 1) & 1]);
        }
        __syncthreads();
    }
    if (tid == 0) d[n - 1] = A[(n - 1) + (size_t)(n - 1) * P].x;
    __syncthreads();

    // ---- 5. the lowest nvec eigenvalues: multisection on Sturm counts
    if (warp == 0) {
        double lo = 1e300, hi = -1e300;
        for (int k = lane; k < n; k += 32) {
            const double left = k > 0 ? fabs(e[k - 1]) : 0.0, right = k + 1 < n ? fabs(e[k]) : 0.0;
            if (k + 1 < n) e2[k] = e[k] * e[k];
            lo = fmin(lo, d[k] - left - right);
            hi = fmax(hi, d[k] + left + right);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
            const double scale = fmax(fabs(lo), fabs(hi));
            bounds[0] = lo - 4.0 * 2.220446049250313e-16 * scale - 1e-300;
            bounds[1] = hi + 4.0 * 2.220446049250313e-16 * scale + 1e-300;
            bounds[2] = scale;
        }
    }
    __syncthreads();
    {
        // eight lanes per eigenvalue, four eigenvalues a warp: a round counts at
        // 16 interior points and keeps the seventeenth of the interval holding it
        constexpr int G = 8, S = 2, NP = G * S;
        const int grp = lane / G, sub = lane % G;
        const double scale = bounds[2];
        const double pivmin = fmax(1e-290, 1e-300 * scale * scale);
        const double tol = 4.0 * 2.220446049250313e-16 * fmax(scale, 1e-300);
        for (int base = warp * (32 / G); base < nvec; base += kBW * (32 / G)) {
            const int i = base + grp;
            const bool valid = i < nvec;
            double a = bounds[0], bb = bounds[1];
            for (int it = 0; it < 64; ++it) {
                const bool active = valid && (bb - a) > tol;
                if (!__any_sync(0xffffffffu, active)) break;
                double x[S];
                int cnt[S];
#pragma unroll
                for (int s = 0; s < S; ++s) x[s] = a + (bb - a) * (sub * S + s + 1) / (NP + 1.0);
                sturm_counts<S>(n, d, e2, x, pivmin, cnt);
                int first = S;
#pragma unroll
                for (int s = S - 1; s >= 0; --s)
                    if (cnt[s] > i) first = s;
                const unsigned ball = __ballot_sync(0xffffffffu, first < S);
                const unsigned gm = (ball >> (grp * G)) & ((1u << G) - 1u);
                const int l = gm ? __ffs(gm) - 1 : G;
                const int fl = __shfl_sync(0xffffffffu, first, grp * G + (l & (G - 1)));
                if (active) {
                    const int mpt = (l == G) ? NP : l * S + fl;
                    const double na = (mpt == 0) ? a : a + (bb - a) * mpt / (NP + 1.0);
                    const double nb = (mpt == NP) ? bb : a + (bb - a) * (mpt + 1) / (NP + 1.0);
                    a = na;
                    bb = nb;
                }
            }
            if (valid && sub == 0) wv[i] = 0.5 * (a + bb);
        }
    }
    __syncthreads();

    // ---- 6. inverse iteration: y_j into Z (real parts), one thread per cluster
    {
        const size_t nn = (size_t)n * nvec;
        double* DL = reinterpret_cast<double*>(sm);
        double* DU = reinterpret_cast<double*>(sm + align16(nn * 8));
        double* DU2 = reinterpret_cast<double*>(sm + 2 * align16(nn * 8));
        double* DI = reinterpret_cast<double*>(sm + 3 * align16(nn * 8));
        double* y = reinterpret_cast<double*>(sm + 4 * align16(nn * 8));
        unsigned char* piv = sm + 5 * align16(nn * 8);
        const int i = tid;
        const double scale = fmax(bounds[2], 1e-300);
        const double ortol = 1e-5 * scale;
        const double eps = 2.220446049250313e-16;
        const double tiny = eps * scale;
        if (i < nvec && !(i > 0 && wv[i] - wv[i - 1] <= ortol)) {
            int jend = i + 1;
            while (jend < nvec && wv[jend] - wv[jend - 1] <= ortol) ++jend;
#define AT(t) ((size_t)(t) * nvec + i)
            double lam_prev = 0.0;
            for (int j = i; j < jend; ++j) {
                double lam = wv[j];
                if (j > i && lam - lam_prev < 10.0 * eps * scale) lam = lam_prev + 10.0 * eps * scale;
                lam_prev = lam;
                // T - lam I = P L U with partial pivoting; T symmetric, off-diagonal e
                double dcur = d[0] - lam, ducur = n > 1 ? e[0] : 0.0;
                for (int t = 0; t + 1 < n; ++t) {
                    const double sub = e[t];
                    const double dnext = d[t + 1] - lam;
                    const double dunext = (t + 2 < n) ? e[t + 1] : 0.0;
                    if (fabs(dcur) >= fabs(sub)) {
                        if (dcur == 0.0) dcur = tiny;
                        const double f = sub / dcur;
                        DL[AT(t)] = f;
                        DU[AT(t)] = ducur;
                        DU2[AT(t)] = 0.0;
                        DI[AT(t)] = 1.0 / clamp_tiny(dcur, tiny);
                        piv[AT(t)] = 0;
                        dcur = dnext - f * ducur;
                        ducur = dunext;
                    } else {
                        const double f = dcur / sub;
                        DL[AT(t)] = f;
                        DU[AT(t)] = dnext;
                        DU2[AT(t)] = dunext;
                        DI[AT(t)] = 1.0 / clamp_tiny(sub, tiny);
                        piv[AT(t)] = 1;
                        dcur = ducur - f * dnext;
                        ducur = -f * dunext;
                    }
                }
                DI[AT(n - 1)] = 1.0 / clamp_tiny(dcur, tiny);
                for (int t = 0; t < n; ++t) y[AT(t)] = 1.0 + 0.25 * sin(0.7 * t + 1.3 * j);
                double ys = 1.0;  // pending normalisation of y
                for (int iter = 0; iter < 3; ++iter) {
                    double ycur = y[AT(0)] * ys;
                    for (int t = 0; t + 1 < n; ++t) {
                        const double ynext = y[AT(t + 1)] * ys;
                        const double f = DL[AT(t)];
                        if (!piv[AT(t)]) {
                            y[AT(t)] = ycur;
                            ycur = ynext - f * ycur;
                        } else {
                            y[AT(t)] = ynext;
                            ycur = ycur - f * ynext;
                        }
                    }
                    double y1 = ycur * DI[AT(n - 1)], y2 = 0.0;
                    y[AT(n - 1)] = y1;
                    double nr = y1 * y1;
                    for (int t = n - 2; t >= 0; --t) {
                        const double val = (y[AT(t)] - DU[AT(t)] * y1 - DU2[AT(t)] * y2) * DI[AT(t)];
                        y[AT(t)] = val;
                        nr += val * val;
                        y2 = y1;
                        y1 = val;
                    }
                    if (j > i) {
                        for (int q = i; q < j; ++q) {
                            const double2* yq = Z + (size_t)q * n;
                            double s = 0.0;
                            for (int t = 0; t < n; ++t) s += yq[t].x * y[AT(t)];
                            for (int t = 0; t < n; ++t) y[AT(t)] -= s * yq[t].x;
                        }
                        nr = 0.0;
                        for (int t = 0; t < n; ++t) nr += y[AT(t)] * y[AT(t)];
                    }
                    ys = 1.0 / sqrt(nr);
                }
                double2* yo = Z + (size_t)j * n;
                for (int t = 0; t < n; ++t) yo[t] = mk(y[AT(t)] * ys, 0.0);
            }
#undef AT
        }
    }
    __syncthreads();

    // ---- 7. z = U^{-1} Q y
    for (int idx = tid; idx < n * n; idx += kBT) {
        const int r = idx % n, k = idx / n;
        if (r > k + 1) A[r + (size_t)k * P] = W2[r + (size_t)k * n];
    }
    __syncthreads();
    constexpr int kCols = 3;  // vectors a warp carries through the reflectors together
    for (int c0 = warp; c0 < nvec; c0 += kCols * kBW) {
        double2 z[kCols][kMaxRowsPerLane];
#pragma unroll
        for (int j = 0; j < kCols; ++j) {
            const int c = c0 + j * kBW;
#pragma unroll
            for (int q = 0; q < kMaxRowsPerLane; ++q) {
                const int r = lane + 32 * q;
                z[j][q] = (c < nvec && r < n) ? Z[r + (size_t)c * n] : mk(0.0, 0.0);
            }
        }
        // Q y = H_0 H_1 ... H_{n-2} y: the last reflector first
        for (int k = n - 2; k >= 0; --k) {
            double2 vr[kMaxRowsPerLane];
#pragma unroll
            for (int q = 0; q < kMaxRowsPerLane; ++q) {
                const int r = lane + 32 * q;
                vr[q] = (r > k && r < n) ? (r == k + 1 ? mk(1.0, 0.0) : A[r + (size_t)k * P]) : mk(0.0, 0.0);
            }
            double2 s[kCols];
#pragma unroll
            for (int j = 0; j < kCols; ++j) {
                s[j] = mk(0.0, 0.0);
#pragma unroll
                for (int q = 0; q < kMaxRowsPerLane; ++q) s[j] = s[j] + cmulc(vr[q], z[j][q]);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int j = 0; j < kCols; ++j) {
                    s[j].x += __shfl_xor_sync(0xffffffffu, s[j].x, o);
                    s[j].y += __shfl_xor_sync(0xffffffffu, s[j].y, o);
                }
            const double2 tk = tau[k];
#pragma unroll
            for (int j = 0; j < kCols; ++j) {
                const double2 ts = cmul(tk, s[j]);
#pragma unroll
                for (int q = 0; q < kMaxRowsPerLane; ++q) z[j][q] = z[j][q] - cmul(vr[q], ts);
            }
        }
#pragma unroll
        for (int j = 0; j < kCols; ++j) {
            const int c = c0 + j * kBW;
            if (c >= nvec) continue;
#pragma unroll
            for (int q = 0; q < kMaxRowsPerLane; ++q) {
                const int r = lane + 32 * q;
                if (r < n) Z[r + (size_t)c * n] = z[j][q];
            }
        }
    }
    __syncthreads();
    for (int idx = tid; idx < n * n; idx += kBT) {
        const int i = idx % n, j = idx / n;
        if (i <= j) A[i + (size_t)j * P] = Uinv[i + (size_t)j * n];
    }
    __syncthreads();
    for (int c = warp; c < nvec; c += kBW) {
        for (int r = lane; r < n; r += 32) xw[r] = Z[r + (size_t)c * n];
        __syncwarp();
        for (int r = lane; r < n; r += 32) {
            double2 s0 = mk(0.0, 0.0), s1 = mk(0.0, 0.0), s2 = mk(0.0, 0.0), s3 = mk(0.0, 0.0);
            int k = r;
            for (; k + 3 < n; k += 4) {
                cfma(s0, A[r + (size_t)k * P], xw[k]);
                cfma(s1, A[r + (size_t)(k + 1) * P], xw[k + 1]);
                cfma(s2, A[r + (size_t)(k + 2) * P], xw[k + 2]);
                cfma(s3, A[r + (size_t)(k + 3) * P], xw[k + 3]);
            }
            for (; k < n; ++k) cfma(s0, A[r + (size_t)k * P], xw[k]);
            Z[r + (size_t)c * n] = (s0 + s1) + (s2 + s3);
        }
        __syncwarp();
    }
    for (int i = tid; i < nvec; i += kBT) pr.w[i] = wv[i];
    if (tid == 0) *pr.info = 0;
}

__global__ void __launch_bounds__(kBT, 1) hegv_block_one(BlockProblem p) { hegv_block_body(p); }

__global__ void __launch_bounds__(kBT, 1) hegv_block_many(const BlockProblem* ps, int count) {
    if ((int)blockIdx.x >= count) return;
    const BlockProblem p = ps[blockIdx.x];
    hegv_block_body(p);
}

// Cholesky and inverse of one Gram matrix (the orthogonalisation's potrf +
// trtri, subspace_manager/serial.hpp:334-339)
__global__ void __launch_bounds__(kBT, 1)
chol_inverse_block(int n, const double2* G, int ldg, double2* Uinv, int* info) {
    extern __shared__ __align__(16) unsigned char sm[];
    const int P = pitch_of(n);
    double2* A = reinterpret_cast<double2*>(sm);
    double* rdiag = reinterpret_cast<double*>(sm + align16((size_t)n * P * 16 + (size_t)kBW * n * 16));
    int* fail = reinterpret_cast<int*>(rdiag + n);
    if (!cholesky_in_smem(n, P, G, ldg, A, rdiag, fail)) {
        if (threadIdx.x == 0) *info = *fail;
        return;
    }
    inverse_to_global(n, P, A, rdiag, Uinv);
    if (threadIdx.x == 0) *info = 0;
}

PerDeviceOnce g_block_attr;

void set_block_attributes() {
    g_block_attr.run([] {
        Q3B_CUDA(cudaFuncSetAttribute(hegv_block_one, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kSmemLimit)));
        Q3B_CUDA(cudaFuncSetAttribute(hegv_block_many, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kSmemLimit)));
        Q3B_CUDA(cudaFuncSetAttribute(chol_inverse_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(kSmemLimit)));
    });
}

bool valid(const BlockProblem& p) {
    return hegv_block_fits(p.n, p.nvec) && p.ld >= p.n && p.H && p.S && p.w && p.Z && p.work && p.info;
}

}  // namespace

size_t hegv_block_smem(int n, int nvec) { return region_a(n, nvec) + vec_bytes(n); }

bool hegv_block_fits(int n, int nvec) {
    return n >= 1 && n <= 32 * kMaxRowsPerLane && nvec >= 1 && nvec <= n &&
           hegv_block_smem(n, nvec) <= kSmemLimit;
}

size_t hegv_block_work_elems(int n) { return 2 * (size_t)n * n; }

static size_t chol_smem(int n) {
    return align16((size_t)n * pitch_of(n) * 16 + (size_t)kBW * n * 16) + (size_t)n * 8 + 16;
}

bool chol_inverse_block_fits(int n) { return n >= 1 && chol_smem(n) <= kSmemLimit; }

void chol_inverse_block(cudaStream_t st, int n, const double2* G, int ldg, double2* Uinv, int* info) {
    if (!chol_inverse_block_fits(n) || ldg < n || !G || !Uinv || !info)
        throw Status(Q3B_ERR_INVALID, "block Cholesky: problem out of range");
    set_block_attributes();
    chol_inverse_block<<<1, kBT, chol_smem(n), st>>>(n, G, ldg, Uinv, info);
    Q3B_LAUNCH_CHECK();
}

void hegv_block(cudaStream_t st, const BlockProblem& p) {
    if (!valid(p)) throw Status(Q3B_ERR_INVALID, "block eigensolver: problem out of range");
    set_block_attributes();
    hegv_block_one<<<1, kBT, hegv_block_smem(p.n, p.nvec), st>>>(p);
    Q3B_LAUNCH_CHECK();
}

void hegv_block_many(cudaStream_t st, const BlockProblem* problems_dev, int count, size_t smem) {
    if (count <= 0) return;
    if (smem > kSmemLimit) throw Status(Q3B_ERR_INVALID, "block eigensolver: problems out of range");
    set_block_attributes();
    hegv_block_many<<<count, kBT, smem, st>>>(problems_dev, count);
    Q3B_LAUNCH_CHECK();
}

}  // namespace dense
}  // namespace q3b
