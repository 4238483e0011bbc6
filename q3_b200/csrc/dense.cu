// FP64 dense kernels for the Davidson subspace; see dense.cuh.
//
// potrf : blocked right-looking upper Cholesky (32x32 blocks): a diagonal
//         block factor + its triangular inverse, a panel solve and a trailing
//         update per block step.
// trtri : U^{-1} by recursive doubling: the diagonal blocks' inverses, then
//         per level the off-diagonal block of each pair, -Inv11 U12 Inv22, as
//         two batched tile products.
// hegv  : H c = w S c reduced to C = U^{-H} H U^{-1} with S = U^H U, as
//         zhegv does (subspace/serial.hpp:18-151 calls zhegv itype 1), solved
//         by heev, back-transformed c = U^{-1} z.
// heev  : Householder tridiagonalisation in one cooperative kernel (one grid
//         barrier per column, each wait bounded), the complex subdiagonal
//         made real by a diagonal phase, eigenvalues by multisection on
//         division-free Sturm counts (one warp per eigenvalue), eigenvectors
//         by inverse iteration in shared memory with Gram-Schmidt inside
//         clusters of close eigenvalues, then Z = Q (phase * Y) by GEMM.
#include <cstring>
#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>
#include <vector>

#include "context.cuh"
#include "dense.cuh"
#include "tridiag.cuh"
#include "q3b.h"

namespace q3b {
namespace dense {
namespace {

constexpr int NB = 32;

__device__ __forceinline__ int vload(const int* p) { return *reinterpret_cast<const volatile int*>(p); }

__device__ __forceinline__ double2 warp_sum(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ------------------------------------------------------------------ potrf
// Diagonal block k, 32x32 threads: warp c, lane r owns element (r, c).  At
// step j every (r, c) with j < r <= c subtracts conj(G(j,r)) G(j,c) / G(j,j)
// (row j of U times its conjugate, taken from the unscaled row) while row j
// is scaled into U: one barrier a step.  The thread that finishes a pivot
// (the diagonal element of the next step) also forms its reciprocal, square
// root and reciprocal square root, so no step waits on a division.  Then
// U^{-1} a column per warp: lane t holds X(t, c) and row r, from the bottom
// up, is a warp sum.
__device__ __forceinline__ void pivot_terms(double piv, int j, int bs, int r0, double* rp, double* sq,
                                            double* isq, int* bad) {
    if (!(piv > 0.0)) {
        if (j < bs) atomicMin(bad, r0 + j + 1);
        piv = 1.0;
    }
    // one reciprocal square root on the step's critical path instead of a
    // square root and two divisions
    const double iq = rsqrt(piv);
    rp[j] = iq * iq;
    sq[j] = piv * iq;
    isq[j] = iq;
}

__global__ void __launch_bounds__(1024, 1)
potrf_diag(int n, int k, double2* A, int lda, double2* dinv, int* info) {
    if (vload(info)) return;
    __shared__ double2 a[NB][NB + 1];  // a[c][r] = G(r, c)
    __shared__ double2 u[NB][NB + 1];  // u[c][r] = U(r, c)
    __shared__ double s_rp[NB], s_sq[NB], s_isq[NB];
    __shared__ int s_bad;
    const int r = threadIdx.x & 31, c = threadIdx.x >> 5;
    const int r0 = k * NB;
    const int bs = min(NB, n - r0);
    {
        double2 v = (r == c) ? mk(1.0, 0.0) : mk(0.0, 0.0);
        if (r < bs && c < bs && r <= c) v = A[(r0 + r) + (long)(r0 + c) * lda];
        a[c][r] = v;
        u[c][r] = mk(0.0, 0.0);
        if (threadIdx.x == 0) s_bad = 0x7fffffff;
    }
    __syncthreads();
    if (threadIdx.x == 0) pivot_terms(a[0][0].x, 0, bs, r0, s_rp, s_sq, s_isq, &s_bad);
    __syncthreads();
    for (int j = 0; j < NB; ++j) {
        if (r == j && c >= j) {
            const double is = s_isq[j];
            u[c][j] = (c == j) ? mk(s_sq[j], 0.0) : mk(a[c][j].x * is, a[c][j].y * is);
        }
        if (j < r && r <= c) {
            const double2 g = cmulc(a[r][j], a[c][j]);  // conj(G(j,r)) G(j,c)
            const double rp = s_rp[j];
            const double2 v = a[c][r] - mk(g.x * rp, g.y * rp);
            a[c][r] = v;
            if (r == c && r == j + 1) pivot_terms(v.x, j + 1, bs, r0, s_rp, s_sq, s_isq, &s_bad);
        }
        __syncthreads();
    }
    // column c of X = U^{-1}; lane t holds X(t, c)
    double2 x = mk(0.0, 0.0);
    for (int rr = c; rr >= 0; --rr) {
        double2 p = (rr < r && r <= c) ? cmul(u[r][rr], x) : mk(0.0, 0.0);
        p = warp_sum(p);
        if (r == rr) {
            const double2 rhs = (rr == c) ? mk(1.0 - p.x, -p.y) : mk(-p.x, -p.y);
            const double iu = s_isq[rr];
            x = mk(rhs.x * iu, rhs.y * iu);
        }
    }
    if (r < bs && c < bs && r <= c) A[(r0 + r) + (long)(r0 + c) * lda] = u[c][r];
    dinv[(long)k * NB * NB + r + c * NB] = x;
    if (threadIdx.x == 0 && s_bad != 0x7fffffff) atomicCAS(info, 0, s_bad);
}

// U(k, j) = U_kk^{-H} G(k, j) for every block column j > k
__global__ void __launch_bounds__(256)
potrf_panel(int n, int k, double2* A, int lda, const double2* dinv, const int* info) {
    if (vload(info)) return;
    __shared__ double2 xk[NB][NB + 1];  // xk[c][r] = Xk(r, c)
    __shared__ double2 g[NB][NB + 1];   // g[c][t] = G(k_t, j_c)
    const int j = k + 1 + blockIdx.x;
    const int r0 = k * NB, c0 = j * NB;
    const int bsk = min(NB, n - r0), bsj = min(NB, n - c0);
    const int tid = threadIdx.x;
    for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
        const int r = idx % NB, c = idx / NB;
        xk[c][r] = dinv[(long)k * NB * NB + r + c * NB];
        g[c][r] = (r < bsk && c < bsj) ? A[(r0 + r) + (long)(c0 + c) * lda] : mk(0.0, 0.0);
    }
    __syncthreads();
    for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
        const int r = idx % NB, c = idx / NB;
        double2 s = mk(0.0, 0.0);
        for (int t = 0; t <= r; ++t) s = s + cmulc(xk[r][t], g[c][t]);
        if (r < bsk && c < bsj) A[(r0 + r) + (long)(c0 + c) * lda] = s;
    }
}

// G(i, j) -= U(k, i)^H U(k, j) for k < i <= j
__global__ void __launch_bounds__(256) potrf_update(int n, int k, double2* A, int lda, const int* info) {
    if (vload(info)) return;
    const int i = k + 1 + blockIdx.x, j = k + 1 + blockIdx.y;
    if (i > j) return;
    __shared__ double2 ui[NB][NB + 1];  // ui[r][t] = U(k_t, i_r)
    __shared__ double2 uj[NB][NB + 1];  // uj[c][t] = U(k_t, j_c)
    const int r0 = k * NB, ci = i * NB, cj = j * NB;
    const int bsk = min(NB, n - r0), bsi = min(NB, n - ci), bsj = min(NB, n - cj);
    const int tid = threadIdx.x;
    for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
        const int t = idx % NB, c = idx / NB;
        ui[c][t] = (t < bsk && c < bsi) ? A[(r0 + t) + (long)(ci + c) * lda] : mk(0.0, 0.0);
        uj[c][t] = (t < bsk && c < bsj) ? A[(r0 + t) + (long)(cj + c) * lda] : mk(0.0, 0.0);
    }
    __syncthreads();
    for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
        const int r = idx % NB, c = idx / NB;
        if (r >= bsi || c >= bsj) continue;
        double2 s = mk(0.0, 0.0);
        for (int t = 0; t < NB; ++t) s = s + cmulc(ui[r][t], uj[c][t]);
        double2* p = A + (ci + r) + (long)(cj + c) * lda;
        *p = *p - s;
    }
}

// ------------------------------------------------------------------ trtri
__global__ void trtri_diag(int n, const double2* dinv, double2* U) {
    const int k = blockIdx.x;
    const int r0 = k * NB, bs = min(NB, n - r0);
    for (int idx = threadIdx.x; idx < NB * NB; idx += blockDim.x) {
        const int r = idx % NB, c = idx / NB;
        if (r < bs && c < bs) U[(r0 + r) + (long)(r0 + c) * n] = dinv[(long)k * NB * NB + r + c * NB];
    }
}

// One level of the recursive triangular inverse.  At level m the diagonal
// blocks of order m are inverted already; pair p joins blocks [r1, r1+m) and
// [r2, r2+m2) (r1 = 2mp, r2 = r1 + m, m2 = min(m, n - r2)) through
//   inv([U11 U12; 0 U22]) = [Inv11, -Inv11 U12 Inv22; 0, Inv22]:
// mode 0 forms T_p = U12 Inv22 (m x m2, ld m, in T), mode 1 writes
// Inv12 = -Inv11 T_p into Ui.  Block (blockIdx.y, blockIdx.z) is a 32x32 tile
// of the product; K runs over 32-chunks, skipping the zero chunks of the
// triangular factor, with the next chunk's tiles loaded into registers while
// the current one is multiplied.
__global__ void __launch_bounds__(256)
trtri_level(int n, int m, int mode, const double2* U, int ldu, double2* Ui, double2* T) {
    const int p = blockIdx.x, ti = blockIdx.y, tj = blockIdx.z;
    const int r1 = 2 * m * p, r2 = r1 + m;
    const int m2 = min(m, n - r2);
    if (m2 <= 0 || tj * NB >= m2) return;
    __shared__ double2 sa[NB][NB + 1];  // sa[k][i] = A(i, k)
    __shared__ double2 sb[NB][NB + 1];  // sb[j][k] = B(k, j)
    double2* Tp = T + (size_t)p * m * m;
    const int kmax = (mode == 0) ? m2 : m;
    const int kc0 = (mode == 0) ? 0 : ti;                               // Inv11 upper triangular
    const int kc1 = (mode == 0) ? min(tj, (m2 - 1) / NB) : (kmax - 1) / NB;  // Inv22 upper triangular
    const int tid = threadIdx.x;
    auto a_at = [&](int i, int k) -> double2 {
        if (k >= kmax) return mk(0.0, 0.0);
        return mode == 0 ? U[(r1 + i) + (long)(r2 + k) * ldu] : Ui[(r1 + i) + (long)(r1 + k) * n];
    };
    auto b_at = [&](int k, int j) -> double2 {
        if (k >= kmax || j >= m2) return mk(0.0, 0.0);
        return mode == 0 ? Ui[(r2 + k) + (long)(r2 + j) * n] : Tp[k + (long)j * m];
    };
    double2 ra[4], rb[4], acc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        acc[q] = mk(0.0, 0.0);
        const int idx = tid + q * 256, x = idx % NB, y = idx / NB;
        ra[q] = (kc0 <= kc1) ? a_at(ti * NB + x, kc0 * NB + y) : mk(0.0, 0.0);
        rb[q] = (kc0 <= kc1) ? b_at(kc0 * NB + x, tj * NB + y) : mk(0.0, 0.0);
    }
    for (int kc = kc0; kc <= kc1; ++kc) {
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int idx = tid + q * 256, x = idx % NB, y = idx / NB;
            sa[y][x] = ra[q];
            sb[y][x] = rb[q];
        }
        __syncthreads();
        if (kc < kc1) {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int idx = tid + q * 256, x = idx % NB, y = idx / NB;
                ra[q] = a_at(ti * NB + x, (kc + 1) * NB + y);
                rb[q] = b_at((kc + 1) * NB + x, tj * NB + y);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int idx = tid + q * 256, i = idx % NB, j = idx / NB;
            double2 v = acc[q];
#pragma unroll 8
            for (int k = 0; k < NB; ++k) v = v + cmul(sa[k][i], sb[j][k]);
            acc[q] = v;
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int idx = tid + q * 256, i = ti * NB + idx % NB, j = tj * NB + idx / NB;
        if (i >= m || j >= m2) continue;
        if (mode == 0) Tp[i + (long)j * m] = acc[q];
        else Ui[(r1 + i) + (long)(r2 + j) * n] = mk(-acc[q].x, -acc[q].y);
    }
}

// ------------------------------------------------------------------ helpers
// dst (n x n, ld n) = full Hermitian matrix from the upper triangle of src (ld lds)
__global__ void hermitian_from_upper(int n, const double2* src, int lds, double2* dst) {
    const long total = (long)n * n;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        const int r = static_cast<int>(idx % n), c = static_cast<int>(idx / n);
        double2 v;
        if (r < c) v = src[r + (long)c * lds];
        else if (r > c) v = conj2(src[c + (long)r * lds]);
        else v = mk(src[r + (long)c * lds].x, 0.0);
        dst[idx] = v;
    }
}

__global__ void copy_matrix(int n, const double2* src, int lds, double2* dst, int ldd) {
    const long total = (long)n * n;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        const int r = static_cast<int>(idx % n), c = static_cast<int>(idx / n);
        dst[r + (long)c * ldd] = src[r + (long)c * lds];
    }
}

inline int grid_for(long n) { return stride_grid(n, 8); }

// ------------------------------------------------------------ grid barrier
// One monotonic arrival counter: the e-th barrier of a launch completes when
// the counter reaches e * nblocks.  Every wait is bounded (about 2 s of
// clock), after which the kernel records an error and all blocks leave.
__device__ unsigned& grid_epoch() {
    __shared__ unsigned s_epoch;
    return s_epoch;
}
__device__ __forceinline__ void grid_sync_init() {
    if (threadIdx.x == 0) grid_epoch() = 0;
}
__device__ __forceinline__ bool grid_sync(unsigned* bar, unsigned nblocks, int* err) {
    __shared__ int s_ok;
    unsigned& s_epoch = grid_epoch();
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned epoch = s_epoch + 1;  // barriers this block has entered
        s_epoch = epoch;
        __threadfence();
        atomicAdd(bar, 1u);
        const unsigned target = epoch * nblocks;
        int ok = 1;
        const long long t0 = clock64();
        while (true) {
            unsigned cur;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(cur) : "l"(bar) : "memory");
            if (cur >= target) break;
            if (vload(err)) {
                ok = 0;
                break;
            }
            if (clock64() - t0 > (1LL << 32)) {
                atomicExch(err, 1);
                ok = 0;
                break;
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ------------------------------------------------------------------ hetrd
// A (n x n, ld n, full Hermitian; read once) reduced to tridiagonal form by
// reflectors H_k = I - tau_k v_k v_k^H on rows/columns k+1..n-1, with
//   d[k] = A_kk,  e[k] = T(k+1, k) (complex),  W = Q^H = H_{n-2} ... H_0,
// so that A = Q T Q^H and an eigenvector of A is W^H times one of T.
// Block b owns columns c = b + G*j (cyclic, G = gridDim.x); it keeps them in
// shared memory for the whole reduction, and its columns of W too when they
// fit (`w_in_smem`), else in global memory.
//
// One grid barrier per column step.  Before it, every block publishes its
// entries of p = tau A v and its share of v^H p, and the owner of column k+1
// publishes that column as it stands before step k's update.  After it, every
// block reads the three together (one L2 latency), forms w, and applies step
// k's rank-2 update to its own copy of column k+1, which is the next step's
// Householder input: no block waits for another between the barriers.  The
// published vectors are double-buffered by step parity; a block can run at
// most one step ahead of another (the next barrier holds it), so nothing is
// overwritten while it is still being read.  Every wait is bounded.
__global__ void __launch_bounds__(256, 1)
hetrd_smem(int n, int cpb, int w_in_smem, const double2* A, double* d, double2* e, double2* W,
           double2* xpre2, double2* pbuf2, double2* partial2, unsigned* bar, int* err) {
    extern __shared__ __align__(16) unsigned char smem[];
    double2* cols = reinterpret_cast<double2*>(smem);   // cpb columns of A
    double2* sv = cols + (size_t)cpb * n;              // v
    double2* sw = sv + n;                              // w
    double2* sx = sw + n;                              // column k, rows k.. (the next v)
    double2* wsm = sx + n;                             // cpb columns of W (if w_in_smem)
    __shared__ double red[8];
    __shared__ double2 redc[8];
    __shared__ double s_tau;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int G = gridDim.x, b = blockIdx.x;
    const int owned = b < n ? (n - b + G - 1) / G : 0;
    grid_sync_init();
    auto wcol = [&](int jj) -> double2* { return w_in_smem ? wsm + (size_t)jj * n : W + (size_t)(b + G * jj) * n; };
    for (int jj = 0; jj < owned; ++jj) {
        const int c = b + G * jj;
        double2* wc = wcol(jj);
        for (int r = tid; r < n; r += blockDim.x) {
            cols[(size_t)jj * n + r] = A[r + (size_t)c * n];
            wc[r] = (r == c) ? mk(1.0, 0.0) : mk(0.0, 0.0);
        }
    }
    for (int r = tid; r < n; r += blockDim.x) sx[r] = A[r];  // column 0
    __syncthreads();
    for (int k = 0; k + 1 < n; ++k) {
        const int m = n - k - 1;
        const int par = k & 1;
        double2* pbuf = pbuf2 + (size_t)par * n;
        double2* partial = partial2 + (size_t)par * G;
        double2* xpre = xpre2 + (size_t)par * n;
        double part = 0.0;
        for (int j = tid; j < m; j += blockDim.x) {
            const double2 x = sx[k + 1 + j];
            sv[j] = x;
            if (j > 0) part += x.x * x.x + x.y * x.y;
        }
        part = warp_sum(part);
        if (lane == 0) red[warp] = part;
        __syncthreads();
        if (tid == 0) {
            double sigma = 0.0;
            for (int q = 0; q < 8; ++q) sigma += red[q];
            const double2 x0 = sv[0];
            double t = 0.0;
            double2 alpha = x0;
            if (m > 1 && sigma > 0.0) {
                const double ax0 = hypot(x0.x, x0.y);
                const double nrm = sqrt(sigma + ax0 * ax0);
                alpha = ax0 > 0.0 ? mk(-nrm * x0.x / ax0, -nrm * x0.y / ax0) : mk(-nrm, 0.0);
                const double2 v0 = x0 - alpha;
                t = 2.0 / (sigma + v0.x * v0.x + v0.y * v0.y);
                sv[0] = v0;
            }
            s_tau = t;
            if (b == 0) {
                d[k] = sx[k].x;
                e[k] = alpha;
            }
        }
        // the owner of column k+1 publishes it as it stands before this step
        if ((k + 1) % G == b) {
            const double2* col = cols + (size_t)((k + 1) / G) * n + (k + 1);
            for (int j = tid; j < m; j += blockDim.x) xpre[j] = col[j];
        }
        __syncthreads();
        const double tk = s_tau;
        // p_i = tau (column i)^H v for the owned columns i > k; this block's share of v^H p
        double2 acc = mk(0.0, 0.0);
        if (tk != 0.0) {
            for (int jj = warp; jj < owned; jj += 8) {
                const int i = b + G * jj;
                if (i <= k) continue;
                const double2* col = cols + (size_t)jj * n + (k + 1);
                double2 sacc = mk(0.0, 0.0);
                for (int j = lane; j < m; j += 32) sacc = sacc + cmulc(col[j], sv[j]);
                sacc = warp_sum(sacc);
                const double2 p = mk(tk * sacc.x, tk * sacc.y);
                if (lane == 0) pbuf[i] = p;
                acc = acc + cmulc(sv[i - k - 1], p);
            }
        }
        if (lane == 0) redc[warp] = acc;
        __syncthreads();
        if (tid == 0) {
            double2 sacc = mk(0.0, 0.0);
            for (int q = 0; q < 8; ++q) sacc = sacc + redc[q];
            partial[b] = sacc;
        }
        if (!grid_sync(bar, G, err)) return;
        // column k+1 before the update, p and the shares, read together
        for (int j = tid; j < m; j += blockDim.x) {
            sx[k + 1 + j] = __ldcg(&xpre[j]);
            if (tk != 0.0) sw[j] = __ldcg(&pbuf[k + 1 + j]);
        }
        if (tk != 0.0 && warp == 0) {
            double2 sacc = mk(0.0, 0.0);
            for (int q = lane; q < G; q += 32) sacc = sacc + __ldcg(&partial[q]);
            sacc = warp_sum(sacc);
            if (lane == 0) redc[0] = sacc;
        }
        __syncthreads();
        if (tk != 0.0) {
            const double half = 0.5 * tk * redc[0].x;  // v^H p is real
            for (int j = tid; j < m; j += blockDim.x) {
                const double2 p = sw[j];
                sw[j] = mk(p.x - half * sv[j].x, p.y - half * sv[j].y);
            }
            __syncthreads();
            // the next step's column: A[k+1+j, k+1] -= v_j conj(w_0) + w_j conj(v_0)
            {
                const double2 v0 = sv[0], w0 = sw[0];
                for (int j = tid; j < m; j += blockDim.x) {
                    const double2 u = cmul(sv[j], conj2(w0)) + cmul(sw[j], conj2(v0));
                    sx[k + 1 + j] = sx[k + 1 + j] - u;
                }
            }
            for (int jj = warp; jj < owned; jj += 8) {
                const int i = b + G * jj;
                // W column: W[k+1:, i'] -= tau v (v^H W[k+1:, i'])
                double2* wc = wcol(jj) + (k + 1);
                double2 sacc = mk(0.0, 0.0);
                for (int j = lane; j < m; j += 32) sacc = sacc + cmulc(sv[j], wc[j]);
                sacc = warp_sum(sacc);
                const double2 f = mk(tk * sacc.x, tk * sacc.y);
                for (int j = lane; j < m; j += 32) wc[j] = wc[j] - cmul(sv[j], f);
                if (i <= k) continue;
                // A[j, i] -= v_j conj(w_i) + w_j conj(v_i)
                const double2 vi = sv[i - k - 1], wi = sw[i - k - 1];
                double2* col = cols + (size_t)jj * n + (k + 1);
                for (int j = lane; j < m; j += 32) {
                    const double2 u = cmul(sv[j], conj2(wi)) + cmul(sw[j], conj2(vi));
                    col[j] = col[j] - u;
                }
            }
        }
        __syncthreads();
    }
    if (b == 0 && tid == 0) {
        d[n - 1] = sx[n - 1].x;
        e[n - 1] = mk(0.0, 0.0);
    }
    if (w_in_smem) {
        for (int jj = 0; jj < owned; ++jj) {
            const int c = b + G * jj;
            for (int r = tid; r < n; r += blockDim.x) W[r + (size_t)c * n] = wsm[(size_t)jj * n + r];
        }
    }
}

// |e|, e^2, Gershgorin bounds and the phases delta_{k+1} = delta_k e_k/|e_k|
// (a prefix product: one warp, chunks of the vector per lane, a shuffle scan
// across lanes)
__global__ void tridiag_prep(int n, const double* d, const double2* e, double* ea, double* e2,
                             double2* phase, double* bounds) {
    const int lane = threadIdx.x;
    if (blockIdx.x != 0 || lane >= 32) return;
    const int chunk = (n + 31) / 32;
    const int k0 = lane * chunk, k1 = min(n, k0 + chunk);
    double lo = 1e300, hi = -1e300;
    for (int k = k0; k < k1; ++k) {
        const double a = (k + 1 < n) ? hypot(e[k].x, e[k].y) : 0.0;
        if (k + 1 < n) {
            ea[k] = a;
            e2[k] = a * a;
        }
        const double left = (k > 0) ? hypot(e[k - 1].x, e[k - 1].y) : 0.0;
        lo = fmin(lo, d[k] - left - a);
        hi = fmax(hi, d[k] + left + a);
    }
    // product of the unit factors u_k = e_k/|e_k| over this lane's chunk
    double2 prod = mk(1.0, 0.0);
    for (int k = k0; k < k1 && k + 1 < n; ++k) {
        const double a = hypot(e[k].x, e[k].y);
        if (a > 0.0) prod = cmul(prod, mk(e[k].x / a, e[k].y / a));
    }
    // exclusive scan of the chunk products across lanes
    double2 incl = prod;
    for (int o = 1; o < 32; o <<= 1) {
        double2 t;
        t.x = __shfl_up_sync(0xffffffffu, incl.x, o);
        t.y = __shfl_up_sync(0xffffffffu, incl.y, o);
        if (lane >= o) incl = cmul(t, incl);
    }
    double2 ph;
    ph.x = __shfl_up_sync(0xffffffffu, incl.x, 1);
    ph.y = __shfl_up_sync(0xffffffffu, incl.y, 1);
    if (lane == 0) ph = mk(1.0, 0.0);
    for (int k = k0; k < k1; ++k) {
        phase[k] = ph;
        if (k + 1 < n) {
            const double a = hypot(e[k].x, e[k].y);
            if (a > 0.0) ph = cmul(ph, mk(e[k].x / a, e[k].y / a));
        }
    }
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

// Yc[:, c] = phase .* Y[:, c] (complex)
__global__ void apply_phase(int n, int nvec, const double2* phase, const double* Y, double2* Yc) {
    const long total = (long)n * nvec;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int r = static_cast<int>(t % n);
        const double2 p = phase[r];
        const double y = Y[t];
        Yc[t] = mk(p.x * y, p.y * y);
    }
}

// one warp per eigenvalue (the lowest nw): multisection of [lo, hi] on Sturm
// counts at 32 x kShifts interior points per round (the interval shrinks
// 65-fold).  The block stages d and e^2 in shared memory when they fit
// (kSturmSmemOrder), so the count's loads do not wait on L1 or L2.
constexpr int kShifts = 2;
constexpr int kSturmSmemOrder = 3072;
__global__ void tridiag_multisect(int n, const double* d, const double* e2, const double* bounds, double* w,
                                  int nw) {
    extern __shared__ double sturm_smem[];
    if (n <= kSturmSmemOrder) {
        for (int k = threadIdx.x; k < n; k += blockDim.x) {
            sturm_smem[k] = d[k];
            sturm_smem[n + k] = e2[k];
        }
        __syncthreads();
        d = sturm_smem;
        e2 = sturm_smem + n;
    }
    const int lane = threadIdx.x & 31;
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= nw) return;
    constexpr int P = 32 * kShifts;  // points per round
    double a = bounds[0], b = bounds[1];
    const double scale = bounds[2];
    const double pivmin = fmax(1e-290, 1e-300 * scale * scale);
    const double tol = 4.0 * 2.220446049250313e-16 * fmax(scale, 1e-300);
    for (int it = 0; it < 64 && (b - a) > tol; ++it) {
        double x[kShifts];
        int cnt[kShifts];
#pragma unroll
        for (int s = 0; s < kShifts; ++s) x[s] = a + (b - a) * (lane * kShifts + s + 1) / (P + 1.0);
        sturm_counts<kShifts>(n, d, e2, x, pivmin, cnt);
        // first point (in order lane*kShifts + s) with more than i eigenvalues below it
        int first = kShifts;
#pragma unroll
        for (int s = kShifts - 1; s >= 0; --s)
            if (cnt[s] > i) first = s;
        const unsigned above = __ballot_sync(0xffffffffu, first < kShifts);
        const int l = above ? __ffs(above) - 1 : 32;
        const int fl = __shfl_sync(0xffffffffu, first, l & 31);
        const int m = (l == 32) ? P : l * kShifts + fl;
        const double na = (m == 0) ? a : a + (b - a) * m / (P + 1.0);
        const double nb = (m == P) ? b : a + (b - a) * (m + 1) / (P + 1.0);
        a = na;
        b = nb;
    }
    if (lane == 0) w[i] = 0.5 * (a + b);
}

// Inverse iteration, one thread per cluster of close eigenvalues;
// Gram-Schmidt inside a cluster.  Vectors of eigenvalues a gap g apart come
// out orthogonal to about eps ||T|| / g without it, so clusters are cut at a
// gap of 1e-5 ||T|| (orthogonality ~1e-11 across clusters).
__global__ void tridiag_invit(int n, const double* d, const double* ea, const double* w,
                              const double* bounds, int nvec, double* Y, double* work) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nvec) return;
    const double scale = fmax(bounds[2], 1e-300);
    const double ortol = 1e-5 * scale;
    if (i > 0 && w[i] - w[i - 1] <= ortol) return;
    int jend = i + 1;
    while (jend < nvec && w[jend] - w[jend - 1] <= ortol) ++jend;
    double* DL = work + (size_t)i * 5 * n;
    double* D = DL + n;
    double* DU = D + n;
    double* DU2 = DU + n;
    int* piv = reinterpret_cast<int*>(DU2 + n);
    const double eps = 2.220446049250313e-16;
    const double tiny = eps * scale;
    double lam_prev = 0.0;
    for (int j = i; j < jend; ++j) {
        double lam = w[j];
        if (j > i && lam - lam_prev < 10.0 * eps * scale) lam = lam_prev + 10.0 * eps * scale;
        lam_prev = lam;
        // LU with partial pivoting of T - lam I
        for (int t = 0; t < n; ++t) {
            D[t] = d[t] - lam;
            if (t + 1 < n) {
                DL[t] = ea[t];
                DU[t] = ea[t];
            }
            DU2[t] = 0.0;
            piv[t] = t;
        }
        for (int t = 0; t + 1 < n; ++t) {
            if (fabs(D[t]) >= fabs(DL[t])) {
                if (D[t] == 0.0) D[t] = tiny;
                const double f = DL[t] / D[t];
                DL[t] = f;
                D[t + 1] -= f * DU[t];
            } else {
                const double f = D[t] / DL[t];
                D[t] = DL[t];
                DL[t] = f;
                const double tmp = DU[t];
                DU[t] = D[t + 1];
                D[t + 1] = tmp - f * D[t + 1];
                if (t + 2 < n) {
                    DU2[t] = DU[t + 1];
                    DU[t + 1] = -f * DU[t + 1];
                }
                piv[t] = t + 1;
            }
        }
        for (int t = 0; t < n; ++t)
            if (fabs(D[t]) < tiny) D[t] = D[t] < 0.0 ? -tiny : tiny;
        double* y = Y + (size_t)j * n;
        for (int t = 0; t < n; ++t) y[t] = 1.0 + 0.25 * sin(0.7 * t + 1.3 * j);
        for (int iter = 0; iter < 3; ++iter) {
            for (int t = 0; t + 1 < n; ++t) {
                if (piv[t] == t) {
                    y[t + 1] -= DL[t] * y[t];
                } else {
                    const double tmp = y[t];
                    y[t] = y[t + 1];
                    y[t + 1] = tmp - DL[t] * y[t];
                }
            }
            y[n - 1] /= D[n - 1];
            if (n > 1) y[n - 2] = (y[n - 2] - DU[n - 2] * y[n - 1]) / D[n - 2];
            for (int t = n - 3; t >= 0; --t) y[t] = (y[t] - DU[t] * y[t + 1] - DU2[t] * y[t + 2]) / D[t];
            for (int q = i; q < j; ++q) {
                const double* yq = Y + (size_t)q * n;
                double s = 0.0;
                for (int t = 0; t < n; ++t) s += yq[t] * y[t];
                for (int t = 0; t < n; ++t) y[t] -= s * yq[t];
            }
            double nr = 0.0;
            for (int t = 0; t < n; ++t) nr += y[t] * y[t];
            nr = 1.0 / sqrt(nr);
            for (int t = 0; t < n; ++t) y[t] *= nr;
        }
    }
}

// The same inverse iteration with each thread's factors and iterate in shared
// memory, laid out [t][thread] (a warp's accesses fall in distinct banks), the
// recurrences carried in registers and the pivots' reciprocals stored, so a
// step of each sweep is a few shared-memory accesses and fused multiply-adds.
// blockDim.x threads (one per eigenvalue) share the block's shared memory:
// 41 bytes per thread and row.
__global__ void tridiag_invit_smem(int n, const double* d, const double* ea, const double* w,
                                   const double* bounds, int nvec, double* Y) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int T = blockDim.x, tid = threadIdx.x;
    double* DL = reinterpret_cast<double*>(smem);
    double* DU = DL + (size_t)n * T;
    double* DU2 = DU + (size_t)n * T;
    double* DI = DU2 + (size_t)n * T;
    double* y = DI + (size_t)n * T;
    unsigned char* piv = reinterpret_cast<unsigned char*>(y + (size_t)n * T);
    const int i = blockIdx.x * T + tid;
    if (i >= nvec) return;
    const double scale = fmax(bounds[2], 1e-300);
    const double ortol = 1e-5 * scale;
    if (i > 0 && w[i] - w[i - 1] <= ortol) return;
    int jend = i + 1;
    while (jend < nvec && w[jend] - w[jend - 1] <= ortol) ++jend;
    const double eps = 2.220446049250313e-16;
    const double tiny = eps * scale;
    double lam_prev = 0.0;
#define AT(t) ((size_t)(t) * T + tid)
    for (int j = i; j < jend; ++j) {
        double lam = w[j];
        if (j > i && lam - lam_prev < 10.0 * eps * scale) lam = lam_prev + 10.0 * eps * scale;
        lam_prev = lam;
        // LU with partial pivoting of T - lam I; (dcur, ducur) = row t's
        // diagonal and superdiagonal as modified by the steps before it
        double dcur = d[0] - lam, ducur = n > 1 ? ea[0] : 0.0;
        for (int t = 0; t + 1 < n; ++t) {
            const double sub = ea[t];
            const double dnext = d[t + 1] - lam;
            const double dunext = (t + 2 < n) ? ea[t + 1] : 0.0;
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
#pragma unroll 4
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
#pragma unroll 4
            for (int t = n - 2; t >= 0; --t) {
                const double v = (y[AT(t)] - DU[AT(t)] * y1 - DU2[AT(t)] * y2) * DI[AT(t)];
                y[AT(t)] = v;
                nr += v * v;
                y2 = y1;
                y1 = v;
            }
            if (j > i) {
                for (int q = i; q < j; ++q) {
                    const double* yq = Y + (size_t)q * n;
                    double s = 0.0;
                    for (int t = 0; t < n; ++t) s += yq[t] * y[AT(t)];
                    for (int t = 0; t < n; ++t) y[AT(t)] -= s * yq[t];
                }
                nr = 0.0;
                for (int t = 0; t < n; ++t) nr += y[AT(t)] * y[AT(t)];
            }
            ys = 1.0 / sqrt(nr);
        }
        double* yo = Y + (size_t)j * n;
        for (int t = 0; t < n; ++t) yo[t] = y[AT(t)] * ys;
    }
#undef AT
}

constexpr size_t kInvitSmemLimit = 200 * 1024;
constexpr int kInvitBytesPerRow = 5 * sizeof(double) + 1;

// elements of the recursive inverse's product buffer: the largest level's
// pairs x m^2
size_t trtri_tbuf_elems(int n) {
    size_t most = 0;
    for (long m = NB; m < n; m *= 2) most = std::max<size_t>(most, (size_t)ceil_div(n, 2 * m) * m * m);
    return most + 1;
}

struct Chol {
    double2* dinv;
    double2* tbuf;  // the recursive inverse's products, n*n/2 at most
    int* info;
};

Chol chol_take(Scratch& ws, int n) {
    const int nblk = ceil_div(n, NB);
    Chol c;
    c.dinv = ws.take<double2>((size_t)nblk * NB * NB);
    c.tbuf = ws.take<double2>(trtri_tbuf_elems(n));
    c.info = ws.take<int>(1);
    return c;
}

void potrf_launch(cudaStream_t st, int n, double2* A, int lda, const Chol& c) {
    const int nblk = ceil_div(n, NB);
    Q3B_CUDA(cudaMemsetAsync(c.info, 0, sizeof(int), st));
    for (int k = 0; k < nblk; ++k) {
        potrf_diag<<<1, 1024, 0, st>>>(n, k, A, lda, c.dinv, c.info);
        Q3B_LAUNCH_CHECK();
        const int m = nblk - k - 1;
        if (m > 0) {
            potrf_panel<<<m, 256, 0, st>>>(n, k, A, lda, c.dinv, c.info);
            Q3B_LAUNCH_CHECK();
            potrf_update<<<dim3(m, m), 256, 0, st>>>(n, k, A, lda, c.info);
            Q3B_LAUNCH_CHECK();
        }
    }
}

int potrf_impl(cudaStream_t st, int n, double2* A, int lda, const Chol& c) {
    potrf_launch(st, n, A, lda, c);
    int* hb = static_cast<int*>(host_readback(sizeof(int)));
    Q3B_CUDA(cudaMemcpyAsync(hb, c.info, sizeof(int), cudaMemcpyDeviceToHost, st));
    Q3B_CUDA(cudaStreamSynchronize(st));
    return hb[0];
}

void trtri_impl(cudaStream_t st, int n, const double2* A, int lda, const Chol& c, double2* Ui) {
    const int nblk = ceil_div(n, NB);
    Q3B_CUDA(cudaMemsetAsync(Ui, 0, (size_t)n * n * sizeof(double2), st));
    trtri_diag<<<nblk, 256, 0, st>>>(n, c.dinv, Ui);
    Q3B_LAUNCH_CHECK();
    for (int m = NB; m < n; m *= 2) {
        const int pairs = ceil_div(n, 2 * m);
        const dim3 grid(pairs, m / NB, m / NB);
        trtri_level<<<grid, 256, 0, st>>>(n, m, 0, A, lda, Ui, c.tbuf);
        Q3B_LAUNCH_CHECK();
        trtri_level<<<grid, 256, 0, st>>>(n, m, 1, A, lda, Ui, c.tbuf);
        Q3B_LAUNCH_CHECK();
    }
}

}  // namespace

size_t potrf_scratch_bytes(int n) {
    const size_t nblk = (size_t)ceil_div(n, NB);
    return nblk * NB * NB * sizeof(double2) + trtri_tbuf_elems(n) * sizeof(double2) + 2048;
}

size_t hegv_scratch_bytes(int n) {
    // hegv: U, U^-1, H, H U^-1 (n x n complex each) and the eigenvector block;
    // heev: W (n x n complex), Y and D Y, five real work vectors per
    // eigenvector; a few length-n vectors; 256-byte alignment slack
    const size_t nn = (size_t)n * n;
    return potrf_scratch_bytes(n) + 5 * nn * sizeof(double2) + nn * (sizeof(double2) + 6 * sizeof(double)) +
           nn * sizeof(double2) + 64 * (size_t)n * sizeof(double2) + 2 * (size_t)device_sms() * sizeof(double2) +
           (size_t)n * sizeof(unsigned) + 64 * 1024;
}

bool order_supported(int n) {
    if (n < 1) return false;
    const int nsm = device_sms();
    const int G = std::max(1, std::min(nsm, (n + 7) / 8));
    const int cpb = (n + G - 1) / G;
    return ((size_t)cpb * n + 3 * (size_t)n) * sizeof(double2) <= 200 * 1024;
}

int potrf(cudaStream_t st, int n, double2* A, int lda, Scratch& ws) {
    Chol c = chol_take(ws, n);
    return potrf_impl(st, n, A, lda, c);
}

void trtri_after_potrf(cudaStream_t st, int n, const double2* A, int lda, double2* Uinv, Scratch& ws) {
    Chol c = chol_take(ws, n);  // the slices potrf took first, still holding its block inverses
    trtri_impl(st, n, A, lda, c, Uinv);
}

namespace {

// Everything heev's launches need, taken from the scratch in a fixed order:
// planning twice from the same scratch state gives the same pointers, which
// the graph replays of hegv rely on.
struct HeevPlan {
    int n = 0, nvec = 0;
    double* d;
    double2* e;
    double2* W;
    double2* xpre;
    double2* pbuf;
    double* ea;
    double* e2;
    double2* phase;
    double* bounds;
    double* Y;
    double* work;
    double2* Yc;
    double2* partial;
    unsigned* bar;
    int* err;
    int G = 1, cpb = 1, w_in_smem = 0;
    size_t smem = 0;
};

HeevPlan heev_plan(int n, int nvec, Scratch& ws) {
    HeevPlan p;
    p.n = n;
    p.nvec = nvec;
    const int nv = nvec > 0 ? nvec : 1;
    p.d = ws.take<double>(n);
    p.e = ws.take<double2>(n);
    p.W = ws.take<double2>((size_t)n * n);
    p.xpre = ws.take<double2>(2 * (size_t)n);
    p.pbuf = ws.take<double2>(2 * (size_t)n);
    p.ea = ws.take<double>(n);
    p.e2 = ws.take<double>(n);
    p.phase = ws.take<double2>(n);
    p.bounds = ws.take<double>(4);
    p.Y = ws.take<double>((size_t)n * nv);
    p.work = ws.take<double>((size_t)5 * n * nv);
    p.Yc = ws.take<double2>((size_t)n * nv);
    int device = 0;
    Q3B_CUDA(cudaGetDevice(&device));
    int nsm = 0;
    Q3B_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    static PerDeviceOnce once_inv;
    once_inv.run([] {
        cudaFuncSetAttribute(tridiag_invit_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInvitSmemLimit);
    });
    // blocks: about 8 columns each, at most one per SM; columns (and W) in shared memory
    p.G = std::max(1, std::min(nsm, (n + 7) / 8));
    p.cpb = (n + p.G - 1) / p.G;
    const size_t limit = 200 * 1024;
    p.smem = ((size_t)p.cpb * n + 3 * (size_t)n) * sizeof(double2);
    if (p.smem > limit)
        throw Status(Q3B_ERR_INVALID, "subspace of order " + std::to_string(n) + " too large for the eigensolver");
    p.w_in_smem = (p.smem + (size_t)p.cpb * n * sizeof(double2) <= limit) ? 1 : 0;
    if (p.w_in_smem) p.smem += (size_t)p.cpb * n * sizeof(double2);
    p.partial = ws.take<double2>(2 * (size_t)p.G);
    p.bar = ws.take<unsigned>(2);
    p.err = ws.take<int>(1);
    static PerDeviceOnce once;
    once.run([limit] {
        cudaFuncSetAttribute(hetrd_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)limit);
        cudaFuncSetAttribute(tridiag_invit_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInvitSmemLimit);
    });
    int per_sm = 0;
    Q3B_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hetrd_smem, 256, p.smem));
    if (per_sm < 1 || per_sm * nsm < p.G) throw Status(Q3B_ERR_INVALID, "eigensolver blocks cannot be co-resident");
    return p;
}

// heev's launches, no host synchronisation (the timeout word is read by the caller)
void heev_launch(cudaStream_t st, const HeevPlan& p, const double2* A, double* w, double2* Z,
                 const GemmWorkspace& gws) {
    const int n = p.n, nvec = p.nvec;
    Q3B_CUDA(cudaMemsetAsync(p.bar, 0, 2 * sizeof(unsigned), st));
    Q3B_CUDA(cudaMemsetAsync(p.err, 0, sizeof(int), st));
    {
        int nn = n, cpb = p.cpb, wis = p.w_in_smem;
        const double2* Ac = A;
        double* d = p.d;
        double2 *e = p.e, *W = p.W, *xpre = p.xpre, *pbuf = p.pbuf, *partial = p.partial;
        unsigned* bar = p.bar;
        int* err = p.err;
        void* args[] = {&nn, &cpb, &wis, &Ac, &d, &e, &W, &xpre, &pbuf, &partial, &bar, &err};
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(p.G);
        cfg.blockDim = dim3(256);
        cfg.dynamicSmemBytes = p.smem;
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        Q3B_CUDA(cudaLaunchKernelExC(&cfg, (const void*)hetrd_smem, args));
        Q3B_LAUNCH_CHECK();
    }
    tridiag_prep<<<1, 32, 0, st>>>(n, p.d, p.e, p.ea, p.e2, p.phase, p.bounds);
    Q3B_LAUNCH_CHECK();
    const int nw = nvec > 0 ? nvec : n;
    const size_t sturm_smem = n <= kSturmSmemOrder ? 2 * (size_t)n * sizeof(double) : 0;
    tridiag_multisect<<<ceil_div((long)nw * 32, 256), 256, sturm_smem, st>>>(n, p.d, p.e2, p.bounds, w, nw);
    Q3B_LAUNCH_CHECK();
    if (nvec > 0) {
        const int T = static_cast<int>(std::min<size_t>(64, kInvitSmemLimit / ((size_t)n * kInvitBytesPerRow)));
        if (T >= 1) {
            const size_t sm = (size_t)n * T * kInvitBytesPerRow;
            tridiag_invit_smem<<<ceil_div(nvec, T), T, sm, st>>>(n, p.d, p.ea, w, p.bounds, nvec, p.Y);
        } else {
            tridiag_invit<<<ceil_div(nvec, 64), 64, 0, st>>>(n, p.d, p.ea, w, p.bounds, nvec, p.Y, p.work);
        }
        Q3B_LAUNCH_CHECK();
        apply_phase<<<grid_for((long)n * nvec), 256, 0, st>>>(n, nvec, p.phase, p.Y, p.Yc);
        Q3B_LAUNCH_CHECK();
        const double2 one = mk(1.0, 0.0), zero = mk(0.0, 0.0);
        cgemm<double>(st, true, n, nvec, n, one, p.W, n, p.Yc, n, zero, Z, n, gws);   // Z = W^H (D Y)
    }
}

int read_flag(cudaStream_t st, const int* flag) {
    int* hb = static_cast<int*>(host_readback(sizeof(int)));
    Q3B_CUDA(cudaMemcpyAsync(hb, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    Q3B_CUDA(cudaStreamSynchronize(st));
    return hb[0];
}

}  // namespace

void heev(cudaStream_t st, int n, double2* A, double* w, double2* Z, int nvec, Scratch& ws,
          const GemmWorkspace& gws) {
    if (n <= 0) return;
    const HeevPlan p = heev_plan(n, nvec, ws);
    heev_launch(st, p, A, w, Z, gws);
    if (read_flag(st, p.err)) throw Status(Q3B_ERR_INTERNAL, "eigensolver grid barrier timed out");
}

HegvGraphs::~HegvGraphs() {
    for (int i = 0; i < count_; ++i)
        if (entries_[i].exec) cudaGraphExecDestroy(entries_[i].exec);
}

bool HegvGraphs::Key::operator==(const Key& o) const {
    return n == o.n && ld == o.ld && nvec == o.nvec && H == o.H && S == o.S && w == o.w && Z == o.Z &&
           ws == o.ws && gws == o.gws && ws_used == o.ws_used && ws_bytes == o.ws_bytes &&
           gws_bytes == o.gws_bytes && st == o.st;
}

HegvGraphs::Entry* HegvGraphs::find(const Key& k) {
    for (int i = 0; i < count_; ++i) {
        if (entries_[i].key == k) {
            entries_[i].used = ++tick_;
            if (entries_[i].exec)
                for (unsigned long long l = 0; l < entries_[i].launches; ++l) count_launch();
            return &entries_[i];
        }
    }
    return nullptr;
}

void HegvGraphs::store(const Key& k, cudaGraphExec_t e) {
    int slot = count_;
    if (count_ == kMax) {
        slot = 0;
        for (int i = 1; i < kMax; ++i)
            if (entries_[i].used < entries_[slot].used) slot = i;
        if (entries_[slot].exec) cudaGraphExecDestroy(entries_[slot].exec);
    } else {
        ++count_;
    }
    entries_[slot] = Entry{k, e, ++tick_, 0, 1};
}

cudaGraphExec_t HegvGraphs::capture(cudaStream_t st, void (*issue)(void*), void* ctx) {
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaGetLastError();
        disabled = true;
        return nullptr;
    }
    const unsigned long long l0 = launches();
    bool ok = true;
    try {
        issue(ctx);
    } catch (const std::exception&) {
        ok = false;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    cudaGraphExec_t exec = nullptr;
    if (ok && e == cudaSuccess && g && cudaGraphInstantiate(&exec, g, 0) == cudaSuccess) {
        captured_launches_ = launches() - l0;
    } else {
        exec = nullptr;
        disabled = true;
    }
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    return exec;
}

namespace {
std::atomic<int> g_block_max_order{kBlockOrderDefault};
}  // namespace

void set_block_max_order(int n) { g_block_max_order.store(n < 0 ? 0 : n); }
int block_max_order() { return g_block_max_order.load(); }

int hegv(cudaStream_t st, int n, const double2* H, const double2* S, int ld, double* w, double2* Z,
         int nvec, Scratch& ws, const GemmWorkspace& gws, HegvGraphs* graphs, double* w_host) {
    if (n <= 0) return 0;
    const int nv = nvec > 0 ? nvec : n;
    if (n <= block_max_order() && hegv_block_fits(n, nv)) {
        // one block: a single launch and one synchronisation (dense_block.cu)
        double2* work = ws.take<double2>(hegv_block_work_elems(n));
        int* info = ws.take<int>(1);
        hegv_block(st, BlockProblem{n, ld, nv, H, S, w, Z, work, info});
        char* hb = static_cast<char*>(host_readback(sizeof(double) + (w_host ? nv * sizeof(double) : 0)));
        int* flag = reinterpret_cast<int*>(hb);
        double* wb = reinterpret_cast<double*>(hb + sizeof(double));
        Q3B_CUDA(cudaMemcpyAsync(flag, info, sizeof(int), cudaMemcpyDeviceToHost, st));
        if (w_host) Q3B_CUDA(cudaMemcpyAsync(wb, w, nv * sizeof(double), cudaMemcpyDeviceToHost, st));
        Q3B_CUDA(cudaStreamSynchronize(st));
        if (w_host) std::memcpy(w_host, wb, nv * sizeof(double));
        return flag[0];
    }
    const size_t used0 = ws.used;
    const size_t nn = (size_t)n * n;
    // every slice first, in a fixed order: the same pointers on every call
    double2* Uw = ws.take<double2>(nn);
    Chol c = chol_take(ws, n);
    double2* Ui = ws.take<double2>(nn);
    double2* Hf = ws.take<double2>(nn);
    double2* W = ws.take<double2>(nn);
    double2* Zc = ws.take<double2>((size_t)n * (nvec > 0 ? nvec : 1));
    const HeevPlan hp = heev_plan(n, nvec, ws);
    auto issue = [&] {
        const double2 one = mk(1.0, 0.0), zero = mk(0.0, 0.0);
        copy_matrix<<<grid_for((long)nn), 256, 0, st>>>(n, S, ld, Uw, n);
        Q3B_LAUNCH_CHECK();
        potrf_launch(st, n, Uw, n, c);
        trtri_impl(st, n, Uw, n, c, Ui);
        hermitian_from_upper<<<grid_for((long)nn), 256, 0, st>>>(n, H, ld, Hf);
        Q3B_LAUNCH_CHECK();
        cgemm<double>(st, false, n, n, n, one, Hf, n, Ui, n, zero, W, n, gws);     // H U^{-1}
        cgemm<double>(st, true, n, n, n, one, Ui, n, W, n, zero, Hf, n, gws);      // U^{-H} H U^{-1}
        // make it exactly Hermitian from its upper triangle
        hermitian_from_upper<<<grid_for((long)nn), 256, 0, st>>>(n, Hf, n, W);
        Q3B_LAUNCH_CHECK();
        heev_launch(st, hp, W, w, Zc, gws);
        if (nvec > 0) cgemm<double>(st, false, n, nvec, n, one, Ui, n, Zc, n, zero, Z, n, gws);
    };
    cudaGraphExec_t ex = nullptr;
    if (graphs) {
        const HegvGraphs::Key key{n, ld, nvec, H, S, w, Z, ws.base, gws.ptr, used0, ws.bytes, gws.bytes, st};
        ex = graphs->get(key, issue);
    }
    if (ex) {
        Q3B_CUDA(cudaGraphLaunch(ex, st));
    } else {
        issue();
    }
    // a failed Cholesky leaves the later steps on garbage: their result is
    // discarded, and every loop in them is bounded
    // status words and eigenvalues read back together, one synchronisation
    const size_t nw = nvec > 0 ? nvec : n;
    char* hb = static_cast<char*>(host_readback(2 * sizeof(double) + (w_host ? nw * sizeof(double) : 0)));
    int* flags = reinterpret_cast<int*>(hb);
    double* wb = reinterpret_cast<double*>(hb + 2 * sizeof(double));
    Q3B_CUDA(cudaMemcpyAsync(&flags[0], c.info, sizeof(int), cudaMemcpyDeviceToHost, st));
    Q3B_CUDA(cudaMemcpyAsync(&flags[1], hp.err, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (w_host) Q3B_CUDA(cudaMemcpyAsync(wb, w, nw * sizeof(double), cudaMemcpyDeviceToHost, st));
    Q3B_CUDA(cudaStreamSynchronize(st));
    if (w_host) std::memcpy(w_host, wb, nw * sizeof(double));
    if (flags[1]) throw Status(Q3B_ERR_INTERNAL, "eigensolver grid barrier timed out");
    return flags[0] ? n + flags[0] : 0;
}

}  // namespace dense
}  // namespace q3b
