#include <algorithm>
// Complex GEMMs on CUDA cores; see cgemm.cuh.
#include <type_traits>

#include "cgemm.cuh"

namespace q3b {
namespace {

constexpr int kBM = 64;
constexpr int kBN = 64;
constexpr int kThreads = 256;

template <typename R> struct GemmTile;
template <> struct GemmTile<double> { static constexpr int BK = 8; };
template <> struct GemmTile<float> { static constexpr int BK = 16; };

// One BM x BN tile of C per block (64x64, or 32x32 for small products),
// (BM/16) x (BN/16) complex outputs per thread.  With kchunk < K the block
// handles K range [z*kchunk, (z+1)*kchunk) and writes its raw sum to part[z]
// (ld M); otherwise it applies alpha/beta into C.
template <typename R, bool CONJ_A, int BM = kBM, int BN = kBN>
__global__ void __launch_bounds__(kThreads)
cgemm_kernel(int M, int N, int K, cplx_t<R> alpha, const cplx_t<R>* __restrict__ A, long lda,
             const cplx_t<R>* __restrict__ B, long ldb, cplx_t<R> beta, cplx_t<R>* C, long ldc,
             int kchunk, cplx_t<R>* part) {
    using T = cplx_t<R>;
    constexpr int BK = GemmTile<R>::BK;
    constexpr int TM = BM / 16, TN = BN / 16;  // outputs per thread
    constexpr int LA = (BK * BM + kThreads - 1) / kThreads;  // complex loads per thread, A tile
    constexpr int LB = (BK * BN + kThreads - 1) / kThreads;
    __shared__ T As[2][BK][BM + 1];
    __shared__ T Bs[2][BK][BN + 1];

    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    // N tiles run fastest: the blocks that share an A tile run together
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kbeg = blockIdx.z * kchunk;
    const int kend = min(K, kbeg + kchunk);

    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = czero<T>();

    T ra[LA], rb[LB];
    auto load = [&](int k0) {
#pragma unroll
        for (int r = 0; r < LA; ++r) {
            const int idx = tid + r * kThreads;
            int k, m;
            if (CONJ_A) {
                k = idx % BK;
                m = idx / BK;
            } else {
                m = idx % BM;
                k = idx / BM;
            }
            const int gk = k0 + k, gm = m0 + m;
            T v = czero<T>();
            if (idx < BK * BM && gk < kend && gm < M) {
                v = CONJ_A ? conj2(A[gk + (long)gm * lda]) : A[gm + (long)gk * lda];
            }
            ra[r] = v;
        }
#pragma unroll
        for (int r = 0; r < LB; ++r) {
            const int idx = tid + r * kThreads;
            const int k = idx % BK, n = idx / BK;
            const int gk = k0 + k, gn = n0 + n;
            rb[r] = (idx < BK * BN && gk < kend && gn < N) ? B[gk + (long)gn * ldb] : czero<T>();
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int r = 0; r < LA; ++r) {
            const int idx = tid + r * kThreads;
            if (idx >= BK * BM) continue;
            int k, m;
            if (CONJ_A) {
                k = idx % BK;
                m = idx / BK;
            } else {
                m = idx % BM;
                k = idx / BM;
            }
            As[buf][k][m] = ra[r];
        }
#pragma unroll
        for (int r = 0; r < LB; ++r) {
            const int idx = tid + r * kThreads;
            if (idx >= BK * BN) continue;
            Bs[buf][idx % BK][idx / BK] = rb[r];
        }
    };

    int buf = 0;
    if (kbeg < kend) {
        load(kbeg);
        store(0);
    }
    __syncthreads();
    for (int k0 = kbeg; k0 < kend; k0 += BK) {
        const bool more = (k0 + BK) < kend;
        if (more) load(k0 + BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            T a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; ++i) a[i] = As[buf][kk][ty + 16 * i];
#pragma unroll
            for (int j = 0; j < TN; ++j) b[j] = Bs[buf][kk][tx + 16 * j];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < TN; ++j) cfma(acc[i][j], a[i], b[j]);
        }
        if (more) store(buf ^ 1);
        __syncthreads();
        buf ^= 1;
    }

    const bool use_beta = (beta.x != R(0) || beta.y != R(0));
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int gm = m0 + ty + 16 * i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int gn = n0 + tx + 16 * j;
            if (gn >= N) continue;
            if (part) {
                part[(long)blockIdx.z * M * N + (long)gn * M + gm] = acc[i][j];
            } else {
                T v = cmul(alpha, acc[i][j]);
                T* c = C + gm + (long)gn * ldc;
                if (use_beta) v = v + cmul(beta, *c);
                *c = v;
            }
        }
    }
}

// C = alpha * sum_z part[z] + beta * C, the splits summed in index order
template <typename R>
__global__ void splitk_reduce(int M, int N, int splits, const cplx_t<R>* __restrict__ part,
                              cplx_t<R> alpha, cplx_t<R> beta, cplx_t<R>* C, long ldc) {
    using T = cplx_t<R>;
    const long total = (long)M * N;
    const bool use_beta = (beta.x != R(0) || beta.y != R(0));
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        const int m = static_cast<int>(idx % M);
        const int n = static_cast<int>(idx / M);
        T s = splits > 0 ? part[idx] : czero<T>();
        for (int z = 1; z < splits; ++z) s = s + part[(long)z * total + idx];
        T v = cmul(alpha, s);
        T* c = C + m + (long)n * ldc;
        if (use_beta) v = v + cmul(beta, *c);
        *c = v;
    }
}

// Products whose 64x64 tiling has fewer tiles than the GPU has SMs (the
// subspace eigensolver's n x n x n products up to n = 767) run on 32x32 tiles:
// four times the blocks and a quarter of the serial K loop per block.
constexpr long kSmallTiles = 148;
inline bool small_tiles(int M, int N) { return (long)ceil_div(M, kBM) * ceil_div(N, kBN) < kSmallTiles; }

// K splits for a product with `tiles` output tiles (never more than for
// 64x64 tiles, which size the workspace)
inline int choose_splits_for(int tiles, int K) {
    const int target = 2 * 148;
    int s = ceil_div(target, tiles);
    const int kmax = ceil_div(K, 128);
    if (s > kmax) s = kmax;
    if (s < 1) s = 1;
    if (s > 64) s = 64;
    return s;
}

template <typename R> int choose_splits(int M, int N, int K) {
    return choose_splits_for(ceil_div(M, kBM) * ceil_div(N, kBN), K);
}

}  // namespace

bool use_tensor_cores(int M, int N, int K) { return (double)M * N * K >= kTensorCoreMinMacs; }

template <typename R> size_t cgemm_workspace_bytes(int M, int N, int K) {
    const int s = choose_splits<R>(M, N, K);
    const size_t simt = s > 1 ? (size_t)s * M * N * sizeof(cplx_t<R>) : 0;
    if constexpr (std::is_same<R, float>::value) return std::max(simt, tc::workspace_bytes(M, N, K));
    return simt;
}

template <typename R>
void cgemm(cudaStream_t st, bool conj_a, int M, int N, int K, cplx_t<R> alpha, const cplx_t<R>* A,
           long lda, const cplx_t<R>* B, long ldb, cplx_t<R> beta, cplx_t<R>* C, long ldc,
           const GemmWorkspace& ws) {
    using T = cplx_t<R>;
    if (M <= 0 || N <= 0) return;
    constexpr int BK = GemmTile<R>::BK;
    if constexpr (std::is_same<R, float>::value) {
        // small products stay on the CUDA cores: a tensor-core block takes a
        // whole SM's shared memory, which small problems, often several at
        // once on separate streams, cannot keep busy
        if (K > 0 && use_tensor_cores(M, N, K)) {
            tc::cgemm(st, conj_a, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, ws);
            return;
        }
    }
    if (K <= 0) {
        // C = beta * C
        dim3 g(ceil_div((long)M * N, 256));
        splitk_reduce<R><<<g, 256, 0, st>>>(M, N, 0, nullptr, alpha, beta, C, ldc);
        Q3B_LAUNCH_CHECK();
        return;
    }
    const bool small = small_tiles(M, N);
    const int bm = small ? 32 : kBM;
    int splits = conj_a ? choose_splits_for(ceil_div(M, bm) * ceil_div(N, bm), K) : 1;
    size_t need = (size_t)splits * M * N * sizeof(T);
    if (splits > 1 && (ws.ptr == nullptr || ws.bytes < need)) splits = 1;
    int kchunk = K;
    if (splits > 1) {
        kchunk = ceil_div(K, splits);
        kchunk = ceil_div(kchunk, BK) * BK;
        splits = ceil_div(K, kchunk);
    }
    if (ceil_div(M, bm) > 65535) throw std::runtime_error("complex GEMM: M too large");
    dim3 grid(ceil_div(N, bm), ceil_div(M, bm), splits);
    T* part = splits > 1 ? static_cast<T*>(ws.ptr) : nullptr;
    if (small) {
        if (conj_a)
            cgemm_kernel<R, true, 32, 32><<<grid, kThreads, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta,
                                                                    C, ldc, kchunk, part);
        else
            cgemm_kernel<R, false, 32, 32><<<grid, kThreads, 0, st>>>(M, N, K, alpha, A, lda, B, ldb,
                                                                     beta, C, ldc, kchunk, part);
    } else if (conj_a) {
        cgemm_kernel<R, true><<<grid, kThreads, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C,
                                                         ldc, kchunk, part);
    } else {
        cgemm_kernel<R, false><<<grid, kThreads, 0, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C,
                                                          ldc, kchunk, part);
    }
    Q3B_LAUNCH_CHECK();
    if (splits > 1) {
        const long total = (long)M * N;
        int blocks = ceil_div(total, 256);
        if (blocks > 4096) blocks = 4096;
        splitk_reduce<R><<<blocks, 256, 0, st>>>(M, N, splits, part, alpha, beta, C, ldc);
        Q3B_LAUNCH_CHECK();
    }
}

template void cgemm<double>(cudaStream_t, bool, int, int, int, double2, const double2*, long,
                            const double2*, long, double2, double2*, long, const GemmWorkspace&);
template void cgemm<float>(cudaStream_t, bool, int, int, int, float2, const float2*, long,
                           const float2*, long, float2, float2*, long, const GemmWorkspace&);
template size_t cgemm_workspace_bytes<double>(int, int, int);
template size_t cgemm_workspace_bytes<float>(int, int, int);

}  // namespace q3b
