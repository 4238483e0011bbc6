#include <algorithm>
// Complex GEMMs on CUDA cores; see cgemm.cuh.
#include <cstdint>
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

// ------------------------------------------------------------------ FP64, large tiles
// BM x 64 tiles of C (BM = 16 TM: 128 or 96), TM x 4 complex outputs per
// thread (outputs m = ty + 16 i, n = tx + 16 j), BK = 8 complex of K per stage, three stages filled by 16-byte
// cp.async copies (one complex each; out-of-range elements are zero-filled).
// Each shared-memory read of a stage feeds 128 DFMA per 24 doubles loaded.
// Shared-memory layouts (complex, padded so a warp's reads fall in distinct
// banks): A as [k][m] (pitch 132) when op(A) = A, as [m][k] (pitch 9) when
// op(A) = A^H; B as [n][k] (pitch 9).
namespace big {
constexpr int BM = 128, BN = 64, BK = 16, STAGES = 3, THREADS = 256;
constexpr int KP = BK + 1;         // [m][k] and [n][k]
template <int TM> struct Shape {   // BM = 16 TM rows of C per block
    static constexpr int bm = 16 * TM;
    static constexpr int a_pitch_n = bm + 4;  // [k][m]
    static constexpr int a_stage = (BK * a_pitch_n > bm * KP ? BK * a_pitch_n : bm * KP);  // complex
    static constexpr int b_stage = BN * KP;
    static constexpr size_t smem = (size_t)STAGES * (a_stage + b_stage) * sizeof(double2);
};

__device__ __forceinline__ void cp16(void* dst, const void* src, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
    const int n = valid ? 16 : 0;  // 0 bytes read: the 16 bytes are zero-filled
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
}  // namespace big

template <bool CONJ_A, int TM>
__global__ void __launch_bounds__(big::THREADS, 1)
zgemm_big(int M, int N, int K, double2 alpha, const double2* __restrict__ A, long lda,
          const double2* __restrict__ B, long ldb, double2 beta, double2* C, long ldc, int kchunk,
          double2* part) {
    using namespace big;
    constexpr int BM = Shape<TM>::bm, A_PITCH_N = Shape<TM>::a_pitch_n, A_STAGE = Shape<TM>::a_stage,
                  B_STAGE = Shape<TM>::b_stage;
    extern __shared__ __align__(16) unsigned char zsm[];
    double2* As = reinterpret_cast<double2*>(zsm);
    double2* Bs = As + STAGES * A_STAGE;
    const int tid = threadIdx.x;
    const int tx = tid % 16, ty = tid / 16;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kbeg = blockIdx.z * kchunk;
    const int kend = min(K, kbeg + kchunk);
    const int nk = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;

    // issue the copies of K block `kb` into stage `s`
    auto fill = [&](int kb, int s) {
        const int k0 = kbeg + kb * BK;
        double2* as = As + s * A_STAGE;
        double2* bs = Bs + s * B_STAGE;
        // A: BM x BK complex, TM / 2 per thread
#pragma unroll
        for (int r = 0; r < (BM * BK) / THREADS; ++r) {
            const int idx = tid + r * THREADS;
            if (CONJ_A) {  // A is K x M: each m holds BK consecutive k
                const int k = idx % BK, m = idx / BK;
                const int gk = k0 + k, gm = m0 + m;
                const bool ok = gk < kend && gm < M;
                cp16(as + m * KP + k, ok ? A + gk + (long)gm * lda : A, ok);
            } else {       // A is M x K: each k holds BM consecutive m
                const int m = idx % BM, k = idx / BM;
                const int gk = k0 + k, gm = m0 + m;
                const bool ok = gk < kend && gm < M;
                cp16(as + k * A_PITCH_N + m, ok ? A + gm + (long)gk * lda : A, ok);
            }
        }
        // B: BK x BN complex, 2 per thread; each n holds BK consecutive k
#pragma unroll
        for (int r = 0; r < (BN * BK) / THREADS; ++r) {
            const int idx = tid + r * THREADS;
            const int k = idx % BK, n = idx / BK;
            const int gk = k0 + k, gn = n0 + n;
            const bool ok = gk < kend && gn < N;
            cp16(bs + n * KP + k, ok ? B + gk + (long)gn * ldb : B, ok);
        }
    };

    double2 acc[TM][4];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < nk) fill(s, s);
        cp_commit();
    }
    for (int kb = 0; kb < nk; ++kb) {
        cp_wait<STAGES - 2>();
        __syncthreads();  // stage kb % STAGES is complete for everyone; stage (kb-1) % STAGES is free
        {
            const int nxt = kb + STAGES - 1;
            if (nxt < nk) fill(nxt, nxt % STAGES);
            cp_commit();
        }
        const double2* as = As + (kb % STAGES) * A_STAGE;
        const double2* bs = Bs + (kb % STAGES) * B_STAGE;
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            double2 a[TM], b[4];
#pragma unroll
            for (int i = 0; i < TM; ++i) {
                const double2 v = CONJ_A ? as[(ty + 16 * i) * KP + kk] : as[kk * A_PITCH_N + ty + 16 * i];
                a[i] = CONJ_A ? conj2(v) : v;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = bs[(tx + 16 * j) * KP + kk];
#pragma unroll
            for (int i = 0; i < TM; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) cfma(acc[i][j], a[i], b[j]);
        }
    }
    cp_wait<0>();

    const bool use_beta = (beta.x != 0.0 || beta.y != 0.0);
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int gm = m0 + ty + 16 * i;
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gn = n0 + tx + 16 * j;
            if (gn >= N) continue;
            if (part) {
                part[(long)blockIdx.z * M * N + (long)gn * M + gm] = acc[i][j];
            } else {
                double2 v = cmul(alpha, acc[i][j]);
                double2* c = C + gm + (long)gn * ldc;
                if (use_beta) v = v + cmul(beta, *c);
                *c = v;
            }
        }
    }
}

// DFMA rate probe: every thread runs 8 independent FMA chains of `iters` steps
// (2 flops each) on values that stay finite; the result is written so the
// chains are not optimised away.
__global__ void __launch_bounds__(256) dfma_probe(int iters, double seed, double* out) {
    double a[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) a[c] = seed + 0.001 * (threadIdx.x + c);
    const double b = 0.999999, d = 1e-7;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < 8; ++c) a[c] = fma(a[c], b, d);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < 8; ++c) s += a[c];
    if (s == 12345.678) out[blockIdx.x] = s;  // never true for these inputs; keeps the chains live
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
inline bool small_tiles(int M, int N) { return (long)ceil_div(M, kBM) * ceil_div(N, kBN) < device_sms(); }

// K splits for a product with `tiles` output tiles (never more than for
// 64x64 tiles, which size the workspace)
inline int choose_splits_for(int tiles, int K) {
    const int target = 2 * device_sms();
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

// FP64 products of at least one 128 x 64 tile take zgemm_big
inline bool big_tiles(int M, int N) { return M >= big::BM && N >= big::BN; }

// K splits of a large-tile C,N product: at most 64, at most one per 256 of K,
// and a workspace of at most 64 MB
constexpr size_t kBigSplitBytes = 64ull << 20;
inline int big_max_splits(int M, int N, int K) {
    const long by_ws = static_cast<long>(kBigSplitBytes / ((size_t)M * N * sizeof(double2)));
    long s = std::min<long>(64, ceil_div(K, 256));
    s = std::min(s, by_ws);
    return s < 1 ? 1 : static_cast<int>(s);
}

template <bool CONJ_A, int TM>
void zgemm_big_run(cudaStream_t st, dim3 grid, int M, int N, int K, double2 alpha, const double2* A, long lda,
                   const double2* B, long ldb, double2 beta, double2* C, long ldc, int kchunk, double2* part) {
    constexpr size_t smem = big::Shape<TM>::smem;
    static_assert(smem <= 227 * 1024, "zgemm_big stages exceed shared memory");
    // the attribute belongs to the function on one device
    static PerDeviceOnce once;
    once.run([] {
        Q3B_CUDA(cudaFuncSetAttribute(zgemm_big<CONJ_A, TM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)big::Shape<TM>::smem));
    });
    zgemm_big<CONJ_A, TM><<<grid, big::THREADS, smem, st>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, kchunk,
                                                             part);
    Q3B_LAUNCH_CHECK();
}

// One 256-thread block of zgemm_big per SM, so the launch runs in waves of
// `sms` blocks.  The tile height (128 or 96 rows) is the one with the least
// rows of work per SM over whole waves; a C,N product splits K into as many
// chunks as fill whole waves (at least two, at most 64).
void zgemm_big_launch(cudaStream_t st, bool conj_a, int M, int N, int K, double2 alpha, const double2* A,
                      long lda, const double2* B, long ldb, double2 beta, double2* C, long ldc,
                      const GemmWorkspace& ws) {
    const int sms = device_sms();
    auto waves = [&](long units) { return (units + sms - 1) / sms; };
    const int t128 = ceil_div(M, 128) * ceil_div(N, big::BN), t96 = ceil_div(M, 96) * ceil_div(N, big::BN);
    int splits = 1, tm = 8, tiles = t128;
    if (conj_a) {
        // the waves of split blocks, per tile height
        auto best_split = [&](int t, int& s_out) {
            long best = -1;
            const int kmax = big_max_splits(M, N, K);
            for (int s = 1; s <= kmax; ++s) {
                const long cost = waves((long)t * s) * ((long)ceil_div(K, s));  // K steps of the busiest SM
                if (best < 0 || cost < best) {
                    best = cost;
                    s_out = s;
                }
            }
            return best;
        };
        int s128 = 1, s96 = 1;
        const long c128 = best_split(t128, s128) * 128, c96 = best_split(t96, s96) * 96;
        if (c96 < c128) {
            tm = 6;
            splits = s96;
            tiles = t96;
        } else {
            splits = s128;
        }
    } else if (waves(t96) * 96 < waves(t128) * 128) {
        tm = 6;
        tiles = t96;
    }
    (void)tiles;
    const size_t need = (size_t)splits * M * N * sizeof(double2);
    if (splits > 1 && (ws.ptr == nullptr || ws.bytes < need)) splits = 1;
    int kchunk = K;
    if (splits > 1) {
        kchunk = ceil_div(K, splits);
        kchunk = ceil_div(kchunk, big::BK) * big::BK;
        splits = ceil_div(K, kchunk);
    }
    const int bm = 16 * tm;
    if (ceil_div(M, bm) > 65535) throw std::runtime_error("complex GEMM: M too large");
    dim3 grid(ceil_div(N, big::BN), ceil_div(M, bm), splits);
    double2* part = splits > 1 ? static_cast<double2*>(ws.ptr) : nullptr;
    if (conj_a) {
        if (tm == 6) zgemm_big_run<true, 6>(st, grid, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, kchunk, part);
        else zgemm_big_run<true, 8>(st, grid, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, kchunk, part);
    } else {
        if (tm == 6) zgemm_big_run<false, 6>(st, grid, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, kchunk, part);
        else zgemm_big_run<false, 8>(st, grid, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, kchunk, part);
    }
    if (splits > 1) {
        const long total = (long)M * N;
        int blocks = ceil_div(total, 256);
        if (blocks > 4096) blocks = 4096;
        splitk_reduce<double><<<blocks, 256, 0, st>>>(M, N, splits, part, alpha, beta, C, ldc);
        Q3B_LAUNCH_CHECK();
    }
}


}  // namespace

bool use_tensor_cores(int M, int N, int K) { return (double)M * N * K >= kTensorCoreMinMacs; }

template <typename R> size_t cgemm_workspace_bytes(int M, int N, int K) {
    const int s = std::max(choose_splits<R>(M, N, K), big_max_splits(M, N, K));
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
    if constexpr (std::is_same<R, double>::value) {
        if (big_tiles(M, N) && reinterpret_cast<uintptr_t>(A) % 16 == 0 &&
            reinterpret_cast<uintptr_t>(B) % 16 == 0) {
            zgemm_big_launch(st, conj_a, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, ws);
            return;
        }
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

double measure_dfma_tflops(cudaStream_t st) {
    int dev = 0, sms = 0;
    Q3B_CUDA(cudaGetDevice(&dev));
    Q3B_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8, iters = 4096;
    double* out = nullptr;
    Q3B_CUDA(cudaMallocAsync(&out, blocks * sizeof(double), st));
    cudaEvent_t e0, e1;
    Q3B_CUDA(cudaEventCreate(&e0));
    Q3B_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        Q3B_CUDA(cudaEventRecord(e0, st));
        dfma_probe<<<blocks, 256, 0, st>>>(iters, 1.0, out);
        Q3B_LAUNCH_CHECK();
        Q3B_CUDA(cudaEventRecord(e1, st));
        Q3B_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        Q3B_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    Q3B_CUDA(cudaFreeAsync(out, st));
    const double flops = 2.0 * 8.0 * iters * 256.0 * blocks;
    return flops / (best * 1e-3) / 1e12;
}

template void cgemm<double>(cudaStream_t, bool, int, int, int, double2, const double2*, long,
                            const double2*, long, double2, double2*, long, const GemmWorkspace&);
template void cgemm<float>(cudaStream_t, bool, int, int, int, float2, const float2*, long,
                           const float2*, long, float2, float2*, long, const GemmWorkspace&);
template size_t cgemm_workspace_bytes<double>(int, int, int);
template size_t cgemm_workspace_bytes<float>(int, int, int);

}  // namespace q3b
