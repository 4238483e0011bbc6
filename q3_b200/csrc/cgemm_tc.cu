// Complex FP32 GEMMs on the 5th-generation tensor cores (tcgen05, sm_100a).
//
//   "C,N":  C = alpha A^H B + beta C    (A: K x M, lda; B: K x N, ldb)
//   "N,N":  C = alpha A B   + beta C    (A: M x K, lda; B: K x N, ldb)
//
// Every real operand x is split into two TF32 numbers, x = hi + lo with
// hi = rn_tf32(x), lo = rn_tf32(x - hi); a real product is hi*hi + hi*lo +
// lo*hi accumulated in FP32 in TMEM (the lo*lo term, ~2^-22 relative, is
// dropped), which keeps FP32 accuracy at tensor-core rate.
//
// Block tile: 128 (M) x 64 (N) complex outputs, K in blocks of 32.  The A
// operand is held as four planes (re hi, re lo, im hi, im lo), 128 rows each;
// the B operand as two planes (hi, lo) of 128 rows: rows 0-63 the real parts
// of the 64 columns, rows 64-127 their imaginary parts.  Each row is 32 TF32
// values = one 128-byte swizzle row (K-major, SWIZZLE_128B).  Per K step of 8
// one thread issues six tcgen05.mma of 128 x 128 x 8:
//   P = Ar [Br | Bi]^T  and  Q = Ai [Br | Bi]^T   (x3 for the split terms)
// into two FP32 accumulators of 128 TMEM columns, and the epilogue forms
//   C,N: Re = P_r + Q_i,  Im = P_i - Q_r      N,N: Re = P_r - Q_i,  Im = P_i + Q_r.
// Two producer groups of four warps each own one of the two stages: a group
// loads a K block with coalesced 16-byte loads (all issued before any
// conversion), splits and de-interleaves it into the planes and signals the
// stage's "full" mbarrier, so one group converts while the other's loads are
// in flight.  The MMA thread (warp 8) commits each stage to an "empty"
// mbarrier.  After the last block all eight producer warps read the
// accumulators with tcgen05.ld (warp w: TMEM lanes 32*(w%4).., column half
// w/4) and write C, or the raw sums of their K range for a fixed-order
// split-K reduction.  Every mbarrier wait is
// bounded; a timeout sets an error word and the block drains and frees TMEM.
#include <cstdint>
#include <mutex>

#include "cgemm.cuh"

namespace q3b {
namespace tc {
namespace {

constexpr int BM = 128;            // complex rows per block (UMMA M)
constexpr int BN = 64;             // complex columns per block (UMMA N)
constexpr int BK = 32;             // K per stage: one 128-byte TF32 row
constexpr int STAGES = 2;
constexpr int PRODUCERS = 128;     // threads of one producer group (4 warps)
constexpr int GROUPS = 2;          // producer groups: group g fills stage g
constexpr int MMA_WARP = 4 * GROUPS;
constexpr int THREADS = GROUPS * PRODUCERS + 32;
static_assert(GROUPS == STAGES, "each producer group owns one stage");
constexpr int A_PLANE = BM * 128;      // bytes of one A plane (BM rows x 128 B)
constexpr int B_PLANE = 2 * BN * 128;  // bytes of one B plane (re rows + im rows)
constexpr int UMMA_N = 2 * BN;         // [Br | Bi]
constexpr int STAGE_BYTES = 4 * A_PLANE + 2 * B_PLANE;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024;  // + alignment slack
// P in columns [0, 128), Q in [128, 256) (one block per SM: TMEM is not shared)
constexpr uint32_t TMEM_COLS = 256;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait on an mbarrier phase; false (and the error word set) on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err) {
    for (int i = 0; i < (1 << 22); ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*reinterpret_cast<volatile int*>(err)) return false;
        if (i > 32) __nanosleep(64);
    }
    atomicExch(err, 1);
    return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// raise the transaction count the barrier's current phase waits for
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// bulk asynchronous copy global -> this block's shared memory, completing
// `bytes` of the barrier's transaction count (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, SWIZZLE_128B, rows of 128 B,
// 8-row groups 1024 B apart (SBO), version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((addr >> 4) & 0x3FFF);
    d |= static_cast<uint64_t>(1) << 16;                 // LBO (unused for swizzled K-major)
    d |= static_cast<uint64_t>((1024 >> 4) & 0x3FFF) << 32;
    d |= static_cast<uint64_t>(1) << 46;                 // version
    d |= static_cast<uint64_t>(2) << 61;                 // SWIZZLE_128B
    return d;
}

// Instruction descriptor: kind::tf32, D f32, A/B tf32 K-major, M = 128, N = 128.
__host__ __device__ constexpr uint32_t instr_desc() {
    return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(UMMA_N >> 3) << 17) |
           (static_cast<uint32_t>(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 16 consecutive TMEM columns of this warp's 32 lanes; the values are valid
// after tmem_wait_ld (several loads may be in flight before one wait)
__device__ __forceinline__ void tmem_ld16_issue(uint32_t taddr, uint32_t* r) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ float tf32_rn(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

// byte offset of (row, k) in a 128B-swizzled K-major plane of TF32
__device__ __forceinline__ uint32_t swz(int row, int k) {
    return static_cast<uint32_t>(row * 128 + ((((k >> 2) ^ (row & 7))) << 4) + ((k & 3) << 2));
}

// Split two complex values (re0, im0, re1, im1) at K positions k, k+1 of one
// operand row into the four planes (re hi, re lo, im hi, im lo).
__device__ __forceinline__ void put_pair(unsigned char* planes, int plane_bytes, int row, int k, float4 v,
                                         bool conj) {
    const float re0 = v.x, re1 = v.z;
    const float im0 = conj ? -v.y : v.y, im1 = conj ? -v.w : v.w;
    const float rh0 = tf32_rn(re0), rh1 = tf32_rn(re1), ih0 = tf32_rn(im0), ih1 = tf32_rn(im1);
    const float rl0 = tf32_rn(re0 - rh0), rl1 = tf32_rn(re1 - rh1);
    const float il0 = tf32_rn(im0 - ih0), il1 = tf32_rn(im1 - ih1);
    const uint32_t o = swz(row, k);
    *reinterpret_cast<float2*>(planes + 0 * plane_bytes + o) = make_float2(rh0, rh1);
    *reinterpret_cast<float2*>(planes + 1 * plane_bytes + o) = make_float2(rl0, rl1);
    *reinterpret_cast<float2*>(planes + 2 * plane_bytes + o) = make_float2(ih0, ih1);
    *reinterpret_cast<float2*>(planes + 3 * plane_bytes + o) = make_float2(il0, il1);
}

// Four K values (k..k+3) of one operand row, as a 16-byte chunk per plane.
__device__ __forceinline__ void put_quad(unsigned char* planes, int plane_bytes, int row, int k, const float2* c) {
    float rh[4], rl[4], ih[4], il[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        rh[j] = tf32_rn(c[j].x);
        rl[j] = tf32_rn(c[j].x - rh[j]);
        ih[j] = tf32_rn(c[j].y);
        il[j] = tf32_rn(c[j].y - ih[j]);
    }
    const uint32_t o = swz(row, k);
    *reinterpret_cast<float4*>(planes + 0 * plane_bytes + o) = make_float4(rh[0], rh[1], rh[2], rh[3]);
    *reinterpret_cast<float4*>(planes + 1 * plane_bytes + o) = make_float4(rl[0], rl[1], rl[2], rl[3]);
    *reinterpret_cast<float4*>(planes + 2 * plane_bytes + o) = make_float4(ih[0], ih[1], ih[2], ih[3]);
    *reinterpret_cast<float4*>(planes + 3 * plane_bytes + o) = make_float4(il[0], il[1], il[2], il[3]);
}

// One K block of a K-contiguous operand (column `row` of X holds K values):
// rows [r0, r0+NROWS) of the tile, K in [k0, k0+32).  Each half-warp reads one
// row's 256 bytes.  All of a thread's loads are issued before any is
// converted, so a K block costs one memory latency, not one per load.
template <int NROWS>
__device__ __forceinline__ void load_kmajor(unsigned char* planes, int plane_bytes, const float2* X, long ldx,
                                            int r0, int rmax, int k0, int kend, int tid) {
    constexpr int ITEMS = NROWS * 16 / PRODUCERS;
    float4 v[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const int idx = tid + i * PRODUCERS;
        const int row = idx >> 4;
        const int kp = (idx & 15) * 2;  // even K offset within the block
        const int gr = r0 + row, gk = k0 + kp;
        float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gr < rmax) {
            const float2* p = X + (long)gr * ldx + gk;
            if (gk + 1 < kend && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
                x = __ldg(reinterpret_cast<const float4*>(p));
            } else {
                if (gk < kend) { const float2 a = __ldg(p); x.x = a.x; x.y = a.y; }
                if (gk + 1 < kend) { const float2 b = __ldg(p + 1); x.z = b.x; x.w = b.y; }
            }
        }
        v[i] = x;
    }
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const int idx = tid + i * PRODUCERS;
        put_pair(planes, plane_bytes, idx >> 4, (idx & 15) * 2, v[i], false);
    }
}

// One K block of an M-contiguous operand (A of "N,N": element (m, k) at
// X[m + k*ldx]): each item is two rows by four K values; loads first.
__device__ __forceinline__ void load_mmajor(unsigned char* planes, int plane_bytes, const float2* X, long ldx,
                                            int m0, int mmax, int k0, int kend, int tid) {
    constexpr int ITEMS = (BM / 2) * (BK / 4) / PRODUCERS;
    float4 v[ITEMS][4];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const int idx = tid + i * PRODUCERS;
        const int mp = idx % (BM / 2);
        const int kq = idx / (BM / 2);
        const int gm = m0 + 2 * mp;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gk = k0 + kq * 4 + j;
            float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
            if (gk < kend && gm < mmax) {
                const float2* p = X + (long)gk * ldx + gm;
                if (gm + 1 < mmax && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
                    x = __ldg(reinterpret_cast<const float4*>(p));
                } else {
                    const float2 a = __ldg(p);
                    x.x = a.x;
                    x.y = a.y;
                    if (gm + 1 < mmax) { const float2 b = __ldg(p + 1); x.z = b.x; x.w = b.y; }
                }
            }
            v[i][j] = x;
        }
    }
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const int idx = tid + i * PRODUCERS;
        const int mp = idx % (BM / 2);
        const int kq = idx / (BM / 2);
        float2 c0[4], c1[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            c0[j] = make_float2(v[i][j].x, v[i][j].y);
            c1[j] = make_float2(v[i][j].z, v[i][j].w);
        }
        put_quad(planes, plane_bytes, 2 * mp, kq * 4, c0);
        put_quad(planes, plane_bytes, 2 * mp + 1, kq * 4, c1);
    }
}

// One K block of B (K-contiguous columns) into the two stacked planes: the
// real parts of column n go to row n of the (hi, lo) planes, the imaginary
// parts to row BN + n.
__device__ __forceinline__ void load_b(unsigned char* planes, const float2* X, long ldx, int n0, int nmax,
                                       int k0, int kend, int tid) {
    constexpr int ITEMS = BN * 16 / PRODUCERS;
    float4 v[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const int idx = tid + i * PRODUCERS;
        const int row = idx >> 4;
        const int kp = (idx & 15) * 2;
        const int gr = n0 + row, gk = k0 + kp;
        float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
        if (gr < nmax) {
            const float2* p = X + (long)gr * ldx + gk;
            if (gk + 1 < kend && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
                x = __ldg(reinterpret_cast<const float4*>(p));
            } else {
                if (gk < kend) { const float2 a = __ldg(p); x.x = a.x; x.y = a.y; }
                if (gk + 1 < kend) { const float2 b = __ldg(p + 1); x.z = b.x; x.w = b.y; }
            }
        }
        v[i] = x;
    }
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const int idx = tid + i * PRODUCERS;
        const int row = idx >> 4, k = (idx & 15) * 2;
        const float4 x = v[i];
        const float rh0 = tf32_rn(x.x), rh1 = tf32_rn(x.z), ih0 = tf32_rn(x.y), ih1 = tf32_rn(x.w);
        const float rl0 = tf32_rn(x.x - rh0), rl1 = tf32_rn(x.z - rh1);
        const float il0 = tf32_rn(x.y - ih0), il1 = tf32_rn(x.w - ih1);
        const uint32_t orr = swz(row, k), oi = swz(BN + row, k);
        *reinterpret_cast<float2*>(planes + orr) = make_float2(rh0, rh1);
        *reinterpret_cast<float2*>(planes + B_PLANE + orr) = make_float2(rl0, rl1);
        *reinterpret_cast<float2*>(planes + oi) = make_float2(ih0, ih1);
        *reinterpret_cast<float2*>(planes + B_PLANE + oi) = make_float2(il0, il1);
    }
}

// One packed A tile (128 rows x 32 K, four 16 KB planes) per block: built in
// shared memory, then written out contiguously.  Tiles are stored K-block
// fastest: tile (mt, kb) at (mt * nkt + kb) * A_TILE bytes.
constexpr int A_TILE = 4 * A_PLANE;
__global__ void __launch_bounds__(256)
pack_a_kernel(int M, int K, const float2* __restrict__ A, long lda, int kmajor, int nkt, unsigned char* out) {
    extern __shared__ __align__(1024) unsigned char tile[];
    const int mt = blockIdx.x / nkt, kb = blockIdx.x % nkt;
    for (int idx = threadIdx.x; idx < BM * BK; idx += blockDim.x) {
        // lanes along the operand's contiguous index, for coalesced reads
        const int r = kmajor ? idx / BK : idx % BM;
        const int k = kmajor ? idx % BK : idx / BM;
        const int gm = mt * BM + r, gk = kb * BK + k;
        float2 x = make_float2(0.f, 0.f);
        if (gm < M && gk < K) x = kmajor ? A[(long)gm * lda + gk] : A[gm + (long)gk * lda];
        const float rh = tf32_rn(x.x), ih = tf32_rn(x.y);
        const uint32_t o = swz(r, k);
        *reinterpret_cast<float*>(tile + 0 * A_PLANE + o) = rh;
        *reinterpret_cast<float*>(tile + 1 * A_PLANE + o) = tf32_rn(x.x - rh);
        *reinterpret_cast<float*>(tile + 2 * A_PLANE + o) = ih;
        *reinterpret_cast<float*>(tile + 3 * A_PLANE + o) = tf32_rn(x.y - ih);
    }
    __syncthreads();
    float4* dst = reinterpret_cast<float4*>(out + (size_t)blockIdx.x * A_TILE);
    const float4* src = reinterpret_cast<const float4*>(tile);
    for (int i = threadIdx.x; i < A_TILE / 16; i += blockDim.x) dst[i] = src[i];
}

// PACKED_A: A's tiles come from a pack_a_kernel image by bulk copies (one
// thread of the stage's producer group issues them), and the group converts
// only B; the stage's barrier waits for the copies' bytes as well.
template <bool CONJ_A, bool PACKED_A>
__global__ void __launch_bounds__(THREADS, 1)
cgemm_tc_kernel(int M, int N, int K, float2 alpha, const float2* __restrict__ A, long lda,
                const unsigned char* __restrict__ Apk, const float2* __restrict__ B, long ldb, float2 beta,
                float2* C, long ldc, int kchunk, float2* part, int* err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[STAGES];
    __shared__ __align__(8) uint64_t empty_bar[STAGES];
    __shared__ __align__(8) uint64_t done_bar;
    __shared__ uint32_t tmem_slot;

    unsigned char* smem = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    // N tiles run fastest, so the blocks that share an A tile run together and
    // all but the first find it in L2
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int kbeg = blockIdx.z * kchunk;
    const int kend = min(K, kbeg + kchunk);
    const int nkb = kend > kbeg ? (kend - kbeg + BK - 1) / BK : 0;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full_bar[s], PRODUCERS);
            mbar_init(&empty_bar[s], 1);
        }
        mbar_init(&done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp < MMA_WARP) {
        // ---------------------------------------------------------- producers
        // group g loads K blocks g, g + GROUPS, ... into stage g: while one
        // group waits on its loads the other converts, so two K blocks are
        // in flight
        const int g = warp / 4, ptid = tid % PRODUCERS;
        for (int kb = g; kb < nkb; kb += GROUPS) {
            const int s = kb % STAGES;
            if (kb >= STAGES && !mbar_wait(&empty_bar[s], ((kb / STAGES) - 1) & 1, err)) break;
            unsigned char* st = smem + s * STAGE_BYTES;
            unsigned char* pa = st;
            unsigned char* pb = st + 4 * A_PLANE;
            const int k0 = kbeg + kb * BK;
            if (PACKED_A) {
                if (ptid == 0) {
                    const int nkt = (K + BK - 1) / BK;
                    const unsigned char* src = Apk + ((size_t)blockIdx.y * nkt + k0 / BK) * A_TILE;
                    mbar_expect_tx(&full_bar[s], A_TILE);
#pragma unroll
                    for (int pl = 0; pl < 4; ++pl)
                        bulk_copy_g2s(pa + pl * A_PLANE, src + pl * A_PLANE, A_PLANE, &full_bar[s]);
                }
            } else if (CONJ_A) {
                load_kmajor<BM>(pa, A_PLANE, A, lda, m0, M, k0, kend, ptid);
            } else {
                load_mmajor(pa, A_PLANE, A, lda, m0, M, k0, kend, ptid);
            }
            load_b(pb, B, ldb, n0, N, k0, kend, ptid);
            fence_async_smem();
            mbar_arrive(&full_bar[s]);
        }
    } else if (lane == 0) {
        // ------------------------------------------------------- MMA issuer (warp MMA_WARP)
        // per K step: P += Ar [Br|Bi]^T, Q += Ai [Br|Bi]^T, each as hi*hi + hi*lo + lo*hi
        bool first = true;
        bool ok = true;
        for (int kb = 0; kb < nkb && ok; ++kb) {
            const int s = kb % STAGES;
            if (!mbar_wait(&full_bar[s], (kb / STAGES) & 1, err)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const uint32_t base = smem_u32(smem + s * STAGE_BYTES);
            const uint32_t a_base = base, b_base = base + 4 * A_PLANE;
#pragma unroll
            for (int ks = 0; ks < BK / 8; ++ks) {
                const uint32_t off = ks * 32;
#pragma unroll
                for (int t = 0; t < 6; ++t) {
                    const int part = t / 3;   // 0: P (A re planes), 1: Q (A im planes)
                    const int term = t % 3;   // 0: hi*hi 1: hi*lo 2: lo*hi
                    const int a_plane = 2 * part + (term == 2 ? 1 : 0);
                    const int b_plane = (term == 1 ? 1 : 0);
                    const uint64_t ad = smem_desc(a_base + a_plane * A_PLANE + off);
                    const uint64_t bd = smem_desc(b_base + b_plane * B_PLANE + off);
                    const uint32_t d = tmem + (part ? UMMA_N : 0);
                    mma_tf32(d, ad, bd, instr_desc(), (first && term == 0) ? 0u : 1u);
                }
                first = false;
            }
            mma_commit(&empty_bar[s]);
        }
        mma_commit(&done_bar);
    }

    // ------------------------------------------------------------ epilogue
    // warp w reads TMEM lanes 32*(w%4).. (its rows) for columns half w/4
    if (warp < MMA_WARP) {
        const bool waited = nkb > 0 && mbar_wait(&done_bar, 0, err);
        const bool have = __all_sync(0xffffffffu, waited);  // tcgen05.ld is warp-collective
        tc_fence_after();
        const int q = warp & 3, h = warp >> 2;
        const int row = m0 + q * 32 + lane;
        const uint32_t lane_addr = tmem + (static_cast<uint32_t>(q * 32) << 16);
        const bool use_beta = (beta.x != 0.f || beta.y != 0.f);
#pragma unroll 1
        for (int c0 = h * (BN / GROUPS); c0 < (h + 1) * (BN / GROUPS); c0 += 16) {
            float pr[16], pi[16], qr[16], qi[16];
            if (have) {
                uint32_t r0[16], r1[16], r2[16], r3[16];
                tmem_ld16_issue(lane_addr + c0, r0);                  // Ar Br
                tmem_ld16_issue(lane_addr + BN + c0, r1);             // Ar Bi
                tmem_ld16_issue(lane_addr + UMMA_N + c0, r2);         // Ai Br
                tmem_ld16_issue(lane_addr + UMMA_N + BN + c0, r3);    // Ai Bi
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    pr[j] = __uint_as_float(r0[j]);
                    pi[j] = __uint_as_float(r1[j]);
                    qr[j] = __uint_as_float(r2[j]);
                    qi[j] = __uint_as_float(r3[j]);
                }
            } else {
#pragma unroll
                for (int j = 0; j < 16; ++j) pr[j] = pi[j] = qr[j] = qi[j] = 0.f;
            }
            if (row < M) {
                // the 16 old values of C are read before any is written, so
                // their latencies overlap
                float2 old[16];
                if (use_beta && !part) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int col = n0 + c0 + j;
                        old[j] = col < N ? C[row + (long)col * ldc] : make_float2(0.f, 0.f);
                    }
                }
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int col = n0 + c0 + j;
                    if (col >= N) break;
                    const float2 acc = CONJ_A ? make_float2(pr[j] + qi[j], pi[j] - qr[j])
                                              : make_float2(pr[j] - qi[j], pi[j] + qr[j]);
                    if (part) {
                        part[(long)blockIdx.z * M * N + (long)col * M + row] = acc;
                    } else {
                        float2 v = make_float2(alpha.x * acc.x - alpha.y * acc.y, alpha.x * acc.y + alpha.y * acc.x);
                        if (use_beta) {
                            const float2 o = old[j];
                            v.x += beta.x * o.x - beta.y * o.y;
                            v.y += beta.x * o.y + beta.y * o.x;
                        }
                        C[row + (long)col * ldc] = v;
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS)
                     : "memory");
    }
}

__global__ void splitk_sum(int M, int N, int splits, const float2* __restrict__ part, float2 alpha, float2 beta,
                           float2* C, long ldc) {
    const long total = (long)M * N;
    const bool use_beta = (beta.x != 0.f || beta.y != 0.f);
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const int m = static_cast<int>(idx % M), n = static_cast<int>(idx / M);
        float2 s = part[idx];
        for (int z = 1; z < splits; ++z) {
            const float2 p = part[(long)z * total + idx];
            s.x += p.x;
            s.y += p.y;
        }
        float2 v = make_float2(alpha.x * s.x - alpha.y * s.y, alpha.x * s.y + alpha.y * s.x);
        float2* cp = C + m + (long)n * ldc;
        if (use_beta) {
            const float2 o = *cp;
            v.x += beta.x * o.x - beta.y * o.y;
            v.y += beta.x * o.y + beta.y * o.x;
        }
        *cp = v;
    }
}

// one block per SM: keep tiles x splits within one wave
int choose_splits(int M, int N, int K) {
    const int tiles = ceil_div(M, BM) * ceil_div(N, BN);
    int s = device_sms() / tiles;
    const int kmax = ceil_div(K, 256);
    if (s > kmax) s = kmax;
    if (s < 1) s = 1;
    if (s > 64) s = 64;
    return s;
}

__device__ int g_tc_error;

}  // namespace

namespace {
thread_local int* t_context_word = nullptr;
}  // namespace

ErrorScope::ErrorScope(int* word) : prev_(t_context_word) { t_context_word = word; }
ErrorScope::~ErrorScope() { t_context_word = prev_; }

int* error_word() {
    if (t_context_word) return t_context_word;
    // per host thread: the device it last asked for and the word's address there
    thread_local int cached_dev = -1;
    thread_local int* cached = nullptr;
    int dev = 0;
    Q3B_CUDA(cudaGetDevice(&dev));
    if (dev != cached_dev || !cached) {
        void* p = nullptr;
        Q3B_CUDA(cudaGetSymbolAddress(&p, g_tc_error));
        cached = static_cast<int*>(p);
        cached_dev = dev;
    }
    return cached;
}

void check_error(cudaStream_t st) {
    int* w = error_word();
    int* hb = static_cast<int*>(host_readback(sizeof(int)));
    Q3B_CUDA(cudaMemcpyAsync(hb, w, sizeof(int), cudaMemcpyDeviceToHost, st));
    Q3B_CUDA(cudaStreamSynchronize(st));
    if (hb[0]) {
        Q3B_CUDA(cudaMemsetAsync(w, 0, sizeof(int), st));
        throw CudaError("a bounded device wait timed out (tensor-core GEMM pipeline or plane-kernel stick copy)");
    }
}

size_t workspace_bytes(int M, int N, int K) {
    const int s = choose_splits(M, N, K);
    return s > 1 ? (size_t)s * M * N * sizeof(float2) : 0;
}

namespace {

template <bool CONJ_A, bool PACKED_A> void set_kernel_smem() {
    cudaFuncSetAttribute(cgemm_tc_kernel<CONJ_A, PACKED_A>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
}

void launch(cudaStream_t st, bool conj_a, int M, int N, int K, float2 alpha, const float2* A, long lda,
            const unsigned char* Apk, const float2* B, long ldb, float2 beta, float2* C, long ldc,
            const GemmWorkspace& ws) {
    int* err = error_word();
    static PerDeviceOnce once;
    once.run([] {
        set_kernel_smem<true, false>();
        set_kernel_smem<false, false>();
        set_kernel_smem<true, true>();
        set_kernel_smem<false, true>();
        cudaFuncSetAttribute(pack_a_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, A_TILE);
    });
    int splits = conj_a ? choose_splits(M, N, K) : 1;
    const size_t need = (size_t)splits * M * N * sizeof(float2);
    if (splits > 1 && (ws.ptr == nullptr || ws.bytes < need)) splits = 1;
    int kchunk = K;
    if (splits > 1) {
        kchunk = ceil_div(ceil_div(K, splits), BK) * BK;
        splits = ceil_div(K, kchunk);
    }
    if (ceil_div(M, BM) > 65535) throw std::runtime_error("tensor-core GEMM: M too large");
    dim3 grid(ceil_div(N, BN), ceil_div(M, BM), splits);
    float2* part = splits > 1 ? static_cast<float2*>(ws.ptr) : nullptr;
#define Q3B_TC_LAUNCH(CA, PA)                                                                             \
    cgemm_tc_kernel<CA, PA><<<grid, THREADS, SMEM_BYTES, st>>>(M, N, K, alpha, A, lda, Apk, B, ldb, beta, C, \
                                                               ldc, kchunk, part, err)
    if (Apk) {
        if (conj_a) Q3B_TC_LAUNCH(true, true);
        else Q3B_TC_LAUNCH(false, true);
    } else {
        if (conj_a) Q3B_TC_LAUNCH(true, false);
        else Q3B_TC_LAUNCH(false, false);
    }
#undef Q3B_TC_LAUNCH
    Q3B_LAUNCH_CHECK();
    if (splits > 1) {
        const long total = (long)M * N;
        int blocks = ceil_div(total, 256);
        if (blocks > 4096) blocks = 4096;
        splitk_sum<<<blocks, 256, 0, st>>>(M, N, splits, part, alpha, beta, C, ldc);
        Q3B_LAUNCH_CHECK();
    }
}

}  // namespace

void cgemm(cudaStream_t st, bool conj_a, int M, int N, int K, float2 alpha, const float2* A, long lda,
           const float2* B, long ldb, float2 beta, float2* C, long ldc, const GemmWorkspace& ws) {
    launch(st, conj_a, M, N, K, alpha, A, lda, nullptr, B, ldb, beta, C, ldc, ws);
}

size_t packed_a_bytes(int M, int K) {
    return (size_t)ceil_div(M, BM) * ceil_div(K, BK) * A_TILE;
}

void pack_a(cudaStream_t st, int M, int K, const float2* A, long lda, bool kmajor, unsigned char* out) {
    if (M <= 0 || K <= 0) return;
    static PerDeviceOnce once;
    once.run([] {
        cudaFuncSetAttribute(pack_a_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, A_TILE);
    });
    const int nkt = ceil_div(K, BK);
    const long tiles = (long)ceil_div(M, BM) * nkt;
    if (tiles > 0x7fffffffL) throw std::runtime_error("tensor-core GEMM: operand too large to pack");
    pack_a_kernel<<<static_cast<unsigned>(tiles), 256, A_TILE, st>>>(M, K, A, lda, kmajor ? 1 : 0, nkt, out);
    Q3B_LAUNCH_CHECK();
}

void cgemm_packed(cudaStream_t st, bool conj_a, int M, int N, int K, float2 alpha, const PackedA& A,
                  const float2* B, long ldb, float2 beta, float2* C, long ldc, const GemmWorkspace& ws) {
    if (!A.tiles || A.M != M || A.K != K) throw std::runtime_error("tensor-core GEMM: packed A of another shape");
    launch(st, conj_a, M, N, K, alpha, nullptr, 0, A.tiles, B, ldb, beta, C, ldc, ws);
}

}  // namespace tc
}  // namespace q3b
