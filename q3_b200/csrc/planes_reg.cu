// Plane pass of the local H|psi> term with every line transform held in
// registers (pass B of hpsi_local.cuh, the register-resident variant).
//
// One block per (w3 position, band) plane, as in the shared-memory kernel, but
// each 1D transform along w1 or w2 is done by a group of L lanes (L = 1 or 2)
// holding the whole line in registers, with the line length a compile-time
// constant so every twiddle is a literal operand:
//   lane j of a line of n = L*m points holds x[L*i + j], i < m;
//   backward: per-lane DFT_m (natural order), twiddle w_n^{j k'}, DFT_L across
//     the L lanes by __shfl_xor_sync  ->  lane t holds X[t*m + k'], k' < m,
//     a contiguous natural block;
//   forward: the adjoint (DFT_L across lanes, conjugate twiddle, DFT_m) takes
//     that block layout back to lane j holding y[L*i + j].
// So rows, columns, V and sticks are all in natural order.  Shared memory
// holds only what has to cross between lanes of different lines:
//   * the plane's sticks, staged in and out with one cp.async.bulk copy each
//     way (X's per-plane stick run is padded to a 16-byte multiple);
//   * the rows that hold sticks, nrows x PITCH (PITCH = 1 mod 16 elements in
//     FP32, 1 mod 8 in FP64, so half- or quarter-warp accesses down a column or
//     along a row fall in distinct banks).
// Phases, one barrier between each:
//   rows backward  (nrows lines along w2): staged sticks -> registers ->
//                  plane rows (all n2 outputs);
//   columns        (n2 lines along w1): stick rows -> registers (other rows are
//                  zero), backward, times V(r)/N at natural (w1, w2), forward,
//                  back to the stick rows only (the others are never read);
//   rows forward   (nrows lines): plane rows -> registers -> the stick outputs
//                  of the row -> staged sticks -> one bulk copy back to X.
// A plane's stick rows are a cyclic interval of w1 from row_lo, and each row's
// sticks a cyclic interval of w2 (the cross-section of the G-sphere's
// projection); the plan orders the sticks row by row along those intervals, so
// a row's sticks are contiguous in X and in the staged copy.  The plan checks
// this shape and falls back to the shared-memory kernel when it does not hold.
#include <cuda_runtime.h>

#include "fft_core.cuh"
#include "hpsi_local.cuh"

namespace q3b {
namespace {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

template <typename T> __device__ __forceinline__ T shfl_xor(T v, int mask);
template <> __device__ __forceinline__ float2 shfl_xor(float2 v, int mask) {
    return mk(__shfl_xor_sync(0xffffffffu, v.x, mask), __shfl_xor_sync(0xffffffffu, v.y, mask));
}
template <> __device__ __forceinline__ double2 shfl_xor(double2 v, int mask) {
    return mk(__shfl_xor_sync(0xffffffffu, v.x, mask), __shfl_xor_sync(0xffffffffu, v.y, mask));
}

// DFT_2 across the lane pair (t, t ^ partner): lane 0 of the pair keeps
// a + b, lane 1 keeps a - b (the same in both directions).
template <typename T> __device__ __forceinline__ T pair_butterfly(T own, int t, int partner) {
    const T other = shfl_xor(own, partner);
    return t == 0 ? own + other : other - own;
}

// In-place DFTs in registers with every index a compile-time constant.
//   dft_ip<N, DIR>:     natural order in; for N = A*B (fft::Split), position
//                       B*k1 + k2 holds X[k1 + A*k2] on return (perm<N>);
//   dft_ip_rev<N, DIR>: the adjoint ordering: position perm<N>(k) holds z[k] on
//                       entry, natural order on return.
// Radix 2-5 are the natural-order kernels of fft_core.cuh.  The sub-DFTs' own
// orders are absorbed by their gathers and scatters, so besides the N values
// only one sub-line of A or B values is live at a time.
template <int N, typename = void> struct Composite { static constexpr bool value = false; };
template <int N> struct Composite<N, decltype((void)fft::Split<N>::A)> { static constexpr bool value = true; };

template <int N> __host__ __device__ constexpr int perm(int k) {
    if constexpr (Composite<N>::value) {
        constexpr int A = fft::Split<N>::A, B = fft::Split<N>::B;
        return B * (k % A) + k / A;
    } else {
        return k;
    }
}

template <int N, int DIR, typename T> __device__ __forceinline__ void dft_ip(T* x) {
    if constexpr (!Composite<N>::value) {
        fft::dft<N, DIR>(x, static_cast<const T*>(nullptr), 0);
    } else {
        constexpr int A = fft::Split<N>::A, B = fft::Split<N>::B;
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) {
            T t[A];
#pragma unroll
            for (int n1 = 0; n1 < A; ++n1) t[n1] = x[n2 + B * n1];
            dft_ip<A, DIR>(t);
#pragma unroll
            for (int k1 = 0; k1 < A; ++k1)
                x[n2 + B * k1] = fft::rotate_const<N, DIR>(t[perm<A>(k1)], (n2 * k1) % N);
        }
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
            T u[B];
#pragma unroll
            for (int n2 = 0; n2 < B; ++n2) u[n2] = x[n2 + B * k1];
            dft_ip<B, DIR>(u);
#pragma unroll
            for (int k2 = 0; k2 < B; ++k2) x[B * k1 + k2] = u[perm<B>(k2)];
        }
    }
}

template <int N, int DIR, typename T> __device__ __forceinline__ void dft_ip_rev(T* x) {
    if constexpr (!Composite<N>::value) {
        fft::dft<N, DIR>(x, static_cast<const T*>(nullptr), 0);
    } else {
        // position B*p + q holds z[p + A*q]; output j = j1 + B*j2
        constexpr int A = fft::Split<N>::A, B = fft::Split<N>::B;
#pragma unroll
        for (int p = 0; p < A; ++p) {
            T u[B];
#pragma unroll
            for (int q = 0; q < B; ++q) u[q] = x[B * p + q];
            dft_ip<B, DIR>(u);
#pragma unroll
            for (int j1 = 0; j1 < B; ++j1)
                x[B * p + j1] = fft::rotate_const<N, DIR>(u[perm<B>(j1)], (p * j1) % N);
        }
#pragma unroll
        for (int j1 = 0; j1 < B; ++j1) {
            T t[A];
#pragma unroll
            for (int p = 0; p < A; ++p) t[p] = x[B * p + j1];
            dft_ip<A, DIR>(t);
#pragma unroll
            for (int j2 = 0; j2 < A; ++j2) x[B * j2 + j1] = t[perm<A>(j2)];
        }
    }
}

// The line transforms of a group of L lanes, n = L*M points, DIR +1 backward,
// -1 forward (fft_core.cuh's convention).  x: the lane's M registers.
//   line_backward: x[i] = sample L*i + t in; on return position perm<M>(k)
//                  holds X[t*M + k];
//   line_forward:  position perm<M>(k) holds X[t*M + k] on entry; on return
//                  x[i] = sample L*i + t.
template <int N, int L, typename T>
__device__ __forceinline__ void line_backward(T (&x)[N / L], int t, int partner) {
    constexpr int M = N / L;
    dft_ip<M, +1>(x);
    if constexpr (L == 2) {
#pragma unroll
        for (int k = 1; k < M; ++k) {
            const T w = fft::rotate_const<N, +1>(x[perm<M>(k)], k);
            x[perm<M>(k)] = t ? w : x[perm<M>(k)];
        }
#pragma unroll
        for (int k = 0; k < M; ++k) x[k] = pair_butterfly(x[k], t, partner);
    }
}

template <int N, int L, typename T>
__device__ __forceinline__ void line_forward(T (&x)[N / L], int t, int partner) {
    constexpr int M = N / L;
    if constexpr (L == 2) {
#pragma unroll
        for (int k = 0; k < M; ++k) x[k] = pair_butterfly(x[k], t, partner);
#pragma unroll
        for (int k = 1; k < M; ++k) {
            const T w = fft::rotate_const<N, -1>(x[perm<M>(k)], k);
            x[perm<M>(k)] = t ? w : x[perm<M>(k)];
        }
    }
    dft_ip_rev<M, -1>(x);
}

}  // namespace

template <typename R, int N, int L> constexpr int reg_plane_threads() {
    return ((N * L + 31) / 32) * 32;
}

template <typename R, int N> constexpr int reg_plane_pitch() {
    // 1 mod 16 elements for 8-byte complex, 1 mod 8 for 16-byte
    constexpr int g = sizeof(R) == 4 ? 16 : 8;
    return N + ((1 - N) % g + g) % g;
}

// Bounded wait on phase 0 of an mbarrier (the stick load); false and the
// error word set when it runs out.
__device__ __forceinline__ bool wait_phase0(uint64_t* bar, int* err) {
    for (int i = 0; i < (1 << 22); ++i) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(smem_addr(bar))
            : "memory");
        if (ok) return true;
        if (i > 16) __nanosleep(32);
    }
    atomicExch(err, 2);
    return false;
}

// One block per (w3 position, band) plane.
template <typename R, int N, int L>
__global__ void __launch_bounds__(reg_plane_threads<R, N, L>())
planes_reg(LocalPlan<R> p, cplx_t<R>* X, int* err) {
    using T = cplx_t<R>;
    constexpr int M = N / L;
    constexpr int PITCH = reg_plane_pitch<R, N>();
    constexpr int PER_WARP = 32 / L;  // lines per warp
    extern __shared__ __align__(128) unsigned char smem[];
    // the staged sticks first (16-byte aligned, the bulk copies' end), then the
    // stick rows and the mbarrier
    T* staged = reinterpret_cast<T*>(smem);
    T* plane = staged + p.xpitch;
    uint64_t* bar = reinterpret_cast<uint64_t*>(plane + (size_t)p.nrows * PITCH);

    const int i3 = blockIdx.x, band = blockIdx.y;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int t = L == 2 ? lane >> 4 : 0;  // lane within the line's group
    const int item = warp * PER_WARP + (L == 2 ? (lane & 15) : lane);
    constexpr int partner = 16;
    T* xp = X + ((size_t)band * p.n3 + i3) * p.xpitch;
    const uint32_t bytes = static_cast<uint32_t>(p.xpitch * sizeof(T));

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_addr(staged)),
            "l"(xp), "r"(bytes), "r"(smem_addr(bar))
            : "memory");
    }
    __syncthreads();  // the barrier is initialised before anyone waits on it
    // every thread waits (bounded) for the sticks; the block leaves together
    // if any wait ran out
    if (!__syncthreads_and(wait_phase0(bar, err) ? 1 : 0)) return;

    const int nrows = p.nrows, n1 = p.n1, n2 = p.n2, row_lo = p.row_lo;

    // rows backward: staged sticks -> plane rows
    if (warp * PER_WARP < nrows) {
        const int s = item < nrows ? item : nrows - 1;
        const int4 iv = p.row_iv[s];  // {w2 start, count, first stick, -}
        T x[M];
#pragma unroll
        for (int i = 0; i < M; ++i) {
            int off = L * i + t - iv.x;
            off += off < 0 ? n2 : 0;
            x[i] = off < iv.y ? staged[iv.z + off] : czero<T>();
        }
        line_backward<N, L>(x, t, partner);
        if (item < nrows) {
            T* row = plane + (size_t)s * PITCH + t * M;
#pragma unroll
            for (int k = 0; k < M; ++k) row[k] = x[perm<M>(k)];
        }
    }
    __syncthreads();

    // columns: backward, V, forward, on the stick rows
    {
        const int c = item < n2 ? item : n2 - 1;
        T x[M];
#pragma unroll
        for (int i = 0; i < M; ++i) {
            int slot = L * i + t - row_lo;
            slot += slot < 0 ? n1 : 0;
            x[i] = slot < nrows ? plane[(size_t)slot * PITCH + c] : czero<T>();
        }
        line_backward<N, L>(x, t, partner);
        const R* vcol = p.vnat + ((size_t)i3 * n1 + (size_t)t * M) * n2 + c;
#pragma unroll
        for (int k = 0; k < M; ++k) {
            const R v = vcol[(size_t)k * n2];
            const T y = x[perm<M>(k)];
            x[perm<M>(k)] = mk(v * y.x, v * y.y);
        }
        line_forward<N, L>(x, t, partner);
        if (item < n2) {
#pragma unroll
            for (int i = 0; i < M; ++i) {
                int slot = L * i + t - row_lo;
                slot += slot < 0 ? n1 : 0;
                if (slot < nrows) plane[(size_t)slot * PITCH + c] = x[i];
            }
        }
    }
    __syncthreads();

    // rows forward: plane rows -> the row's sticks -> staged
    if (warp * PER_WARP < nrows) {
        const int s = item < nrows ? item : nrows - 1;
        const int4 iv = p.row_iv[s];
        T x[M];
        const T* row = plane + (size_t)s * PITCH + t * M;
#pragma unroll
        for (int k = 0; k < M; ++k) x[perm<M>(k)] = row[k];
        line_forward<N, L>(x, t, partner);
        if (item < nrows) {
#pragma unroll
            for (int i = 0; i < M; ++i) {
                int off = L * i + t - iv.x;
                off += off < 0 ? n2 : 0;
                if (off < iv.y) staged[iv.z + off] = x[i];
            }
        }
    }
    // the staged sticks were written through the generic proxy; make them
    // visible to the bulk copy's async proxy before it reads them
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
        asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(xp),
                     "r"(smem_addr(staged)), "r"(bytes)
                     : "memory");
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        // complete before the block (and its shared memory) goes away
        asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
}

template <typename R, int N, int L> size_t reg_plane_smem(const LocalPlan<R>& p) {
    return (size_t)(p.xpitch + (size_t)p.nrows * reg_plane_pitch<R, N>()) * sizeof(cplx_t<R>) + sizeof(uint64_t);
}

namespace {

// the grids with a register kernel; anything else takes the shared-memory one
#define Q3B_REG_PLANE_SIZES(X) X(24) X(40) X(80) X(108)

template <typename R, int N, int L> bool launch_one(const LocalPlan<R>& p, cplx_t<R>* X, int nb, cudaStream_t st,
                                                    int* err) {
    if (N % L != 0) return false;
    // the bulk copies move 16-byte multiples between 16-byte aligned addresses
    if (reinterpret_cast<uintptr_t>(X) % 16 != 0 || reinterpret_cast<uintptr_t>(p.vnat) % 16 != 0 ||
        ((size_t)p.xpitch * sizeof(cplx_t<R>)) % 16 != 0)
        return false;
    const size_t smem = reg_plane_smem<R, N, L>(p);
    if (smem > 227 * 1024) return false;
    // the attribute belongs to the function on one device: raised to the most
    // any plane may ask for, once per device (contexts on other threads launch
    // with other sizes at the same time, so it is never set to one launch's size)
    static PerDeviceOnce once;
    once.run([] {
        Q3B_CUDA(cudaFuncSetAttribute(planes_reg<R, N, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      227 * 1024));
    });
    planes_reg<R, N, L><<<dim3(p.n3, nb), reg_plane_threads<R, N, L>(), smem, st>>>(p, X, err);
    return true;
}

}  // namespace

// Launch the register plane kernel with `lanes` lanes per line (1 or 2) when
// the plan has one for its grid; false when it has none.
template <typename R>
bool launch_planes_reg(const LocalPlan<R>& p, cplx_t<R>* X, int nb, int lanes, cudaStream_t st, int* err) {
    if (!p.row_iv || p.n1 != p.n2) return false;
    switch (p.n1) {
#define Q3B_REG_CASE(NN)                                              \
    case NN:                                                          \
        if (lanes == 1) return launch_one<R, NN, 1>(p, X, nb, st, err); \
        if (lanes == 2) return launch_one<R, NN, 2>(p, X, nb, st, err); \
        return false;
        Q3B_REG_PLANE_SIZES(Q3B_REG_CASE)
#undef Q3B_REG_CASE
        default: return false;
    }
}

bool has_planes_reg(int n1, int n2, int lanes) {
    if (n1 != n2 || (lanes != 1 && lanes != 2)) return false;
    switch (n1) {
#define Q3B_REG_HAS(NN) case NN: return NN % lanes == 0;
        Q3B_REG_PLANE_SIZES(Q3B_REG_HAS)
#undef Q3B_REG_HAS
        default: return false;
    }
}

template bool launch_planes_reg<double>(const LocalPlan<double>&, double2*, int, int, cudaStream_t, int*);
template bool launch_planes_reg<float>(const LocalPlan<float>&, float2*, int, int, cudaStream_t, int*);

}  // namespace q3b
