// Kinetic + local-potential part of H|psi>; see hpsi_local.cuh.
//
// Follows SerialPlanewaveHamiltonianApplicator::apply_hamiltonian_batch
// (hamiltonian_applicator/serial.hpp:450-477): hpsi = KE*psi, scatter psi by
// the G->grid map, unnormalised backward 3D FFT, multiply by V/N, unnormalised
// forward 3D FFT, hpsi += grid[map].  The 3D transforms are factored into
// stick (w3) and plane (w1, w2) transforms that never touch empty sticks.
#include <mutex>
#include <type_traits>

#include "fft_core.cuh"
#include "hpsi_local.cuh"

namespace q3b {
namespace {

constexpr int kStickThreads = 256;
constexpr int kLoadBatch = 4;      // global loads a stick-kernel thread keeps in flight
constexpr int kRowMaskWords = 16;  // one word per item of the first column pass (nb1 <= 16)

// Shared-memory set-up of the plane kernels: rowb[i] = w1 * p2 of the i-th
// row holding sticks; colmask[q] bit r set when row q + nb1*r holds sticks
// (the ItemMask of the column passes).  Ends with a barrier.
template <typename R>
__device__ __forceinline__ void stick_rows_setup(const LocalPlan<R>& p, int* rowb, unsigned* colmask) {
    for (int i = threadIdx.x; i < kRowMaskWords; i += blockDim.x) colmask[i] = 0u;
    __syncthreads();
    for (int i = threadIdx.x; i < p.nrows; i += blockDim.x) {
        const int b = p.row_base[i];
        rowb[i] = b;
        const int w1 = b / p.p2;
        atomicOr(&colmask[w1 % p.nb1], 1u << (w1 / p.nb1));
    }
    __syncthreads();
}

// zero the rows that hold sticks, a warp per row
template <typename T, typename R>
__device__ __forceinline__ void zero_stick_rows(const LocalPlan<R>& p, const int* rowb, T* plane) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int r = threadIdx.x >> 5; r < p.nrows; r += nw) {
        T* row = plane + rowb[r];
        for (int c = lane; c < p.p2; c += 32) row[c] = czero<T>();
    }
}

// V/N of one plane in the layout the plane kernel meets it: [w1][w2 position]
// with the w2 positions of the digit-reversed order the row transform leaves.
template <typename R> struct VEpilogue {
    const R* vp;
    int n2;
    template <typename T> __device__ __forceinline__ T operator()(int l, int j, T v) const {
        return vp[j * n2 + l] * v;
    }
};

// Kernels are instantiated twice: for lines whose factors are all <= 10
// (MAXR 10, within 64 registers a thread in FP32) and for any supported line
// (MAXR 16).
constexpr int kSmallR = 10;

// pass A: scatter + backward transform along w3, store X[band][w3 pos][stick]
// (w3 in the transform's digit-reversed order, which pass C undoes)
template <typename R, int MAXR>
__global__ void __launch_bounds__(kStickThreads)
sticks_backward(LocalPlan<R> p, const cplx_t<R>* __restrict__ psi, long ldpsi, cplx_t<R>* X) {
    using T = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem[];
    T* tw = reinterpret_cast<T*>(smem);
    T* lines = tw + p.n3;
    const int band = blockIdx.y;
    const int s0 = blockIdx.x * p.sg;
    const int ns = min(p.sg, p.nsticks - s0);
    for (int i = threadIdx.x; i < p.n3; i += blockDim.x) tw[i] = p.tw3[i];
    for (int i = threadIdx.x; i < ns * p.p3; i += blockDim.x) lines[i] = czero<T>();
    __syncthreads();
    const T* ps = psi + (long)band * ldpsi;
    const int e0 = p.stick_start[s0], e1 = p.stick_start[s0 + ns];
    // kLoadBatch gathers in flight per thread before any is stored
    for (int eb = e0 + threadIdx.x; eb < e1; eb += kLoadBatch * blockDim.x) {
        T v[kLoadBatch];
        int at[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int e = eb + u * blockDim.x;
            at[u] = -1;
            if (e < e1) {
                at[u] = (p.entry_stick[e] - s0) * p.p3 + p.entry_w3[e];
                v[u] = ps[p.entry_g[e]];
            }
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u)
            if (at[u] >= 0) lines[at[u]] = v[u];
    }
    __syncthreads();
    fft::LineGeom g{p.n3, p.na3, p.nb3, ns, p.p3, 1, nullptr};
    fft::backward<MAXR>(lines, g, tw);
    T* xb = X + (long)band * p.n3 * p.xpitch;
    for (int idx = threadIdx.x; idx < ns * p.n3; idx += blockDim.x) {
        const int s = idx % ns, i3 = idx / ns;
        xb[(long)i3 * p.xpitch + s0 + s] = lines[s * p.p3 + i3];
    }
}

// pass B: one (band, w3) plane per block of NT threads: rows backward (their
// w2 left digit-reversed), columns backward, V, columns forward (fused round
// trip), rows forward.  Every pass is in place; one barrier between passes.
// Register budget: 64 per thread in FP32 (four 256-thread planes of an 80x80
// grid fit an SM's shared memory), 128 in FP64.
template <typename R, int NT, int MAXR> constexpr int plane_min_blocks() {
    constexpr int regs = MAXR <= kSmallR ? (sizeof(R) == 4 ? 64 : 128) : (sizeof(R) == 4 ? 96 : 168);
    return 65536 / (NT * regs) > 0 ? 65536 / (NT * regs) : 1;
}

template <typename R, int NT, int MAXR>
__global__ void __launch_bounds__(NT, (plane_min_blocks<R, NT, MAXR>())) planes(LocalPlan<R> p, cplx_t<R>* X) {
    using T = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem[];
    T* tw1 = reinterpret_cast<T*>(smem);
    T* tw2 = tw1 + p.n1;
    T* plane = tw2 + p.n2;
    int* rowb = reinterpret_cast<int*>(plane + (long)p.n1 * p.p2);
    unsigned* colmask = reinterpret_cast<unsigned*>(rowb + p.nrows);  // see stick_rows_setup
    const int i3 = blockIdx.x, band = blockIdx.y;
    for (int i = threadIdx.x; i < p.n1; i += NT) tw1[i] = p.tw1[i];
    for (int i = threadIdx.x; i < p.n2; i += NT) tw2[i] = p.tw2[i];
    stick_rows_setup(p, rowb, colmask);
    // only the rows that hold sticks are read before they are written: the
    // column transform reads the others as zero, and writes back only these
    zero_stick_rows(p, rowb, plane);
    __syncthreads();
    T* xp = X + ((long)band * p.n3 + i3) * p.xpitch;
    for (int s = threadIdx.x; s < p.nsticks; s += NT) plane[p.stick_pos[s]] = xp[s];
    __syncthreads();
    fft::LineGeom gr{p.n2, p.na2, p.nb2, p.nrows, 0, 1, rowb};
    fft::LineGeom gc{p.n1, p.na1, p.nb1, p.n2, 1, p.p2, nullptr};
    fft::backward<MAXR>(plane, gr, tw2);
    fft::roundtrip<MAXR>(plane, gc, tw1, VEpilogue<R>{p.vplane + (long)i3 * p.n1 * p.n2, p.n2},
                         fft::ItemMask{colmask});
    fft::forward<MAXR>(plane, gr, tw2);
    for (int s = threadIdx.x; s < p.nsticks; s += NT) xp[s] = plane[p.stick_pos[s]];
}

// pass C: forward transform along w3, gather the sphere, add the kinetic term
template <typename R, int MAXR>
__global__ void __launch_bounds__(kStickThreads)
sticks_forward(LocalPlan<R> p, const cplx_t<R>* __restrict__ X, const cplx_t<R>* __restrict__ psi,
               long ldpsi, cplx_t<R>* hpsi, long ldh) {
    using T = cplx_t<R>;
    extern __shared__ __align__(16) unsigned char smem[];
    T* tw = reinterpret_cast<T*>(smem);
    T* lines = tw + p.n3;
    const int band = blockIdx.y;
    const int s0 = blockIdx.x * p.sg;
    const int ns = min(p.sg, p.nsticks - s0);
    for (int i = threadIdx.x; i < p.n3; i += blockDim.x) tw[i] = p.tw3[i];
    const T* xb = X + (long)band * p.n3 * p.xpitch;
    const int total = ns * p.n3;
    for (int ib = threadIdx.x; ib < total; ib += kLoadBatch * blockDim.x) {
        T v[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int idx = ib + u * blockDim.x;
            if (idx < total) v[u] = xb[(long)(idx / ns) * p.xpitch + s0 + idx % ns];
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int idx = ib + u * blockDim.x;
            if (idx < total) lines[(idx % ns) * p.p3 + idx / ns] = v[u];
        }
    }
    __syncthreads();
    fft::LineGeom g{p.n3, p.na3, p.nb3, ns, p.p3, 1, nullptr};
    fft::forward<MAXR>(lines, g, tw);
    const T* ps = psi + (long)band * ldpsi;
    T* hs = hpsi + (long)band * ldh;
    const int e0 = p.stick_start[s0], e1 = p.stick_start[s0 + ns];
    for (int eb = e0 + threadIdx.x; eb < e1; eb += kLoadBatch * blockDim.x) {
        int gi[kLoadBatch];
        R ke[kLoadBatch];
        T x[kLoadBatch], v[kLoadBatch];
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            const int e = eb + u * blockDim.x;
            gi[u] = -1;
            if (e < e1) {
                gi[u] = p.entry_g[e];
                v[u] = lines[(p.entry_stick[e] - s0) * p.p3 + p.entry_w3[e]];
            }
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u) {
            if (gi[u] >= 0) {
                ke[u] = p.ke[gi[u]];
                x[u] = ps[gi[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < kLoadBatch; ++u)
            if (gi[u] >= 0) hs[gi[u]] = ke[u] * x[u] + v[u];
    }
}

// G outside the grid get the kinetic term only (serial.hpp:451-462 skip them)
template <typename R>
__global__ void kinetic_unmapped(LocalPlan<R> p, const cplx_t<R>* psi, long ldpsi, cplx_t<R>* hpsi,
                                 long ldh, int nvec) {
    const long total = (long)p.nunmapped * nvec;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        const int i = static_cast<int>(idx % p.nunmapped);
        const long b = idx / p.nunmapped;
        const int gi = p.unmapped_g[i];
        hpsi[b * ldh + gi] = p.ke[gi] * psi[b * ldpsi + gi];
    }
}

template <typename R> size_t stick_smem_bytes(const LocalPlan<R>& p) {
    return (size_t)(p.n3 + p.sg * p.p3) * sizeof(cplx_t<R>);
}

template <typename R, int MAXR> void set_limits_for() {
    const int lim = 227 * 1024;
    const void* pk[3] = {reinterpret_cast<const void*>(planes<R, 128, MAXR>),
                         reinterpret_cast<const void*>(planes<R, 256, MAXR>),
                         reinterpret_cast<const void*>(planes<R, 512, MAXR>)};
    for (const void* k : pk) {
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
        cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    }
    cudaFuncSetAttribute(sticks_backward<R, MAXR>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
    cudaFuncSetAttribute(sticks_forward<R, MAXR>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

template <typename R> void set_smem_limits() {
    static PerDeviceOnce once;
    once.run([] {
        set_limits_for<R, kSmallR>();
        set_limits_for<R, 16>();
    });
}

template <typename R, int NT, int MAXR>
void launch_planes(dim3 grid, size_t smem, cudaStream_t st, const LocalPlan<R>& p, cplx_t<R>* X) {
    planes<R, NT, MAXR><<<grid, NT, smem, st>>>(p, X);
}

// Charge density (accumulator.hpp:375-545, non-Gamma): the backward half of
// the plane pass.  Block (plane position i3, band group g) transforms each
// band of its group on plane i3 (rows holding sticks, then all columns, both
// left in digit-reversed order) and adds w_b |psi(r)|^2 into its own slab of
// `partial` ([g][i3][w1 pos][w2 pos]); one block per slab, bands in order, so
// the sums are deterministic.  Bands of weight 0 are skipped.
constexpr int kAccBatch = 16;

template <int MAXR>
__global__ void __launch_bounds__(256, 2) planes_density(LocalPlan<double> p, const double2* X, int nb,
                                                      const double* w, double* partial, int groups) {
    using T = double2;
    extern __shared__ __align__(16) unsigned char smem[];
    T* tw1 = reinterpret_cast<T*>(smem);
    T* tw2 = tw1 + p.n1;
    T* plane = tw2 + p.n2;
    int* rowb = reinterpret_cast<int*>(plane + (long)p.n1 * p.p2);
    unsigned* colmask = reinterpret_cast<unsigned*>(rowb + p.nrows);
    const int i3 = blockIdx.x, g = blockIdx.y;
    const int per = (nb + groups - 1) / groups;
    const int b0 = g * per, b1 = min(nb, b0 + per);
    for (int i = threadIdx.x; i < p.n1; i += blockDim.x) tw1[i] = p.tw1[i];
    for (int i = threadIdx.x; i < p.n2; i += blockDim.x) tw2[i] = p.tw2[i];
    stick_rows_setup(p, rowb, colmask);
    const int nplane = p.n1 * p.n2;
    double* acc = partial + ((size_t)g * p.n3 + i3) * nplane;
    fft::LineGeom gr{p.n2, p.na2, p.nb2, p.nrows, 0, 1, rowb};
    fft::LineGeom gc{p.n1, p.na1, p.nb1, p.n2, 1, p.p2, nullptr};
    for (int b = b0; b < b1; ++b) {
        const double wb = w[b];
        if (wb == 0.0) continue;
        zero_stick_rows(p, rowb, plane);
        __syncthreads();
        const T* xp = X + ((long)b * p.n3 + i3) * p.xpitch;
        for (int s = threadIdx.x; s < p.nsticks; s += blockDim.x) plane[p.stick_pos[s]] = xp[s];
        __syncthreads();
        fft::backward<MAXR>(plane, gr, tw2);
        fft::run_a<+1, MAXR>(plane, gc, tw1, fft::ItemMask{colmask}, fft::AllPositions{});
        __syncthreads();
        fft::run_b<+1, MAXR>(plane, gc, tw1);
        __syncthreads();
        // the slab's loads are issued kAccBatch at a time, so that as many are
        // in flight per thread rather than one load's latency per position
        for (int i0 = threadIdx.x; i0 < nplane; i0 += kAccBatch * blockDim.x) {
            double old[kAccBatch];
#pragma unroll
            for (int j = 0; j < kAccBatch; ++j) {
                const int i = i0 + j * blockDim.x;
                old[j] = i < nplane ? acc[i] : 0.0;
            }
#pragma unroll
            for (int j = 0; j < kAccBatch; ++j) {
                const int i = i0 + j * blockDim.x;
                if (i < nplane) {
                    const int row = i / p.n2;
                    const T v = plane[row * p.p2 + (i - row * p.n2)];
                    acc[i] = old[j] + wb * (v.x * v.x + v.y * v.y);
                }
            }
        }
        __syncthreads();
    }
}

// rho[(w1*N2 + w2)*N3 + w3] += sum over groups (in order) of the partial at
// the digit-reversed positions of (w1, w2, w3)
__global__ void density_reduce(LocalPlan<double> p, int groups, const double* partial, double* rho) {
    const long n = (long)p.n1 * p.n2 * p.n3;
    const long nplane = (long)p.n1 * p.n2;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < n; idx += (long)gridDim.x * blockDim.x) {
        const int w3 = static_cast<int>(idx % p.n3);
        const int w2 = static_cast<int>((idx / p.n3) % p.n2);
        const int w1 = static_cast<int>(idx / ((long)p.n3 * p.n2));
        const int q1 = p.nb1 * (w1 % p.na1) + w1 / p.na1;
        const int q2 = p.nb2 * (w2 % p.na2) + w2 / p.na2;
        const int q3 = p.nb3 * (w3 % p.na3) + w3 / p.na3;
        const long off = (long)q3 * nplane + (long)q1 * p.n2 + q2;
        double s = 0.0;
        for (int g = 0; g < groups; ++g) s += partial[(long)g * p.n3 * nplane + off];
        rho[idx] += s;
    }
}

}  // namespace

template <typename R> size_t plane_smem_bytes(const LocalPlan<R>& p) {
    return (size_t)(p.n1 + p.n2 + (size_t)p.n1 * p.p2) * sizeof(cplx_t<R>) +
           (size_t)p.nrows * sizeof(int) + kRowMaskWords * sizeof(unsigned);
}

PhaseTimer::PhaseTimer() {
    for (int i = 0; i < 2 * kMax; ++i) Q3B_CUDA(cudaEventCreate(&ev[i]));
}
PhaseTimer::~PhaseTimer() {
    for (int i = 0; i < 2 * kMax; ++i) cudaEventDestroy(ev[i]);
}
void PhaseTimer::begin(int c) {
    if (used >= kMax) return;
    cls[used] = c;
    Q3B_CUDA(cudaEventRecord(ev[2 * used], st));
}
void PhaseTimer::end() {
    if (used >= kMax) return;
    Q3B_CUDA(cudaEventRecord(ev[2 * used + 1], st));
    ++used;
}
void PhaseTimer::collect(double* ms, int* count) {
    Q3B_CUDA(cudaStreamSynchronize(st));
    for (int c = 0; c < NCLASS; ++c) {
        ms[c] = 0.0;
        count[c] = 0;
    }
    for (int i = 0; i < used; ++i) {
        float t = 0.f;
        Q3B_CUDA(cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]));
        ms[cls[i]] += t;
        count[cls[i]] += 1;
    }
}

template <typename R>
void apply_local(cudaStream_t st, const LocalPlan<R>& p, const cplx_t<R>* psi, long ldpsi,
                 cplx_t<R>* hpsi, long ldh, int nvec, cplx_t<R>* X, int chunk, PhaseTimer* tm) {
    if (nvec <= 0) return;
    set_smem_limits<R>();
    if (chunk < 1) chunk = 1;
    const size_t smem_s = stick_smem_bytes(p);
    const size_t smem_p = plane_smem_bytes(p);
    const int nsg = ceil_div(p.nsticks, p.sg);
    for (int b0 = 0; b0 < nvec; b0 += chunk) {
        const int nb = nvec - b0 < chunk ? nvec - b0 : chunk;
        const cplx_t<R>* ps = psi + (long)b0 * ldpsi;
        cplx_t<R>* hs = hpsi + (long)b0 * ldh;
        if (p.nsticks > 0) {
            if (tm) tm->begin(PhaseTimer::STICKS_BACKWARD);
            const bool small3 = p.na3 <= kSmallR && p.nb3 <= kSmallR;
            if (small3)
                sticks_backward<R, kSmallR><<<dim3(nsg, nb), kStickThreads, smem_s, st>>>(p, ps, ldpsi, X);
            else
                sticks_backward<R, 16><<<dim3(nsg, nb), kStickThreads, smem_s, st>>>(p, ps, ldpsi, X);
            Q3B_LAUNCH_CHECK();
            if (tm) tm->end();
            if (tm) tm->begin(PhaseTimer::PLANES);
            const dim3 gp(p.n3, nb);
            const bool small12 = p.na1 <= kSmallR && p.nb1 <= kSmallR && p.na2 <= kSmallR && p.nb2 <= kSmallR;
            if (p.variant > 0 && launch_planes_reg<R>(p, X, nb, p.variant, st, p.err)) {
                // the register kernel took the plane pass
            } else if (small12) {
                if (p.plane_threads >= 512) launch_planes<R, 512, kSmallR>(gp, smem_p, st, p, X);
                else if (p.plane_threads >= 256) launch_planes<R, 256, kSmallR>(gp, smem_p, st, p, X);
                else launch_planes<R, 128, kSmallR>(gp, smem_p, st, p, X);
            } else {
                if (p.plane_threads >= 512) launch_planes<R, 512, 16>(gp, smem_p, st, p, X);
                else if (p.plane_threads >= 256) launch_planes<R, 256, 16>(gp, smem_p, st, p, X);
                else launch_planes<R, 128, 16>(gp, smem_p, st, p, X);
            }
            Q3B_LAUNCH_CHECK();
            if (tm) tm->end();
            if (tm) tm->begin(PhaseTimer::STICKS_FORWARD);
            if (small3)
                sticks_forward<R, kSmallR><<<dim3(nsg, nb), kStickThreads, smem_s, st>>>(p, X, ps, ldpsi, hs, ldh);
            else
                sticks_forward<R, 16><<<dim3(nsg, nb), kStickThreads, smem_s, st>>>(p, X, ps, ldpsi, hs, ldh);
            Q3B_LAUNCH_CHECK();
            if (tm) tm->end();
        }
    }
    if (p.nunmapped > 0) {
        const long total = (long)p.nunmapped * nvec;
        int blocks = ceil_div(total, 256);
        if (blocks > 1024) blocks = 1024;
        kinetic_unmapped<R><<<blocks, 256, 0, st>>>(p, psi, ldpsi, hpsi, ldh, nvec);
        Q3B_LAUNCH_CHECK();
    }
}

namespace {

// the partial slabs of the density stay below this many bytes, so that they
// stay in L2 beside a stick chunk (48 MB) while the bands add into them
constexpr size_t kDensityPartialBytes = 32ull << 20;

bool density_small_factors(const LocalPlan<double>& p) {
    return p.na1 <= kSmallR && p.nb1 <= kSmallR && p.na2 <= kSmallR && p.nb2 <= kSmallR;
}

void set_density_limits() {
    static PerDeviceOnce once;
    once.run([] {
        cudaFuncSetAttribute(planes_density<kSmallR>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
        cudaFuncSetAttribute(planes_density<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    });
}

}  // namespace

// A density block runs its group's bands one after another on one plane, so a
// launch of n3 * groups blocks takes ceil(n3 * groups / resident blocks) waves
// of ceil(nvec / groups) band-planes each.  The group count is the one that
// minimises that product (the smallest on a tie), within the slab budget: on
// an 80^3 grid with two resident blocks per SM, a 39-band chunk runs as 7
// groups of 6 bands in 2 waves (12 band-planes a block), where 4 groups of 10
// would take 2 waves of 10 band-planes, the second with 24 blocks on 148 SMs.
int density_groups(const LocalPlan<double>& p, int nvec) {
    if (nvec < 1) return 1;
    set_density_limits();
    int per_sm = 0, dev = 0, sms = 0;
    if (density_small_factors(p))
        Q3B_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, planes_density<kSmallR>, 256,
                                                               plane_smem_bytes(p)));
    else
        Q3B_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, planes_density<16>, 256, plane_smem_bytes(p)));
    Q3B_CUDA(cudaGetDevice(&dev));
    Q3B_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long slots = (long)(per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
    const size_t slab = (size_t)p.n1 * p.n2 * p.n3 * sizeof(double);
    long gmax = static_cast<long>(kDensityPartialBytes / slab);
    if (gmax > nvec) gmax = nvec;
    if (gmax < 1) gmax = 1;
    int best = 1;
    long best_cost = -1;
    for (int g = 1; g <= gmax; ++g) {
        const long cost = (long)ceil_div((long)p.n3 * g, slots) * ceil_div(nvec, g);
        if (best_cost < 0 || cost < best_cost) {
            best_cost = cost;
            best = g;
        }
    }
    return best;
}

void accumulate_density(cudaStream_t st, const LocalPlan<double>& p, const double2* psi, long ldpsi, int nvec,
                        const double* w, double2* X, int chunk, double* partial, int groups, double* rho) {
    if (nvec <= 0 || p.nsticks == 0) return;
    set_smem_limits<double>();
    set_density_limits();
    if (chunk < 1) chunk = 1;
    const size_t smem_s = stick_smem_bytes(p);
    const size_t smem_p = plane_smem_bytes(p);
    const int nsg = ceil_div(p.nsticks, p.sg);
    const bool small3 = p.na3 <= kSmallR && p.nb3 <= kSmallR;
    const bool small12 = density_small_factors(p);
    Q3B_CUDA(cudaMemsetAsync(partial, 0, (size_t)groups * p.n1 * p.n2 * p.n3 * sizeof(double), st));
    for (int b0 = 0; b0 < nvec; b0 += chunk) {
        const int nb = nvec - b0 < chunk ? nvec - b0 : chunk;
        const double2* ps = psi + (long)b0 * ldpsi;
        if (small3)
            sticks_backward<double, kSmallR><<<dim3(nsg, nb), kStickThreads, smem_s, st>>>(p, ps, ldpsi, X);
        else
            sticks_backward<double, 16><<<dim3(nsg, nb), kStickThreads, smem_s, st>>>(p, ps, ldpsi, X);
        Q3B_LAUNCH_CHECK();
        const int gb = nb < groups ? nb : groups;
        // every chunk adds into the same slabs; a chunk with fewer bands than
        // groups leaves the remaining slabs as they are
        if (small12)
            planes_density<kSmallR><<<dim3(p.n3, gb), 256, smem_p, st>>>(p, X, nb, w + b0, partial, gb);
        else
            planes_density<16><<<dim3(p.n3, gb), 256, smem_p, st>>>(p, X, nb, w + b0, partial, gb);
        Q3B_LAUNCH_CHECK();
    }
    const long n = (long)p.n1 * p.n2 * p.n3;
    int blocks = ceil_div(n, 256);
    if (blocks > 4096) blocks = 4096;
    density_reduce<<<blocks, 256, 0, st>>>(p, groups, partial, rho);
    Q3B_LAUNCH_CHECK();
}

template void apply_local<double>(cudaStream_t, const LocalPlan<double>&, const double2*, long,
                                  double2*, long, int, double2*, int, PhaseTimer*);
template void apply_local<float>(cudaStream_t, const LocalPlan<float>&, const float2*, long,
                                 float2*, long, int, float2*, int, PhaseTimer*);
template size_t plane_smem_bytes<double>(const LocalPlan<double>&);
template size_t plane_smem_bytes<float>(const LocalPlan<float>&);

}  // namespace q3b
