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
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        lines[(p.entry_stick[e] - s0) * p.p3 + p.entry_w3[e]] = ps[p.entry_g[e]];
    }
    __syncthreads();
    fft::LineGeom g{p.n3, p.na3, p.nb3, ns, p.p3, 1, nullptr};
    fft::backward<MAXR>(lines, g, tw);
    T* xb = X + (long)band * p.n3 * p.nsticks;
    for (int idx = threadIdx.x; idx < ns * p.n3; idx += blockDim.x) {
        const int s = idx % ns, i3 = idx / ns;
        xb[(long)i3 * p.nsticks + s0 + s] = lines[s * p.p3 + i3];
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
    const int i3 = blockIdx.x, band = blockIdx.y;
    for (int i = threadIdx.x; i < p.n1; i += NT) tw1[i] = p.tw1[i];
    for (int i = threadIdx.x; i < p.n2; i += NT) tw2[i] = p.tw2[i];
    for (int i = threadIdx.x; i < p.nrows; i += NT) rowb[i] = p.row_base[i];
    for (int i = threadIdx.x; i < p.n1 * p.p2; i += NT) plane[i] = czero<T>();
    __syncthreads();
    T* xp = X + ((long)band * p.n3 + i3) * p.nsticks;
    for (int s = threadIdx.x; s < p.nsticks; s += NT) plane[p.stick_pos[s]] = xp[s];
    __syncthreads();
    fft::LineGeom gr{p.n2, p.na2, p.nb2, p.nrows, 0, 1, rowb};
    fft::LineGeom gc{p.n1, p.na1, p.nb1, p.n2, 1, p.p2, nullptr};
    fft::backward<MAXR>(plane, gr, tw2);
    fft::roundtrip<MAXR>(plane, gc, tw1, VEpilogue<R>{p.vplane + (long)i3 * p.n1 * p.n2, p.n2});
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
    const T* xb = X + (long)band * p.n3 * p.nsticks;
    for (int idx = threadIdx.x; idx < ns * p.n3; idx += blockDim.x) {
        const int s = idx % ns, i3 = idx / ns;
        lines[s * p.p3 + i3] = xb[(long)i3 * p.nsticks + s0 + s];
    }
    __syncthreads();
    fft::LineGeom g{p.n3, p.na3, p.nb3, ns, p.p3, 1, nullptr};
    fft::forward<MAXR>(lines, g, tw);
    const T* ps = psi + (long)band * ldpsi;
    T* hs = hpsi + (long)band * ldh;
    const int e0 = p.stick_start[s0], e1 = p.stick_start[s0 + ns];
    for (int e = e0 + threadIdx.x; e < e1; e += blockDim.x) {
        const int gi = p.entry_g[e];
        const T v = lines[(p.entry_stick[e] - s0) * p.p3 + p.entry_w3[e]];
        hs[gi] = p.ke[gi] * ps[gi] + v;
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
    static std::once_flag once;
    std::call_once(once, [] {
        set_limits_for<R, kSmallR>();
        set_limits_for<R, 16>();
    });
}

template <typename R, int NT, int MAXR>
void launch_planes(dim3 grid, size_t smem, cudaStream_t st, const LocalPlan<R>& p, cplx_t<R>* X) {
    planes<R, NT, MAXR><<<grid, NT, smem, st>>>(p, X);
}

}  // namespace

template <typename R> size_t plane_smem_bytes(const LocalPlan<R>& p) {
    return (size_t)(p.n1 + p.n2 + (size_t)p.n1 * p.p2) * sizeof(cplx_t<R>) +
           (size_t)p.nrows * sizeof(int);
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
            if (small12) {
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

template void apply_local<double>(cudaStream_t, const LocalPlan<double>&, const double2*, long,
                                  double2*, long, int, double2*, int, PhaseTimer*);
template void apply_local<float>(cudaStream_t, const LocalPlan<float>&, const float2*, long,
                                 float2*, long, int, float2*, int, PhaseTimer*);
template size_t plane_smem_bytes<double>(const LocalPlan<double>&);
template size_t plane_smem_bytes<float>(const LocalPlan<float>&);

}  // namespace q3b
