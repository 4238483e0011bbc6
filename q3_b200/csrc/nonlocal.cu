#include <type_traits>
// Kleinman-Bylander term and small elementwise helpers.
//
// hpsi += beta D beta^H psi, as SerialPlanewaveHamiltonianApplicator does it
// (hamiltonian_applicator/serial.hpp:567-700): B = beta^H psi ("C","N"),
// B' = D B with D block-diagonal by atom (serial.hpp:602-679), then
// hpsi += beta B' ("N","N", beta = 1).
#include "nonlocal.cuh"

namespace q3b {
namespace {

// B'[p, v] = sum_q D_atom(p)[p - s, q - s] B[q, v] over the atom's block
template <typename R>
__global__ void apply_d_blocks(int P, int nvec, const int* __restrict__ pstart,
                               const int* __restrict__ psize, const int* __restrict__ poff,
                               const R* __restrict__ dpk, const cplx_t<R>* __restrict__ B,
                               cplx_t<R>* __restrict__ Bp) {
    using T = cplx_t<R>;
    const long total = (long)P * nvec;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        const int p = static_cast<int>(idx % P);
        const long v = idx / P;
        const int s = pstart[p], m = psize[p], off = poff[p];
        const int r = p - s;
        T acc = czero<T>();
        for (int c = 0; c < m; ++c) {
            const R d = dpk[off + r + c * m];
            const T b = B[v * P + s + c];
            acc.x += d * b.x;
            acc.y += d * b.y;
        }
        Bp[v * P + p] = acc;
    }
}

template <typename RI, typename RO>
__global__ void convert_kernel(long n, const cplx_t<RI>* __restrict__ in, cplx_t<RO>* __restrict__ out) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const cplx_t<RI> v = in[i];
        out[i] = mk(static_cast<RO>(v.x), static_cast<RO>(v.y));
    }
}

inline int grid_for(long n) { return stride_grid(n, 16); }

}  // namespace

template <typename R>
void apply_nonlocal(cudaStream_t st, const NonlocalData<R>& nl, int npw, int nvec,
                    const cplx_t<R>* psi, long ldpsi, cplx_t<R>* hpsi, long ldh, cplx_t<R>* Bm,
                    cplx_t<R>* Bp, const GemmWorkspace& ws, PhaseTimer* tm) {
    using T = cplx_t<R>;
    if (nl.nproj <= 0 || nvec <= 0) return;
    const T one = mk(R(1), R(0)), zero = mk(R(0), R(0));
    if (tm) tm->begin(PhaseTimer::PROJ_OVERLAP);
    if constexpr (std::is_same<R, float>::value) {
        if (nl.beta_overlap.tiles && use_tensor_cores(nl.nproj, nvec, npw))
            tc::cgemm_packed(st, true, nl.nproj, nvec, npw, one, nl.beta_overlap, psi, ldpsi, zero, Bm, nl.nproj, ws);
        else
            cgemm<R>(st, true, nl.nproj, nvec, npw, one, nl.beta, npw, psi, ldpsi, zero, Bm, nl.nproj, ws);
    } else {
        cgemm<R>(st, true, nl.nproj, nvec, npw, one, nl.beta, npw, psi, ldpsi, zero, Bm, nl.nproj, ws);
    }
    if (tm) tm->end();
    if (tm) tm->begin(PhaseTimer::D_APPLY);
    apply_d_blocks<R><<<grid_for((long)nl.nproj * nvec), 256, 0, st>>>(
        nl.nproj, nvec, nl.pstart, nl.psize, nl.poff, nl.dpk, Bm, Bp);
    Q3B_LAUNCH_CHECK();
    if (tm) tm->end();
    if (tm) tm->begin(PhaseTimer::PROJ_ACCUM);
    if constexpr (std::is_same<R, float>::value) {
        if (nl.beta_accum.tiles && use_tensor_cores(npw, nvec, nl.nproj))
            tc::cgemm_packed(st, false, npw, nvec, nl.nproj, one, nl.beta_accum, Bp, nl.nproj, one, hpsi, ldh, ws);
        else
            cgemm<R>(st, false, npw, nvec, nl.nproj, one, nl.beta, npw, Bp, nl.nproj, one, hpsi, ldh, ws);
    } else {
        cgemm<R>(st, false, npw, nvec, nl.nproj, one, nl.beta, npw, Bp, nl.nproj, one, hpsi, ldh, ws);
    }
    if (tm) tm->end();
}

template <typename RI, typename RO>
void convert(cudaStream_t st, long n, const cplx_t<RI>* in, cplx_t<RO>* out) {
    if (n <= 0) return;
    convert_kernel<RI, RO><<<grid_for(n), 256, 0, st>>>(n, in, out);
    Q3B_LAUNCH_CHECK();
}

template void apply_nonlocal<double>(cudaStream_t, const NonlocalData<double>&, int, int,
                                     const double2*, long, double2*, long, double2*, double2*,
                                     const GemmWorkspace&, PhaseTimer*);
template void apply_nonlocal<float>(cudaStream_t, const NonlocalData<float>&, int, int,
                                    const float2*, long, float2*, long, float2*, float2*,
                                    const GemmWorkspace&, PhaseTimer*);
template void convert<double, float>(cudaStream_t, long, const double2*, float2*);
template void convert<float, double>(cudaStream_t, long, const float2*, double2*);
template void convert<double, double>(cudaStream_t, long, const double2*, double2*);

}  // namespace q3b
