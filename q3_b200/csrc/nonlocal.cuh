// Kleinman-Bylander nonlocal term of H|psi>; see nonlocal.cu.
#pragma once

#include "cgemm.cuh"
#include "common.cuh"
#include "hpsi_local.cuh"

namespace q3b {

template <typename R> struct NonlocalData {
    int nproj = 0;
    const cplx_t<R>* beta = nullptr;  // npw x nproj, ld npw
    const int* pstart = nullptr;      // first projector of p's atom block
    const int* psize = nullptr;       // size of p's atom block
    const int* poff = nullptr;        // offset of p's block in dpk
    const R* dpk = nullptr;           // packed column-major D blocks (Ry)
    // FP32 only: beta pre-split into the tensor-core kernel's A tiles, for
    // beta^H psi (rows = projectors) and for beta B' (rows = plane waves)
    tc::PackedA beta_overlap{}, beta_accum{};
};

// hpsi += beta D beta^H psi.  Bm, Bp: nproj x nvec scratch each.
template <typename R>
void apply_nonlocal(cudaStream_t st, const NonlocalData<R>& nl, int npw, int nvec,
                    const cplx_t<R>* psi, long ldpsi, cplx_t<R>* hpsi, long ldh, cplx_t<R>* Bm,
                    cplx_t<R>* Bp, const GemmWorkspace& ws, PhaseTimer* timer = nullptr);

// out = (RO) in, n complex values
template <typename RI, typename RO>
void convert(cudaStream_t st, long n, const cplx_t<RI>* in, cplx_t<RO>* out);

}  // namespace q3b
