// Ultrasoft overlap operator S psi = psi + sum_ij beta_i q_ij <beta_j|psi>, as
// UltrasoftPseudopotentialOverlapOperator::apply_batch does it
// (diagonalizer/planewave/internal/overlap/pseudopotential/ultrasoft/init.hpp:189-345):
// S psi starts as a copy of psi, B = beta^H psi, B' = Q B with Q block-diagonal
// by atom, S psi += beta B'.  The projector products are the same ones the
// nonlocal term of H runs (tensor-core GEMMs on the pre-split projectors in
// FP32), with Q in place of D.
#include "context.cuh"
#include "nonlocal.cuh"
#include "q3b.h"

namespace q3b {
namespace {

// out = psi + (double) corr
__global__ void add_widened(long n, const double2* __restrict__ psi, const float2* __restrict__ corr,
                            double2* __restrict__ out) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double2 p = psi[i];
        const float2 c = corr[i];
        out[i] = mk(p.x + static_cast<double>(c.x), p.y + static_cast<double>(c.y));
    }
}

inline int blocks_for(long n) { return stride_grid(n, 16); }

}  // namespace

void apply_s_device(Context& c, const double2* psi, double2* spsi, int nvec, int precision) {
    c.require_ready();
    if (!c.kp.has_q) throw Status(Q3B_ERR_STATE, "no overlap blocks set for this k-point (q3b_set_overlap_blocks)");
    if (nvec <= 0) return;
    const int npw = c.kp.npw, P = c.kp.nproj;
    const size_t n = (size_t)npw * nvec;
    if (precision == Q3B_FP64) {
        if (spsi != psi)
            Q3B_CUDA(cudaMemcpyAsync(spsi, psi, n * sizeof(double2), cudaMemcpyDeviceToDevice, c.stream));
        const size_t pb = (size_t)P * nvec * sizeof(double2);
        c.ws_bm.reserve(&c, pb);
        c.ws_bp.reserve(&c, pb);
        GemmWorkspace ws = c.gemm_ws(cgemm_workspace_bytes<double>(P, nvec, npw));
        apply_nonlocal<double>(c.stream, c.overlap<double>(), npw, nvec, psi, npw, spsi, npw,
                               c.ws_bm.as<double2>(), c.ws_bp.as<double2>(), ws);
    } else if (precision == Q3B_MIXED) {
        // the correction beta Q beta^H psi in FP32, added to the FP64 copy of psi
        c.ws_conv_in.reserve(&c, n * sizeof(float2));
        c.ws_conv_out.reserve(&c, n * sizeof(float2));
        convert<double, float>(c.stream, (long)n, psi, c.ws_conv_in.as<float2>());
        Q3B_CUDA(cudaMemsetAsync(c.ws_conv_out.ptr, 0, n * sizeof(float2), c.stream));
        const size_t pb = (size_t)P * nvec * sizeof(float2);
        c.ws_bm.reserve(&c, pb);
        c.ws_bp.reserve(&c, pb);
        GemmWorkspace ws = c.gemm_ws(cgemm_workspace_bytes<float>(P, nvec, npw));
        apply_nonlocal<float>(c.stream, c.overlap<float>(), npw, nvec, c.ws_conv_in.as<float2>(), npw,
                              c.ws_conv_out.as<float2>(), npw, c.ws_bm.as<float2>(), c.ws_bp.as<float2>(), ws);
        add_widened<<<blocks_for((long)n), 256, 0, c.stream>>>((long)n, psi, c.ws_conv_out.as<float2>(), spsi);
        Q3B_LAUNCH_CHECK();
    } else {
        throw Status(Q3B_ERR_INVALID, "unknown precision");
    }
}

}  // namespace q3b

using q3b::Context;

namespace {
template <typename F> int overlap_guarded(q3b_context* c, F&& f) {
    if (!c) return Q3B_ERR_INVALID;
    try {
        Q3B_CUDA(cudaSetDevice(c->impl.device));
        q3b::tc::ErrorScope scope(c->impl.err_word.as<int>());
        f(c->impl);
        return Q3B_OK;
    } catch (const std::exception& e) {
        return q3b::fail(c, e);
    }
}
}  // namespace

int q3b_set_overlap_blocks(q3b_context* ctx, const double* q_blocks_host) {
    return overlap_guarded(ctx, [&](Context& c) { c.set_overlap_blocks(q_blocks_host); });
}

int q3b_apply_s(q3b_context* ctx, const q3b_cplx128* psi_dev, q3b_cplx128* spsi_dev, int nvec, int precision) {
    return overlap_guarded(ctx, [&](Context& c) {
        if (nvec < 0 || (nvec > 0 && (!psi_dev || !spsi_dev))) throw q3b::Status(Q3B_ERR_INVALID, "bad vectors");
        q3b::apply_s_device(c, reinterpret_cast<const double2*>(psi_dev), reinterpret_cast<double2*>(spsi_dev),
                            nvec, precision);
    });
}
