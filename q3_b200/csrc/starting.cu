// Starting-subspace rotation of one k-point (StartingSubspaceSolver,
// wavefunction/planewave/starting_subspace_solver.hpp:29-59; the initializer
// that drives it, wavefunction/planewave/norm_conserving/initializer.hpp:
// 250-385): H on the starting vectors chi, the projections chi^H H chi and
// chi^H chi, the generalised eigenproblem, and the rotation chi c.  FP64, on
// the library's own H|psi>, complex GEMM and dense eigensolver.  chi and H chi
// live in the context's ws_start between the calls.
#include "context.cuh"
#include "dense.cuh"
#include "q3b.h"

namespace {

template <typename F> int guarded_start(q3b_context* ctx, F&& f) {
    if (!ctx) return Q3B_ERR_INVALID;
    try {
        Q3B_CUDA(cudaSetDevice(ctx->impl.device));
        q3b::tc::ErrorScope scope(ctx->impl.err_word.as<int>());
        f(ctx->impl);
        return Q3B_OK;
    } catch (const std::exception& e) {
        return q3b::fail(ctx, e);
    }
}

const double2 kOne = {1.0, 0.0}, kZero = {0.0, 0.0};

// chi at the start of ws_start, H chi after it
double2* chi_of(q3b::Context& c) { return c.ws_start.as<double2>(); }
double2* hchi_of(q3b::Context& c) { return c.ws_start.as<double2>() + (size_t)c.start_npw * c.start_n; }

void start_apply(q3b::Context& c, const double2* chi, int nchi) {
    c.require_ready();
    if (nchi <= 0 || !chi) throw q3b::Status(Q3B_ERR_INVALID, "starting vectors: need nchi > 0 and a buffer");
    const int npw = c.kp.npw;
    const size_t n = (size_t)npw * nchi;
    c.start_n = 0;
    c.ws_start.reserve(&c, 2 * n * sizeof(double2));
    c.start_n = nchi;
    c.start_npw = npw;
    Q3B_CUDA(cudaMemcpyAsync(chi_of(c), chi, n * sizeof(double2), cudaMemcpyHostToDevice, c.stream));
    c.apply_h<double>(chi_of(c), npw, hchi_of(c), npw, nchi);
}

void require_started(const q3b::Context& c) {
    if (c.start_n <= 0 || c.start_npw != c.kp.npw || !c.kp.valid)
        throw q3b::Status(Q3B_ERR_STATE, "call q3b_start_apply on the prepared k-point first");
}

// H (n x n) and S (n x n), ld n, on the device
void start_project_dev(q3b::Context& c, double2* H, double2* S) {
    const int n = c.start_n, npw = c.start_npw;
    q3b::GemmWorkspace g = c.gemm_ws(q3b::cgemm_workspace_bytes<double>(n, n, npw));
    q3b::cgemm<double>(c.stream, true, n, n, npw, kOne, chi_of(c), npw, hchi_of(c), npw, kZero, H, n, g);
    q3b::cgemm<double>(c.stream, true, n, n, npw, kOne, chi_of(c), npw, chi_of(c), npw, kZero, S, n, g);
}

void start_rotate_dev(q3b::Context& c, const double2* C, int ldc, int nb, double2* bands) {
    const int n = c.start_n, npw = c.start_npw;
    q3b::GemmWorkspace g = c.gemm_ws(q3b::cgemm_workspace_bytes<double>(npw, nb, n));
    q3b::cgemm<double>(c.stream, false, npw, nb, n, kOne, chi_of(c), npw, C, ldc, kZero, bands, npw, g);
}

}  // namespace

extern "C" {

int q3b_start_apply(q3b_context* ctx, const q3b_cplx128* chi_host, int nchi) {
    return guarded_start(ctx, [&](q3b::Context& c) {
        start_apply(c, reinterpret_cast<const double2*>(chi_host), nchi);
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
        q3b::tc::check_error(c.stream);
    });
}

int q3b_start_project(q3b_context* ctx, q3b_cplx128* h_host, q3b_cplx128* s_host) {
    return guarded_start(ctx, [&](q3b::Context& c) {
        require_started(c);
        if (!h_host || !s_host) throw q3b::Status(Q3B_ERR_INVALID, "null output matrix");
        const size_t nn = (size_t)c.start_n * c.start_n;
        c.ws_solver.reserve(&c, 2 * nn * sizeof(double2));
        double2* H = c.ws_solver.as<double2>();
        double2* S = H + nn;
        start_project_dev(c, H, S);
        Q3B_CUDA(cudaMemcpyAsync(h_host, H, nn * sizeof(double2), cudaMemcpyDeviceToHost, c.stream));
        Q3B_CUDA(cudaMemcpyAsync(s_host, S, nn * sizeof(double2), cudaMemcpyDeviceToHost, c.stream));
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int q3b_start_rotate(q3b_context* ctx, const q3b_cplx128* coefficients_host, int nb, q3b_cplx128* bands_dev) {
    return guarded_start(ctx, [&](q3b::Context& c) {
        require_started(c);
        if (nb <= 0 || !coefficients_host || !bands_dev) throw q3b::Status(Q3B_ERR_INVALID, "bad rotation arguments");
        const size_t nc = (size_t)c.start_n * nb;
        c.ws_solver.reserve(&c, nc * sizeof(double2));
        double2* C = c.ws_solver.as<double2>();
        Q3B_CUDA(cudaMemcpyAsync(C, coefficients_host, nc * sizeof(double2), cudaMemcpyHostToDevice, c.stream));
        start_rotate_dev(c, C, c.start_n, nb, reinterpret_cast<double2*>(bands_dev));
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int q3b_starting_subspace(q3b_context* ctx, const q3b_cplx128* chi_host, int nchi, int nb,
                          q3b_cplx128* bands_dev, double* eigenvalues_host) {
    return guarded_start(ctx, [&](q3b::Context& c) {
        if (nb <= 0 || nb > nchi || !bands_dev || !eigenvalues_host)
            throw q3b::Status(Q3B_ERR_INVALID, "need 0 < nb <= nchi and output buffers");
        start_apply(c, reinterpret_cast<const double2*>(chi_host), nchi);
        const int n = nchi;
        const size_t nn = (size_t)n * n;
        c.ws_solver.reserve(&c, (3 * nn) * sizeof(double2) + (size_t)n * sizeof(double) + 256);
        double2* H = c.ws_solver.as<double2>();
        double2* S = H + nn;
        double2* Z = S + nn;
        double* w = reinterpret_cast<double*>(Z + nn);
        start_project_dev(c, H, S);
        c.ws_dense.reserve(&c, q3b::dense::hegv_scratch_bytes(n));
        q3b::dense::Scratch ws{c.ws_dense.as<char>(), c.ws_dense.bytes, 0};
        q3b::GemmWorkspace g = c.gemm_ws(q3b::cgemm_workspace_bytes<double>(n, n, n));
        const int info = q3b::dense::hegv(c.stream, n, H, S, n, w, Z, nb, ws, g, &c.hegv_graphs);
        if (info != 0)
            throw q3b::Status(Q3B_ERR_LINALG, "overlap of the starting vectors is not positive definite (info " +
                                                  std::to_string(info) + ")");
        start_rotate_dev(c, Z, n, nb, reinterpret_cast<double2*>(bands_dev));
        Q3B_CUDA(cudaMemcpyAsync(eigenvalues_host, w, nb * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
        q3b::tc::check_error(c.stream);
    });
}

}  // extern "C"
