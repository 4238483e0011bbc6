#include <type_traits>
#include <algorithm>
// extern "C" entry points of libq3b (include/q3b.h).  Every call converts
// exceptions to a status code and keeps the message on the context.
#include <chrono>

#include "context.cuh"
#include "q3b.h"

using q3b::Context;

namespace {

template <typename F> int guarded(q3b_context* c, F&& f) {
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

template <typename R, typename CT>
void gemm_entry(Context& c, char ta, char tb, int m, int n, int k, CT alpha, const CT* a, int lda,
                       const CT* b, int ldb, CT beta, CT* cc, int ldc) {
    using T = q3b::cplx_t<R>;
    const bool conj = (ta == 'C' || ta == 'c');
    if (!(conj || ta == 'N' || ta == 'n') || !(tb == 'N' || tb == 'n'))
        throw q3b::Status(Q3B_ERR_INVALID, "gemm: transpose_a must be N or C and transpose_b N");
    if (m < 0 || n < 0 || k < 0) throw q3b::Status(Q3B_ERR_INVALID, "gemm: negative size");
    if (m == 0 || n == 0) return;
    if ((k > 0 && (!a || !b)) || !cc) throw q3b::Status(Q3B_ERR_INVALID, "gemm: null matrix");
    if (lda < (conj ? k : m) || ldb < k || ldc < m || lda < 1 || ldb < 1)
        throw q3b::Status(Q3B_ERR_INVALID, "gemm: leading dimension too small");
    q3b::GemmWorkspace ws = c.gemm_ws(conj ? q3b::cgemm_workspace_bytes<R>(m, n, k) : 0);
    if constexpr (std::is_same<R, float>::value) {
        // the single-precision entry point always runs on the tensor cores
        // (the library's own products route small ones to the CUDA cores)
        if (k > 0) {
            q3b::tc::cgemm(c.stream, conj, m, n, k, T{alpha.re, alpha.im}, reinterpret_cast<const T*>(a), lda,
                           reinterpret_cast<const T*>(b), ldb, T{beta.re, beta.im}, reinterpret_cast<T*>(cc), ldc,
                           ws);
            return;
        }
    }
    q3b::cgemm<R>(c.stream, conj, m, n, k, T{alpha.re, alpha.im}, reinterpret_cast<const T*>(a), lda,
                  reinterpret_cast<const T*>(b), ldb, T{beta.re, beta.im}, reinterpret_cast<T*>(cc), ldc, ws);
}

}  // namespace

extern "C" {

int q3b_context_create(int device, size_t hbm_budget_bytes, q3b_context** out) {
    if (!out) return Q3B_ERR_INVALID;
    *out = nullptr;
    try {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
            cudaGetLastError();
            return Q3B_ERR_CUDA;
        }
        *out = new q3b_context(device, hbm_budget_bytes);
        return Q3B_OK;
    } catch (const std::exception&) {
        return Q3B_ERR_CUDA;
    }
}

int q3b_context_destroy(q3b_context* ctx) {
    if (!ctx) return Q3B_ERR_INVALID;
    delete ctx;
    return Q3B_OK;
}

const char* q3b_last_error(const q3b_context* ctx) {
    return ctx ? ctx->impl.err.c_str() : "null context";
}

void* q3b_get_stream(q3b_context* ctx) { return ctx ? static_cast<void*>(ctx->impl.stream) : nullptr; }

int q3b_set_stream(q3b_context* ctx, void* s) {
    return guarded(ctx, [&](Context& c) {
        c.stream = s ? static_cast<cudaStream_t>(s) : c.own_stream;
    });
}

int q3b_synchronize(q3b_context* ctx) {
    return guarded(ctx, [&](Context& c) {
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
        q3b::tc::check_error(c.stream);
    });
}

size_t q3b_device_bytes(const q3b_context* ctx) { return ctx ? ctx->impl.held : 0; }

int q3b_set_potential(q3b_context* ctx, const double* v, int n1, int n2, int n3) {
    return guarded(ctx, [&](Context& c) { c.set_potential(v, n1, n2, n3); });
}

int q3b_set_potential_dense(q3b_context* ctx, const double* v, int d1, int d2, int d3, int n1, int n2, int n3) {
    return guarded(ctx, [&](Context& c) { c.set_potential_dense(v, d1, d2, d3, n1, n2, n3); });
}

int q3b_set_d_blocks(q3b_context* ctx, const double* d_blocks_host) {
    return guarded(ctx, [&](Context& c) { c.set_d_blocks(d_blocks_host); });
}

int q3b_invalidate_potential(q3b_context* ctx) {
    return guarded(ctx, [&](Context& c) { c.pot_valid = false; });
}

int q3b_potential_valid(const q3b_context* ctx) { return ctx && ctx->impl.pot_valid ? 1 : 0; }

int q3b_prepare_kpoint(q3b_context* ctx, int npw, const int32_t* g2g, const double* ke,
                       const q3b_cplx128* beta, int nproj, int natoms, const int32_t* offs,
                       const double* dblk) {
    return guarded(ctx, [&](Context& c) {
        c.prepare_kpoint(npw, g2g, ke, reinterpret_cast<const double2*>(beta), nproj, natoms, offs,
                         dblk);
    });
}

int q3b_apply_h(q3b_context* ctx, const q3b_cplx128* psi, q3b_cplx128* hpsi, int nvec, int precision) {
    return guarded(ctx, [&](Context& c) {
        if (nvec < 0 || (nvec > 0 && (!psi || !hpsi))) throw q3b::Status(Q3B_ERR_INVALID, "bad vectors");
        const int npw = c.kp.npw;
        if (precision == Q3B_FP64) {
            c.apply_h<double>(reinterpret_cast<const double2*>(psi), npw,
                              reinterpret_cast<double2*>(hpsi), npw, nvec);
        } else if (precision == Q3B_MIXED) {
            c.require_ready();
            const size_t n = (size_t)npw * nvec;
            c.ws_conv_in.reserve(&c, n * sizeof(float2));
            c.ws_conv_out.reserve(&c, n * sizeof(float2));
            q3b::convert<double, float>(c.stream, n, reinterpret_cast<const double2*>(psi),
                                        c.ws_conv_in.as<float2>());
            c.apply_h<float>(c.ws_conv_in.as<float2>(), npw, c.ws_conv_out.as<float2>(), npw, nvec);
            q3b::convert<float, double>(c.stream, n, c.ws_conv_out.as<float2>(),
                                        reinterpret_cast<double2*>(hpsi));
        } else {
            throw q3b::Status(Q3B_ERR_INVALID, "unknown precision");
        }
    });
}

int q3b_apply_h_f32(q3b_context* ctx, const q3b_cplx64* psi, q3b_cplx64* hpsi, int nvec) {
    return guarded(ctx, [&](Context& c) {
        if (nvec < 0 || (nvec > 0 && (!psi || !hpsi))) throw q3b::Status(Q3B_ERR_INVALID, "bad vectors");
        c.apply_h<float>(reinterpret_cast<const float2*>(psi), c.kp.npw,
                         reinterpret_cast<float2*>(hpsi), c.kp.npw, nvec);
    });
}

// Host vectors in and out.  The bands go through in chunks on three streams:
// chunk i's copy in, its application on the context's stream and its copy out
// run while chunk i+1 is copied in and chunk i-1 copied out, so the two copy
// directions and the kernels overlap.  Pinned host buffers make the copies
// asynchronous; pageable ones still work, serialised by the driver.
int q3b_apply_h_host(q3b_context* ctx, const q3b_cplx128* psi, q3b_cplx128* hpsi, int nvec,
                     int precision) {
    return guarded(ctx, [&](Context& c) {
        c.require_ready();
        if (nvec <= 0) return;
        if (!psi || !hpsi) throw q3b::Status(Q3B_ERR_INVALID, "bad vectors");
        const int npw = c.kp.npw;
        const size_t n = (size_t)npw * nvec;
        c.ws_host_io.reserve(&c, 2 * n * sizeof(double2));
        double2* din = c.ws_host_io.as<double2>();
        double2* dout = din + n;
        c.ensure_io_streams();
        const int nchunk = nvec >= 32 ? Context::kIoChunks : 1;
        const int per = (nvec + nchunk - 1) / nchunk;
        const auto* hin = reinterpret_cast<const double2*>(psi);
        auto* hout = reinterpret_cast<double2*>(hpsi);
        for (int i = 0; i < nchunk; ++i) {
            const int b0 = i * per, nb = std::min(per, nvec - b0);
            if (nb <= 0) break;
            const size_t off = (size_t)b0 * npw, bytes = (size_t)nb * npw * sizeof(double2);
            Q3B_CUDA(cudaMemcpyAsync(din + off, hin + off, bytes, cudaMemcpyHostToDevice, c.io_in));
            Q3B_CUDA(cudaEventRecord(c.io_ev_in[i], c.io_in));
        }
        for (int i = 0; i < nchunk; ++i) {
            const int b0 = i * per, nb = std::min(per, nvec - b0);
            if (nb <= 0) break;
            const size_t off = (size_t)b0 * npw, bytes = (size_t)nb * npw * sizeof(double2);
            Q3B_CUDA(cudaStreamWaitEvent(c.stream, c.io_ev_in[i], 0));
            const int rc = q3b_apply_h(ctx, reinterpret_cast<q3b_cplx128*>(din + off),
                                       reinterpret_cast<q3b_cplx128*>(dout + off), nb, precision);
            if (rc != Q3B_OK) {
                cudaStreamSynchronize(c.io_in);
                throw q3b::Status(rc, c.err);
            }
            Q3B_CUDA(cudaEventRecord(c.io_ev_out[i], c.stream));
            Q3B_CUDA(cudaStreamWaitEvent(c.io_out, c.io_ev_out[i], 0));
            Q3B_CUDA(cudaMemcpyAsync(hout + off, dout + off, bytes, cudaMemcpyDeviceToHost, c.io_out));
        }
        Q3B_CUDA(cudaStreamSynchronize(c.io_out));
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
        q3b::tc::check_error(c.stream);
    });
}

int q3b_graph_stats(q3b_context* ctx, int* captures, int* replays) {
    if (!ctx) return Q3B_ERR_INVALID;
    if (captures) *captures = ctx->impl.hegv_graphs.captures;
    if (replays) *replays = ctx->impl.hegv_graphs.replays;
    return Q3B_OK;
}

int q3b_set_local_kernel(q3b_context* ctx, int precision, int choice) {
    return guarded(ctx, [&](Context& c) {
        c.require_ready();
        if (precision == Q3B_FP64) c.set_local_kernel<double>(choice);
        else if (precision == Q3B_MIXED) c.set_local_kernel<float>(choice);
        else throw q3b::Status(Q3B_ERR_INVALID, "unknown precision");
    });
}

int q3b_get_local_kernel(q3b_context* ctx, int precision, int* choice) {
    return guarded(ctx, [&](Context& c) {
        c.require_ready();
        if (!choice) throw q3b::Status(Q3B_ERR_INVALID, "null output");
        if (precision == Q3B_FP64) *choice = c.local_kernel<double>();
        else if (precision == Q3B_MIXED) *choice = c.local_kernel<float>();
        else throw q3b::Status(Q3B_ERR_INVALID, "unknown precision");
    });
}

int q3b_accumulate_density(q3b_context* ctx, const q3b_cplx128* psi, int nvec, const double* weights,
                           double* rho) {
    return guarded(ctx, [&](Context& c) {
        c.require_ready();
        if (nvec < 0 || (nvec > 0 && (!psi || !weights || !rho))) throw q3b::Status(Q3B_ERR_INVALID, "bad arguments");
        if (nvec == 0) return;
        const q3b::LocalPlan<double>& lp = c.local_plan<double>();
        const int chunk = c.sticks_chunk<double>(nvec);
        const int groups = q3b::density_groups(lp, chunk);
        const size_t n = (size_t)lp.n1 * lp.n2 * lp.n3;
        const size_t pbytes = ((groups * n * sizeof(double)) + 255) & ~size_t(255);
        c.ws_density.reserve(&c, pbytes + (size_t)nvec * sizeof(double));
        double* partial = c.ws_density.as<double>();
        double* w = reinterpret_cast<double*>(c.ws_density.as<char>() + pbytes);
        q3b::upload_async(w, weights, (size_t)nvec * sizeof(double), c.stream);
        c.ws_sticks.reserve(&c, (size_t)chunk * q3b::sticks_bytes_per_band(lp));
        q3b::accumulate_density(c.stream, lp, reinterpret_cast<const double2*>(psi), c.kp.npw, nvec, w,
                                c.ws_sticks.as<double2>(), chunk, partial, groups, rho);
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int q3b_apply_h_timed(q3b_context* ctx, const void* psi, void* hpsi, int nvec, int fp32,
                      q3b_apply_timing* timing) {
    return guarded(ctx, [&](Context& c) {
        if (nvec < 0 || (nvec > 0 && (!psi || !hpsi))) throw q3b::Status(Q3B_ERR_INVALID, "bad vectors");
        q3b::PhaseTimer tm;
        tm.st = c.stream;
        const int npw = c.kp.npw;
        if (fp32)
            c.apply_h<float>(static_cast<const float2*>(psi), npw, static_cast<float2*>(hpsi), npw, nvec, &tm);
        else
            c.apply_h<double>(static_cast<const double2*>(psi), npw, static_cast<double2*>(hpsi), npw, nvec, &tm);
        double ms[q3b::PhaseTimer::NCLASS];
        int cnt[q3b::PhaseTimer::NCLASS];
        tm.collect(ms, cnt);
        q3b::tc::check_error(c.stream);
        if (timing) {
            timing->sticks_backward_ms = ms[0];
            timing->planes_ms = ms[1];
            timing->sticks_forward_ms = ms[2];
            timing->projector_overlap_ms = ms[3];
            timing->d_apply_ms = ms[4];
            timing->projector_accumulate_ms = ms[5];
            for (int i = 0; i < 6; ++i) timing->launches[i] = cnt[i];
        }
    });
}

unsigned long long q3b_kernel_launches(void) { return q3b::launches(); }

int q3b_measure_fp64_rate(q3b_context* ctx, double* tflops) {
    return guarded(ctx, [&](Context& c) {
        if (!tflops) throw q3b::Status(Q3B_ERR_INVALID, "null output");
        *tflops = q3b::measure_dfma_tflops(c.stream);
    });
}

int q3b_gemm(q3b_context* ctx, char ta, char tb, int m, int n, int k, q3b_cplx128 alpha, const q3b_cplx128* a,
             int lda, const q3b_cplx128* b, int ldb, q3b_cplx128 beta, q3b_cplx128* cc, int ldc) {
    return guarded(ctx, [&](Context& c) { gemm_entry<double>(c, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, cc, ldc); });
}

int q3b_gemm_single(q3b_context* ctx, char ta, char tb, int m, int n, int k, q3b_cplx64 alpha, const q3b_cplx64* a,
                    int lda, const q3b_cplx64* b, int ldb, q3b_cplx64 beta, q3b_cplx64* cc, int ldc) {
    return guarded(ctx, [&](Context& c) { gemm_entry<float>(c, ta, tb, m, n, k, alpha, a, lda, b, ldb, beta, cc, ldc); });
}

}  // extern "C"

// ---------------------------------------------------------------- Davidson
#include "davidson.cuh"
#include "dense.cuh"

extern "C" {

void q3b_davidson_default_opts(q3b_davidson_opts* o) {
    if (!o) return;
    o->tolerance = 1e-2;           // initial_eigenvalue_tolerance (tolerances.hpp:224)
    o->max_iterations = 20;        // davidson.hpp:1156
    o->basis_expansion_factor = 2; // davidson.hpp:864
    o->occupied_bands = 0;         // 0: every band is occupied
    o->precision = Q3B_FP64;
    o->refine_sweeps = 0;          // MIXED: refinement up to max_iterations
    o->mixed_tolerance = 1e-6;
    o->profile_stages = 0;
    o->eigenvalue_history = nullptr;
    o->history_rows = 0;
    o->mixed_expansion_factor = 0;
}

int q3b_davidson_solve_dev(q3b_context* ctx, q3b_cplx128* bands, double* eig, int nb,
                           const q3b_davidson_opts* opts, q3b_davidson_stats* stats) {
    return guarded(ctx, [&](Context& c) {
        if (!bands || !eig || !opts) throw q3b::Status(Q3B_ERR_INVALID, "null argument");
        q3b::davidson_solve(c, reinterpret_cast<double2*>(bands), eig, nb, *opts, stats);
    });
}

int q3b_davidson_solve(q3b_context* ctx, q3b_cplx128* bands, double* eig, int nb,
                       const q3b_davidson_opts* opts, q3b_davidson_stats* stats) {
    return guarded(ctx, [&](Context& c) {
        if (!bands || !eig || !opts) throw q3b::Status(Q3B_ERR_INVALID, "null argument");
        c.require_ready();
        if (nb <= 0 || nb > c.band_npw()) throw q3b::Status(Q3B_ERR_INVALID, "band count must be in [1, npw]");
        const size_t bytes = (size_t)c.band_npw() * nb * sizeof(double2);
        c.ws_bands.reserve(&c, bytes);
        Q3B_CUDA(cudaMemcpyAsync(c.ws_bands.ptr, bands, bytes, cudaMemcpyHostToDevice, c.stream));
        q3b::davidson_solve(c, c.ws_bands.as<double2>(), eig, nb, *opts, stats);
        Q3B_CUDA(cudaMemcpyAsync(bands, c.ws_bands.ptr, bytes, cudaMemcpyDeviceToHost, c.stream));
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int q3b_hegv_lowest(q3b_context* ctx, int n, const q3b_cplx128* h, const q3b_cplx128* s, int ld, int nvec,
                    double* w, q3b_cplx128* evec) {
    return guarded(ctx, [&](Context& c) {
        if (n < 0 || ld < n || nvec < 1 || nvec > n || (n > 0 && (!h || !s || !w || !evec)))
            throw q3b::Status(Q3B_ERR_INVALID, "bad hegv arguments");
        if (n == 0) return;
        c.ws_dense.reserve(&c, q3b::dense::hegv_scratch_bytes(n));
        q3b::dense::Scratch ws{c.ws_dense.as<char>(), c.ws_dense.bytes, 0};
        q3b::GemmWorkspace g = c.gemm_ws(q3b::cgemm_workspace_bytes<double>(n, n, n));
        const int info = q3b::dense::hegv(c.stream, n, reinterpret_cast<const double2*>(h),
                                          reinterpret_cast<const double2*>(s), ld, w,
                                          reinterpret_cast<double2*>(evec), nvec, ws, g, &c.hegv_graphs);
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
        if (info != 0)
            throw q3b::Status(Q3B_ERR_LINALG, "overlap matrix not positive definite (info " +
                                                  std::to_string(info) + ")");
    });
}

int q3b_hegv_batched(q3b_context* ctx, int count, const int* n, const q3b_cplx128* const* h,
                     const q3b_cplx128* const* s, const int* ld, const int* nvec, double* const* w,
                     q3b_cplx128* const* evec, int* info_host) {
    return guarded(ctx, [&](Context& c) {
        if (count < 0 || (count > 0 && (!n || !h || !s || !ld || !nvec || !w || !evec || !info_host)))
            throw q3b::Status(Q3B_ERR_INVALID, "bad batched hegv arguments");
        if (count == 0) return;
        std::vector<q3b::dense::BlockProblem> probs(count);
        size_t work = 0, smem = 0;
        for (int i = 0; i < count; ++i) {
            if (!q3b::dense::hegv_block_fits(n[i], nvec[i]) || ld[i] < n[i] || !h[i] || !s[i] || !w[i] || !evec[i])
                throw q3b::Status(Q3B_ERR_INVALID, "batched hegv: problem " + std::to_string(i) +
                                                       " does not fit one block");
            work += (q3b::dense::hegv_block_work_elems(n[i]) + 16) & ~size_t(15);
            smem = std::max(smem, q3b::dense::hegv_block_smem(n[i], nvec[i]));
        }
        // scratch: the problems' work areas, their status words and the descriptors
        const size_t desc_off = work * sizeof(double2);
        const size_t info_off = (desc_off + count * sizeof(q3b::dense::BlockProblem) + 255) & ~size_t(255);
        c.ws_dense.reserve(&c, info_off + count * sizeof(int));
        char* base = c.ws_dense.as<char>();
        double2* wk = reinterpret_cast<double2*>(base);
        int* info = reinterpret_cast<int*>(base + info_off);
        for (int i = 0; i < count; ++i) {
            probs[i] = q3b::dense::BlockProblem{n[i], ld[i], nvec[i], reinterpret_cast<const double2*>(h[i]),
                                                reinterpret_cast<const double2*>(s[i]), w[i],
                                                reinterpret_cast<double2*>(evec[i]), wk, info + i};
            wk += (q3b::dense::hegv_block_work_elems(n[i]) + 16) & ~size_t(15);
        }
        auto* dev_probs = reinterpret_cast<q3b::dense::BlockProblem*>(base + desc_off);
        Q3B_CUDA(cudaMemcpyAsync(dev_probs, probs.data(), count * sizeof(q3b::dense::BlockProblem),
                                 cudaMemcpyHostToDevice, c.stream));
        q3b::dense::hegv_block_many(c.stream, dev_probs, count, smem);
        Q3B_CUDA(cudaMemcpyAsync(info_host, info, count * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int q3b_set_block_eigensolver_order(int max_order) {
    const int prev = q3b::dense::block_max_order();
    q3b::dense::set_block_max_order(max_order);
    return prev;
}

int q3b_hegv(q3b_context* ctx, int n, const q3b_cplx128* h, const q3b_cplx128* s, int ld, double* w,
             q3b_cplx128* evec) {
    return guarded(ctx, [&](Context& c) {
        if (n < 0 || ld < n || (n > 0 && (!h || !s || !w || !evec)))
            throw q3b::Status(Q3B_ERR_INVALID, "bad hegv arguments");
        if (n == 0) return;
        c.ws_dense.reserve(&c, q3b::dense::hegv_scratch_bytes(n));
        q3b::dense::Scratch ws{c.ws_dense.as<char>(), c.ws_dense.bytes, 0};
        q3b::GemmWorkspace g = c.gemm_ws(q3b::cgemm_workspace_bytes<double>(n, n, n));
        const int info = q3b::dense::hegv(c.stream, n, reinterpret_cast<const double2*>(h),
                                          reinterpret_cast<const double2*>(s), ld, w,
                                          reinterpret_cast<double2*>(evec), n, ws, g, &c.hegv_graphs);
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
        if (info != 0)
            throw q3b::Status(Q3B_ERR_LINALG, "overlap matrix not positive definite (info " +
                                                  std::to_string(info) + ")");
    });
}

}  // extern "C"
