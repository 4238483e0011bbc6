// Device-resident block Davidson.
//
// The loop control is the reference's (PlanewaveDavidsonDiagonalizer::solve,
// davidson.hpp:324-841) with the norm-conserving branches of its serial
// subspace manager (subspace_manager/serial.hpp): seed from the given bands,
// fill from lowest-kinetic-energy plane waves; per iteration diagonalise the
// subspace (generalized, FP64), test |eps_i - eps_i(prev)| < tol, build the
// TPA-preconditioned corrections of the unconverged bands into the free basis
// columns, project them out and Cholesky-QR them (MGS fallback), apply H,
// extend H_sub / S_sub, collapse to nb Ritz vectors when the basis is full.
//
// Everything stays on the GPU: V, HV (S|V> aliases V for norm-conserving
// pseudopotentials), H_sub, S_sub, the eigenvectors.  The host reads only
// scalars: Cholesky info, the nb eigenvalues, MGS norms.
//
// Precision: Davidson<double> is the FP64 solver.  Davidson<float> keeps the
// vectors and the GEMMs in FP32 and the subspace (H_sub, S_sub, Cholesky,
// eigensolve) in FP64; the MIXED solve runs it to a loose tolerance, then
// hands its Ritz vectors to Davidson<double> for the FP64 refinement sweeps.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <numeric>
#include <vector>

#include "batcher.cuh"
#include "davidson.cuh"
#include "dense.cuh"
#include "gamma.cuh"
#include "nonlocal.cuh"

namespace q3b {
namespace {

constexpr double kNormThreshold = 1e-14;    // tolerances.hpp:39
constexpr double kPrecondFloor = 1e-4;      // tolerances.hpp:50
constexpr double kEmptyRelax = 5.0;         // tolerances.hpp:65
constexpr double kEmptyFloor = 1e-5;        // tolerances.hpp:66
constexpr double kStallBelow = 1e-5;        // Ry: the FP32 phase may stop on a plateau below this
constexpr int kFlatIterations = 4;          // FP32 phase: iterations without a new band-energy low
// FP32 phase: the occupied Ritz values' sum fell by less than kCrawlRelative of the
// sum of their magnitudes over the last kCrawlWindow iterations
constexpr int kCrawlWindow = 16;
constexpr double kCrawlRelative = 2e-6;

inline int grid_for(long n) { return stride_grid(n, 16); }

// R[:, j] /= max(0.5 (1 + x + sqrt(1 + (x-1)^2)), 1e-4), x = KE - eps_j
// (subspace_manager/serial.hpp:1138-1156)
template <typename R>
__global__ void precondition_kernel(int npw, int ncols, const double* __restrict__ ke,
                                    const double* __restrict__ eps, cplx_t<R>* X) {
    const long total = (long)npw * ncols;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        const int g = static_cast<int>(idx % npw);
        const int j = static_cast<int>(idx / npw);
        const double x = ke[g] - eps[j];
        double den = 0.5 * (1.0 + x + sqrt(1.0 + (x - 1.0) * (x - 1.0)));
        if (den < kPrecondFloor) den = kPrecondFloor;
        const R inv = static_cast<R>(1.0 / den);
        cplx_t<R> v = X[idx];
        v.x *= inv;
        v.y *= inv;
        X[idx] = v;
    }
}

// out[:, j] = evec[:, idx[j]] (ld n), outneg = -eps_j * out[:, j], in precision R
template <typename R>
__global__ void pack_coefficients(int n, int ncols, const double2* __restrict__ evec,
                                  const int* __restrict__ idx, const double* __restrict__ w,
                                  cplx_t<R>* out, cplx_t<R>* outneg, double* eps) {
    const long total = (long)n * ncols;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
         t += (long)gridDim.x * blockDim.x) {
        const int r = static_cast<int>(t % n);
        const int j = static_cast<int>(t / n);
        const int b = idx[j];
        const double2 v = evec[r + (long)b * n];
        const double e = w[b];
        out[t] = mk(static_cast<R>(v.x), static_cast<R>(v.y));
        outneg[t] = mk(static_cast<R>(-e * v.x), static_cast<R>(-e * v.y));
        if (r == 0) eps[j] = e;
    }
}

template <typename R>
__global__ void unit_vectors(int npw, int count, const int* __restrict__ gidx, cplx_t<R>* V) {
    const long total = (long)npw * count;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
         t += (long)gridDim.x * blockDim.x) {
        const int g = static_cast<int>(t % npw);
        const int j = static_cast<int>(t / npw);
        V[t] = (g == gidx[j]) ? mk(R(1), R(0)) : mk(R(0), R(0));
    }
}

template <typename R>
__global__ void scale_vector(long n, cplx_t<R>* v, double s) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        cplx_t<R> x = v[i];
        x.x = static_cast<R>(x.x * s);
        x.y = static_cast<R>(x.y * s);
        v[i] = x;
    }
}

// dst (double2, ld ldd) = src (R, ld lds), an M x N block
template <typename R>
__global__ void widen_block(int M, int N, const cplx_t<R>* __restrict__ src, int lds, double2* dst, int ldd) {
    const long total = (long)M * N;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
         t += (long)gridDim.x * blockDim.x) {
        const int r = static_cast<int>(t % M), c = static_cast<int>(t / M);
        const cplx_t<R> v = src[r + (long)c * lds];
        dst[r + (long)c * ldd] = mk((double)v.x, (double)v.y);
    }
}

template <typename R>
__global__ void narrow_block(int M, int N, const double2* __restrict__ src, int lds, cplx_t<R>* dst, int ldd) {
    const long total = (long)M * N;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
         t += (long)gridDim.x * blockDim.x) {
        const int r = static_cast<int>(t % M), c = static_cast<int>(t / M);
        const double2 v = src[r + (long)c * lds];
        dst[r + (long)c * ldd] = mk(static_cast<R>(v.x), static_cast<R>(v.y));
    }
}

// out[j] = ||X[:, j]||, one block per column, fixed-order reduction; with
// gamma the half-sphere norm sqrt(2 sum |x|^2 - |x_0|^2)
template <typename R>
__global__ void column_norms(int npw, const cplx_t<R>* __restrict__ X, double* out, int gamma = 0) {
    const cplx_t<R>* x = X + (long)blockIdx.x * npw;
    double s = 0.0;
    for (int g = threadIdx.x; g < npw; g += blockDim.x) {
        const cplx_t<R> v = x[g];
        s += (double)v.x * v.x + (double)v.y * v.y;
    }
    __shared__ double red[256];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double t = red[0];
        if (gamma) {
            const cplx_t<R> v0 = x[0];
            t = 2.0 * t - ((double)v0.x * v0.x + (double)v0.y * v0.y);
        }
        out[blockIdx.x] = sqrt(t > 0.0 ? t : 0.0);
    }
}

// Gamma-only inner products of half-sphere vectors (the subspace manager's
// gamma branches, e.g. subspace_manager/serial.hpp:72-110): C = 2 Re(A^H B)
// less the origin's Re(conj(A_0) B_0), real
template <typename T>
__global__ void gamma_inner_fix(int M, int N, const T* __restrict__ A, long lda, const T* __restrict__ B, long ldb,
                                T* C, long ldc) {
    const long total = (long)M * N;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x) {
        const int i = static_cast<int>(t % M), j = static_cast<int>(t / M);
        const T c = C[i + (long)j * ldc];
        const T a0 = A[(long)i * lda], b0 = B[(long)j * ldb];
        const double re = 2.0 * (double)c.x - ((double)a0.x * b0.x + (double)a0.y * b0.y);
        C[i + (long)j * ldc] = mk(static_cast<decltype(c.x)>(re), static_cast<decltype(c.x)>(0));
    }
}

__global__ void set_identity(int n, double2* E) {
    const long total = (long)n * n;
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total; t += (long)gridDim.x * blockDim.x)
        E[t] = (t % n == t / n) ? mk(1.0, 0.0) : mk(0.0, 0.0);
}

// Host-side stage clock in the spirit of the reference's stage_time_point
// (davidson.hpp:942-956): the stream is drained before each reading, so a
// stage is charged for the device work it queued.
struct StageClock {
    cudaStream_t st = nullptr;
    double* ms = nullptr;  // 8 stages, or null when not profiling
    std::chrono::steady_clock::time_point t;
    void start() {
        if (!ms) return;
        Q3B_CUDA(cudaStreamSynchronize(st));
        t = std::chrono::steady_clock::now();
    }
    void stop(int stage) {
        if (!ms) return;
        Q3B_CUDA(cudaStreamSynchronize(st));
        const auto now = std::chrono::steady_clock::now();
        ms[stage] += std::chrono::duration<double, std::milli>(now - t).count();
        t = now;
    }
};
enum Stage { SEED = 0, DIAG, CORR, ORTHO, HAPPLY, UPDATE, COLLAPSE, EXTRACT };

// carve one device buffer into slices
struct Carve {
    char* base;
    size_t off = 0;
    template <typename T> T* take(size_t count) {
        off = (off + 255) & ~size_t(255);
        T* p = reinterpret_cast<T*>(base + off);
        off += count * sizeof(T);
        return p;
    }
};

template <typename R> class Davidson {
  public:
    using T = cplx_t<R>;

    Davidson(Context& c, int nb, int expansion, DevBuf& mem, DevBuf& dmem)
        : c_(c), st_(c.stream), npw_(c.band_npw()), nb_(nb) {
        maxn_ = std::max(std::min(expansion * nb, npw_), nb);  // davidson.hpp:401-404
        us_ = c.kp.has_q;
        gamma_ = c.gamma_half > 0;
        const size_t vecs = (size_t)npw_ * maxn_;
        const size_t mm = (size_t)maxn_ * maxn_;
        // Gamma-only: band pairs packed into full-sphere vectors for H and S
        const size_t gvecs = gamma_ ? (size_t)c.kp.npw * ((maxn_ + 1) / 2) : 0;
        size_t bytes = (us_ ? 3 : 2) * vecs * sizeof(T) + (size_t)npw_ * maxn_ * sizeof(T)  // V, HV, [SV], tmp
                       + 2 * gvecs * sizeof(T)                                            // packed pairs
                       + 2 * mm * sizeof(double2)                                 // Hs, Ss
                       + 3 * mm * sizeof(double2)                                 // evec, gram64, uinv64
                       + 5 * mm * sizeof(T)                                       // evecR, cpack, cneg, coef, uinvR
                       + 4 * (size_t)maxn_ * sizeof(double) + (size_t)maxn_ * sizeof(int) + 512 +
                       (size_t)npw_ * sizeof(double) + 32 * 256;
        mem.reserve(&c, bytes);
        Carve cv{mem.as<char>()};
        V_ = cv.take<T>(vecs);
        HV_ = cv.take<T>(vecs);
        // S|V> has a buffer of its own only when S is not the identity
        // (subspace_manager/serial.hpp:54-60 aliases it otherwise)
        SV_ = us_ ? cv.take<T>(vecs) : V_;
        if (gamma_) {
            gphi_ = cv.take<T>(gvecs);
            ghphi_ = cv.take<T>(gvecs);
        }
        tmp_ = cv.take<T>((size_t)npw_ * maxn_);
        Hs_ = cv.take<double2>(mm);
        Ss_ = cv.take<double2>(mm);
        evec_ = cv.take<double2>(mm);
        gram_ = cv.take<double2>(mm);
        uinv_ = cv.take<double2>(mm);
        evecR_ = cv.take<T>(mm);
        cpack_ = cv.take<T>(mm);
        cneg_ = cv.take<T>(mm);
        coef_ = cv.take<T>(mm);
        uinvR_ = cv.take<T>(mm);
        w_ = cv.take<double>(maxn_);
        eps_ = cv.take<double>(maxn_);
        norms_ = cv.take<double>(maxn_);
        idx_ = cv.take<int>(maxn_);
        dinfo_ = cv.take<int>(4);
        ke_ = c.kp.ke64.as<double>();
        dmem.reserve(&c, dense::hegv_scratch_bytes(maxn_) + dense::potrf_scratch_bytes(maxn_));
        dscratch_.base = dmem.as<char>();
        dscratch_.bytes = dmem.bytes;
        Q3B_CUDA(cudaMemsetAsync(Hs_, 0, mm * sizeof(double2), st_));
        Q3B_CUDA(cudaMemsetAsync(Ss_, 0, mm * sizeof(double2), st_));
    }

    int maxn() const { return maxn_; }
    T* V() { return V_; }
    T* scratch() { return tmp_; }

    // ------------------------------------------------------------ GEMM
    void gemm(bool conj, int M, int N, int K, T alpha, const T* A, long lda, const T* B, long ldb, T beta,
              T* C, long ldc) {
        GemmWorkspace ws = c_.gemm_ws(conj ? cgemm_workspace_bytes<R>(M, N, K) : 0);
        cgemm<R>(st_, conj, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc, ws);
    }
    // inner products A^H B (K = npw): on a Gamma-only k-point the real
    // half-sphere form
    void inner(int M, int N, const T* A, const T* B, T* C, long ldc) {
        gemm(true, M, N, npw_, one(), A, npw_, B, npw_, zero(), C, ldc);
        if (gamma_) {
            gamma_inner_fix<T><<<grid_for((long)M * N), 256, 0, st_>>>(M, N, A, npw_, B, npw_, C, ldc);
            Q3B_LAUNCH_CHECK();
        }
    }
    static T one() { return mk(R(1), R(0)); }
    static T zero() { return mk(R(0), R(0)); }
    static T mone() { return mk(R(-1), R(0)); }

    // --------------------------------------- orthogonalize_batch (serial.hpp:41-553)
    int orthogonalize(int start, int ncand) {
        if (ncand == 0) return 0;
        T* Tc = V_ + (size_t)start * npw_;
        T* STc = SV_ + (size_t)start * npw_;
        if (gamma_) {
            gamma_real_origin<T><<<1, 256, 0, st_>>>(ncand, Tc, npw_);
            Q3B_LAUNCH_CHECK();
        }
        apply_overlap(start, ncand);                                    // serial.hpp:62-68
        if (start > 0) {
            // C = V^H (S T); T -= V C, and S T -= (S V) C when S|V> is its own buffer
            inner(start, ncand, V_, STc, coef_, start);
            gemm(false, npw_, ncand, start, mone(), V_, npw_, coef_, start, one(), Tc, npw_);
            if (us_) gemm(false, npw_, ncand, start, mone(), SV_, npw_, coef_, start, one(), STc, npw_);
        }
        // Cholesky QR, the Gram matrix T^H S T and its factor in FP64
        inner(ncand, ncand, Tc, STc, coef_, ncand);
        widen(ncand, ncand, coef_, ncand, gram_, ncand);
        const int info = cholesky_inverse(ncand);
        if (info == 0) {
            const T* U = narrowed(ncand, ncand, uinv_, ncand, uinvR_);
            gemm(false, npw_, ncand, ncand, one(), Tc, npw_, U, ncand, zero(), tmp_, npw_);
            Q3B_CUDA(cudaMemcpyAsync(Tc, tmp_, (size_t)npw_ * ncand * sizeof(T), cudaMemcpyDeviceToDevice, st_));
            if (us_) {
                gemm(false, npw_, ncand, ncand, one(), STc, npw_, U, ncand, zero(), tmp_, npw_);
                Q3B_CUDA(cudaMemcpyAsync(STc, tmp_, (size_t)npw_ * ncand * sizeof(T), cudaMemcpyDeviceToDevice,
                                         st_));
            }
            return ncand;
        }
        if (us_) return mgs_overlap(start, ncand);
        // modified Gram-Schmidt fallback (serial.hpp:370-552)
        int accepted = 0;
        for (int cidx = 0; cidx < ncand; ++cidx) {
            const int src = start + cidx, dst = start + accepted;
            T* v = V_ + (size_t)dst * npw_;
            if (dst != src)
                Q3B_CUDA(cudaMemcpyAsync(v, V_ + (size_t)src * npw_, npw_ * sizeof(T), cudaMemcpyDeviceToDevice, st_));
            const int nex = dst - start;
            if (nex > 0) {
                inner(nex, 1, Tc, v, coef_, nex);
                gemm(false, npw_, 1, nex, mone(), Tc, npw_, coef_, nex, one(), v, npw_);
            }
            column_norms<R><<<1, 256, 0, st_>>>(npw_, v, norms_, gamma_ ? 1 : 0);
            Q3B_LAUNCH_CHECK();
            double* hb = static_cast<double*>(host_readback(sizeof(double)));
            Q3B_CUDA(cudaMemcpyAsync(hb, norms_, sizeof(double), cudaMemcpyDeviceToHost, st_));
            Q3B_CUDA(cudaStreamSynchronize(st_));
            const double nrm = hb[0];
            const double n2 = nrm * nrm;
            if (n2 > kNormThreshold) {
                scale_vector<R><<<grid_for(npw_), 256, 0, st_>>>(npw_, v, 1.0 / nrm);
                Q3B_LAUNCH_CHECK();
                ++accepted;
            }
        }
        return accepted;
    }

    // gram_ = U^H U and uinv_ = U^{-1} (ld n); LAPACK's potrf info (0: positive definite)
    int cholesky_inverse(int n) {
        if (n <= dense::block_max_order() && dense::chol_inverse_block_fits(n)) {
            dense::chol_inverse_block(st_, n, gram_, n, uinv_, dinfo_);
            int* h = static_cast<int*>(host_readback(sizeof(int)));
            Q3B_CUDA(cudaMemcpyAsync(h, dinfo_, sizeof(int), cudaMemcpyDeviceToHost, st_));
            Q3B_CUDA(cudaStreamSynchronize(st_));
            return h[0];
        }
        dscratch_.used = 0;
        const int info = dense::potrf(st_, n, gram_, n, dscratch_);
        if (info == 0) {
            // the same scratch still holds the diagonal-block inverses potrf left
            dscratch_.used = 0;
            dense::trtri_after_potrf(st_, n, gram_, n, uinv_, dscratch_);
        }
        return info;
    }

    // ------------------------------------ update_subspace_matrices (serial.hpp:555-678)
    void update(int start, int nnew, int total) {
        if (nnew <= 0) return;
        const T* Hn = HV_ + (size_t)start * npw_;
        const T* Sn = SV_ + (size_t)start * npw_;
        if constexpr (std::is_same<R, double>::value) {
            inner(total, nnew, V_, Hn, Hs_ + (size_t)start * maxn_, maxn_);
            inner(total, nnew, V_, Sn, Ss_ + (size_t)start * maxn_, maxn_);
        } else {
            inner(total, nnew, V_, Hn, coef_, total);
            widen(total, nnew, coef_, total, Hs_ + (size_t)start * maxn_, maxn_);
            inner(total, nnew, V_, Sn, coef_, total);
            widen(total, nnew, coef_, total, Ss_ + (size_t)start * maxn_, maxn_);
        }
    }

    // --------------------------------------- diagonalize_subspace (serial.hpp:680-756)
    // eigenvalues to w_ (and, when `publish`, to the host copy the loop's
    // convergence test reads), eigenvectors (first nvec) to evec_ (ld n).  The
    // collapse diagonalises for its rotation only and does not publish, as the
    // reference keeps those eigenvalues local (serial.hpp:838).
    int diagonalize(int n, const double2* H, const double2* S, int ld, bool publish = true) {
        dscratch_.used = 0;
        const int nvec = std::min(nb_, n);
        if (c_.batcher && EigenBatcher::takes(n, nvec)) {
            // in a batch with the other workers' solves (batcher.cuh)
            double2* work = dscratch_.take<double2>(dense::hegv_block_work_elems(n));
            int* info = dscratch_.take<int>(1);
            wread_.assign(n, 0.0);
            const int st = c_.batcher->solve(dense::BlockProblem{n, ld, nvec, H, S, w_, evec_, work, info}, st_,
                                              wread_.data());
            if (st == 0 && publish) whost_.assign(wread_.begin(), wread_.begin() + nvec);
            return st;
        }
        GemmWorkspace gws = c_.gemm_ws(cgemm_workspace_bytes<double>(n, n, n));
        // the lowest nvec eigenvalues come back in the solve's own status read
        wread_.assign(n, 0.0);
        const int info = dense::hegv(st_, n, H, S, ld, w_, evec_, nvec, dscratch_, gws, &c_.hegv_graphs,
                                     wread_.data());
        if (info == 0 && publish) whost_.assign(wread_.begin(), wread_.begin() + nvec);
        return info;
    }

    // ------------------------------------ build_correction_vectors (serial.hpp:995-1132)
    int corrections(int basis, const std::vector<int>& bands, int maxcand) {
        int ncand = std::min<int>(static_cast<int>(bands.size()), maxcand);
        if (ncand <= 0) return 0;
        upload_async(idx_, bands.data(), ncand * sizeof(int), st_);
        pack_coefficients<R><<<grid_for((long)basis * ncand), 256, 0, st_>>>(basis, ncand, evec_, idx_, w_,
                                                                             cpack_, cneg_, eps_);
        Q3B_LAUNCH_CHECK();
        T* Rc = V_ + (size_t)basis * npw_;
        gemm(false, npw_, ncand, basis, one(), SV_, npw_, cneg_, basis, zero(), Rc, npw_);  // -(SV)c eps
        gemm(false, npw_, ncand, basis, one(), HV_, npw_, cpack_, basis, one(), Rc, npw_);  // + (HV)c
        precondition_kernel<R><<<grid_for((long)npw_ * ncand), 256, 0, st_>>>(npw_, ncand, ke_, eps_, Rc);
        Q3B_LAUNCH_CHECK();
        return ncand;
    }

    // rotate V and HV onto the first nb eigenvectors of the last diagonalisation
    void rotate(int basis) {
        const T* C = narrowed(basis, nb_, evec_, basis, evecR_);
        const size_t bytes = (size_t)npw_ * nb_ * sizeof(T);
        gemm(false, npw_, nb_, basis, one(), V_, npw_, C, basis, zero(), tmp_, npw_);
        Q3B_CUDA(cudaMemcpyAsync(V_, tmp_, bytes, cudaMemcpyDeviceToDevice, st_));
        gemm(false, npw_, nb_, basis, one(), HV_, npw_, C, basis, zero(), tmp_, npw_);
        Q3B_CUDA(cudaMemcpyAsync(HV_, tmp_, bytes, cudaMemcpyDeviceToDevice, st_));
        if (us_) {
            gemm(false, npw_, nb_, basis, one(), SV_, npw_, C, basis, zero(), tmp_, npw_);
            Q3B_CUDA(cudaMemcpyAsync(SV_, tmp_, bytes, cudaMemcpyDeviceToDevice, st_));
        }
    }

    // --------------------------------------- collapse_subspace (serial.hpp:825-945)
    int collapse(int basis, bool from_held) {
        int info = -1;
        if (from_held) info = diagonalize(basis, Hs_, Ss_, maxn_, false);
        if (info != 0) {
            // rebuild the subspace from the vectors
            T* h = coef_;
            inner(basis, basis, V_, HV_, h, basis);
            widen(basis, basis, h, basis, gram_, basis);
            inner(basis, basis, V_, SV_, h, basis);
            widen(basis, basis, h, basis, uinv_, basis);
            info = diagonalize(basis, gram_, uinv_, basis, false);
            if (info != 0) throw Status(Q3B_ERR_LINALG, "subspace eigensolver failed in the collapse");
        }
        rotate(basis);
        const size_t mm = (size_t)maxn_ * maxn_;
        Q3B_CUDA(cudaMemsetAsync(Hs_, 0, mm * sizeof(double2), st_));
        Q3B_CUDA(cudaMemsetAsync(Ss_, 0, mm * sizeof(double2), st_));
        update(0, nb_, nb_);
        // The next iteration's subspace is the nb Ritz vectors just formed: its
        // matrices are diag(w) and the identity to rounding, so its eigenpairs
        // are these eigenvalues (left in w_[0, nb)) and unit vectors.
        // the collapse's eigenvalues were read back by its subspace solve
        collapse_w_.assign(wread_.begin(), wread_.begin() + nb_);
        reuse_collapse_ = true;
        return nb_;
    }

    // psi = V c[:, :nb] into out (npw x nb), the FP64 residual norms ||HVc - eps Vc||
    void extract(int basis, T* out, double* resid_max) {
        const T* C = narrowed(basis, nb_, evec_, basis, evecR_);
        gemm(false, npw_, nb_, basis, one(), V_, npw_, C, basis, zero(), out, npw_);
        if (resid_max) {
            const std::vector<double> r = residual_norms(basis);
            *resid_max = *std::max_element(r.begin(), r.end());
        }
    }

    // ||(HV) c_b - eps_b (SV) c_b|| of the current Ritz pairs, every band (on the host)
    std::vector<double> residual_norms(int basis) {
        std::vector<int> all(nb_);
        std::iota(all.begin(), all.end(), 0);
        upload_async(idx_, all.data(), nb_ * sizeof(int), st_);
        pack_coefficients<R><<<grid_for((long)basis * nb_), 256, 0, st_>>>(basis, nb_, evec_, idx_, w_, cpack_,
                                                                           cneg_, eps_);
        Q3B_LAUNCH_CHECK();
        gemm(false, npw_, nb_, basis, one(), SV_, npw_, cneg_, basis, zero(), tmp_, npw_);
        gemm(false, npw_, nb_, basis, one(), HV_, npw_, cpack_, basis, one(), tmp_, npw_);
        column_norms<R><<<nb_, 256, 0, st_>>>(npw_, tmp_, norms_, gamma_ ? 1 : 0);
        Q3B_LAUNCH_CHECK();
        double* h = static_cast<double*>(host_readback(nb_ * sizeof(double)));
        Q3B_CUDA(cudaMemcpyAsync(h, norms_, nb_ * sizeof(double), cudaMemcpyDeviceToHost, st_));
        Q3B_CUDA(cudaStreamSynchronize(st_));
        return std::vector<double>(h, h + nb_);
    }

    // Residual gate of the mixed solve's refinement (0: off, the reference's test
    // alone): when every band passes the eigenvalue-change test, the occupied bands
    // whose squared residual norm exceeds the gate stay unconverged.  A band's
    // eigenvalue error is at most about ||r||^2 / (its gap to the rest of the
    // spectrum), while a slowly converging band can change by less than the
    // tolerance per iteration and still be far from its limit.
    void set_residual_gate(double g) { resid_gate_ = g; }

    // S|V> for columns [first, first+count): V + beta Q beta^H V (the
    // ultrasoft operator, overlap/pseudopotential/ultrasoft/init.hpp:189-345)
    void apply_overlap(int first, int count) {
        if (!us_ || count <= 0) return;
        const T* v = V_ + (size_t)first * npw_;
        T* sv = SV_ + (size_t)first * npw_;
        const int nfull = c_.kp.npw;
        // on a Gamma-only k-point the band pairs go through S on the full sphere
        const int nv = gamma_ ? (count + 1) / 2 : count;
        const T* in = v;
        T* out = sv;
        if (gamma_) {
            gamma_pack<T><<<gamma_blocks((long)npw_ * nv), 256, 0, st_>>>(npw_, count, v, npw_, gphi_, nfull);
            Q3B_LAUNCH_CHECK();
            in = gphi_;
            out = ghphi_;
        }
        const int len = gamma_ ? nfull : npw_;
        Q3B_CUDA(cudaMemcpyAsync(out, in, (size_t)len * nv * sizeof(T), cudaMemcpyDeviceToDevice, st_));
        const int P = c_.kp.nproj;
        const size_t pb = (size_t)P * nv * sizeof(T);
        c_.ws_bm.reserve(&c_, pb);
        c_.ws_bp.reserve(&c_, pb);
        GemmWorkspace ws = c_.gemm_ws(cgemm_workspace_bytes<R>(P, nv, len));
        apply_nonlocal<R>(st_, c_.overlap<R>(), len, nv, in, len, out, len, c_.ws_bm.as<T>(), c_.ws_bp.as<T>(), ws);
        if (gamma_) {
            gamma_unpack<T><<<gamma_blocks((long)npw_ * nv), 256, 0, st_>>>(npw_, count, ghphi_, nfull, sv, npw_);
            Q3B_LAUNCH_CHECK();
        }
    }

    // modified Gram-Schmidt in the S metric (the Cholesky-QR fallback,
    // serial.hpp:370-552, with S|v> carried beside every v)
    int mgs_overlap(int start, int ncand) {
        int accepted = 0;
        for (int cidx = 0; cidx < ncand; ++cidx) {
            const int src = start + cidx, dst = start + accepted;
            T* v = V_ + (size_t)dst * npw_;
            T* sv = SV_ + (size_t)dst * npw_;
            if (dst != src) {
                Q3B_CUDA(cudaMemcpyAsync(v, V_ + (size_t)src * npw_, npw_ * sizeof(T), cudaMemcpyDeviceToDevice, st_));
                Q3B_CUDA(cudaMemcpyAsync(sv, SV_ + (size_t)src * npw_, npw_ * sizeof(T), cudaMemcpyDeviceToDevice,
                                         st_));
            }
            const int nex = dst - start;
            if (nex > 0) {
                const T* B = V_ + (size_t)start * npw_;
                const T* SB = SV_ + (size_t)start * npw_;
                inner(nex, 1, B, sv, coef_, nex);
                gemm(false, npw_, 1, nex, mone(), B, npw_, coef_, nex, one(), v, npw_);
                gemm(false, npw_, 1, nex, mone(), SB, npw_, coef_, nex, one(), sv, npw_);
            }
            // ||v||_S^2 = Re v^H S v
            inner(1, 1, v, sv, coef_, 1);
            T* hb = static_cast<T*>(host_readback(sizeof(T)));
            Q3B_CUDA(cudaMemcpyAsync(hb, coef_, sizeof(T), cudaMemcpyDeviceToHost, st_));
            Q3B_CUDA(cudaStreamSynchronize(st_));
            const double n2 = static_cast<double>(hb[0].x);
            if (n2 > kNormThreshold) {
                const double inv = 1.0 / std::sqrt(n2);
                scale_vector<R><<<grid_for(npw_), 256, 0, st_>>>(npw_, v, inv);
                Q3B_LAUNCH_CHECK();
                scale_vector<R><<<grid_for(npw_), 256, 0, st_>>>(npw_, sv, inv);
                Q3B_LAUNCH_CHECK();
                ++accepted;
            }
        }
        return accepted;
    }

    void apply(int first, int count) {
        if (count <= 0) return;
        if (gamma_) {
            // two bands per full-sphere vector (hamiltonian_applicator/serial.hpp:283-418)
            const int nfull = c_.kp.npw, np = (count + 1) / 2;
            gamma_pack<T><<<gamma_blocks((long)npw_ * np), 256, 0, st_>>>(npw_, count, V_ + (size_t)first * npw_,
                                                                         npw_, gphi_, nfull);
            Q3B_LAUNCH_CHECK();
            c_.apply_h<R>(gphi_, nfull, ghphi_, nfull, np);
            gamma_unpack<T><<<gamma_blocks((long)npw_ * np), 256, 0, st_>>>(npw_, count, ghphi_, nfull,
                                                                           HV_ + (size_t)first * npw_, npw_);
            Q3B_LAUNCH_CHECK();
        } else {
            c_.apply_h<R>(V_ + (size_t)first * npw_, npw_, HV_ + (size_t)first * npw_, npw_, count);
        }
        happly_ += count;
    }

    std::vector<double> subspace_diagonal(int n) {
        double2* d = static_cast<double2*>(host_readback(n * sizeof(double2)));
        Q3B_CUDA(cudaMemcpy2DAsync(d, sizeof(double2), Hs_, (maxn_ + 1) * sizeof(double2),
                                   sizeof(double2), n, cudaMemcpyDeviceToHost, st_));
        Q3B_CUDA(cudaStreamSynchronize(st_));
        std::vector<double> r(n);
        for (int i = 0; i < n; ++i) r[i] = d[i].x;
        return r;
    }

    // The solve of davidson.hpp:324-841 on bands already in V[:, :nb].
    // Returns the eigenvalues; the eigenvectors go to `out`.
    struct Result {
        std::vector<double> eig;
        int iterations = 0, unconverged = 0, collapses = 0;
        double resid = 0.0;
        bool stagnated = false;
    };

    // stagnate: stop (with the Ritz pairs of this iteration) once the largest
    // eigenvalue change has stopped halving for three iterations while below
    // kStallBelow -- near the FP32 resolution of the eigenvalues, where the FP32
    // phase of the mixed solve can go no further -- or once the sum of the
    // occupied Ritz values has set no new low for kFlatIterations iterations.
    // In exact arithmetic that sum never rises (the Ritz values fall as the
    // basis grows and are kept across a collapse), so a sum that stops falling
    // is the FP32 H|psi> accuracy floor (about 1e-4 Ry on the 80^3 and 108^3
    // cells), below which further FP32 iterations leave the eigenvalues as
    // they are.
    Result solve(int seeded, const std::vector<double>& stored, double tol, int max_it, int occupied,
                 T* out, bool want_resid, double* stage_ms = nullptr, bool stagnate = false) {
        Result res;
        StageClock clk{st_, stage_ms};
        reuse_collapse_ = false;
        clk.start();
        int basis = orthogonalize(0, seeded);                            // :1000-1045
        apply(0, basis);
        if (basis < nb_) {                                                // :1047-1101
            const std::vector<double>& ke = c_.kp.ke_host;
            std::vector<int> order(npw_);
            std::iota(order.begin(), order.end(), 0);
            std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ke[a] < ke[b]; });
            const int start = basis;
            std::vector<int> gsel;
            for (int band = start; band < nb_; ++band) gsel.push_back(order[band]);
            const int ncand = static_cast<int>(gsel.size());
            upload_async(idx_, gsel.data(), ncand * sizeof(int), st_);
            unit_vectors<R><<<grid_for((long)npw_ * ncand), 256, 0, st_>>>(npw_, ncand, idx_,
                                                                           V_ + (size_t)basis * npw_);
            Q3B_LAUNCH_CHECK();
            basis += orthogonalize(basis, ncand);
            apply(start, basis - start);
        }
        if (basis < nb_)
            throw Status(Q3B_ERR_LINALG, "could not build " + std::to_string(nb_) +
                                             " independent starting vectors");
        update(0, basis, basis);                                          // :459-469
        clk.stop(SEED);
        std::vector<double> prev(nb_, 0.0);
        std::vector<double> history;
        bool have_stored = false;
        for (double e : stored) have_stored = have_stored || e != 0.0;
        if (have_stored) {
            prev = stored;                                                // :483-487
        } else {
            std::vector<double> dg = subspace_diagonal(std::min(nb_, basis));
            std::copy(dg.begin(), dg.end(), prev.begin());                // :488-494
        }
        const double empty_tol = std::max(kEmptyRelax * tol, kEmptyFloor);
        double low = 0.0;
        int since_low = 0;
        std::vector<double> sums;  // the occupied Ritz values' sum, per iteration
        for (int it = 0; it < max_it; ++it) {                            // :498
            int info = 0;
            if (reuse_collapse_ && basis == nb_) {
                whost_ = collapse_w_;
                set_identity<<<grid_for((long)nb_ * nb_), 256, 0, st_>>>(nb_, evec_);
                Q3B_LAUNCH_CHECK();
            } else {
                info = diagonalize(basis, Hs_, Ss_, maxn_);
            }
            reuse_collapse_ = false;
            if (info != 0 && basis > nb_) {                               // :521-590
                basis = collapse(basis, false);
                ++res.collapses;
                info = diagonalize(basis, Hs_, Ss_, maxn_);
                if (info != 0) {
                    whost_.assign(std::max(basis, nb_), 0.0);
                    std::copy(prev.begin(), prev.end(), whost_.begin());
                }
            } else if (info != 0) {
                throw Status(Q3B_ERR_LINALG, "subspace eigensolver failed");
            }
            clk.stop(DIAG);
            ++res.iterations;
            if (history_) history_->insert(history_->end(), whost_.begin(), whost_.begin() + nb_);
            std::vector<int> unconv;
            double maxchange = 0.0;
            for (int b = 0; b < nb_; ++b) {                               // :615-629
                const double change = std::fabs(whost_[b] - prev[b]);
                maxchange = std::max(maxchange, change);
                const double tb = b < occupied ? tol : empty_tol;
                if (!(it != 0 && change < tb)) unconv.push_back(b);
            }
            res.unconverged = static_cast<int>(unconv.size());
            if (it != 0) history.push_back(maxchange);
            const size_t h = history.size();
            double occ_sum = 0.0, occ_abs = 0.0;
            for (int b = 0; b < occupied; ++b) {
                occ_sum += whost_[b];
                occ_abs += std::fabs(whost_[b]);
            }
            sums.push_back(occ_sum);
            const bool crawling = sums.size() > (size_t)kCrawlWindow &&
                                  sums[sums.size() - 1 - kCrawlWindow] - occ_sum < kCrawlRelative * occ_abs;
            if (it == 0 || occ_sum < low) {
                low = occ_sum;
                since_low = 0;
            } else {
                ++since_low;
            }
            const bool stalled = stagnate && ((h >= 4 && history[h - 1] < kStallBelow &&
                                               history[h - 1] > 0.5 * history[h - 4]) ||
                                              since_low >= kFlatIterations || crawling);
            if (unconv.empty() && !stalled && resid_gate_ > 0.0) {
                const std::vector<double> r = residual_norms(basis);
                for (int b = 0; b < occupied; ++b)
                    if (r[b] * r[b] > resid_gate_) unconv.push_back(b);
                res.unconverged = static_cast<int>(unconv.size());
            }
            if (unconv.empty() || stalled) {                              // :649-668
                res.stagnated = stalled && !unconv.empty();
                extract(basis, out, want_resid ? &res.resid : nullptr);
                clk.stop(EXTRACT);
                res.eig.assign(whost_.begin(), whost_.begin() + nb_);
                return res;
            }
            const int ncand = corrections(basis, unconv, maxn_ - basis);  // :689-703
            clk.stop(CORR);
            const int acc = orthogonalize(basis, ncand);                  // :705-712
            clk.stop(ORTHO);
            apply(basis, acc);                                            // :728-738
            clk.stop(HAPPLY);
            const int old = basis;
            basis += acc;
            if (acc > 0) update(old, acc, basis);                         // :743-760
            clk.stop(UPDATE);
            if (basis >= maxn_) {                                         // :763-808
                basis = collapse(basis, true);
                ++res.collapses;
            }
            clk.stop(COLLAPSE);
            for (int b = 0; b < nb_; ++b) prev[b] = whost_[b];
        }
        int info = 0;                                                     // :816-840
        if (reuse_collapse_ && basis == nb_) {
            whost_ = collapse_w_;
            set_identity<<<grid_for((long)nb_ * nb_), 256, 0, st_>>>(nb_, evec_);
            Q3B_LAUNCH_CHECK();
        } else {
            info = diagonalize(basis, Hs_, Ss_, maxn_);
        }
        reuse_collapse_ = false;
        if (info != 0) throw Status(Q3B_ERR_LINALG, "subspace eigensolver failed at exit");
        clk.stop(DIAG);
        extract(basis, out, want_resid ? &res.resid : nullptr);
        clk.stop(EXTRACT);
        res.eig.assign(whost_.begin(), whost_.begin() + nb_);
        return res;
    }

    int happly() const { return happly_; }

    // keep the Ritz values of every iteration (nb per iteration) in *h
    void record_history(std::vector<double>* h) { history_ = h; }

  private:
    void widen(int M, int N, const T* src, int lds, double2* dst, int ldd) {
        widen_block<R><<<grid_for((long)M * N), 256, 0, st_>>>(M, N, src, lds, dst, ldd);
        Q3B_LAUNCH_CHECK();
    }
    const T* narrowed(int M, int N, const double2* src, int lds, T* buf) {
        if constexpr (std::is_same<R, double>::value) {
            (void)M;
            (void)N;
            (void)lds;
            (void)buf;
            return src;
        } else {
            narrow_block<R><<<grid_for((long)M * N), 256, 0, st_>>>(M, N, src, lds, buf, M);
            Q3B_LAUNCH_CHECK();
            return buf;
        }
    }

    Context& c_;
    cudaStream_t st_;
    int npw_, nb_, maxn_ = 0;
    int happly_ = 0;
    T *V_, *HV_, *SV_, *tmp_, *evecR_, *cpack_, *cneg_, *coef_, *uinvR_;
    T *gphi_ = nullptr, *ghphi_ = nullptr;  // packed band pairs (Gamma-only)
    bool us_ = false;     // S is not the identity (ultrasoft overlap blocks set)
    bool gamma_ = false;  // half-sphere vectors of a Gamma-only k-point
    double2 *Hs_, *Ss_, *evec_, *gram_, *uinv_;
    double *w_, *eps_, *norms_;
    int* idx_;
    int* dinfo_ = nullptr;  // status word of the block Cholesky
    const double* ke_;
    dense::Scratch dscratch_;
    std::vector<double> whost_;
    std::vector<double>* history_ = nullptr;
    std::vector<double> collapse_w_;
    std::vector<double> wread_;  // eigenvalues of the last subspace solve, on the host
    bool reuse_collapse_ = false;
    double resid_gate_ = 0.0;
};

}  // namespace

int mixed_bands(int nb, int npw) { return std::min(npw, nb + std::max(2, (nb + 7) / 8)); }

// The basis factor of the mixed solve's FP32 phase: a larger basis cuts that
// phase's iterations (config 1: 94 -> 36 at factor 4), and with them its
// subspace eigensolves, which both precisions pay once per iteration.  The
// FP64 path and the mixed solve's FP64 refinement keep the reference's factor.
int basis_factor(const q3b_davidson_opts& o, int nb, int npw) {
    if (o.precision != Q3B_MIXED) return o.basis_expansion_factor;
    int factor = o.mixed_expansion_factor;
    if (factor <= 0) {
        factor = o.basis_expansion_factor;
        for (int f : {4, 3})
            if (f > factor && dense::order_supported(std::min(f * mixed_bands(nb, npw), npw))) {
                factor = f;
                break;
            }
    }
    if (factor < 2) throw Status(Q3B_ERR_INVALID, "mixed_expansion_factor must be >= 2");
    return factor;
}

void davidson_solve(Context& c, double2* bands_dev, double* eig_host, int nb, const q3b_davidson_opts& o,
                    q3b_davidson_stats* stats) {
    c.require_ready();
    const int npw = c.band_npw();
    if (nb <= 0 || nb > npw) throw Status(Q3B_ERR_INVALID, "band count must be in [1, npw]");
    if (o.basis_expansion_factor < 2) throw Status(Q3B_ERR_INVALID, "basis_expansion_factor must be >= 2");
    if (!(o.tolerance > 0.0)) throw Status(Q3B_ERR_INVALID, "tolerance must be positive");
    const auto t0 = std::chrono::steady_clock::now();
    const int occupied = o.occupied_bands > 0 ? std::min(o.occupied_bands, nb) : nb;
    std::vector<double> stored(eig_host, eig_host + nb);
    q3b_davidson_stats s{};
    const size_t band_bytes = (size_t)npw * nb * sizeof(double2);
    if (o.history_rows < 0 || (o.history_rows > 0 && !o.eigenvalue_history))
        throw Status(Q3B_ERR_INVALID, "eigenvalue_history needs history_rows >= 0 and a buffer");
    std::vector<double> hist;
    std::vector<double>* rec = o.history_rows > 0 ? &hist : nullptr;
    size_t hist_width = (size_t)nb;
    if (o.precision == Q3B_FP64) {
        Davidson<double> dv(c, nb, o.basis_expansion_factor, c.ws_solver, c.ws_dense);
        dv.record_history(rec);
        Q3B_CUDA(cudaMemcpyAsync(dv.V(), bands_dev, band_bytes, cudaMemcpyDeviceToDevice, c.stream));
        auto r = dv.solve(nb, stored, o.tolerance, std::max(1, o.max_iterations), occupied, bands_dev, true,
                          o.profile_stages ? s.stage_ms : nullptr);
        std::copy(r.eig.begin(), r.eig.end(), eig_host);
        s.iterations = s.fp64_iterations = r.iterations;
        s.h_applications = dv.happly();
        s.unconverged = r.unconverged;
        s.collapses = r.collapses;
        s.max_residual_norm = r.resid;
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
        s.fp64_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    } else if (o.precision == Q3B_MIXED) {
        const int factor = basis_factor(o, nb, npw);
        // With the larger basis, both phases solve for nbi = nb + a few buffer bands,
        // held to the loose tolerance of empty bands; the lowest nb are returned.
        // Without them the FP32 phase, which ends sooner with the larger basis, hands
        // over a block whose top band (its gap to the first band outside the block
        // is small) converges so slowly in the refinement that its eigenvalue change
        // can drop below the tolerance while it is still 1e-8 to 1e-7 Ry from its
        // limit.  At the reference's factor the solve is the plain two-phase one.
        const int nbi = factor > o.basis_expansion_factor ? mixed_bands(nb, npw) : nb;
        c.ws_mixed.reserve(&c, (size_t)npw * nbi * sizeof(double2));
        double2* mix = c.ws_mixed.as<double2>();
        std::vector<double> stored_i(nbi, 0.0);
        std::copy(stored.begin(), stored.end(), stored_i.begin());
        // FP32 phase to the loose tolerance
        std::vector<double> eig32;
        int it32 = 0, h32 = 0, col32 = 0;
        {
            Davidson<float> dv(c, nbi, factor, c.ws_solver, c.ws_dense);
            dv.record_history(rec);
            convert<double, float>(c.stream, (long)npw * nb, bands_dev, dv.V());
            const double tol32 = o.mixed_tolerance > 0.0 ? o.mixed_tolerance : 1e-6;
            auto r = dv.solve(nb, stored_i, std::max(tol32, o.tolerance), std::max(1, o.max_iterations),
                              occupied, dv.scratch(), false, o.profile_stages ? s.stage_ms : nullptr, true);
            // widen the FP32 Ritz vectors for the refinement
            convert<float, double>(c.stream, (long)npw * nbi, dv.scratch(), mix);
            eig32 = r.eig;
            it32 = r.iterations;
            h32 = dv.happly();
            col32 = r.collapses;
        }
        // FP64 refinement sweeps from the FP32 Ritz pairs, at the reference's factor
        const auto t64 = std::chrono::steady_clock::now();
        Davidson<double> dv(c, nbi, o.basis_expansion_factor, c.ws_solver, c.ws_dense);
        dv.record_history(rec);
        // a tenth of the tolerance: an eigenvalue within about tol / (10 gap) of its limit
        dv.set_residual_gate(0.1 * o.tolerance);
        Q3B_CUDA(cudaMemcpyAsync(dv.V(), mix, (size_t)npw * nbi * sizeof(double2), cudaMemcpyDeviceToDevice,
                                 c.stream));
        const int sweeps = o.refine_sweeps > 0 ? o.refine_sweeps : std::max(1, o.max_iterations);
        auto r = dv.solve(nbi, eig32, o.tolerance, sweeps, occupied, mix, true,
                          o.profile_stages ? s.stage_ms : nullptr);
        Q3B_CUDA(cudaMemcpyAsync(bands_dev, mix, band_bytes, cudaMemcpyDeviceToDevice, c.stream));
        std::copy(r.eig.begin(), r.eig.begin() + nb, eig_host);
        s.iterations = it32 + r.iterations;
        s.fp64_iterations = r.iterations;
        s.h_applications = h32 + dv.happly();
        s.unconverged = r.unconverged;
        s.collapses = col32 + r.collapses;
        s.max_residual_norm = r.resid;
        Q3B_CUDA(cudaStreamSynchronize(c.stream));
        s.fp64_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t64).count();
        hist_width = nbi;
    } else {
        throw Status(Q3B_ERR_INVALID, "unknown precision");
    }
    Q3B_CUDA(cudaStreamSynchronize(c.stream));
    tc::check_error(c.stream);
    s.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rec) {
        // rows of hist_width values (the mixed solve's buffer bands after the nb)
        const size_t rows = std::min(hist.size() / (size_t)hist_width, (size_t)o.history_rows);
        for (size_t i = 0; i < rows; ++i)
            std::copy(hist.begin() + i * hist_width, hist.begin() + i * hist_width + nb,
                      o.eigenvalue_history + i * nb);
    }
    if (stats) *stats = s;
}

}  // namespace q3b
