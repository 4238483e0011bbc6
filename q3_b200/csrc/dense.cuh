// FP64 small dense linear algebra on the device for the Davidson subspace
// (n <= a few thousand): Cholesky, triangular inverse, generalized Hermitian
// eigensolver.  These replace the reference's zpotrf / ztrsm / zhegv calls
// (subspace_manager/serial.hpp:334-339, subspace/serial.hpp:18-151).
#pragma once

#include <type_traits>

#include "cgemm.cuh"
#include "common.cuh"

namespace q3b {

class Context;

namespace dense {

struct Scratch {
    // grow-only device workspace handed out in slices
    char* base = nullptr;
    size_t bytes = 0;
    size_t used = 0;
    template <typename T> T* take(size_t count) {
        size_t off = (used + 255) & ~size_t(255);
        used = off + count * sizeof(T);
        if (used > bytes) throw std::runtime_error("dense scratch too small");
        return reinterpret_cast<T*>(base + off);
    }
};

// bytes of scratch hegv / potrf need for order n
size_t hegv_scratch_bytes(int n);
size_t potrf_scratch_bytes(int n);

// Upper Cholesky A = U^H U in place (upper triangle of A, ld lda).  Returns
// LAPACK's info: 0, or j+1 when the leading minor of order j+1 is not
// positive definite.  Synchronises the stream to read info.
int potrf(cudaStream_t st, int n, double2* A, int lda, Scratch& ws);

// Uinv = U^{-1} (n x n, ld n, zero below the diagonal) from the upper factor
// left in A by potrf.  ws must be handed in as it was handed to potrf (same
// base and `used`), so that the block inverses potrf stored are found again.
void trtri_after_potrf(cudaStream_t st, int n, const double2* A, int lda, double2* Uinv, Scratch& ws);

// Captured CUDA graphs of hegv's launch sequence (about 3 n/32 + 15 launches,
// no host synchronisation inside), keyed by every argument the sequence
// depends on, the last few kept.  A caller that solves problems of the same
// shape on the same buffers again and again (a Davidson loop) replays one
// graph per solve.  If the runtime refuses a capture, graphs are turned off
// and the launches are issued directly.
class HegvGraphs {
  public:
    HegvGraphs() = default;
    HegvGraphs(const HegvGraphs&) = delete;
    HegvGraphs& operator=(const HegvGraphs&) = delete;
    ~HegvGraphs();
    struct Key {
        int n, ld, nvec;
        const void *H, *S, *w, *Z, *ws, *gws;
        size_t ws_used, ws_bytes, gws_bytes;
        cudaStream_t st;
        bool operator==(const Key& o) const;
    };
    // the executable graph for `k`, capturing `issue` on the stream when new;
    // nullptr when graphs are off
    template <typename F> cudaGraphExec_t get(const Key& k, F&& issue);
    bool disabled = false;
    int captures = 0, replays = 0;

  private:
    struct Entry {
        Key key;
        cudaGraphExec_t exec;
        unsigned long long used;
        unsigned long long launches;  // kernels in the graph (the library's launch count)
        int seen;
    };
    static constexpr int kMax = 16;
    static constexpr int kCaptureAfter = 3;
    // below this order the sequence is short and the solves are often many
    // at once on other streams (serving), where instantiating graphs costs
    // more than the launches it saves
    static constexpr int kMinOrder = 256;
    Entry entries_[kMax];
    int count_ = 0;
    unsigned long long tick_ = 0;
    unsigned long long captured_launches_ = 0;
    cudaGraphExec_t capture(cudaStream_t st, void (*issue)(void*), void* ctx);
    Entry* find(const Key& k);
    void store(const Key& k, cudaGraphExec_t e);
};

// A key is only counted the first kCaptureAfter - 1 times it is seen (the
// caller launches directly); then it is captured and replayed from there on,
// so shapes that come and go (a Davidson basis that shrinks as bands
// converge) pay no capture and instantiation.
template <typename F> cudaGraphExec_t HegvGraphs::get(const Key& k, F&& issue) {
    if (disabled || k.n < kMinOrder) return nullptr;
    Entry* hit = find(k);
    if (hit && hit->exec) {
        ++replays;
        return hit->exec;
    }
    if (!hit) {
        store(k, nullptr);
        return nullptr;
    }
    if (++hit->seen < kCaptureAfter) return nullptr;
    using FF = std::remove_reference_t<F>;
    cudaGraphExec_t e = capture(k.st, [](void* f) { (*static_cast<FF*>(f))(); }, &issue);
    if (e) {
        hit->exec = e;
        hit->launches = captured_launches_;
        ++captures;
    }
    return e;
}

// Generalized Hermitian eigenproblem H c = w S c (itype 1; upper triangles of
// H and S, ld ld).  The lowest nvec eigenvalues ascending in w (device; all n
// when nvec is 0), their S-orthonormal eigenvectors in Z (n x nvec, ld n).  Returns 0, or n + j
// when S is not positive definite (zhegv's convention).  With `graphs`, the
// launch sequence is replayed from a captured graph when one matches.
// With w_host, the eigenvalues are also copied to the host in the same
// synchronisation that reads the status words.
int hegv(cudaStream_t st, int n, const double2* H, const double2* S, int ld, double* w, double2* Z,
         int nvec, Scratch& ws, const GemmWorkspace& gws, HegvGraphs* graphs = nullptr,
         double* w_host = nullptr);

// One problem of the block eigensolver (dense_block.cu): H c = w S c of order
// n <= 128 (upper triangles, ld ld), the lowest nvec eigenpairs into w and Z
// (n x nvec, ld n), status into *info (0, or n + j as hegv); `work` holds
// hegv_block_work_elems(n) complex values.  Device pointers.
struct BlockProblem {
    int n, ld, nvec;
    const double2* H;
    const double2* S;
    double* w;
    double2* Z;
    double2* work;
    int* info;
};
size_t hegv_block_smem(int n, int nvec);
// whether a block holds a problem of this order and vector count
bool hegv_block_fits(int n, int nvec);
size_t hegv_block_work_elems(int n);
// one problem, one block of 512 threads; no host synchronisation
void hegv_block(cudaStream_t st, const BlockProblem& p);
// `count` problems (descriptors in device memory, each checked by
// hegv_block_fits), one block each; smem = the largest hegv_block_smem of them
void hegv_block_many(cudaStream_t st, const BlockProblem* problems_dev, int count, size_t smem);

// G = U^H U (upper triangle of G, ld ldg) and Uinv = U^{-1} (n x n, ld n, zero
// below the diagonal) in one block; *info = 0, or k+1 when the leading minor of
// order k+1 is not positive definite (potrf's info).  No host synchronisation.
bool chol_inverse_block_fits(int n);
void chol_inverse_block(cudaStream_t st, int n, const double2* G, int ldg, double2* Uinv, int* info);

// hegv runs problems up to this order on one block (when hegv_block_fits);
// 0 keeps every order on the multi-kernel path
constexpr int kBlockOrderDefault = 64;
void set_block_max_order(int n);
int block_max_order();

// Whether hegv/heev take a problem of order n on the current device (the
// tridiagonalisation keeps its blocks' columns in shared memory).
bool order_supported(int n);

// Standard Hermitian eigenproblem of a full (both triangles) matrix A (n x n,
// ld n; read only).  The lowest nvec eigenvalues ascending in w (all n when
// nvec is 0), their eigenvectors in Z (ld n).
void heev(cudaStream_t st, int n, double2* A, double* w, double2* Z, int nvec, Scratch& ws,
          const GemmWorkspace& gws);

}  // namespace dense
}  // namespace q3b
