// FP64 small dense linear algebra on the device for the Davidson subspace
// (n <= a few thousand): Cholesky, triangular inverse, generalized Hermitian
// eigensolver.  These replace the reference's zpotrf / ztrsm / zhegv calls
// (subspace_manager/serial.hpp:334-339, subspace/serial.hpp:18-151).
#pragma once

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

// Generalized Hermitian eigenproblem H c = w S c (itype 1; upper triangles of
// H and S, ld ld).  Eigenvalues ascending in w (n, device), the first nvec
// S-orthonormal eigenvectors in Z (n x nvec, ld n).  Returns 0, or n + j
// when S is not positive definite (zhegv's convention).
int hegv(cudaStream_t st, int n, const double2* H, const double2* S, int ld, double* w, double2* Z,
         int nvec, Scratch& ws, const GemmWorkspace& gws);

// Standard Hermitian eigenproblem of a full (both triangles) matrix A (n x n,
// ld n; read only).  Eigenvalues ascending in w, the first nvec eigenvectors
// in Z (ld n).
void heev(cudaStream_t st, int n, double2* A, double* w, double2* Z, int nvec, Scratch& ws,
          const GemmWorkspace& gws);

}  // namespace dense
}  // namespace q3b
