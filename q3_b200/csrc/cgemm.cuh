// Complex GEMMs on CUDA cores (FP64 DFMA / FP32 FFMA), column-major like the
// reference's ZGEMM calls.
//
//   C(M x N) = alpha * op(A) * B + beta * C
//   op(A) = A   (A is M x K, lda)         -- "N,N": beta|psi>, V c, ...
//   op(A) = A^H (A is K x M, lda)         -- "C,N": <beta|psi>, V^H HV, Gram
//
// The "C,N" products reduce over the long plane-wave axis; they split K across
// blockIdx.z into a workspace and a second kernel sums the splits in a fixed
// order, so the result does not depend on how many other problems share the
// launch or on timing.
#pragma once

#include "common.cuh"

namespace q3b {

struct GemmWorkspace {
    void* ptr = nullptr;
    size_t bytes = 0;
};

template <typename R>
void cgemm(cudaStream_t st, bool conj_a, int M, int N, int K, cplx_t<R> alpha, const cplx_t<R>* A,
           long lda, const cplx_t<R>* B, long ldb, cplx_t<R> beta, cplx_t<R>* C, long ldc,
           const GemmWorkspace& ws);

// bytes of workspace cgemm may use for a C,N product of this shape
template <typename R> size_t cgemm_workspace_bytes(int M, int N, int K);

// The FP32 products run on the tensor cores (cgemm_tc.cu).
namespace tc {
void cgemm(cudaStream_t st, bool conj_a, int M, int N, int K, float2 alpha, const float2* A, long lda,
           const float2* B, long ldb, float2 beta, float2* C, long ldc, const GemmWorkspace& ws);
size_t workspace_bytes(int M, int N, int K);
// device word the tensor-core kernels set when a pipeline wait times out
int* error_word();
// read (and clear) it; throws CudaError when it was set.  Synchronises st.
void check_error(cudaStream_t st);
}  // namespace tc

}  // namespace q3b
