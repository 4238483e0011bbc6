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

// DFMA throughput of the current device (TFLOP/s), from a probe kernel of
// independent FMA chains (the FP64 roofline's denominator)
double measure_dfma_tflops(cudaStream_t st);

// bytes of workspace cgemm may use for a C,N product of this shape
template <typename R> size_t cgemm_workspace_bytes(int M, int N, int K);

// FP32 products of at least this many complex multiply-adds (M N K) run on
// the tensor cores, smaller ones on the CUDA cores
constexpr double kTensorCoreMinMacs = 67108864.0;  // 2^26
bool use_tensor_cores(int M, int N, int K);

// The FP32 products run on the tensor cores (cgemm_tc.cu).
namespace tc {
void cgemm(cudaStream_t st, bool conj_a, int M, int N, int K, float2 alpha, const float2* A, long lda,
           const float2* B, long ldb, float2 beta, float2* C, long ldc, const GemmWorkspace& ws);

// An A operand converted once into the shared-memory image the tensor-core
// kernel's stages take (TF32 hi/lo planes, 128B-swizzled, tiles of 128 rows x
// 32 K), for operands used many times, such as a k-point's projectors: the
// kernel then moves its A tiles with bulk asynchronous copies and converts
// only B.  Rows are M of the product, K its reduction index.
struct PackedA {
    const unsigned char* tiles = nullptr;
    int M = 0, K = 0;
};
size_t packed_a_bytes(int M, int K);
// kmajor: element (m, k) at A[m * lda + k] (the "C,N" operand, A^H's source);
// else at A[m + k * lda] (the "N,N" operand).  out: packed_a_bytes(M, K).
void pack_a(cudaStream_t st, int M, int K, const float2* A, long lda, bool kmajor, unsigned char* out);
// cgemm with a packed A (same meaning of conj_a and the other arguments)
void cgemm_packed(cudaStream_t st, bool conj_a, int M, int N, int K, float2 alpha, const PackedA& A,
                  const float2* B, long ldb, float2 beta, float2* C, long ldc, const GemmWorkspace& ws);
size_t workspace_bytes(int M, int N, int K);
// device word the tensor-core kernels set when a pipeline wait times out: the
// word of the context the calling thread works for (ErrorScope), so that
// contexts used by different threads at once report only their own timeouts;
// a process-wide word per device outside any context
int* error_word();
struct ErrorScope {
    explicit ErrorScope(int* word);
    ~ErrorScope();
    ErrorScope(const ErrorScope&) = delete;
    ErrorScope& operator=(const ErrorScope&) = delete;

  private:
    int* prev_;
};
// read (and clear) it; throws CudaError when it was set.  Synchronises st.
void check_error(cudaStream_t st);
}  // namespace tc

}  // namespace q3b
