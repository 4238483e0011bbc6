// Shared helpers for the q3b sm_100a kernels: complex arithmetic on float2 /
// double2, error plumbing, launch checks.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <stdexcept>
#include <string>

namespace q3b {

template <typename R> struct CplxOf;
template <> struct CplxOf<double> { using T = double2; };
template <> struct CplxOf<float> { using T = float2; };
template <typename R> using cplx_t = typename CplxOf<R>::T;

__host__ __device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__host__ __device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }

__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return mk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return mk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator*(double s, double2 a) { return mk(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return mk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return mk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) { return mk(s * a.x, s * a.y); }

// complex product a*b
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return mk(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return mk(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// conj(a)*b
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
    return mk(fma(a.x, b.x, a.y * b.y), fma(a.x, b.y, -a.y * b.x));
}
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return mk(fmaf(a.x, b.x, a.y * b.y), fmaf(a.x, b.y, -a.y * b.x));
}
__host__ __device__ __forceinline__ double2 conj2(double2 a) { return mk(a.x, -a.y); }
__host__ __device__ __forceinline__ float2 conj2(float2 a) { return mk(a.x, -a.y); }
// i*a
__host__ __device__ __forceinline__ double2 mul_i(double2 a) { return mk(-a.y, a.x); }
__host__ __device__ __forceinline__ float2 mul_i(float2 a) { return mk(-a.y, a.x); }

// acc += a*b
__device__ __forceinline__ void cfma(double2& acc, double2 a, double2 b) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
__device__ __forceinline__ void cfma(float2& acc, float2 a, float2 b) {
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
}

template <typename T> __host__ __device__ __forceinline__ T czero();
template <> __host__ __device__ __forceinline__ double2 czero<double2>() { return mk(0.0, 0.0); }
template <> __host__ __device__ __forceinline__ float2 czero<float2>() { return mk(0.0f, 0.0f); }

struct CudaError : std::runtime_error {
    explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

#define Q3B_CUDA(call)                                                                         \
    do {                                                                                       \
        cudaError_t q3b_err_ = (call);                                                         \
        if (q3b_err_ != cudaSuccess) {                                                         \
            throw ::q3b::CudaError(std::string(#call) + ": " + cudaGetErrorString(q3b_err_)); \
        }                                                                                      \
    } while (0)

// every kernel launch of the library is followed by Q3B_LAUNCH_CHECK(), which
// also counts it (q3b_kernel_launches)
void count_launch();
#define Q3B_LAUNCH_CHECK()          \
    do {                            \
        ::q3b::count_launch();      \
        Q3B_CUDA(cudaGetLastError()); \
    } while (0)

// Pinned host memory of the calling host thread, at least `bytes` long, for
// small device->host reads (status words, eigenvalues, norms).  A read into
// pageable memory is staged by the driver through memory it shares between
// threads, and several threads solving at once on their own streams then wait
// on each other's reads; a pinned destination is written by the copy engine
// directly.  The block stays valid until the next call from the same thread.
void* host_readback(size_t bytes);

// Copies `bytes` of host memory to `dst` on `st` through the calling thread's
// pinned staging block (same reason), for the small uploads inside the solver
// loop.  The host data is taken at the call; the block is reused only after
// the stream has consumed the previous copy.  The large one-off copies of a
// request's setup stay on the driver's pageable path, which pipelines its
// staging with the transfer (faster there with several threads at once).
void upload_async(void* dst, const void* src, size_t bytes, cudaStream_t st);

inline int ceil_div(long a, long b) { return static_cast<int>((a + b - 1) / b); }

// Streaming multiprocessors of the current device (looked up once per device).
int device_sms();

// Grid of `threads`-thread blocks for a grid-stride loop over n items: one
// block per `threads` items, at most `per_sm` blocks per SM of the device.
inline int stride_grid(long n, int per_sm, int threads = 256) {
    long b = (n + threads - 1) / threads;
    const long cap = (long)device_sms() * per_sm;
    if (b > cap) b = cap;
    return static_cast<int>(b < 1 ? 1 : b);
}

// Runs a set-up step (function attributes, which belong to a function on one
// device) the first time it is called with each device current.
class PerDeviceOnce {
  public:
    template <typename F> void run(F&& f) {
        int dev = 0;
        Q3B_CUDA(cudaGetDevice(&dev));
        std::lock_guard<std::mutex> lk(mu_);
        if (dev >= 0 && dev < 64 && ((done_ >> dev) & 1ull)) return;
        f();
        if (dev >= 0 && dev < 64) done_ |= 1ull << dev;
    }

  private:
    std::mutex mu_;
    unsigned long long done_ = 0;
};

}  // namespace q3b
