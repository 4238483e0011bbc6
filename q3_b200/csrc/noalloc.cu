// q3b_apply_h_noalloc: FP64 H|psi> that allocates no device memory.
//
// Some callers cannot call cudaMalloc while they apply H: runtimes that own
// all device memory through a pool of their own, and runtimes that forbid
// allocation after start-up.  This entry point serves them.  Its
// scratch -- the stick buffer of the sticks/planes transform and the two
// projector-coefficient blocks of the nonlocal term -- lives in one
// file-scope __device__ array of kNoallocScratchBytes (32 MiB), which every
// GPU that loads the library holds until the process exits.  Bands are taken
// in batches sized to that array; a k-point whose single band does not fit is
// rejected.  The projector product runs without a split-K workspace.
//
// Host code cannot pass the array's name to a kernel: in host code it is a
// host-side stand-in, not a device address.  The first call on each device
// (with that device current) resolves the address with cudaGetSymbolAddress;
// that first call should come before any stream capture.  All calls share the
// array and the last call's contents stay in it; every element a call reads
// it has written first in that call, so nothing needs clearing, but calls
// whose work overlaps on the GPU (other streams, other threads) race on it.
#include <mutex>

#include "context.cuh"
#include "q3b.h"

namespace q3b {
namespace {

constexpr size_t kNoallocScratchBytes = 32ull << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

void* scratch_address(int device) {
    static void* addr[kMaxDevices] = {};
    static std::mutex mu;
    if (device < 0 || device >= kMaxDevices) throw Status(Q3B_ERR_INVALID, "device index out of range");
    std::lock_guard<std::mutex> lk(mu);
    if (!addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            throw Status(Q3B_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        }
        addr[device] = p;
    }
    return addr[device];
}

}  // namespace
}  // namespace q3b

extern "C" int q3b_apply_h_noalloc(q3b_context* ctx, const q3b_cplx128* psi, q3b_cplx128* hpsi, int nvec) {
    if (!ctx) return Q3B_ERR_INVALID;
    q3b::Context& c = ctx->impl;
    try {
        Q3B_CUDA(cudaSetDevice(c.device));
        q3b::tc::ErrorScope scope(c.err_word.as<int>());
        c.require_ready();
        if (nvec < 0 || (nvec > 0 && (!psi || !hpsi))) throw q3b::Status(Q3B_ERR_INVALID, "bad vectors");
        if (nvec == 0) return Q3B_OK;
        const q3b::LocalPlan<double>& lp = c.local_plan<double>();
        const int npw = c.kp.npw, P = c.kp.nproj;
        const size_t sticks = q3b::sticks_bytes_per_band(lp);
        const size_t proj = 2 * (size_t)P * sizeof(double2);
        const size_t per_band = ((sticks + 255) & ~size_t(255)) + proj;
        const size_t cap = q3b::kNoallocScratchBytes - 1024;
        if (per_band > cap) {
            throw q3b::Status(Q3B_ERR_INVALID,
                              "q3b_apply_h_noalloc: one band needs " + std::to_string(per_band) +
                                  " bytes of scratch, above its fixed " +
                                  std::to_string(q3b::kNoallocScratchBytes) + "-byte buffer");
        }
        const int batch = static_cast<int>(cap / per_band);
        char* base = static_cast<char*>(q3b::scratch_address(c.device));
        const auto* x = reinterpret_cast<const double2*>(psi);
        auto* y = reinterpret_cast<double2*>(hpsi);
        for (int b0 = 0; b0 < nvec; b0 += batch) {
            const int nb = nvec - b0 < batch ? nvec - b0 : batch;
            double2* X = reinterpret_cast<double2*>(base);
            const size_t xbytes = ((nb * sticks) + 255) & ~size_t(255);
            double2* Bm = reinterpret_cast<double2*>(base + xbytes);
            double2* Bp = Bm + (size_t)P * nb;
            q3b::apply_local<double>(c.stream, lp, x + (size_t)b0 * npw, npw, y + (size_t)b0 * npw, npw,
                                     nb, X, nb);
            if (P > 0) {
                q3b::apply_nonlocal<double>(c.stream, c.nonlocal<double>(), npw, nb,
                                            x + (size_t)b0 * npw, npw, y + (size_t)b0 * npw, npw, Bm,
                                            Bp, q3b::GemmWorkspace{});
            }
        }
        return Q3B_OK;
    } catch (const std::exception& e) {
        return q3b::fail(ctx, e);
    }
}
