// The state behind a q3b_context: device, stream, HBM accounting, the
// potential, the prepared k-point (plane-wave list, sticks plan, projectors)
// and grow-only workspaces.
#pragma once

#include <string>
#include <vector>

#include "cgemm.cuh"
#include "common.cuh"
#include "dense.cuh"
#include "hpsi_local.cuh"
#include "nonlocal.cuh"

struct q3b_context;

namespace q3b {

struct Status : std::runtime_error {
    int code;
    Status(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

class Context;
class EigenBatcher;

// A device allocation charged to its context's HBM budget.
struct DevBuf {
    Context* ctx = nullptr;
    void* ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf();
    void release();
    // grow to at least `need` bytes (contents are not kept)
    void reserve(Context* c, size_t need);
    template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

struct KPoint {
    int npw = 0;
    int nproj = 0;
    int natoms = 0;
    bool valid = false;
    std::vector<int> g_to_grid;     // host copy, for replanning on a new grid
    std::vector<double> ke_host;
    DevBuf ke64, ke32;
    DevBuf beta64, beta32;
    DevBuf beta_pk_overlap, beta_pk_accum;  // beta32 as packed tensor-core A tiles
    DevBuf pstart, psize, poff, dpk64, dpk32;
    size_t dpk_len = 0;             // packed block entries (D, and Q when set)
    bool has_q = false;             // ultrasoft overlap blocks set for this k-point
    DevBuf qpk64, qpk32;
    // sticks plan
    DevBuf stick_start, entry_g, entry_w3, entry_stick, stick_pos, row_base, unmapped;
    DevBuf row_iv;  // int4 per stick row (LocalPlan::row_iv), when the sticks allow it
    DevBuf tw64[3], tw32[3];
    LocalPlan<double> lp64{};
    LocalPlan<float> lp32{};
    bool tuned64 = false, tuned32 = false;
};

class Context {
  public:
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    size_t budget = 0;
    size_t held = 0;
    std::string err;

    int n1 = 0, n2 = 0, n3 = 0;
    bool pot_valid = false;
    std::vector<double> v_host;     // V(r) as given, reference layout
    DevBuf v64, v32;                // V/N, [w3 pos][w1][w2 pos] (see LocalPlan::vplane)
    DevBuf v64nat, v32nat;          // V/N, [w3 pos][w1][w2] (LocalPlan::vnat)
    DevBuf err_word;                // device error word of this context's kernels (bounded waits)

    KPoint kp;

    // workspaces
    DevBuf ws_sticks, ws_gemm, ws_bm, ws_bp, ws_conv_in, ws_conv_out, ws_host_io;
    DevBuf ws_solver, ws_dense, ws_bands, ws_tune;
    DevBuf ws_mixed;  // FP64 bands of a mixed solve between its phases (buffer bands included)
    // replays of the dense eigensolver's launch sequence (one per context)
    dense::HegvGraphs hegv_graphs;
    // when set (a serving worker's context), the Davidson's subspace eigensolves
    // that fit one block go through this batcher, shared with the other workers
    EigenBatcher* batcher = nullptr;
    // charge density: per-group partial sums and the band weights
    DevBuf ws_density;
    // starting-subspace rotation: chi and H chi of the last q3b_start_apply
    DevBuf ws_start;
    int start_n = 0;
    int start_npw = 0;
    // Gamma-only k-point: the half sphere's length (0 when the k-point was
    // prepared with the full sphere) and the packed band pairs of q3b_apply_h_gamma
    int gamma_half = 0;
    DevBuf ws_gamma;
    // length of a band vector of the prepared k-point (the half sphere at Gamma)
    int band_npw() const { return gamma_half > 0 ? gamma_half : kp.npw; }

    // copy streams and events of q3b_apply_h_host's pipelined chunks
    static constexpr int kIoChunks = 4;
    cudaStream_t io_in = nullptr, io_out = nullptr;
    cudaEvent_t io_ev_in[kIoChunks] = {}, io_ev_out[kIoChunks] = {};
    void ensure_io_streams();

    explicit Context(int dev, size_t hbm_budget);
    ~Context();

    void set_potential(const double* v, int a, int b, int c);
    // V(r) on a density grid d1 x d2 x d3 restricted to the wavefunction grid a x b x c
    void set_potential_dense(const double* v, int d1, int d2, int d3, int a, int b, int c);
    void prepare_kpoint(int npw, const int32_t* g2g, const double* ke, const double2* beta, int nproj,
                        int natoms, const int32_t* offs, const double* dblk, bool beta_on_device = false);
    void require_ready() const;

    template <typename R> const LocalPlan<R>& local_plan() const;
    template <typename R> NonlocalData<R> nonlocal() const;
    // the same projectors with the ultrasoft overlap blocks Q in place of D
    template <typename R> NonlocalData<R> overlap() const;
    void set_overlap_blocks(const double* qblk);
    // the D blocks of the prepared k-point (another spin channel), layout unchanged
    void set_d_blocks(const double* dblk);
    template <typename R> int sticks_chunk(int nvec) const;

    // H|psi> on device vectors in precision R (the solver's building block)
    template <typename R>
    void apply_h(const cplx_t<R>* psi, long ldpsi, cplx_t<R>* hpsi, long ldh, int nvec,
                 PhaseTimer* timer = nullptr);

    GemmWorkspace gemm_ws(size_t need);

    // Autotuner: time the candidate plane kernels on a few bands of this
    // k-point and keep the fastest (once per plan and precision).
    template <typename R> void tune_local();
    // override of the tuner's plane kernel (q3b_set_local_kernel) and the choice in force
    template <typename R> void set_local_kernel(int choice);
    template <typename R> int local_kernel();

  private:
    void build_plan();
};

// convert an exception into a status code and message
int fail(q3b_context* c, const std::exception& e);

// kernel launches issued by the library so far
unsigned long long launches();

}  // namespace q3b

namespace q3b {
// S psi = psi + beta Q beta^H psi on device vectors of the prepared plan
// (npw x nvec, FP64 in and out; MIXED computes the correction in FP32)
void apply_s_device(Context& c, const double2* psi, double2* spsi, int nvec, int precision);
}  // namespace q3b

struct q3b_context {
    q3b::Context impl;
    q3b_context(int dev, size_t budget) : impl(dev, budget) {}
};
