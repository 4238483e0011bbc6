// Kinetic + local-potential part of H|psi> on the sticks/planes layout.
//
// A k-point's G-sphere occupies S "sticks" (grid columns (w1, w2) along the
// contiguous axis w3).  One application for a chunk of bands is three kernels:
//   A  sticks, backward: scatter psi into each stick, 1D transform along w3,
//      store X[band][w3][stick];
//   B  planes: per (band, w3) plane in shared memory, scatter the S stick
//      values, 2D backward transform (rows w1 that hold sticks, then all
//      columns), multiply by V(r)/N, 2D forward transform, gather back;
//   C  sticks, forward: 1D forward transform along w3, gather the sphere and
//      write hpsi = |k+G|^2 psi + (local term).
// Nothing outside the sticks is stored or moved through HBM.
#pragma once

#include "common.cuh"

namespace q3b {

template <typename R> struct LocalPlan {
    using T = cplx_t<R>;
    int n1, n2, n3;
    int npw;
    int nsticks;
    int nrows;          // distinct w1 among the sticks
    int p2;             // pitch of a plane row in shared memory (odd)
    int p3;             // pitch of a stick line in shared memory (odd)
    int na1, nb1, na2, nb2, na3, nb3;
    int sg;             // sticks per block in passes A and C
    int plane_threads;  // threads per block of the plane kernel (128, 256, 512)
    int nunmapped;      // G outside the grid: kinetic term only
    const int* stick_start;  // nsticks+1, ranges into the entry arrays
    const int* entry_g;      // G index (caller's order) of each sphere entry
    const int* entry_w3;
    const int* entry_stick;
    const int* stick_pos;    // w1*p2 + w2
    const int* row_base;     // w1*p2 of each used row
    const int* unmapped_g;
    const T* tw1;            // w_n^m = exp(-2 pi i m/n), one table per axis
    const T* tw2;
    const T* tw3;
    const R* ke;             // |k+G|^2 (Ry), caller's order
    const R* vplane;         // V(r)/N laid out [w3 pos][w1][w2 pos], with the w3 and w2
                             // positions of the backward transform's digit-reversed order
    // stick buffer X[band][w3 pos][stick]: sticks of one (band, w3) plane are
    // xpitch apart (nsticks rounded up to an even count, so every plane's run
    // starts on a 16-byte boundary for the bulk copies of planes_reg.cu)
    int xpitch;
    // Register plane kernel (planes_reg.cu): the stick rows are the cyclic
    // interval row_lo .. row_lo + nrows - 1 of w1, row slot s holding
    // row_iv[s] = {first w2, count, first stick, 0} (its sticks a cyclic
    // interval of w2, numbered consecutively).  row_iv is null when the
    // k-point's sticks do not have that shape.
    int row_lo;
    const int4* row_iv;
    const R* vnat;           // V(r)/N laid out [w3 pos][w1][w2], w1 and w2 natural
    int variant;             // plane kernel: 0 shared-memory (plane_threads), L > 0 register with L lanes a line
    int* err;                // the context's device error word (bounded waits that ran out)
};

// the register plane kernel: whether there is one for an n1 x n2 plane with
// `lanes` lanes a line, and its launch (false when the plan or grid has none)
bool has_planes_reg(int n1, int n2, int lanes);
template <typename R>
bool launch_planes_reg(const LocalPlan<R>& p, cplx_t<R>* X, int nb, int lanes, cudaStream_t st, int* err);

// bytes of the stick buffer per band
template <typename R> inline size_t sticks_bytes_per_band(const LocalPlan<R>& p) {
    return (size_t)p.n3 * p.xpitch * sizeof(cplx_t<R>);
}

// Per-kernel-class CUDA-event timing of one application (diagnostics).
struct PhaseTimer {
    enum { STICKS_BACKWARD = 0, PLANES, STICKS_FORWARD, PROJ_OVERLAP, D_APPLY, PROJ_ACCUM, NCLASS };
    static constexpr int kMax = 256;
    cudaEvent_t ev[2 * kMax];
    int cls[kMax];
    int used = 0;
    cudaStream_t st = nullptr;
    PhaseTimer();
    ~PhaseTimer();
    void begin(int c);   // record the start of a launch of class c
    void end();          // record its end
    // synchronise and sum the durations per class (ms) and count launches
    void collect(double* ms, int* count);
};

// hpsi[:, b] = KE*psi[:, b] + local term, for nvec bands (column stride ld).
// X must hold chunk*sticks_bytes_per_band bytes.
template <typename R>
void apply_local(cudaStream_t st, const LocalPlan<R>& p, const cplx_t<R>* psi, long ldpsi,
                 cplx_t<R>* hpsi, long ldh, int nvec, cplx_t<R>* X, int chunk,
                 PhaseTimer* timer = nullptr);

// Charge density: rho (N doubles, natural grid order) += sum_b w[b] |psi_b(r)|^2,
// psi_b(r) the unnormalised backward transform of band b scattered onto the
// grid.  w: nvec device weights (0 skips a band).  X: chunk *
// sticks_bytes_per_band; partial: groups * N doubles with groups from
// density_groups(p, chunk), the bands of one launch.
int density_groups(const LocalPlan<double>& p, int nvec);
void accumulate_density(cudaStream_t st, const LocalPlan<double>& p, const double2* psi, long ldpsi, int nvec,
                        const double* w, double2* X, int chunk, double* partial, int groups, double* rho);

// shared-memory footprint of the plane kernel (for capacity checks)
template <typename R> size_t plane_smem_bytes(const LocalPlan<R>& p);

}  // namespace q3b
