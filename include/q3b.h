/*
 * q3b -- B200 (sm_100a) plane-wave H|psi> and block-Davidson, C ABI.
 *
 * A drop-in for the reference's operator interfaces of this path:
 *   PlanewaveHamiltonianApplicator
 *     (src/layer_4_computation/diagonalizer/planewave/internal/hamiltonian_applicator/init.hpp:28-153)
 *   PlanewaveDavidsonDiagonalizer::solve + PlanewaveSubspaceManager
 *     (src/layer_4_computation/diagonalizer/planewave/davidson.hpp:324-841,
 *      .../internal/subspace_manager/init.hpp:30-184)
 *
 * Conventions (the reference's): column-major, vector-contiguous arrays,
 * psi[g + v*npw]; complex numbers are (re, im) pairs of double (cplx128) or
 * float (cplx64); energies in Rydberg; the G-sphere order is the caller's
 * (the reference sorts it by kinetic energy).  Pointers named *_dev are device
 * pointers on the context's GPU; *_host are host pointers.  The caller owns
 * every buffer it passes; the context owns its device workspaces.
 *
 * Errors: every call returns Q3B_OK (0) or an error code; q3b_last_error()
 * returns the message of the context's last failure.  No C++ exception
 * crosses this boundary.  One context per host thread.
 *
 * Work is queued on the context's stream (q3b_get_stream / q3b_set_stream);
 * calls that return host data synchronise that stream before returning.
 */
#ifndef Q3B_H
#define Q3B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct q3b_context q3b_context;
typedef struct { double re, im; } q3b_cplx128;
typedef struct { float re, im; } q3b_cplx64;

enum q3b_status {
    Q3B_OK = 0,
    Q3B_ERR_INVALID = 1,   /* bad argument or unsupported size        */
    Q3B_ERR_CUDA = 2,      /* a CUDA runtime error                    */
    Q3B_ERR_STATE = 3,     /* call out of order (no potential, ...)   */
    Q3B_ERR_MEMORY = 4,    /* device allocation or HBM budget refused */
    Q3B_ERR_LINALG = 5,    /* subspace eigensolver / Cholesky failure */
    Q3B_ERR_INTERNAL = 6
};

enum q3b_precision {
    Q3B_FP64 = 0,          /* everything in FP64                       */
    Q3B_MIXED = 1          /* FP32 bulk, FP64 subspace + refinement    */
};

/* ---- context ------------------------------------------------------------ */

/* Create a context on CUDA device `device`.  hbm_budget_bytes caps the device
 * memory the context may hold (0 = no cap). */
int q3b_context_create(int device, size_t hbm_budget_bytes, q3b_context** out);
int q3b_context_destroy(q3b_context* ctx);
const char* q3b_last_error(const q3b_context* ctx);
/* cudaStream_t of the context, as void* */
void* q3b_get_stream(q3b_context* ctx);
/* Queue the context's work on an existing stream (NULL: its own stream). */
int q3b_set_stream(q3b_context* ctx, void* cuda_stream);
int q3b_synchronize(q3b_context* ctx);
/* Bytes of device memory the context holds now. */
size_t q3b_device_bytes(const q3b_context* ctx);

/* ---- PlanewaveHamiltonianApplicator ------------------------------------- */

/* update_potential (init.hpp:40; serial.hpp:64-78): V(r) on the wavefunction
 * grid, n1*n2*n3 values in the reference's flat order (i1*n2+i2)*n3+i3, Ry.
 * The 1/N scaling of the reference's cached potential is applied inside. */
int q3b_set_potential(q3b_context* ctx, const double* v_r_host, int n1, int n2, int n3);

/* update_potential when the density grid is larger than the wavefunction grid
 * (serial.hpp:64-78 -> compute_smooth_grid_potential_from_dense and
 * inverse_fft_smooth_potential, planewave_potential_utils.hpp:33-135): V(r) on
 * the density grid d1 x d2 x d3 (flat (i1*d2+i2)*d3+i3, Ry) is restricted to the
 * wavefunction grid n1 x n2 x n3 by G-space truncation (forward transform, the
 * coefficients of Miller indices -n/2 < m <= n/2 per axis, inverse transform,
 * real part) on the device, then taken as q3b_set_potential takes it.  Each
 * n_i must be at most d_i; equal grids are the identity. */
int q3b_set_potential_dense(q3b_context* ctx, const double* v_dense_host, int d1, int d2, int d3, int n1,
                            int n2, int n3);

/* invalidate_smooth_potential_cache (init.hpp:90) / is_smooth_potential_cache_valid (:96) */
int q3b_invalidate_potential(q3b_context* ctx);
int q3b_potential_valid(const q3b_context* ctx);

/* prepare_kpoint (init.hpp:47-50; serial.hpp:84-105) plus the projector set the
 * reference reads from its store (kleinman_bylander_projector_set.hpp:20-23):
 *   g_to_grid_host   npw flat grid indices ((w1*n2+w2)*n3+w3), -1 outside the grid
 *   ke_host          npw kinetic factors |k+G|^2 (Ry)
 *   beta_host        npw x nproj projectors, column-major (ld npw); may be NULL if nproj == 0
 *   atom_proj_offsets_host  natoms+1 offsets: atom a owns projectors [off[a], off[a+1])
 *   d_blocks_host    per-atom D blocks (Ry), packed one after another, each
 *                    m x m column-major with m = off[a+1]-off[a]
 *                    (serial.hpp:602-647; entries |D| <= 1e-15 are dropped). */
int q3b_prepare_kpoint(q3b_context* ctx, int npw, const int32_t* g_to_grid_host,
                       const double* ke_host, const q3b_cplx128* beta_host, int nproj,
                       int natoms, const int32_t* atom_proj_offsets_host,
                       const double* d_blocks_host);

/* set_spin_channel (init.hpp:75-80): the D blocks of the prepared k-point for
 * another spin channel, packed as d_blocks_host of q3b_prepare_kpoint (the
 * same atoms and projector offsets; entries |D| <= 1e-15 dropped).  The
 * reference reads D_ij(spin) when it rebuilds its block D after a channel
 * change (serial.hpp:602-647); the channel's V(r) comes through
 * q3b_set_potential as in the reference.  The projectors stay on the device. */
int q3b_set_d_blocks(q3b_context* ctx, const double* d_blocks_host);

/* apply_batch (init.hpp:59-61; serial.hpp:110-155): hpsi = H psi for nvec
 * vectors, device pointers, FP64 in and out.  precision Q3B_MIXED runs the
 * transforms and projector products in FP32 (inputs rounded, outputs widened).
 * Asynchronous: the work is queued on the context's stream (q3b_get_stream)
 * and the call returns; psi must be ready on that stream, and hpsi is ready
 * after q3b_synchronize or an event recorded on it (the reference's GPU form
 * synchronises the device instead, gpu.hpp:305). */
int q3b_apply_h(q3b_context* ctx, const q3b_cplx128* psi_dev, q3b_cplx128* hpsi_dev, int nvec,
                int precision);

/* The same product on FP32 vectors (the mixed solver's own storage). */
int q3b_apply_h_f32(q3b_context* ctx, const q3b_cplx64* psi_dev, q3b_cplx64* hpsi_dev, int nvec);

/* apply_batch with host buffers: copies in, applies, copies out, synchronises. */
int q3b_apply_h_host(q3b_context* ctx, const q3b_cplx128* psi_host, q3b_cplx128* hpsi_host,
                     int nvec, int precision);

/* q3b_apply_h (FP64) for callers that cannot allocate device memory during the
 * call: runtimes that own all device memory through their own pool, or that
 * forbid allocation once started.  No
 * counterpart in the reference.  Its scratch (the stick buffer and the
 * projector coefficients) is one fixed 32 MiB __device__ array that every GPU
 * loading the library holds until exit; bands are processed in batches that
 * fit it, and a k-point whose single band needs more is rejected with
 * Q3B_ERR_INVALID.  The first call on a device looks the array up (with that
 * device current) and should come before any stream capture.  Calls share the
 * array, so calls that overlap on the GPU race.  Inputs and outputs are the
 * caller's device buffers, as for q3b_apply_h. */
int q3b_apply_h_noalloc(q3b_context* ctx, const q3b_cplx128* psi_dev, q3b_cplx128* hpsi_dev,
                        int nvec);

/* ---- complex GEMMs of the subspace algebra --------------------------------- */

/* The reference's GPU BLAS products (GPUBLAS::gemm / gemm_single,
 * src/layer_0_core/math/linear_algebra/gpu/blas/init.hpp:70-82,136-148) as the
 * path uses them: C = alpha op(A) B + beta C, column-major, device pointers,
 * transpose_a 'N' or 'C', transpose_b 'N'.  q3b_gemm runs in FP64 on the CUDA
 * cores; q3b_gemm_single runs on the tensor cores (TF32 split into hi + lo,
 * three products, FP32 accumulation: FP32 accuracy).  Queued on the stream. */
int q3b_gemm(q3b_context* ctx, char transpose_a, char transpose_b, int m, int n, int k,
             q3b_cplx128 alpha, const q3b_cplx128* a_dev, int lda, const q3b_cplx128* b_dev, int ldb,
             q3b_cplx128 beta, q3b_cplx128* c_dev, int ldc);
int q3b_gemm_single(q3b_context* ctx, char transpose_a, char transpose_b, int m, int n, int k,
                    q3b_cplx64 alpha, const q3b_cplx64* a_dev, int lda, const q3b_cplx64* b_dev, int ldb,
                    q3b_cplx64 beta, q3b_cplx64* c_dev, int ldc);

/* ---- diagnostics ---------------------------------------------------------- */

/* Per-kernel device time of one application, CUDA events around each launch
 * (the reference's hamiltonian_fft / nonlocal / projector_overlap timers,
 * counters.hpp:36-52, split by kernel). */
typedef struct {
    double sticks_backward_ms;       /* scatter + backward transform along w3     */
    double planes_ms;                /* 2D transforms + V(r) product              */
    double sticks_forward_ms;        /* forward transform along w3 + gather + KE  */
    double projector_overlap_ms;     /* <beta|psi>                                */
    double d_apply_ms;               /* D blocks                                  */
    double projector_accumulate_ms;  /* hpsi += beta (D <beta|psi>)              */
    int launches[6];                 /* launches of each of the six classes       */
} q3b_apply_timing;

/* q3b_apply_h (fp32 == 0, cplx128 vectors) or q3b_apply_h_f32 (fp32 != 0,
 * cplx64 vectors) with the timing above; synchronises the stream. */
int q3b_apply_h_timed(q3b_context* ctx, const void* psi_dev, void* hpsi_dev, int nvec, int fp32,
                      q3b_apply_timing* timing);

/* The FP64 FMA throughput of the context's GPU in TFLOP/s, measured by a
 * probe kernel of independent DFMA chains (a few milliseconds): the
 * denominator of the FP64 GEMMs' roofline.  No counterpart in the reference
 * (diagnostics). */
int q3b_measure_fp64_rate(q3b_context* ctx, double* tflops);

/* Kernel launches the library has issued in this process (all contexts). */
unsigned long long q3b_kernel_launches(void);

/* ---- PlanewaveDavidsonDiagonalizer::solve -------------------------------- */

typedef struct {
    double tolerance;            /* eigenvalue-change tolerance, Ry (davidson.hpp:608-629)  */
    int max_iterations;          /* set_maximum_iterations (davidson.hpp:270-272), default 20 */
    int basis_expansion_factor;  /* set_basis_expansion_factor (davidson.hpp:260-264), >= 2 */
    int occupied_bands;          /* bands held to `tolerance`; the rest to max(5 tol, 1e-5)  */
    int precision;               /* Q3B_FP64 or Q3B_MIXED                                   */
    int refine_sweeps;           /* MIXED: max FP64 refinement iterations at the end; 0 (the
                                    default) allows max_iterations of them                   */
    double mixed_tolerance;      /* MIXED: eigenvalue-change tolerance of the FP32 phase, Ry;
                                    the phase also ends once the change stops falling       */
    int profile_stages;          /* nonzero: fill q3b_davidson_stats.stage_ms (drains the
                                    stream at every stage boundary)                         */
    double* eigenvalue_history;  /* optional host array of history_rows x nb (row-major): row
                                    i = the nb Ritz values (Ry) of iteration i's subspace
                                    solve, the FP32 phase's iterations first under MIXED;
                                    rows past the iterations run are left as they are.  The
                                    serving API ignores it.                                  */
    int history_rows;            /* rows of eigenvalue_history (0: no history)              */
    int mixed_expansion_factor;  /* MIXED: basis expansion factor of the FP32 phase (no
                                    counterpart in the reference; the FP64 refinement takes
                                    basis_expansion_factor); 0 (the default) takes 4, else 3,
                                    when that subspace order is within the eigensolver's
                                    limit, else basis_expansion_factor                      */
} q3b_davidson_opts;

typedef struct {
    int iterations;              /* Davidson iterations run (both phases)                   */
    int fp64_iterations;         /* of which in FP64                                        */
    int h_applications;          /* band applications of H                                  */
    int unconverged;             /* bands short of the tolerance at exit                    */
    int collapses;
    double max_residual_norm;    /* max_i ||H psi_i - eps_i psi_i|| of the returned bands   */
    double seconds;              /* wall time of the solve                                   */
    double stage_ms[8];          /* with profile_stages: seed, diagonalize, correction,
                                    orthogonalize, hamiltonian, subspace_update, collapse,
                                    extract (the reference's DavidsonTimingAccumulator
                                    stages, counters.hpp:36-52)                             */
    double fp64_seconds;         /* MIXED: wall time of the FP64 refinement phase           */
} q3b_davidson_stats;

void q3b_davidson_default_opts(q3b_davidson_opts* opts);

/* Solve for the nb lowest eigenpairs at the prepared k-point.  With overlap
 * blocks set (q3b_set_overlap_blocks) the problem is H c = eps S c and the bands
 * come back S-orthonormal; on a k-point prepared with q3b_prepare_kpoint_gamma
 * the bands are half-sphere vectors (npw = npw_half) under the real inner
 * product 2 Re(a^H b) - Re(conj(a_0) b_0).
 *   bands_host   npw x nb (ld npw): in, the starting bands (the reference seeds
 *                from the stored bands, davidson.hpp:1000-1045; zero columns are
 *                replaced by lowest-kinetic-energy plane waves, :1047-1101);
 *                out, the eigenvectors.
 *   eigenvalues_host  nb: in, stored eigenvalues (all zero = none); out, Ry. */
int q3b_davidson_solve(q3b_context* ctx, q3b_cplx128* bands_host, double* eigenvalues_host,
                       int nb, const q3b_davidson_opts* opts, q3b_davidson_stats* stats);

/* Same, with the bands already on the device (npw x nb, ld npw). */
int q3b_davidson_solve_dev(q3b_context* ctx, q3b_cplx128* bands_dev, double* eigenvalues_host,
                           int nb, const q3b_davidson_opts* opts, q3b_davidson_stats* stats);

/* ---- serving: continuous batching of band-solve requests ------------------- */

/* A request: one cell at one k-point, everything q3b_set_potential,
 * q3b_prepare_kpoint and q3b_davidson_solve take, all host pointers (copied at
 * submission).  No counterpart in the reference, which solves k-points one
 * after another from its SCF loop (iterator/.../pseudopotential/init.hpp:1059). */
typedef struct {
    int n1, n2, n3;
    const double* v_r;
    int npw;
    const int32_t* g_to_grid;
    const double* ke;
    int nproj;
    const q3b_cplx128* beta;
    int natoms;
    const int32_t* atom_proj_offsets;
    const double* d_blocks;
    int nb;
    const q3b_cplx128* bands;        /* starting bands, npw x nb                    */
    const double* eigenvalues;       /* stored eigenvalues, nb; NULL = none         */
    const q3b_davidson_opts* opts;   /* NULL = q3b_davidson_default_opts            */
} q3b_request;

typedef struct {
    double queue_ms;                 /* submission to start                        */
    double solve_ms;                 /* start to finish                            */
    double latency_ms;               /* submission to finish                       */
    size_t estimated_bytes;          /* device memory charged to the HBM budget     */
} q3b_request_times;

typedef struct q3b_server q3b_server;

/* A server on CUDA device `device` with `workers` concurrent solves (each its
 * own context and stream).  A queued request starts, oldest first, when a
 * worker is free and its memory estimate fits hbm_budget_bytes beside the
 * running ones (0 = no budget; one request always runs). */
int q3b_server_create(int device, size_t hbm_budget_bytes, int workers, q3b_server** out);
int q3b_server_destroy(q3b_server* server);
const char* q3b_server_last_error(const q3b_server* server);
int q3b_server_submit(q3b_server* server, const q3b_request* request, int* id_out);
/* 1 finished, 0 pending, -1 unknown id */
int q3b_server_poll(q3b_server* server, int id);
/* Block until request `id` is done; copy out the eigenvectors (npw x nb), the
 * eigenvalues (nb), its statistics and times (any may be NULL) and forget it.
 * Returns the solve's status. */
int q3b_server_wait(q3b_server* server, int id, q3b_cplx128* bands_out, double* eigenvalues_out,
                    q3b_davidson_stats* stats, q3b_request_times* times);

/* Batch the running solves' subspace eigensolves (enable != 0): each Davidson
 * iteration's generalized eigenproblem of order <= about 110 is solved in one
 * launch together with those of the other workers that reach the same step,
 * one thread block per problem; a batch waits up to wait_us microseconds
 * (0: 200) for workers busy elsewhere.  Only while the server is idle
 * (Q3B_ERR_STATE otherwise).  A problem that fits one block is solved the same
 * way whatever batch it joins, so results do not depend on the mix. */
int q3b_server_set_batching(q3b_server* server, int enable, int wait_us);
/* batches launched and problems they solved so far */
int q3b_server_batch_stats(q3b_server* server, long* batches, long* problems);

/* ---- dense FP64 subspace kernels (PlanewaveSubspaceManager pieces) ---------- */

/* diagonalize_subspace (subspace_manager/init.hpp:82; subspace/serial.hpp:18-151):
 * the generalized Hermitian problem H c = eps S c, itype 1, on device matrices
 * with leading dimension ld; only the upper triangles are read.  Writes n
 * eigenvalues (ascending) to w_dev and the S-orthonormal eigenvectors to
 * evec_dev (ld n).  Returns Q3B_ERR_LINALG (LAPACK's info != 0 case) when S is
 * not positive definite. */
int q3b_hegv(q3b_context* ctx, int n, const q3b_cplx128* h_dev, const q3b_cplx128* s_dev, int ld,
             double* w_dev, q3b_cplx128* evec_dev);

/* The same for the lowest nvec eigenpairs only (the Davidson's use,
 * davidson.hpp:512-520): nvec eigenvalues to w_dev, evec_dev n x nvec (ld n). */
int q3b_hegv_lowest(q3b_context* ctx, int n, const q3b_cplx128* h_dev, const q3b_cplx128* s_dev, int ld,
                    int nvec, double* w_dev, q3b_cplx128* evec_dev);

/* Many small problems in one launch, one thread block each (no counterpart in
 * the reference, which solves one subspace at a time).  Problem i is
 * H_i c = eps S_i c of order n[i] <= 128 with leading dimension ld[i], its
 * lowest nvec[i] eigenpairs into w_dev[i] and evec_dev[i] (ld n[i]); the
 * arrays of pointers and sizes are host arrays of `count` entries.  info_host[i]
 * gets 0 or n[i] + j (S_i not positive definite at order j, zhegv's info).
 * Returns Q3B_ERR_INVALID when a problem does not fit one block. */
int q3b_hegv_batched(q3b_context* ctx, int count, const int* n, const q3b_cplx128* const* h_dev,
                     const q3b_cplx128* const* s_dev, const int* ld, const int* nvec, double* const* w_dev,
                     q3b_cplx128* const* evec_dev, int* info_host);

/* Largest order the subspace eigensolver solves in one thread block (the
 * others take the multi-kernel path); 0 sends every order to the multi-kernel
 * path.  Process-wide; returns the previous value.  Default 64, up to which the
 * one-block solve is the faster of the two on a B200. */
int q3b_set_block_eigensolver_order(int max_order);

/* Counters of the context's CUDA-graph replays of the dense eigensolver: graphs
 * captured and replays served (either pointer may be NULL).  The launch
 * sequence of q3b_hegv and of the Davidson subspace solves of order >= 256 is
 * captured the third time the same problem shape meets the same buffers and
 * replayed after that.  No counterpart in the reference (diagnostics). */
int q3b_graph_stats(q3b_context* ctx, int* captures, int* replays);

/* The plane-pass kernel of the local term for the prepared k-point, by
 * precision (Q3B_FP64 or Q3B_MIXED's FP32 product).  choice: 0 hands it back
 * to the autotuner (the default: the candidates are timed once per grid and
 * precision); 128, 256 or 512 selects the shared-memory kernel with that many
 * threads a plane; -1 or -2 the register kernel with one or two lanes a line,
 * which exists for some grids only (Q3B_ERR_INVALID when not for this one).
 * q3b_get_local_kernel reports the choice in force, tuning first if needed.
 * No counterpart in the reference (its FFT is a library call). */
int q3b_set_local_kernel(q3b_context* ctx, int precision, int choice);
int q3b_get_local_kernel(q3b_context* ctx, int precision, int* choice);

/* ---- projector set built on the device (ProjectorSetBuilder) ---------------- */

/* q3b_prepare_kpoint with the Kleinman-Bylander projector matrix built on the
 * device instead of passed in (compute_kleinman_bylander_projectors,
 * pseudopotential/planewave/internal/projector.hpp:42-199; device builder
 * projector_set_builder_gpu.hpp):
 *   beta_{a,i,m}(G) = Omega^{-1/2} (-i)^l f_i(|k+G|) Y_lm(k+G) exp(-i (k+G).r_a),
 * f_i by 4-point Lagrange interpolation of a uniform table (q = 0, dq, 2dq,
 * ...), Y_lm real with the Condon-Shortley phase, projectors atom by atom,
 * beta by beta, m = 0, 1, -1, 2, -2, ....  Units: kpg_cart (npw x 3, k+G per
 * plane wave, x y z) in bohr^-1, positions (natoms x 3) in bohr, the volume
 * in bohr^3, dq in bohr^-1.  Species s has nbeta_of_species[s] beta functions;
 * beta_l and beta_tables (nq values each) list them species by species.
 * d_blocks: per-atom D blocks in the projector order above (Ry), as for
 * q3b_prepare_kpoint.  l <= 4. */
int q3b_prepare_kpoint_build(q3b_context* ctx, int npw, const int32_t* g_to_grid, const double* ke,
                             const double* kpg_cart, double cell_volume, int natoms, const double* positions,
                             const int32_t* species_of_atom, int nspecies, const int32_t* nbeta_of_species,
                             const int32_t* beta_l, int nq, double dq, const double* beta_tables,
                             const double* d_blocks);
/* The projector matrix (npw x P, column-major) the context holds for its
 * prepared k-point, copied to device memory `beta_dev`; P to *nproj. */
int q3b_get_projectors(q3b_context* ctx, q3b_cplx128* beta_dev, int* nproj);

/* ---- charge density (PlanewaveChargeDensityAccumulator) --------------------- */

/* accumulate_on_rho_grid, non-Gamma branch
 * (charge_density/planewave/internal/accumulator.hpp:375-545), for the context's
 * prepared k-point on its grid: rho[(w1*N2 + w2)*N3 + w3] +=
 * sum_b weights[b] |psi_b(r)|^2, psi_b(r) the unnormalised backward transform
 * of band b (npw x nvec device vectors, FP64) scattered by the G -> grid map.
 * weights (host, nvec) fold the k-point weight, the occupation and 1/volume;
 * a band of weight 0 is skipped, as the reference skips unoccupied bands.
 * rho: N1*N2*N3 doubles on the device, added to, so that k-points accumulate.
 * Deterministic: the band sums have a fixed order. */
int q3b_accumulate_density(q3b_context* ctx, const q3b_cplx128* psi_dev, int nvec, const double* weights_host,
                           double* rho_dev);

/* ---- starting-subspace rotation (StartingSubspaceSolver) -------------------- */

/* The three large steps of the starting rotation of one k-point's bands
 * (wavefunction/planewave/starting_subspace_solver.hpp:29-59, driven by
 * wavefunction/planewave/norm_conserving/initializer.hpp:250-385), FP64, on
 * the context's prepared k-point; the overlap is the identity (norm-conserving).
 *
 * apply_hamiltonian: copy the nchi starting vectors chi (host, npw x nchi,
 * column-major) to the device and apply H; chi and H chi stay on the device
 * for the two calls below. */
int q3b_start_apply(q3b_context* ctx, const q3b_cplx128* chi_host, int nchi);
/* project: H_ij = chi_i^H (H chi)_j and S_ij = chi_i^H chi_j, each nchi x nchi,
 * column-major, into host arrays. */
int q3b_start_project(q3b_context* ctx, q3b_cplx128* h_host, q3b_cplx128* s_host);
/* rotate_into_bands: band n = chi (column n of coefficients), coefficients on
 * the host (nchi x nb, ld nchi), bands written to DEVICE memory (npw x nb), as
 * the reference stores them in the quantum system's device block: only the
 * coefficients cross to the device. */
int q3b_start_rotate(q3b_context* ctx, const q3b_cplx128* coefficients_host, int nb,
                     q3b_cplx128* bands_dev);
/* The whole rotation on the device: q3b_start_apply, the projections, the
 * generalized problem (zhegv itype 1 on the upper triangles, as the
 * initializer calls it), bands = chi c[:, :nb] into bands_dev and the nb
 * lowest eigenvalues (Ry) into eigenvalues_host.  Returns Q3B_ERR_LINALG when
 * the starting vectors' overlap is not positive definite. */
int q3b_starting_subspace(q3b_context* ctx, const q3b_cplx128* chi_host, int nchi, int nb,
                          q3b_cplx128* bands_dev, double* eigenvalues_host);

/* ---------------------------------------------------------------- Gamma-only k-point
 * The reference's Gamma-only basis stores each band on the half sphere of G
 * (the origin at index 0, then one of each +G/-G pair; basis/planewave/init.hpp:60-67)
 * and applies H two real bands per complex transform
 * (hamiltonian_applicator/serial.hpp:283-418) with real projector overlaps
 * 2 Re(beta^H psi) less the origin's term (serial.hpp:519-566).
 *
 * prepare_kpoint for such a k-point (k = 0):
 *   g_to_grid_host        npw_half grid indices of +G (-1 outside the grid); entry 0 the origin
 *   g_minus_to_grid_host  npw_half grid indices of -G (serial.hpp:889-900); entry 0 equal to
 *                         g_to_grid_host[0]
 *   ke_host, beta_host    on the half sphere (npw_half x nproj, column-major); the projectors
 *                         of a Gamma-only k-point satisfy beta(-G) = conj(beta(G)), which the
 *                         library uses to extend them to the full sphere
 *   atom offsets and D blocks as for q3b_prepare_kpoint.
 * The library keeps the full-sphere plan (2 npw_half - 1 plane waves); q3b_apply_h
 * then takes full-sphere vectors in the order [half sphere, mirrors of entries 1..]. */
int q3b_prepare_kpoint_gamma(q3b_context* ctx, int npw_half, const int32_t* g_to_grid_host,
                             const int32_t* g_minus_to_grid_host, const double* ke_host,
                             const q3b_cplx128* beta_host, int nproj, int natoms,
                             const int32_t* atom_proj_offsets_host, const double* d_blocks_host);

/* apply_batch on a Gamma-only k-point (serial.hpp:283-418 and :519-566):
 * hpsi = H psi for nvec half-sphere vectors (device, npw_half x nvec,
 * column-major), bands 2p and 2p+1 through one complex transform.  The origin
 * is packed as (Re psi_a(0), Re psi_b(0)) and hpsi(0) is real, as in the
 * reference; a last band without a partner goes alone (the reference's
 * single-band path).  Asynchronous on the context's stream, like q3b_apply_h. */
int q3b_apply_h_gamma(q3b_context* ctx, const q3b_cplx128* psi_dev, q3b_cplx128* hpsi_dev, int nvec,
                      int precision);

/* ---------------------------------------------------------------- ultrasoft overlap S
 * UltrasoftPseudopotentialOverlapOperator (diagonalizer/planewave/internal/overlap/
 * pseudopotential/ultrasoft/init.hpp:27-470): S psi = psi + sum_ij beta_i q_ij <beta_j|psi>.
 *
 * set the per-atom blocks q_ij of the prepared k-point (Ry-free, dimensionless), packed as
 * the D blocks of q3b_prepare_kpoint (one m x m column-major block per atom; the reference's
 * build_q_matrix, init.hpp:416-466, sets q_ab for equal l and m; entries |q| <= 1e-15 dropped).
 * Preparing a k-point clears them. */
int q3b_set_overlap_blocks(q3b_context* ctx, const double* q_blocks_host);

/* apply_batch (init.hpp:189-345): spsi = S psi for nvec device vectors (npw x nvec,
 * FP64 in and out; may be the same array).  Q3B_MIXED forms the correction
 * beta Q beta^H psi with the FP32 tensor-core products and adds it to psi in FP64.
 * Asynchronous on the context's stream. */
int q3b_apply_s(q3b_context* ctx, const q3b_cplx128* psi_dev, q3b_cplx128* spsi_dev, int nvec,
                int precision);

/* The same on a Gamma-only k-point (init.hpp:212-270): half-sphere vectors, two bands
 * per pass, separated as in q3b_apply_h_gamma. */
int q3b_apply_s_gamma(q3b_context* ctx, const q3b_cplx128* psi_dev, q3b_cplx128* spsi_dev, int nvec,
                      int precision);

#ifdef __cplusplus
}
#endif

#endif /* Q3B_H */
