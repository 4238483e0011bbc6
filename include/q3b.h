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

/* apply_batch (init.hpp:59-61; serial.hpp:110-155): hpsi = H psi for nvec
 * vectors, device pointers, FP64 in and out.  precision Q3B_MIXED runs the
 * transforms and projector products in FP32 (inputs rounded, outputs widened). */
int q3b_apply_h(q3b_context* ctx, const q3b_cplx128* psi_dev, q3b_cplx128* hpsi_dev, int nvec,
                int precision);

/* The same product on FP32 vectors (the mixed solver's own storage). */
int q3b_apply_h_f32(q3b_context* ctx, const q3b_cplx64* psi_dev, q3b_cplx64* hpsi_dev, int nvec);

/* apply_batch with host buffers: copies in, applies, copies out, synchronises. */
int q3b_apply_h_host(q3b_context* ctx, const q3b_cplx128* psi_host, q3b_cplx128* hpsi_host,
                     int nvec, int precision);

#ifdef __cplusplus
}
#endif

#endif /* Q3B_H */
