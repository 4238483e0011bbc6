// Device-resident block Davidson; see davidson.cu.
#pragma once

#include "context.cuh"
#include "q3b.h"

namespace q3b {

// Solve at the context's prepared k-point.  bands_dev: npw x nb (ld npw), in =
// starting bands, out = eigenvectors; eig_host: in = stored eigenvalues (all
// zero = none), out = eigenvalues (Ry).
void davidson_solve(Context& c, double2* bands_dev, double* eig_host, int nb,
                    const q3b_davidson_opts& opts, q3b_davidson_stats* stats);

// The basis expansion factor of a solve with these options (under Q3B_MIXED,
// that of its FP32 phase: see q3b_davidson_opts; its FP64 refinement takes
// basis_expansion_factor).
int basis_factor(const q3b_davidson_opts& opts, int nb, int npw);

// Bands a mixed solve carries for nb wanted ones: nb plus max(2, nb/8) buffer
// bands held to the loose tolerance of empty bands (at most npw).
int mixed_bands(int nb, int npw);

}  // namespace q3b
