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

}  // namespace q3b
