// Real symmetric tridiagonal helpers shared by the eigensolvers (dense.cu,
// dense_block.cu): Sturm counts for bisection and a pivot clamp for inverse
// iteration.
#pragma once

#include <cuda_runtime.h>

namespace q3b {
namespace dense {

// numbers of eigenvalues of the real tridiagonal (d, e2) below x[0..S).  The
// count is the number of sign changes along p_0 = 1, p_1, ..., p_n with
// p_k = (d_k - x) p_{k-1} - e2_{k-1} p_{k-2} (the leading principal minors of
// T - x I); the ratio p_k / p_{k-1} is the pivot of the LDL^T form, and a
// ratio below pivmin in magnitude is replaced by -pivmin, as in the LDL^T
// count.  No division: each step rescales the pair by the power of two of
// p_{k-1} (exact), which keeps both in range, so the dependent chain per step
// is one FMA, a select and a multiply.  S independent recurrences interleave.
__device__ __forceinline__ double pow2_inverse_exponent(double p) {
    // the exponent field sits in bits 20..30 of the high word: 32-bit integer
    // work only
    const int e = (__double2hiint(p) >> 20) & 0x7ff;
    return __hiloint2double((2046 - e) << 20, 0);
}

template <int S>
__device__ __forceinline__ void sturm_counts(int n, const double* d, const double* e2, const double* x,
                                             double pivmin, int* c) {
    double p[S], pm[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        pm[s] = 1.0;
        p[s] = d[0] - x[s];
        if (fabs(p[s]) < pivmin) p[s] = -pivmin;
        c[s] = p[s] < 0.0;
    }
#pragma unroll 4
    for (int k = 1; k < n; ++k) {
        const double dk = d[k], ek = e2[k - 1];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const double sc = pow2_inverse_exponent(p[s]);
            double q = fma(dk - x[s], p[s], -ek * pm[s]);
            if (fabs(q) < pivmin * fabs(p[s])) q = -pivmin * p[s];
            c[s] += (q < 0.0) != (p[s] < 0.0);
            pm[s] = p[s] * sc;
            p[s] = q * sc;
        }
    }
}

__device__ __forceinline__ double clamp_tiny(double x, double tiny) {
    return fabs(x) < tiny ? (x < 0.0 ? -tiny : tiny) : x;
}

}  // namespace dense
}  // namespace q3b
