// Band pairs of a Gamma-only k-point as full-sphere vectors (see gamma.cu):
// pair p = bands (2p, 2p+1) of half-sphere vectors (npw_half each, the origin
// at entry 0) becomes one vector of the full-sphere plan, +G of half entry h
// at h and -G at nhalf-1+h.
#pragma once

#include "common.cuh"

namespace q3b {

template <typename T>
__global__ void gamma_pack(int nhalf, int nvec, const T* __restrict__ psi, long ldpsi, T* __restrict__ phi,
                           long ldphi) {
    const int npair = (nvec + 1) / 2;
    const long total = (long)nhalf * npair;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        const int h = static_cast<int>(idx % nhalf), p = static_cast<int>(idx / nhalf);
        const int b1 = 2 * p, b2 = 2 * p + 1;
        const T a = psi[h + (long)b1 * ldpsi];
        T* out = phi + (long)p * ldphi;
        if (b2 < nvec) {
            const T b = psi[h + (long)b2 * ldpsi];
            if (h == 0) {
                out[0] = mk(a.x, b.x);                           // (Re a(0), Re b(0))
            } else {
                out[h] = mk(a.x - b.y, a.y + b.x);               // a + i b
                out[nhalf - 1 + h] = mk(a.x + b.y, b.x - a.y);   // conj(a) + i conj(b)
            }
        } else {
            out[h] = a;
            if (h > 0) out[nhalf - 1 + h] = conj2(a);
        }
    }
}

// a = (F(+G) + conj F(-G)) / 2, b = -i (F(+G) - conj F(-G)) / 2; at the
// origin (Re F, Im F); a band without a partner reads F(+G), and the real part
// of F at the origin (the reference keeps F(0) as computed, which is real for
// a state that is real in real space up to rounding; an imaginary rounding
// residue there would leave the half-sphere space, on which the pair packing
// sees only Re psi(0))
template <typename T>
__global__ void gamma_unpack(int nhalf, int nvec, const T* __restrict__ F, long ldf, T* __restrict__ hpsi,
                             long ldh) {
    using R = decltype(T{}.x);
    const int npair = (nvec + 1) / 2;
    const long total = (long)nhalf * npair;
    for (long idx = blockIdx.x * (long)blockDim.x + threadIdx.x; idx < total;
         idx += (long)gridDim.x * blockDim.x) {
        const int h = static_cast<int>(idx % nhalf), p = static_cast<int>(idx / nhalf);
        const int b1 = 2 * p, b2 = 2 * p + 1;
        const T* f = F + (long)p * ldf;
        const T fp = f[h];
        if (b2 < nvec) {
            if (h == 0) {
                hpsi[(long)b1 * ldh] = mk(fp.x, R(0));
                hpsi[(long)b2 * ldh] = mk(fp.y, R(0));
            } else {
                const T fm = conj2(f[nhalf - 1 + h]);
                const T s = mk(R(0.5) * (fp.x + fm.x), R(0.5) * (fp.y + fm.y));
                const T d = mk(R(0.5) * (fp.x - fm.x), R(0.5) * (fp.y - fm.y));
                hpsi[h + (long)b1 * ldh] = s;
                hpsi[h + (long)b2 * ldh] = mk(d.y, -d.x);
            }
        } else {
            hpsi[h + (long)b1 * ldh] = h == 0 ? mk(fp.x, R(0)) : fp;
        }
    }
}

// keep half-sphere vectors in the space the pair packing represents: a real
// origin coefficient
template <typename T>
__global__ void gamma_real_origin(int ncols, T* V, long ldv) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < ncols; j += gridDim.x * blockDim.x) V[(long)j * ldv].y = 0;
}

inline int gamma_blocks(long n) { return stride_grid(n, 16); }

}  // namespace q3b
