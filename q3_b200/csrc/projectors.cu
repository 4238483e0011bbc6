// Kleinman-Bylander projector set of a k-point, built on the device.
//
// compute_kleinman_bylander_projectors (pseudopotential/planewave/internal/
// projector.hpp:42-199; the device form is projector_set_builder_gpu.hpp):
//
//   beta_{a,i,m}(G) = Omega^{-1/2} (-i)^l  f_i(|k+G|)  Y_lm(k+G)  exp(-i (k+G).r_a)
//
// f_i: the species' beta function, 4-point Lagrange on a uniform q table
// (math/interpolation/lagrange.hpp:31-47, uniform_q_grid_table.hpp:54-63);
// Y_lm: real spherical harmonics with the Condon-Shortley phase, from the
// normalised associated-Legendre recursion (math/spherical/harmonics.hpp:
// 217-330); projectors atom by atom, beta by beta, m = 0, 1, -1, 2, -2, ...
// One thread per plane wave and projector chunk: its Y_lm once, the phase once
// per atom, the radial value once per beta; writes are coalesced along G.  The
// matrix then goes into the k-point's plan like a host-supplied one, so a
// k-point's projectors never cross the bus.
#include <algorithm>
#include <cmath>
#include <vector>

#include "context.cuh"
#include "q3b.h"

namespace q3b {
namespace {

constexpr int kMaxL = 4;                        // l <= 4
constexpr int kMaxLM = (kMaxL + 1) * (kMaxL + 1);
constexpr int kProjectorsPerBlock = 64;

__device__ __forceinline__ int lm_index(int l, int m) {
    return m == 0 ? l * l : (m > 0 ? l * l + 2 * m - 1 : l * l - 2 * m);
}

// harmonics.hpp:262-329 for one vector
__device__ void real_ylm(int lmax, double vx, double vy, double vz, double* y) {
    const double g = sqrt(vx * vx + vy * vy + vz * vz);
    const bool degenerate = g < 1e-9;
    const double ct = degenerate ? 0.0 : vz / g;
    const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
    const double phi = degenerate ? copysign(3.14159265358979323846 / 2.0, vy) : atan2(vy, vx);
    double q[(kMaxL + 1) * (kMaxL + 2) / 2];
    auto qi = [](int l, int m) { return l * (l + 1) / 2 + m; };
    q[0] = 1.0;
    if (lmax >= 1) {
        q[qi(1, 0)] = ct;
        q[qi(1, 1)] = -st / sqrt(2.0);
    }
    for (int l = 2; l <= lmax; ++l) {
        for (int m = 0; m <= l - 2; ++m) {
            const double den = sqrt(static_cast<double>(l * l - m * m));
            q[qi(l, m)] = ct * (2 * l - 1) / den * q[qi(l - 1, m)] -
                          sqrt(static_cast<double>((l - 1) * (l - 1) - m * m)) / den * q[qi(l - 2, m)];
        }
        const double diag = sqrt(static_cast<double>(2 * l - 1));
        const double prev = q[qi(l - 1, l - 1)];
        q[qi(l, l - 1)] = ct * diag * prev;
        q[qi(l, l)] = -diag / sqrt(static_cast<double>(2 * l)) * st * prev;
    }
    const double four_pi = 4.0 * 3.14159265358979323846;
    y[0] = q[0] / sqrt(four_pi);
    for (int l = 1; l <= lmax; ++l) {
        const double norm = sqrt(static_cast<double>(2 * l + 1) / four_pi);
        y[lm_index(l, 0)] = norm * q[qi(l, 0)];
        const double off = norm * sqrt(2.0);
        for (int m = 1; m <= l; ++m) {
            const double v = q[qi(l, m)];
            y[lm_index(l, m)] = off * v * cos(m * phi);
            y[lm_index(l, -m)] = off * v * sin(m * phi);
        }
    }
}

// uniform_q_grid_table.hpp:54-63 with lagrange.hpp:31-47
__device__ __forceinline__ double interpolate(const double* t, int nq, double q, double dq) {
    if (nq <= 0) return 0.0;
    if (q < 1e-10) return t[0];
    const double f = q / dq;
    const int b = static_cast<int>(f);
    const double x = f - b;
    if (b + 3 >= nq) return 0.0;
    const double w1 = 1.0 - x, w2 = 2.0 - x, w3 = 3.0 - x;
    return t[b] * w1 * w2 * w3 / 6.0 + t[b + 1] * x * w2 * w3 / 2.0 - t[b + 2] * x * w1 * w3 / 2.0 +
           t[b + 3] * x * w1 * w2 / 6.0;
}

// projector p: atom, table offset (species, beta), l, lm slot
struct ProjectorMap {
    const int* atom;
    const int* table;
    const int* l;
    const int* lm;
};

__global__ void __launch_bounds__(128)
build_projectors(int npw, const double* __restrict__ kpg, int lmax, double inv_sqrt_volume,
                 const double* __restrict__ pos, int nproj, ProjectorMap map, const double* __restrict__ tables,
                 int nq, double dq, double2* beta) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= npw) return;
    const double vx = kpg[3 * g], vy = kpg[3 * g + 1], vz = kpg[3 * g + 2];
    double y[kMaxLM];
    real_ylm(lmax, vx, vy, vz, y);
    const double q = sqrt(vx * vx + vy * vy + vz * vz);
    const int p0 = blockIdx.y * kProjectorsPerBlock, p1 = min(nproj, p0 + kProjectorsPerBlock);
    int atom = -1, tab = -1;
    double2 sf = mk(0.0, 0.0);
    double radial = 0.0;
    for (int p = p0; p < p1; ++p) {
        const int a = map.atom[p];
        if (a != atom) {
            atom = a;
            double s, c;
            sincos(vx * pos[3 * a] + vy * pos[3 * a + 1] + vz * pos[3 * a + 2], &s, &c);
            sf = mk(c, -s);                                   // exp(-i (k+G).r)
        }
        if (map.table[p] != tab) {
            tab = map.table[p];
            radial = interpolate(tables + (size_t)tab * nq, nq, q, dq);
        }
        const int l = map.l[p];
        const double r = radial * y[map.lm[p]];
        const double2 ang = (l & 3) == 0 ? mk(1.0, 0.0)
                          : (l & 3) == 1 ? mk(0.0, -1.0)
                          : (l & 3) == 2 ? mk(-1.0, 0.0) : mk(0.0, 1.0);  // (-i)^l
        const double2 pre = mk(inv_sqrt_volume * ang.x, inv_sqrt_volume * ang.y);
        beta[(size_t)p * npw + g] = cmul(mk(r * sf.x, r * sf.y), pre);
    }
}

}  // namespace
}  // namespace q3b

extern "C" int q3b_prepare_kpoint_build(q3b_context* ctx, int npw, const int32_t* g_to_grid, const double* ke,
                                        const double* kpg_cart, double cell_volume, int natoms,
                                        const double* positions, const int32_t* species_of_atom, int nspecies,
                                        const int32_t* nbeta_of_species, const int32_t* beta_l, int nq, double dq,
                                        const double* beta_tables, const double* d_blocks) {
    if (!ctx) return Q3B_ERR_INVALID;
    q3b::Context& c = ctx->impl;
    try {
        Q3B_CUDA(cudaSetDevice(c.device));
        q3b::tc::ErrorScope scope(c.err_word.as<int>());
        if (npw <= 0 || !kpg_cart || !(cell_volume > 0.0) || natoms < 0 || nspecies < 0 || nq < 0 ||
            (natoms > 0 && (!positions || !species_of_atom || !d_blocks)) || (nspecies > 0 && !nbeta_of_species) ||
            (nq > 0 && !(dq > 0.0)))
            throw q3b::Status(Q3B_ERR_INVALID, "q3b_prepare_kpoint_build: bad arguments");
        // projector map: atoms in order, their species' betas in order, m = 0, 1, -1, ...
        std::vector<int> beta_first(nspecies + 1, 0);
        for (int s = 0; s < nspecies; ++s) {
            if (nbeta_of_species[s] < 0) throw q3b::Status(Q3B_ERR_INVALID, "negative beta count");
            beta_first[s + 1] = beta_first[s] + nbeta_of_species[s];
        }
        if (beta_first[nspecies] > 0 && (!beta_l || !beta_tables))
            throw q3b::Status(Q3B_ERR_INVALID, "q3b_prepare_kpoint_build: beta functions missing");
        std::vector<int> patom, ptab, pl, plm, offs(1, 0);
        int lmax = 0;
        for (int a = 0; a < natoms; ++a) {
            const int s = species_of_atom[a];
            if (s < 0 || s >= nspecies) throw q3b::Status(Q3B_ERR_INVALID, "species index out of range");
            for (int i = beta_first[s]; i < beta_first[s + 1]; ++i) {
                const int l = beta_l[i];
                if (l < 0 || l > q3b::kMaxL) throw q3b::Status(Q3B_ERR_INVALID, "beta angular momentum above 4");
                lmax = std::max(lmax, l);
                for (int k = 0; k <= 2 * l; ++k) {
                    const int m = k == 0 ? 0 : ((k & 1) ? (k + 1) / 2 : -(k / 2));
                    patom.push_back(a);
                    ptab.push_back(i);
                    pl.push_back(l);
                    plm.push_back(m == 0 ? l * l : (m > 0 ? l * l + 2 * m - 1 : l * l - 2 * m));
                }
            }
            offs.push_back(static_cast<int>(patom.size()));
        }
        const int nproj = static_cast<int>(patom.size());
        if (nproj == 0) {
            c.prepare_kpoint(npw, g_to_grid, ke, nullptr, 0, 0, nullptr, nullptr);
            return Q3B_OK;
        }
        const size_t ntab = (size_t)beta_first[nspecies] * nq;
        // device staging: inputs, the map and the matrix, in one buffer
        auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
        const size_t b_kpg = al((size_t)npw * 3 * sizeof(double)), b_pos = al((size_t)natoms * 3 * sizeof(double));
        const size_t b_tab = al(std::max<size_t>(ntab, 1) * sizeof(double)), b_map = al((size_t)nproj * sizeof(int));
        const size_t b_beta = al((size_t)npw * nproj * sizeof(double2));
        c.ws_tune.reserve(&c, b_kpg + b_pos + b_tab + 4 * b_map + b_beta);
        char* base = c.ws_tune.as<char>();
        double* d_kpg = reinterpret_cast<double*>(base);
        double* d_pos = reinterpret_cast<double*>(base + b_kpg);
        double* d_tab = reinterpret_cast<double*>(base + b_kpg + b_pos);
        int* d_map = reinterpret_cast<int*>(base + b_kpg + b_pos + b_tab);
        double2* d_beta = reinterpret_cast<double2*>(base + b_kpg + b_pos + b_tab + 4 * b_map);
        const size_t mstride = b_map / sizeof(int);
        Q3B_CUDA(cudaMemcpyAsync(d_kpg, kpg_cart, (size_t)npw * 3 * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        Q3B_CUDA(cudaMemcpyAsync(d_pos, positions, (size_t)natoms * 3 * sizeof(double), cudaMemcpyHostToDevice,
                                 c.stream));
        if (ntab) Q3B_CUDA(cudaMemcpyAsync(d_tab, beta_tables, ntab * sizeof(double), cudaMemcpyHostToDevice, c.stream));
        const std::vector<int>* parts[4] = {&patom, &ptab, &pl, &plm};
        for (int k = 0; k < 4; ++k)
            Q3B_CUDA(cudaMemcpyAsync(d_map + k * mstride, parts[k]->data(), (size_t)nproj * sizeof(int),
                                     cudaMemcpyHostToDevice, c.stream));
        const q3b::ProjectorMap map{d_map, d_map + mstride, d_map + 2 * mstride, d_map + 3 * mstride};
        const dim3 grid(q3b::ceil_div(npw, 128), q3b::ceil_div(nproj, q3b::kProjectorsPerBlock));
        q3b::build_projectors<<<grid, 128, 0, c.stream>>>(npw, d_kpg, lmax, 1.0 / std::sqrt(cell_volume), d_pos,
                                                         nproj, map, d_tab, nq, dq, d_beta);
        Q3B_LAUNCH_CHECK();
        c.prepare_kpoint(npw, g_to_grid, ke, d_beta, nproj, natoms, offs.data(), d_blocks, true);
        c.ws_tune.release();
        return Q3B_OK;
    } catch (const std::exception& e) {
        return q3b::fail(ctx, e);
    }
}

extern "C" int q3b_get_projectors(q3b_context* ctx, q3b_cplx128* beta_dev, int* nproj) {
    if (!ctx) return Q3B_ERR_INVALID;
    q3b::Context& c = ctx->impl;
    try {
        Q3B_CUDA(cudaSetDevice(c.device));
        q3b::tc::ErrorScope scope(c.err_word.as<int>());
        c.require_ready();
        if (nproj) *nproj = c.kp.nproj;
        if (beta_dev && c.kp.nproj > 0) {
            Q3B_CUDA(cudaMemcpyAsync(beta_dev, c.kp.beta64.ptr, (size_t)c.kp.npw * c.kp.nproj * sizeof(double2),
                                     cudaMemcpyDeviceToDevice, c.stream));
            Q3B_CUDA(cudaStreamSynchronize(c.stream));
        }
        return Q3B_OK;
    } catch (const std::exception& e) {
        return q3b::fail(ctx, e);
    }
}
