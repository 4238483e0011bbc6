// Gamma-only H|psi> on half-sphere coefficient vectors.
//
// At k = 0 the reference stores a wavefunction that is real in real space by
// the half sphere of G (the origin first, one of each pair +G/-G), and applies
// H two bands at a time: band pair (a, b) is transformed as the one complex
// function a(r) + i b(r), whose coefficients are a(G) + i b(G) at +G and
// conj(a(G)) + i conj(b(G)) at -G, and the two results are separated by the
// +G/-G symmetry (hamiltonian_applicator/serial.hpp:283-418).  The nonlocal
// term is real there too: 2 Re(beta^H psi) over the half sphere less the
// origin's term (serial.hpp:519-566).
//
// Here the pair's full-sphere vector phi is built on the device and the
// full-sphere H|psi> of the prepared k-point (sticks/planes transforms,
// tensor-core projector GEMMs) is applied to the pairs: half the transforms
// of the bands, as in the reference.  Because the projectors of a Gamma-only
// k-point satisfy beta(-G) = conj(beta(G)), beta^H phi = x_a + i x_b with x_a,
// x_b the reference's real overlaps, and the separation of the results gives
// each band its own kinetic, local and nonlocal terms.  The origin is packed
// as (Re a(0), Re b(0)) and read back as (Re, Im), as in the reference.  A last
// band without a partner is packed alone (a at +G, conj(a) at -G, a(0) as is)
// and read from +G, the reference's single-band path (its origin read as the
// real part); its nonlocal term then uses a(0) as given, where the reference
// takes Re a(0) (the two agree for a state that is real in real space, whose
// a(0) is real).
#include "context.cuh"
#include "gamma.cuh"
#include "nonlocal.cuh"
#include "q3b.h"


using q3b::Context;

namespace {
template <typename F> int gamma_guarded(q3b_context* c, F&& f) {
    if (!c) return Q3B_ERR_INVALID;
    try {
        Q3B_CUDA(cudaSetDevice(c->impl.device));
        q3b::tc::ErrorScope scope(c->impl.err_word.as<int>());
        f(c->impl);
        return Q3B_OK;
    } catch (const std::exception& e) {
        return q3b::fail(c, e);
    }
}
}  // namespace

int q3b_prepare_kpoint_gamma(q3b_context* ctx, int npw_half, const int32_t* g2g, const int32_t* g2g_minus,
                             const double* ke, const q3b_cplx128* beta, int nproj, int natoms,
                             const int32_t* offs, const double* dblk) {
    return gamma_guarded(ctx, [&](Context& c) {
        if (npw_half <= 0 || !g2g || !g2g_minus || !ke)
            throw q3b::Status(Q3B_ERR_INVALID, "bad half-sphere plane-wave list");
        if (g2g[0] != g2g_minus[0])
            throw q3b::Status(Q3B_ERR_INVALID, "entry 0 of the half sphere must be the origin (its own -G)");
        if (nproj < 0 || (nproj > 0 && !beta)) throw q3b::Status(Q3B_ERR_INVALID, "bad projector set");
        const int nfull = 2 * npw_half - 1;
        std::vector<int32_t> gf(nfull);
        std::vector<double> kf(nfull);
        for (int h = 0; h < npw_half; ++h) {
            gf[h] = g2g[h];
            kf[h] = ke[h];
            if (h > 0) {
                // a G outside the grid takes its mirror out with it (serial.hpp:344-349)
                gf[npw_half - 1 + h] = g2g[h] >= 0 ? g2g_minus[h] : -1;
                kf[npw_half - 1 + h] = ke[h];
            }
        }
        std::vector<double2> bf;
        if (nproj > 0) {
            const auto* b = reinterpret_cast<const double2*>(beta);
            bf.resize((size_t)nfull * nproj);
            for (int j = 0; j < nproj; ++j) {
                const double2* src = b + (size_t)j * npw_half;
                double2* dst = bf.data() + (size_t)j * nfull;
                for (int h = 0; h < npw_half; ++h) {
                    dst[h] = src[h];
                    if (h > 0) dst[npw_half - 1 + h] = q3b::conj2(src[h]);  // beta(-G) = conj(beta(G))
                }
            }
        }
        c.prepare_kpoint(nfull, gf.data(), kf.data(), nproj ? bf.data() : nullptr, nproj, natoms, offs, dblk);
        c.gamma_half = npw_half;
    });
}

int q3b_apply_h_gamma(q3b_context* ctx, const q3b_cplx128* psi, q3b_cplx128* hpsi, int nvec, int precision) {
    return gamma_guarded(ctx, [&](Context& c) {
        c.require_ready();
        if (c.gamma_half <= 0) throw q3b::Status(Q3B_ERR_STATE, "the k-point was not prepared as Gamma-only");
        if (nvec < 0 || (nvec > 0 && (!psi || !hpsi))) throw q3b::Status(Q3B_ERR_INVALID, "bad vectors");
        if (nvec == 0) return;
        if (precision != Q3B_FP64 && precision != Q3B_MIXED) throw q3b::Status(Q3B_ERR_INVALID, "unknown precision");
        const int nhalf = c.gamma_half, nfull = c.kp.npw;
        const int npair = (nvec + 1) / 2;
        const size_t n = (size_t)nfull * npair;
        c.ws_gamma.reserve(&c, 2 * n * sizeof(double2));
        double2* phi = c.ws_gamma.as<double2>();
        double2* hphi = phi + n;
        const long work = (long)nhalf * npair;
        q3b::gamma_pack<<<q3b::gamma_blocks(work), 256, 0, c.stream>>>(
            nhalf, nvec, reinterpret_cast<const double2*>(psi), nhalf, phi, nfull);
        Q3B_LAUNCH_CHECK();
        if (precision == Q3B_FP64) {
            c.apply_h<double>(phi, nfull, hphi, nfull, npair);
        } else {
            c.ws_conv_in.reserve(&c, n * sizeof(float2));
            c.ws_conv_out.reserve(&c, n * sizeof(float2));
            q3b::convert<double, float>(c.stream, (long)n, phi, c.ws_conv_in.as<float2>());
            c.apply_h<float>(c.ws_conv_in.as<float2>(), nfull, c.ws_conv_out.as<float2>(), nfull, npair);
            q3b::convert<float, double>(c.stream, (long)n, c.ws_conv_out.as<float2>(), hphi);
        }
        q3b::gamma_unpack<<<q3b::gamma_blocks(work), 256, 0, c.stream>>>(
            nhalf, nvec, hphi, nfull, reinterpret_cast<double2*>(hpsi), nhalf);
        Q3B_LAUNCH_CHECK();
    });
}

// The ultrasoft overlap operator on a Gamma-only k-point (ultrasoft/init.hpp:
// 212-270 forms the real overlaps 2 Re(beta^H psi) less the origin's term):
// the band pairs through S psi = psi + beta Q beta^H psi of the full-sphere
// plan, separated as for H.
int q3b_apply_s_gamma(q3b_context* ctx, const q3b_cplx128* psi, q3b_cplx128* spsi, int nvec, int precision) {
    return gamma_guarded(ctx, [&](Context& c) {
        c.require_ready();
        if (c.gamma_half <= 0) throw q3b::Status(Q3B_ERR_STATE, "the k-point was not prepared as Gamma-only");
        if (nvec < 0 || (nvec > 0 && (!psi || !spsi))) throw q3b::Status(Q3B_ERR_INVALID, "bad vectors");
        if (nvec == 0) return;
        const int nhalf = c.gamma_half, nfull = c.kp.npw;
        const int npair = (nvec + 1) / 2;
        const size_t n = (size_t)nfull * npair;
        c.ws_gamma.reserve(&c, 2 * n * sizeof(double2));
        double2* phi = c.ws_gamma.as<double2>();
        double2* sphi = phi + n;
        const long work = (long)nhalf * npair;
        q3b::gamma_pack<<<q3b::gamma_blocks(work), 256, 0, c.stream>>>(
            nhalf, nvec, reinterpret_cast<const double2*>(psi), nhalf, phi, nfull);
        Q3B_LAUNCH_CHECK();
        q3b::apply_s_device(c, phi, sphi, npair, precision);
        q3b::gamma_unpack<<<q3b::gamma_blocks(work), 256, 0, c.stream>>>(
            nhalf, nvec, sphi, nfull, reinterpret_cast<double2*>(spsi), nhalf);
        Q3B_LAUNCH_CHECK();
    });
}
