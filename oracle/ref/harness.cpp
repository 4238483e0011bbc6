// Test-oracle harness: runs the reference's own CPU H|psi> and Davidson on a
// synthetic cell and writes every input and output as raw little-endian arrays.
//
// This file is test infrastructure.  It is compiled against the reference's
// header-only sources (oracle/ref/Makefile), never shipped, and only the fixture
// scripts under tests/golden/ and the CPU baseline of bench.py run it.
//
// What it drives (all reference code, unmodified):
//   * Crystal, PlanewaveBasis::generate, PlanewaveBasis::compute_gk
//     (src/layer_1_structure/crystal/crystal.hpp, src/layer_3_representation/basis/planewave/init.hpp:60-108,191-206);
//   * NormConservingPlanewaveKohnShamQuantumSystem::init over an in-memory species
//     (quantum_system/kohn_sham/planewave/norm_conserving/init.hpp:50-56);
//   * SerialProjectorSetBuilder (the projector matrix of a k-point, as
//     ProjectorSetProvider builds it, diagonalizer/planewave/internal/projector_set_provider.hpp:47-64);
//   * SerialPlanewaveHamiltonianApplicator::update_potential / prepare_kpoint / apply_batch
//     (hamiltonian_applicator/serial.hpp:64-153,440-700);
//   * PlanewaveDavidsonDiagonalizer::solve (diagonalizer/planewave/davidson.hpp:324-841).
//
// The FFT grids are forced to the case's N1 x N2 x N3 (a grid factory whose grids ignore the
// sizer).  The density grid is the same grid unless the case names a larger one
// ("density_grid D1 D2 D3"); V(r) is then given on that grid and update_potential restricts
// it to the wavefunction grid (serial.hpp:64-78, planewave_potential_utils.hpp:33-135).
//
// The species: beta_l(r) = r^l exp(-r^2/w^2) given as r*beta on a logarithmic radial mesh,
// D diagonal (Ry); the reference tabulates beta(q) by its own spherical Bessel transform.
//
// Usage: harness CASE_FILE OUT_DIR
// The case file is "key value..." lines (oracle/ref/run.py, write_case, writes them).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <map>
#include <memory>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "layer_0_core/math/transform/spherical_bessel.hpp"
#include "layer_1_structure/crystal/crystal.hpp"
#include "layer_1_structure/reciprocal_space/kpoints_grid.hpp"
#include "layer_3_representation/basis/planewave/init.hpp"
#include "layer_3_representation/pseudopotential/set.hpp"
#include "layer_3_representation/pseudopotential/planewave/projector_set_builder_serial.hpp"
#include "layer_3_representation/quantum_system/kohn_sham/planewave/norm_conserving/init.hpp"
#include "layer_4_computation/diagonalizer/planewave/davidson.hpp"
#include "layer_4_computation/diagonalizer/planewave/internal/hamiltonian_applicator/serial.hpp"
#include "layer_0_core/execution/serial.hpp"
#include "layer_3_representation/basis/planewave/internal/fft/fft_grid_factory.hpp"

using namespace q3;

namespace {

// ------------------------------------------------------------------ case file

struct Case {
    std::map<std::string, std::vector<std::string>> kv;
    const std::vector<std::string>& at(const std::string& k) const {
        auto it = kv.find(k);
        if (it == kv.end()) throw std::runtime_error("case file lacks key: " + k);
        return it->second;
    }
    bool has(const std::string& k) const { return kv.count(k) != 0; }
    double num(const std::string& k, int i = 0) const { return std::stod(at(k).at(i)); }
    int integer(const std::string& k, int i = 0) const { return std::stoi(at(k).at(i)); }
    std::string str(const std::string& k) const { return at(k).at(0); }
};

Case read_case(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open " + path);
    Case c;
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream ss(line);
        std::string key, tok;
        ss >> key;
        std::vector<std::string> vals;
        while (ss >> tok) vals.push_back(tok);
        // repeated keys (atom, kpoint, beta) append rows
        auto& slot = c.kv[key];
        slot.insert(slot.end(), vals.begin(), vals.end());
    }
    return c;
}

template <typename T> void write_array(const std::string& path, const T* data, std::size_t count) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + path);
    if (count && std::fwrite(data, sizeof(T), count, f) != count) throw std::runtime_error("short write " + path);
    std::fclose(f);
}

template <typename T> std::vector<T> read_array(const std::string& path, std::size_t count) {
    std::vector<T> out(count);
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot read " + path);
    if (count && std::fread(out.data(), sizeof(T), count, f) != count) throw std::runtime_error("short read " + path);
    std::fclose(f);
    return out;
}

// --------------------------------------------------------- forced FFT grids

// The wavefunction grid n1 x n2 x n3 and the density grid d1 x d2 x d3 (the same
// unless the case names a larger one: update_potential then restricts V(r) from
// the density grid to the wavefunction grid, serial.hpp:64-78, 853-870).
class ForcedGridFactory : public FFTGridFactory {
  public:
    ForcedGridFactory(int n1, int n2, int n3, int d1, int d2, int d3)
        : n1_(n1), n2_(n2), n3_(n3), d1_(d1), d2_(d2), d3_(d3) {}
    std::unique_ptr<FFTGrid> create_fft_grid() const override {
        return std::make_unique<Forced>(n1_, n2_, n3_);
    }
    std::unique_ptr<FFTGrid> create_density_fft_grid() const override {
        return std::make_unique<Forced>(d1_, d2_, d3_);
    }

  private:
    class Forced : public SerialFFTGrid {
      public:
        Forced(int n1, int n2, int n3) : n1_(n1), n2_(n2), n3_(n3) {}
        void init(int, int, int, bool planning = false) override {
            SerialFFTGrid::init(n1_, n2_, n3_, planning);
        }
      private:
        int n1_, n2_, n3_;
    };
    int n1_, n2_, n3_, d1_, d2_, d3_;
};

// ------------------------------------------------------- synthetic species

std::unique_ptr<Pseudopotential> make_species(const Case& c) {
    auto pp = std::make_unique<Pseudopotential>();
    pp->element = "X";
    pp->pseudopotential_type = "NC";
    pp->xc_functional = "PZ";
    pp->valence_charge = c.num("valence");
    // logarithmic mesh r_i = exp(xmin + i dx), dr/di = r_i dx
    const double xmin = c.num("mesh", 0), dx = c.num("mesh", 1);
    const int mesh = c.integer("mesh", 2);
    const double width = c.num("beta_width");
    const double rcut = c.num("beta_rcut");
    pp->mesh_size = mesh;
    pp->radial_grid.resize(mesh);
    pp->radial_grid_derivative.resize(mesh);
    for (int i = 0; i < mesh; ++i) {
        double r = std::exp(xmin + i * dx);
        pp->radial_grid[i] = r;
        pp->radial_grid_derivative[i] = r * dx;
    }
    int kkbeta = mesh;
    for (int i = 0; i < mesh; ++i)
        if (pp->radial_grid[i] > rcut) { kkbeta = i; break; }
    if (kkbeta % 2 == 0) kkbeta += 1;  // Simpson wants an odd count
    kkbeta = std::min(kkbeta, mesh);
    const auto& ls = c.at("beta_l");
    const auto& ds = c.at("beta_d");
    const int nbeta = static_cast<int>(ls.size());
    pp->number_of_projectors = nbeta;
    int lmax = 0;
    for (int b = 0; b < nbeta; ++b) {
        Projector p;
        p.angular_momentum = std::stoi(ls[b]);
        lmax = std::max(lmax, p.angular_momentum);
        p.number_of_radial_cutoff_points = kkbeta;
        p.radial_values.assign(mesh, 0.0);
        for (int i = 0; i < kkbeta; ++i) {
            double r = pp->radial_grid[i];
            p.radial_values[i] = std::pow(r, p.angular_momentum + 1) * std::exp(-(r * r) / (width * width));
        }
        pp->projectors.push_back(std::move(p));
    }
    pp->maximum_angular_momentum = lmax;
    pp->d_ion_matrix.assign(nbeta, std::vector<Real>(nbeta, 0.0));
    for (int b = 0; b < nbeta; ++b) pp->d_ion_matrix[b][b] = std::stod(ds[b]);
    // The local part is handed to the applicator as V(r); the species' own V_loc(r) and
    // atomic charge only feed tables this harness never reads.  Smooth placeholders.
    pp->potential_local.radial_values.resize(mesh);
    pp->charge_atomic.radial_values.resize(mesh);
    for (int i = 0; i < mesh; ++i) {
        double r = pp->radial_grid[i];
        pp->potential_local.radial_values[i] = -2.0 * pp->valence_charge * std::erf(r) / r;
        pp->charge_atomic.radial_values[i] = pp->valence_charge * 4.0 * r * r * std::exp(-r * r) / std::sqrt(M_PI);
    }
    pp->has_nonlinear_core_correction = false;
    pp->number_of_wavefunctions = 0;
    return pp;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s CASE_FILE OUT_DIR\n", argv[0]);
        return 2;
    }
    try {
        const Case c = read_case(argv[1]);
        const std::string out = argv[2];
        const int n1 = c.integer("grid", 0), n2 = c.integer("grid", 1), n3 = c.integer("grid", 2);
        const double alat = c.num("alat");
        const bool dense = c.has("density_grid");
        const int d1 = dense ? c.integer("density_grid", 0) : n1, d2 = dense ? c.integer("density_grid", 1) : n2,
                  d3 = dense ? c.integer("density_grid", 2) : n3;
        ForcedGridFactory grids(n1, n2, n3, d1, d2, d3);

        // --- crystal: lattice rows in bohr, atoms fractional, one species
        Crystal crystal;
        crystal.set_from_lattice_type(1, alat);
        Matrix3x3 lat;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) lat[i][j] = c.num("lattice", 3 * i + j) / alat;
        crystal.set_lattice(lat);
        PseudopotentialSet pp_set;
        pp_set.push_back(make_species(c));
        crystal.add_species({"X", 28.0, pp_set[0].valence_charge, "synthetic"});
        const auto& atoms = c.at("atom");
        const int natoms = static_cast<int>(atoms.size() / 3);
        for (int a = 0; a < natoms; ++a)
            crystal.add_atom({0, {std::stod(atoms[3 * a]), std::stod(atoms[3 * a + 1]), std::stod(atoms[3 * a + 2])}});
        crystal.compute_derived_quantities();

        // --- basis
        const double ecut = c.num("ecutwfc");
        PlanewaveBasis basis;
        basis.generate(grids, crystal, ecut, 4.0 * ecut, /*is_gamma_only=*/false,
                       /*use_measured_fft_planning=*/false);
        if (basis.fft_wave().grid_dimension_1() != n1 || basis.fft_wave().grid_dimension_3() != n3)
            throw std::runtime_error("the FFT grid was not forced");

        NormConservingPlanewaveKohnShamQuantumSystem system;
        system.init(crystal, basis, pp_set);
        const auto& nc_basis = system.pseudopotential_basis();

        // --- k-points (reciprocal-lattice coordinates)
        const auto& kv = c.at("kpoint");
        const int nk = static_cast<int>(kv.size() / 3);
        KPointsGrid kgrid;
        for (int k = 0; k < nk; ++k) {
            KPoint kp;
            kp.coordinates = {std::stod(kv[3 * k]), std::stod(kv[3 * k + 1]), std::stod(kv[3 * k + 2])};
            kp.weight = 2.0 / nk;
            kgrid.add_kpoint(kp);
        }

        // --- potential V(r), flat (i1*N2 + i2)*N3 + i3, Ry
        const std::size_t N = static_cast<std::size_t>(n1) * n2 * n3;
        // V(r) on the density grid, flat (i1*D2 + i2)*D3 + i3
        std::vector<Real> v_r = read_array<double>(c.str("potential"), static_cast<std::size_t>(d1) * d2 * d3);

        // --- beta(q) tables exactly as the reference tabulates them
        {
            const auto& table = nc_basis.beta_function_table();
            std::vector<Real> q = table.q_grid().q_point_values();
            const auto& pp = pp_set[0];
            std::vector<double> all;
            for (int b = 0; b < pp.number_of_projectors; ++b) {
                std::vector<Real> f;
                transform_spherical_bessel(pp.radial_grid, pp.radial_grid_derivative,
                                           pp.projectors[b].radial_values, pp.projectors[b].angular_momentum,
                                           pp.projectors[b].number_of_radial_cutoff_points, q, f);
                // the interpolant is defined below the last three nodes (lagrange.hpp:38-39)
                for (std::size_t j = 0; j + 3 < q.size(); ++j) {
                    if (std::abs(f[j] - table.interpolate(0, b, q[j])) > 1e-12 * (1.0 + std::abs(f[j])))
                        throw std::runtime_error("beta table does not reproduce");
                }
                all.insert(all.end(), f.begin(), f.end());
            }
            write_array(out + "/beta_tables.f64", all.data(), all.size());
            double meta[3] = {table.q_spacing(), static_cast<double>(q.size()), crystal.cell_volume()};
            write_array(out + "/beta_meta.f64", meta, 3);
        }

        // per-k plane waves, maps, projectors, D blocks
        std::vector<std::vector<int>> gidx(nk);
        std::vector<std::vector<Real>> ke(nk);
        std::vector<int> npw_of(nk);
        for (int k = 0; k < nk; ++k) {
            basis.compute_gk(kgrid[k].coordinates, crystal, gidx[k], ke[k]);
            npw_of[k] = static_cast<int>(gidx[k].size());
        }
        write_array(out + "/npw.i32", npw_of.data(), npw_of.size());

        const int nb = c.integer("nbands");
        const std::string mode = c.str("mode");
        execution::SerialExecutionPolicy exec;

        SerialPlanewaveHamiltonianApplicator applicator(crystal, basis, kgrid, system, exec);
        applicator.update_potential(v_r);

        // per-atom D blocks through the same accessor the applicator uses (serial.hpp:610-647)
        std::vector<double> dblocks;
        std::vector<int> offsets{0};
        for (int a = 0; a < crystal.number_of_atoms(); ++a) {
            int s = crystal.species_type_index(a);
            int m = nc_basis.number_of_projector_channels(s);
            for (int j = 0; j < m; ++j)
                for (int i = 0; i < m; ++i) dblocks.push_back(system.d_matrix_element(a, s, i, j, 0));
            offsets.push_back(offsets.back() + m);
        }
        write_array(out + "/d_blocks.f64", dblocks.data(), dblocks.size());
        write_array(out + "/atom_offsets.i32", offsets.data(), offsets.size());
        // scaled potential V/N as the applicator holds it
        write_array(out + "/v_scaled.f64", applicator.cached_scaled_potential().data(), N);

        const bool dump_projectors = c.has("dump_projectors") && c.integer("dump_projectors") != 0;
        for (int k = 0; k < nk; ++k) {
            const std::string tag = out + "/k" + std::to_string(k);
            std::vector<int> miller(3 * static_cast<std::size_t>(npw_of[k]));
            std::vector<double> kpg(3 * static_cast<std::size_t>(npw_of[k]));
            const auto& gv = basis.g_vectors();
            const auto& b = crystal.reciprocal_lattice_vectors();
            const double tpiba = crystal.two_pi_over_lattice_parameter();
            const auto& kc = kgrid[k].coordinates;
            for (int g = 0; g < npw_of[k]; ++g) {
                const auto& G = gv[gidx[k][g]];
                miller[3 * g] = static_cast<int>(std::lround(G.miller.x));
                miller[3 * g + 1] = static_cast<int>(std::lround(G.miller.y));
                miller[3 * g + 2] = static_cast<int>(std::lround(G.miller.z));
                for (int d = 0; d < 3; ++d)
                    kpg[3 * g + d] = tpiba * ((G.miller.x + kc.x) * b[0][d] + (G.miller.y + kc.y) * b[1][d] +
                                              (G.miller.z + kc.z) * b[2][d]);
            }
            write_array(tag + "_miller.i32", miller.data(), miller.size());
            write_array(tag + "_kpg.f64", kpg.data(), kpg.size());
            write_array(tag + "_ke.f64", ke[k].data(), ke[k].size());
            applicator.prepare_kpoint(k, npw_of[k], gidx[k], ke[k]);
            write_array(tag + "_g_to_grid.i32", applicator.g_to_fft_mapping().data(), npw_of[k]);
            if (dump_projectors) {
                KleinmanBylanderProjectorSet set;
                SerialProjectorSetBuilder builder(crystal, basis, nc_basis);
                builder.build(kc, gidx[k], npw_of[k], set);
                const std::size_t P = static_cast<std::size_t>(set.number_of_projectors());
                write_array(tag + "_beta.c128", reinterpret_cast<const double*>(set.host()),
                            2 * P * static_cast<std::size_t>(npw_of[k]));
            }
        }
        {
            std::vector<double> tau(3 * static_cast<std::size_t>(natoms));
            for (int a = 0; a < natoms; ++a) {
                Vector3D r = crystal.convert_from_crystal_to_cartesian(a);  // units of alat
                tau[3 * a] = r.x * alat; tau[3 * a + 1] = r.y * alat; tau[3 * a + 2] = r.z * alat;
            }
            write_array(out + "/positions.f64", tau.data(), tau.size());
        }

        // starting vectors: given per k (npw x nvec, column-major) as psi files
        if (mode == "hpsi" || mode == "both") {
            const int nvec = c.integer("hpsi_vectors");
            for (int k = 0; k < nk; ++k) {
                const std::string tag = out + "/k" + std::to_string(k);
                auto psi = read_array<Complex>(tag + "_psi.c128", static_cast<std::size_t>(npw_of[k]) * nvec);
                std::vector<Complex> hpsi(psi.size());
                applicator.prepare_kpoint(k, npw_of[k], gidx[k], ke[k]);
                // wall time of each application (the CPU baseline reads these)
                const int repeats = c.has("hpsi_repeats") ? c.integer("hpsi_repeats") : 1;
                std::vector<double> ms(repeats);
                for (int r = 0; r < repeats; ++r) {
                    auto t0 = std::chrono::steady_clock::now();
                    applicator.apply_batch(psi.data(), hpsi.data(), nvec);
                    auto t1 = std::chrono::steady_clock::now();
                    ms[r] = std::chrono::duration<double, std::milli>(t1 - t0).count();
                }
                write_array(tag + "_hpsi.c128", hpsi.data(), hpsi.size());
                write_array(tag + "_hpsi_ms.f64", ms.data(), ms.size());
            }
        }
        if (mode == "davidson" || mode == "both") {
            const double tol = c.num("tolerance");
            const int max_iter = c.integer("max_iterations");
            system.set_number_of_bands(nb);
            system.set_kpoint_grid(&kgrid);
            system.set_basis(&basis);
            system.set_number_of_electrons(2.0 * nb);  // every band occupied: the tight tolerance
            system.allocate_electronic_states(npw_of);
            std::vector<int> kset;
            for (const auto& s : c.at("davidson_kpoints")) kset.push_back(std::stoi(s));
            for (int k : kset) {
                const std::string tag = out + "/k" + std::to_string(k);
                auto psi0 = read_array<Complex>(tag + "_psi0.c128", static_cast<std::size_t>(npw_of[k]) * nb);
                std::copy(psi0.begin(), psi0.end(), system.mutable_band_block(k));
                PlanewaveDavidsonDiagonalizer dav(exec);
                dav.set_tolerance(tol);
                dav.set_maximum_iterations(max_iter);
                ProfilingCounters::instance().davidson_iteration_count = 0;
                auto t0 = std::chrono::steady_clock::now();
                dav.solve(k, k, npw_of[k], nb, gidx[k], ke[k], v_r, crystal, kgrid, basis, system, system);
                double solve_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
                write_array(tag + "_solve_ms.f64", &solve_ms, 1);
                std::vector<double> eig(nb);
                for (int i = 0; i < nb; ++i) eig[i] = system.eigenvalue(k, i);
                write_array(tag + "_eig.f64", eig.data(), eig.size());
                write_array(tag + "_bands.c128", system.band_block(k), static_cast<std::size_t>(npw_of[k]) * nb);
                int stats[2] = {static_cast<int>(ProfilingCounters::instance().davidson_iteration_count),
                                dav.number_of_unconverged_bands()};
                write_array(tag + "_stats.i32", stats, 2);
            }
        }
        std::printf("ok\n");
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "harness: %s\n", e.what());
        return 1;
    }
}
