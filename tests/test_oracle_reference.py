"""The oracle against the reference's own CPU code (CPU only).

tests/golden/ref_config*.npz hold outputs of the reference's compiled C++
(SerialPlanewaveHamiltonianApplicator::apply_batch, PlanewaveDavidsonDiagonalizer::solve,
SerialProjectorSetBuilder; made by tests/golden/make_ref_golden.py).  Here the numpy
restatement in oracle/ reproduces them on the same inputs: H|psi> to 1e-13 relative, the
projector set to 1e-13, and the Davidson eigenvalues and iteration counts of the same
trajectory.  This is what pins the oracle that the GPU tests compare against.
"""
from pathlib import Path

import numpy as np
import pytest

from oracle import davidson as odav
from oracle import hpsi as ohpsi
from tests.golden import ref_fixtures as RF


def _need(cid):
    if not RF.path(cid).exists():
        pytest.skip(f"{RF.path(cid).name} not generated")
    return RF.load(cid)


def _kp_with_beta(rk, beta):
    rk.beta = beta
    return rk


def test_fixture_inputs_regenerate():
    # the seeded recipe still gives the potential and plane-wave sets the reference saw
    for cid in (0, 2, 1, 3):
        if not RF.path(cid).exists():
            continue
        g = RF.load(cid)
        sy = RF.system(cid)
        assert np.allclose(RF.v_checksum(sy.v_r), g["v_checksum"], rtol=1e-13, atol=0)
        for k in range(len(sy.kpoints)):
            p = RF.perm_of(g, k)
            assert np.array_equal(np.sort(p), np.arange(sy.kpoints[k].npw))


def test_config0_inputs_match_reference():
    g = _need(0)
    sy = RF.system(0)
    rk = RF.kpoint(sy, g)
    assert np.array_equal(rk.miller, g["miller"])
    assert np.array_equal(rk.g_to_grid, g["g_to_grid"])
    assert np.max(np.abs(rk.ke - g["ke"])) < 1e-13
    assert np.max(np.abs(rk.kpg - g["kpg"])) < 1e-13


def test_config0_projectors_match_reference_builder():
    g = _need(0)
    sy = RF.system(0)
    rk = RF.kpoint(sy, g)
    beta = RF.oracle_projectors(sy, g, rk)
    assert beta.shape == g["beta"].shape
    assert np.max(np.abs(beta - g["beta"])) / np.max(np.abs(g["beta"])) < 1e-13


def test_config0_hpsi_matches_reference():
    g = _need(0)
    sy = RF.system(0)
    rk = _kp_with_beta(RF.kpoint(sy, g), np.asfortranarray(g["beta"]))
    got = ohpsi.apply_h(rk.psi0, rk, sy.v_r, sy.cell.grid)
    ref = g["hpsi"]
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-13


@pytest.mark.parametrize("tol,key", [(1e-10, "tol10"), (1e-12, "tol12")])
def test_config0_davidson_matches_reference(tol, key):
    g = _need(0)
    sy = RF.system(0)
    rk = _kp_with_beta(RF.kpoint(sy, g), np.asfortranarray(g["beta"]))
    res = odav.solve(lambda v: ohpsi.apply_h(v, rk, sy.v_r, sy.cell.grid), rk.ke, rk.psi0,
                     sy.nbands, tol, max_iterations=200)
    assert res.iterations == int(g[f"iterations_{key}"])
    assert np.max(np.abs(res.eigenvalues - g[f"eig_{key}"])) < 1e-12


def test_config1_hpsi_matches_reference():
    g = _need(1)
    sy = RF.system(1)
    rk = RF.kpoint(sy, g)
    rk.beta = RF.oracle_projectors(sy, g, rk)
    psi = rk.psi0[:, :RF.GRAM_BANDS]
    h = ohpsi.apply_h(psi, rk, sy.v_r, sy.cell.grid, threads=8)
    scale = np.max(np.abs(g["hpsi_band0"]))
    assert np.max(np.abs(h[:, 0] - g["hpsi_band0"])) / scale < 1e-12
    for name, val in (("gram_psi_hpsi", psi.conj().T @ h), ("gram_hpsi_hpsi", h.conj().T @ h),
                      ("sketch", RF.sketch_columns(rk.npw).conj().T @ h)):
        ref = g[name]
        assert np.max(np.abs(val - ref)) / np.max(np.abs(ref)) < 1e-12, name


def test_config2_kpoint_davidson_matches_reference():
    g = _need(2)
    sy = RF.system(2)
    k = 5
    rk = RF.kpoint(sy, g, k)
    rk.beta = RF.oracle_projectors(sy, g, rk)
    res = odav.solve(lambda v: ohpsi.apply_h(v, rk, sy.v_r, sy.cell.grid, threads=8), rk.ke, rk.psi0,
                     sy.nbands, 1e-10, max_iterations=300)
    assert res.iterations == int(g["iterations_tol10"][k])
    assert np.max(np.abs(res.eigenvalues - g["eig_tol10"][k])) < 1e-11


def test_config0_dense_potential_matches_reference():
    # V(r) given on a 48x36x40 density grid: the reference restricts it to the 24^3
    # wavefunction grid by G-space truncation before it applies H
    if not RF.path("0_dense").exists():
        pytest.skip("ref_config0_dense.npz not generated")
    g = RF.load("0_dense")
    sy = RF.system(0)
    vd = RF.dense_potential(sy, tuple(g["density_grid"]))
    assert np.allclose(RF.v_checksum(vd), g["v_dense_checksum"], rtol=1e-13, atol=0)
    vs = ohpsi.restrict_potential(vd, tuple(g["density_grid"]), sy.cell.grid)
    assert np.max(np.abs(ohpsi.scaled_potential(vs) - g["v_scaled"])) / np.max(np.abs(g["v_scaled"])) < 1e-13
    g0 = _need(0)
    rk = _kp_with_beta(RF.kpoint(sy, g0), np.asfortranarray(g0["beta"]))
    assert np.array_equal(RF.perm_of(g), RF.perm_of(g0))
    got = ohpsi.apply_h(rk.psi0, rk, vs, sy.cell.grid)
    assert np.max(np.abs(got - g["hpsi"])) / np.max(np.abs(g["hpsi"])) < 1e-13


@pytest.mark.parametrize("dense,smooth", [((48, 36, 40), (24, 24, 24)), ((25, 31, 50), (20, 24, 27)),
                                          ((16, 16, 16), (16, 16, 16))])
def test_restriction_keeps_band_limited_potentials(dense, smooth):
    # a V(r) whose Fourier components all lie strictly inside the wavefunction grid's
    # Miller range is sampled, not changed, by the restriction
    rng = np.random.default_rng(7)
    r = np.meshgrid(*[np.arange(d) / d for d in dense], indexing="ij")
    v = np.full(dense, 0.3)
    for _ in range(6):
        m = [int(rng.integers(-((n - 1) // 2), (n - 1) // 2 + 1)) for n in smooth]
        ph = 2 * np.pi * sum(mi * ri for mi, ri in zip(m, r))
        v += rng.normal() * np.cos(ph + rng.uniform(0, 2 * np.pi))
    got = ohpsi.restrict_potential(v.reshape(-1), dense, smooth)
    rs = np.meshgrid(*[np.arange(n) / n for n in smooth], indexing="ij")
    rng = np.random.default_rng(7)
    want = np.full(smooth, 0.3)
    for _ in range(6):
        m = [int(rng.integers(-((n - 1) // 2), (n - 1) // 2 + 1)) for n in smooth]
        ph = 2 * np.pi * sum(mi * ri for mi, ri in zip(m, rs))
        want += rng.normal() * np.cos(ph + rng.uniform(0, 2 * np.pi))
    assert np.max(np.abs(got - want.reshape(-1))) < 1e-12
