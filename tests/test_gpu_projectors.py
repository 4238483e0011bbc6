"""Kleinman-Bylander projector set built on the device (ProjectorSetBuilder).

The device matrix against the oracle's restatement of
compute_kleinman_bylander_projectors (projector.hpp:42-199) on the same
tables, to 1e-13 relative, for the synthetic cells' s and p channels and for
random tables up to l = 4; H|psi> through the device-built set against the
oracle's; and the eigenvalues against those of the closed-form projectors the
tables sample (equal up to the tables' interpolation error).
"""
import numpy as np
import pytest

from oracle import hpsi as ohpsi
from oracle import projectors as oproj
from q3_b200 import synthetic
from q3_b200._lib import FP64, Q3BError

pytestmark = pytest.mark.gpu

DQ = 0.01


def _tables(qmax, dq=DQ):
    """The synthetic cells' channels (2 s, 2 p) sampled on a uniform q grid."""
    q = np.arange(0.0, qmax + 5 * dq, dq)
    tabs = [synthetic._radial_transform(l, q) for (l, _ch) in synthetic.CHANNELS]
    return [[l for (l, _ch) in synthetic.CHANNELS]], np.array(tabs)


def _inputs(sy, k=0):
    kp = sy.kpoints[k]
    kpg = (kp.miller + kp.k_frac[None, :]) @ sy.cell.reciprocal
    pos = sy.cell.positions_frac @ sy.cell.lattice
    return kp, kpg, pos


def _build(sy, k=0, beta_l=None, tables=None, species=None, dq=DQ):
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    kp, kpg, pos = _inputs(sy, k)
    if beta_l is None:
        beta_l, tables = _tables(np.max(np.linalg.norm(kpg, axis=1)), dq)
    if species is None:
        species = np.zeros(pos.shape[0], dtype=np.int32)
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    nper = [sum(2 * l + 1 for l in beta_l[s]) for s in species]
    dblk = np.concatenate([np.diag(np.linspace(-1.0, 1.0, n)).reshape(-1, order="F") for n in nper])
    ap.prepare_kpoint_build(k, kp.npw, kp.g_to_grid, kp.ke, kpg, sy.cell.volume, pos, species, beta_l,
                            tables, dq, dblk)
    return ap, kpg, pos, beta_l, tables, species, dblk


@pytest.mark.parametrize("cid", [0, "small_k"])
def test_device_projectors_match_oracle(cuda_device, cid):
    sy = synthetic.config(0) if cid == 0 else synthetic.small_system(
        grid=(15, 16, 18), a=7.5, ecut=9.0, nbands=5, natoms=3, seed=3, k_frac=(0.25, 0.0, 0.125))
    ap, kpg, pos, beta_l, tables, species, _ = _build(sy)
    got = ap.projectors().cpu().numpy().T
    tabs = [[tables[i] for i in range(len(beta_l[0]))]]
    ref = oproj.build(kpg, sy.cell.volume, pos, species, beta_l, tabs, DQ)
    assert got.shape == ref.shape
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-13


def test_higher_l_and_two_species(cuda_device):
    sy = synthetic.small_system(grid=(12, 12, 12), a=7.0, ecut=8.0, nbands=4, natoms=3, seed=8,
                                k_frac=(0.1, 0.2, 0.3))
    rng = np.random.default_rng(12)
    beta_l = [[2, 4, 0], [3, 1]]
    kp, kpg, pos = _inputs(sy)
    nq = int(np.max(np.linalg.norm(kpg, axis=1)) / 0.02) + 8
    tables = rng.standard_normal((5, nq))
    species = np.array([1, 0, 1], dtype=np.int32)
    ap, kpg, pos, _, _, _, _ = _build(sy, beta_l=beta_l, tables=tables, species=species, dq=0.02)
    got = ap.projectors().cpu().numpy().T
    tabs = [[tables[0], tables[1], tables[2]], [tables[3], tables[4]]]
    ref = oproj.build(kpg, sy.cell.volume, pos, species, beta_l, tabs, 0.02)
    assert got.shape == (kp.npw, 2 * (7 + 3) + (5 + 9 + 1))
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-13


def test_hpsi_with_device_projectors(cuda_device):
    import torch
    sy = synthetic.config(0)
    ap, kpg, pos, beta_l, tables, species, dblk = _build(sy)
    kp = sy.kpoints[0]
    beta = oproj.build(kpg, sy.cell.volume, pos, species, beta_l, [[t for t in tables]], DQ)
    psi = sy.psi0[0]
    x = torch.from_numpy(np.ascontiguousarray(psi.T)).to("cuda")
    y = torch.empty_like(x)
    ap.apply_batch(x, y, psi.shape[1], FP64)
    got = y.cpu().numpy().T
    loc = ohpsi.apply_local(psi, kp.ke, kp.g_to_grid, sy.v_r, sy.cell.grid)
    offs = np.cumsum([0] + [8] * pos.shape[0]).astype(np.int32)
    ref = loc + ohpsi.apply_nonlocal(psi, beta, dblk, offs)
    assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-12


def test_eigenvalues_match_closed_form_projectors(cuda_device):
    """Same Hamiltonian up to a rotation inside each p shell and the tables'
    interpolation: the lowest eigenvalues agree."""
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    from q3_b200.davidson import PlanewaveDavidsonDiagonalizer
    sy = synthetic.config(0)
    kp, kpg, pos = _inputs(sy)
    beta_l, tables = _tables(np.max(np.linalg.norm(kpg, axis=1)), 0.002)
    species = np.zeros(pos.shape[0], dtype=np.int32)
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_kpoint_build(0, kp.npw, kp.g_to_grid, kp.ke, kpg, sy.cell.volume, pos, species, beta_l, tables,
                            0.002, kp.d_blocks)
    d = PlanewaveDavidsonDiagonalizer(ap)
    d.set_tolerance(1e-11)
    d.set_maximum_iterations(200)
    w_dev = d.solve(sy.psi0[0], sy.nbands).eigenvalues
    ap2 = PlanewaveHamiltonianApplicator()
    ap2.update_potential(sy.v_r, sy.cell.grid)
    ap2.prepare_system_kpoint(sy)
    d2 = PlanewaveDavidsonDiagonalizer(ap2)
    d2.set_tolerance(1e-11)
    d2.set_maximum_iterations(200)
    w_ref = d2.solve(sy.psi0[0], sy.nbands).eigenvalues
    assert np.max(np.abs(w_dev - w_ref)) < 1e-6


def test_rejects_l_above_four(cuda_device):
    sy = synthetic.config(0)
    kp, kpg, pos = _inputs(sy)
    with pytest.raises(Q3BError):
        _build(sy, beta_l=[[5]], tables=np.zeros((1, 50)), species=np.zeros(pos.shape[0], dtype=np.int32))
