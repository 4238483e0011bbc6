"""Gamma-only H|psi> (half-sphere vectors, two bands per transform) on the GPU,
through the C ABI, against the oracle restatement of the reference's Gamma path.

Bar: FP64 within 1e-12 relative; mixed within 2e-5 relative.
"""
import numpy as np
import pytest

from oracle import gamma as og
from q3_b200 import synthetic
from q3_b200._lib import FP64, MIXED, Q3BError

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _real_space_real(rng, npw, nb):
    """Half-sphere coefficients of states that are real in real space: psi(0) real."""
    psi = rng.standard_normal((npw, nb)) + 1j * rng.standard_normal((npw, nb))
    psi[0] = psi[0].real
    return psi


def _prepared(sy):
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    g = synthetic.gamma_kpoint(sy)
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_kpoint_gamma(g.npw, g.g_to_grid, g.minus_g_to_grid, g.ke, g.beta, g.atom_proj_offsets,
                            g.d_blocks)
    return ap, g


def _apply(ap, psi, precision):
    import torch
    x = torch.from_numpy(np.ascontiguousarray(psi.T)).to("cuda")
    y = torch.empty_like(x)
    ap.apply_batch_gamma(x, y, psi.shape[1], precision)
    torch.cuda.synchronize()
    return y.cpu().numpy().T


def _oracle(sy, g, psi):
    return og.apply_h_gamma(psi, g.ke, g.g_to_grid, g.minus_g_to_grid, g.beta, g.d_blocks,
                            g.atom_proj_offsets, sy.v_r, sy.cell.grid)


@pytest.mark.parametrize("nb", [1, 2, 5, 8])
def test_gamma_small(cuda_device, nb):
    sy = synthetic.small_system(grid=(16, 16, 16), a=8.0, ecut=10.0, natoms=3, nbands=nb)
    ap, g = _prepared(sy)
    psi = _real_space_real(np.random.default_rng(nb), g.npw, nb)
    ref = _oracle(sy, g, psi)
    assert _rel(_apply(ap, psi, FP64), ref) < 1e-12
    assert _rel(_apply(ap, psi, MIXED), ref) < 2e-5


def test_gamma_config0_matches_full_sphere(cuda_device):
    """The FCC cell at Gamma: the half-sphere result equals the full-sphere H|psi> of the same
    real-space-real states, restricted to the half sphere."""
    import torch
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    sy = synthetic.config(0)
    ap, g = _prepared(sy)
    kp = sy.kpoints[0]
    nb = 7
    psi = _real_space_real(np.random.default_rng(3), g.npw, nb)
    got = _apply(ap, psi, FP64)
    assert _rel(got, _oracle(sy, g, psi)) < 1e-12
    key = {tuple(m): i for i, m in enumerate(kp.miller)}
    mirror = np.array([key[tuple(-kp.miller[i])] for i in g.index])
    full = np.zeros((kp.npw, nb), complex)
    full[g.index] = psi
    full[mirror[1:]] = np.conj(psi[1:])
    fa = PlanewaveHamiltonianApplicator()
    fa.update_potential(sy.v_r, sy.cell.grid)
    fa.prepare_system_kpoint(sy)
    x = torch.from_numpy(np.ascontiguousarray(full.T)).to("cuda")
    y = torch.empty_like(x)
    fa.apply_batch(x, y, nb)
    torch.cuda.synchronize()
    hf = y.cpu().numpy().T
    assert _rel(got, hf[g.index]) < 1e-12


def test_gamma_wide_radix_grid(cuda_device):
    sy = synthetic.small_system(grid=(20, 96, 15), a=7.0, ecut=8.0, natoms=3, nbands=6)
    ap, g = _prepared(sy)
    psi = _real_space_real(np.random.default_rng(11), g.npw, 6)
    assert _rel(_apply(ap, psi, FP64), _oracle(sy, g, psi)) < 1e-12


def test_gamma_needs_a_gamma_prepare(cuda_device):
    import torch
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    sy = synthetic.small_system()
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_system_kpoint(sy)
    x = torch.zeros(2, 10, dtype=torch.complex128, device="cuda")
    with pytest.raises(Q3BError):
        ap.apply_batch_gamma(x, x.clone(), 2)
    g = synthetic.gamma_kpoint(sy)
    bad = g.minus_g_to_grid.copy()
    bad[0] = bad[1]
    with pytest.raises(Q3BError):          # entry 0 must be the origin
        ap.prepare_kpoint_gamma(g.npw, g.g_to_grid, bad, g.ke)
