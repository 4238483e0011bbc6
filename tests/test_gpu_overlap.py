"""Ultrasoft overlap operator S on the GPU, through the C ABI, against the oracle
restatement (full sphere and Gamma-only half sphere).

Bar: FP64 within 1e-12 relative; mixed within 2e-5 relative (of |S psi|).
"""
import numpy as np
import pytest

from oracle import overlap as oov
from q3_b200 import synthetic
from q3_b200._lib import FP64, MIXED, Q3BError

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _run(ap, psi, precision, gamma=False):
    import torch
    x = torch.from_numpy(np.ascontiguousarray(psi.T)).to("cuda")
    y = torch.empty_like(x)
    ap.apply_overlap(x, y, psi.shape[1], precision, gamma=gamma)
    torch.cuda.synchronize()
    return y.cpu().numpy().T


def test_overlap_full_sphere(cuda_device):
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    sy = synthetic.small_system(grid=(16, 16, 16), a=8.0, ecut=10.0, natoms=3, nbands=6,
                                k_frac=(0.25, 0.0, 0.125))
    kp = sy.kpoints[0]
    q = synthetic.overlap_blocks(sy)
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_system_kpoint(sy)
    psi = sy.psi0[0]
    with pytest.raises(Q3BError):            # no blocks set yet
        _run(ap, psi, FP64)
    ap.set_overlap_blocks(q)
    ref = oov.apply_s(psi, kp.beta, q, kp.atom_proj_offsets)
    assert _rel(_run(ap, psi, FP64), ref) < 1e-12
    assert _rel(_run(ap, psi, MIXED), ref) < 2e-5
    # S is Hermitian and, with these small q, positive definite
    s = oov.apply_s(np.eye(kp.npw, dtype=complex), kp.beta, q, kp.atom_proj_offsets)
    assert np.allclose(s, s.conj().T, atol=1e-13)
    assert np.min(np.linalg.eigvalsh(s)) > 0.0


def test_overlap_config1_subset(cuda_device):
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    sy = synthetic.config(1, nbands=32)
    kp = sy.kpoints[0]
    q = synthetic.overlap_blocks(sy)
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_system_kpoint(sy)
    ap.set_overlap_blocks(q)
    psi = sy.psi0[0]
    ref = oov.apply_s(psi, kp.beta, q, kp.atom_proj_offsets)
    assert _rel(_run(ap, psi, FP64), ref) < 1e-12
    assert _rel(_run(ap, psi, MIXED), ref) < 2e-5


@pytest.mark.parametrize("nb", [3, 4])
def test_overlap_gamma(cuda_device, nb):
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    sy = synthetic.small_system(grid=(16, 16, 16), a=8.0, ecut=10.0, natoms=3, nbands=nb)
    g = synthetic.gamma_kpoint(sy)
    q = synthetic.overlap_blocks(sy)
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_kpoint_gamma(g.npw, g.g_to_grid, g.minus_g_to_grid, g.ke, g.beta, g.atom_proj_offsets,
                            g.d_blocks)
    ap.set_overlap_blocks(q)
    rng = np.random.default_rng(nb)
    psi = rng.standard_normal((g.npw, nb)) + 1j * rng.standard_normal((g.npw, nb))
    psi[0] = psi[0].real
    ref = oov.apply_s_gamma(psi, g.beta, q, g.atom_proj_offsets)
    assert _rel(_run(ap, psi, FP64, gamma=True), ref) < 1e-12
    assert _rel(_run(ap, psi, MIXED, gamma=True), ref) < 2e-5
