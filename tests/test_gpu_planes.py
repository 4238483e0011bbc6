"""Every plane-pass kernel of the local term against the oracle.

The autotuner picks one plane kernel per grid and precision; here each
candidate is forced through q3b_set_local_kernel (the shared-memory kernel at
128, 256 and 512 threads, the register kernel with one and two lanes a line)
and H|psi> is compared with the CPU oracle on grids with a register kernel (24,
40, 80, 108), at Gamma and at a shifted k-point (where the sphere's sticks are
off-centre cyclic intervals).  A k-point whose sticks are not row intervals has
no register kernel and keeps the shared-memory one.

Bars as in test_gpu_hpsi.py: FP64 1e-12, FP32 2e-5 relative to the largest entry.
"""
import numpy as np
import pytest

from oracle import hpsi as ohpsi
from q3_b200 import synthetic
from q3_b200._lib import FP64, MIXED, Q3BError

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 2e-5
CHOICES = [128, 256, 512, -1, -2]

GRIDS = {
    24: dict(grid=(24, 24, 24), a=10.26, ecut=30.0, natoms=2),
    40: dict(grid=(40, 40, 40), a=10.26, ecut=30.0, natoms=3, k_frac=(0.375, -0.125, 0.25)),
    80: dict(grid=(80, 80, 80), a=20.5, ecut=30.0, natoms=4),
    108: dict(grid=(108, 108, 108), a=25.8, ecut=36.0, natoms=3, k_frac=(0.125, 0.25, -0.375)),
}


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _apply(ap, psi, precision):
    import torch
    x = torch.from_numpy(np.asfortranarray(psi).T.copy()).to("cuda")
    y = torch.empty_like(x)
    ap.apply_batch(x, y, psi.shape[1], precision)
    torch.cuda.synchronize()
    return y.cpu().numpy().T


@pytest.fixture(scope="module", params=sorted(GRIDS))
def case(request):
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    sy = synthetic.small_system(nbands=6, seed=11, **GRIDS[request.param])
    kp = sy.kpoints[0]
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_system_kpoint(sy)
    ref = ohpsi.apply_h(sy.psi0[0], kp, sy.v_r, sy.cell.grid, threads=8)
    return sy, ap, ref


@pytest.mark.parametrize("choice", CHOICES)
def test_plane_kernel_matches_oracle(cuda_device, case, choice):
    sy, ap, ref = case
    for precision, tol in ((FP64, FP64_TOL), (MIXED, FP32_TOL)):
        ap.set_local_kernel(choice, precision)
        assert ap.local_kernel(precision) == choice
        assert _rel(_apply(ap, sy.psi0[0], precision), ref) < tol, (choice, precision)
    for precision in (FP64, MIXED):
        ap.set_local_kernel(0, precision)           # back to the tuner
        assert ap.local_kernel(precision) in CHOICES


def test_sticks_without_row_intervals_keep_the_shared_memory_kernel(cuda_device):
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    sy = synthetic.small_system(nbands=4, seed=5, grid=(24, 24, 24), a=10.26, ecut=30.0, natoms=2)
    kp = sy.kpoints[0]
    # drop the plane waves of one stick in the middle of a row: that row's sticks
    # are no longer one cyclic interval
    row = kp.miller[:, 0] == 0
    target = np.flatnonzero(row & (kp.miller[:, 1] == 2))
    keep = np.ones(kp.npw, dtype=bool)
    keep[target] = False
    assert target.size > 0 and np.any(row & (kp.miller[:, 1] == 3))
    sub = synthetic.KPoint(kp.k_frac, kp.miller[keep], kp.ke[keep], kp.g_to_grid[keep],
                           np.asfortranarray(kp.beta[keep]), kp.d_blocks, kp.atom_proj_offsets)
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_kpoint(0, sub.npw, sub.g_to_grid, sub.ke, sub.beta, sub.atom_proj_offsets, sub.d_blocks)
    with pytest.raises(Q3BError):
        ap.set_local_kernel(-1, FP64)
    assert ap.local_kernel(FP64) > 0
    psi = np.asfortranarray(sy.psi0[0][keep])
    ref = ohpsi.apply_h(psi, sub, sy.v_r, sy.cell.grid)
    assert _rel(_apply(ap, psi, FP64), ref) < FP64_TOL
