"""H|psi> on the GPU (through the C ABI) against the CPU oracle.

Bar: FP64 within 1e-12 relative (max-norm over the batch, relative to the
largest |H psi| entry); FP32 ("mixed") within 2e-5 relative.
"""
import numpy as np
import pytest

from oracle import hpsi as ohpsi
from q3_b200 import synthetic
from q3_b200._lib import FP64, MIXED, Q3BError

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 2e-5


def _applicator(system, k=0):
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(system.v_r, system.cell.grid)
    ap.prepare_system_kpoint(system, k)
    return ap


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _run(ap, psi, precision=FP64):
    import torch
    x = torch.from_numpy(np.asfortranarray(psi).T.copy()).to("cuda")  # rows = bands
    y = torch.empty_like(x)
    ap.apply_batch(x, y, psi.shape[1], precision)
    torch.cuda.synchronize()
    return y.cpu().numpy().T


CASES = [
    dict(grid=(12, 12, 12), a=7.0, ecut=8.0, natoms=2),
    dict(grid=(16, 16, 16), a=8.0, ecut=10.0, natoms=3),
    dict(grid=(24, 20, 18), a=9.0, ecut=9.0, natoms=4),
    dict(grid=(15, 15, 15), a=7.5, ecut=9.0, natoms=2, k_frac=(0.25, 0.125, 0.375)),
    # lines with a factor above 10 (75 = 15 x 5, 96 = 12 x 8, 16 x 16): the
    # kernels built for radices up to 16
    dict(grid=(75, 16, 18), a=7.0, ecut=8.0, natoms=2),
    dict(grid=(20, 96, 15), a=7.0, ecut=8.0, natoms=3, k_frac=(0.5, 0.0, 0.25)),
    dict(grid=(256, 12, 12), a=7.0, ecut=8.0, natoms=2),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c["grid"])))
def test_hpsi_fp64_small(cuda_device, case):
    sy = synthetic.small_system(nbands=5, **case)
    kp = sy.kpoints[0]
    ap = _applicator(sy)
    rng = np.random.default_rng(1)
    psi = rng.standard_normal((kp.npw, 7)) + 1j * rng.standard_normal((kp.npw, 7))
    ref = ohpsi.apply_h(psi, kp, sy.v_r, sy.cell.grid)
    got = _run(ap, psi)
    assert _rel(got, ref) < FP64_TOL
    assert _rel(_run(ap, psi, MIXED), ref) < FP32_TOL


def test_hpsi_config0_fp64_and_mixed(cuda_device):
    sy = synthetic.config(0)
    kp = sy.kpoints[0]
    ap = _applicator(sy)
    psi = sy.psi0[0]
    ref = ohpsi.apply_h(psi, kp, sy.v_r, sy.cell.grid)
    assert _rel(_run(ap, psi, FP64), ref) < FP64_TOL
    assert _rel(_run(ap, psi, MIXED), ref) < FP32_TOL


def test_hpsi_config0_golden(cuda_device):
    from pathlib import Path
    g = np.load(Path(__file__).parent / "golden" / "config0_hpsi.npz")
    sy = synthetic.config(0)
    assert np.array_equal(sy.kpoints[0].g_to_grid, g["g_to_grid"])
    ap = _applicator(sy)
    got = _run(ap, g["psi"])
    assert _rel(got, g["hpsi"]) < FP64_TOL


def test_hpsi_config1_all_bands(cuda_device):
    # the 64-atom 80^3 cell with 512 projectors, the whole 256-band block
    sy = synthetic.config(1)
    kp = sy.kpoints[0]
    ap = _applicator(sy)
    psi = sy.psi0[0]
    ref = ohpsi.apply_h(psi, kp, sy.v_r, sy.cell.grid, threads=8)
    assert _rel(_run(ap, psi, FP64), ref) < FP64_TOL
    assert _rel(_run(ap, psi, MIXED), ref) < FP32_TOL


def test_hpsi_linearity_and_hermiticity_config1(cuda_device):
    # size-independent properties at the full band count: H(a x + b y) = a Hx + b Hy
    # and <x|H y> = <H x|y>
    import torch
    sy = synthetic.config(1, nbands=256)
    ap = _applicator(sy)
    npw = sy.kpoints[0].npw
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(256, npw, dtype=torch.complex128, device="cuda", generator=g)
    y = torch.randn(256, npw, dtype=torch.complex128, device="cuda", generator=g)
    a, b = 0.7 - 0.2j, -1.3 + 0.4j
    hx, hy, hz = torch.empty_like(x), torch.empty_like(y), torch.empty_like(x)
    ap.apply_batch(x, hx, 256)
    ap.apply_batch(y, hy, 256)
    ap.apply_batch(a * x + b * y, hz, 256)
    torch.cuda.synchronize()
    lin = (hz - (a * hx + b * hy)).abs().max() / hz.abs().max()
    assert float(lin) < 1e-12
    lhs = (x.conj() * hy).sum(dim=1)
    rhs = (hx.conj() * y).sum(dim=1)
    herm = (lhs - rhs).abs().max() / lhs.abs().max()
    assert float(herm) < 1e-12


def test_hpsi_empty_batch_and_errors(cuda_device):
    import torch
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    ap = PlanewaveHamiltonianApplicator()
    x = torch.zeros(1, 8, dtype=torch.complex128, device="cuda")
    with pytest.raises(Q3BError):          # no potential / k-point yet
        ap.apply_batch(x, x.clone(), 1)
    sy = synthetic.small_system()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_system_kpoint(sy)
    y = torch.zeros(0, sy.kpoints[0].npw, dtype=torch.complex128, device="cuda")
    ap.apply_batch(y, y.clone(), 0)        # empty batch is a no-op
    with pytest.raises(Q3BError):          # unsupported grid length (7)
        ap.update_potential(np.zeros(7 * 8 * 8), (7, 8, 8))


@pytest.mark.parametrize("nvec", [8, 37, 64])
def test_host_buffer_path_matches_device_path(cuda_device, nvec):
    """q3b_apply_h_host (host vectors, chunked copy/compute pipeline for
    32 bands and more) against q3b_apply_h on device vectors."""
    sy = synthetic.small_system(grid=(16, 16, 16), a=8.0, ecut=12.0, nbands=nvec, natoms=3, seed=5)
    ap = _applicator(sy)
    psi = sy.psi0[0][:, :nvec]
    for prec, tol in ((FP64, 1e-13), (MIXED, 1e-6)):
        dev = _run(ap, psi, prec)
        host = ap.apply_batch_host(psi, nvec, prec)
        assert _rel(host, dev) < tol
    ref = ohpsi.apply_h(psi, sy.kpoints[0], sy.v_r, sy.cell.grid)
    assert _rel(ap.apply_batch_host(psi, nvec, FP64), ref) < FP64_TOL


def test_spin_channel_d_blocks(cuda_device):
    # set_spin_channel: the other channel's D blocks replace the prepared ones, and H|psi>
    # is then the oracle's with those blocks (the projectors stay on the device)
    import dataclasses
    sy = synthetic.small_system(nbands=5, grid=(16, 16, 16), a=8.0, ecut=10.0, natoms=3)
    kp = sy.kpoints[0]
    ap = _applicator(sy)
    rng = np.random.default_rng(4)
    psi = rng.standard_normal((kp.npw, 6)) + 1j * rng.standard_normal((kp.npw, 6))
    d_down = kp.d_blocks * 0.5 + rng.uniform(-0.1, 0.1, size=kp.d_blocks.shape) * (kp.d_blocks != 0)
    ap.set_d_blocks(d_down)
    kp_down = dataclasses.replace(kp, d_blocks=d_down)
    for precision, tol in ((FP64, FP64_TOL), (MIXED, FP32_TOL)):
        assert _rel(_run(ap, psi, precision), ohpsi.apply_h(psi, kp_down, sy.v_r, sy.cell.grid)) < tol
    ap.set_d_blocks(kp.d_blocks)
    assert _rel(_run(ap, psi), ohpsi.apply_h(psi, kp, sy.v_r, sy.cell.grid)) < FP64_TOL
