"""Starting-subspace rotation (StartingSubspaceSolver) on the GPU.

The first two tests restate the reference's own tests of this interface
(test_starting_subspace_solver_gpu.cpp:61-145 and :147-166) with the same
inputs: an H that is diagonal in the plane waves, H_gg = 1 + g/2, which this
library's applicator is exactly when V = 0, there are no projectors and the
kinetic energies are set to 1 + g/2.  The projections and the rotation must
equal the direct sums to 1e-11 and 1e-12, the reference's tolerances.  The
third runs the whole rotation on a real cell against the CPU oracle:
eigenvalues within 1e-10 Ry, the same band subspace.
"""
import numpy as np
import pytest

from oracle import hpsi as ohpsi
from oracle import starting as ostart
from q3_b200 import synthetic
from q3_b200._lib import Q3BError

pytestmark = pytest.mark.gpu


def _diagonal_applicator(npw, grid=(8, 8, 8)):
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(np.zeros(int(np.prod(grid))), grid)
    g2g = (np.arange(npw) * 7) % int(np.prod(grid))      # distinct grid points
    ke = 1.0 + 0.5 * np.arange(npw)
    ap.prepare_kpoint(0, npw, g2g, ke)
    return ap


def test_projects_and_rotates_as_the_direct_sums_do(cuda_device):
    from q3_b200.starting import StartingSubspaceSolver
    npw, nvec, nb = 37, 5, 3
    g = np.arange(npw)[:, None]
    v = np.arange(nvec)[None, :]
    chi = np.sin(0.3 * (g + 1) * (v + 1)) + 1j * np.cos(0.7 * (g + 2) + 0.2 * v)
    ap = _diagonal_applicator(npw)
    sol = StartingSubspaceSolver(ap)
    sol.apply_hamiltonian(chi, nvec)
    h, s = sol.project()
    diag = 1.0 + 0.5 * np.arange(npw)
    assert np.max(np.abs(h - chi.conj().T @ (diag[:, None] * chi))) < 1e-11
    assert np.max(np.abs(s - chi.conj().T @ chi)) < 1e-11
    b = np.arange(nb)[None, :]
    vv = np.arange(nvec)[:, None]
    coef = (0.1 * (vv + 1) - 0.05 * b) + 1j * (0.03 * (b + 1) * (vv - 2))
    bands = sol.rotate_into_bands(coef, nb).cpu().numpy().T
    assert np.max(np.abs(bands - chi @ coef)) < 1e-12


def test_refuses_a_band_block_of_another_shape(cuda_device):
    from q3_b200.starting import StartingSubspaceSolver
    ap = _diagonal_applicator(7)
    sol = StartingSubspaceSolver(ap)
    sol.apply_hamiltonian(np.ones((7, 2), dtype=np.complex128), 2)
    g2g = (np.arange(8) * 7) % 512
    ap.prepare_kpoint(0, 8, g2g, 1.0 + 0.5 * np.arange(8))   # another k-point shape
    with pytest.raises(Q3BError):
        sol.rotate_into_bands(np.ones((2, 2), dtype=np.complex128), 2)


@pytest.mark.parametrize("cid", [0, 2])
def test_rotation_matches_oracle(cuda_device, cid):
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    from q3_b200.starting import rotate_starting_vectors
    sy = synthetic.config(cid, nk=1) if cid == 2 else synthetic.config(cid)
    kp = sy.kpoints[0]
    nb = sy.nbands
    nchi = 2 * nb
    rng = np.random.default_rng(4321 + cid)
    chi = rng.standard_normal((kp.npw, nchi)) + 1j * rng.standard_normal((kp.npw, nchi))
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_system_kpoint(sy)
    eig, bands = rotate_starting_vectors(ap, chi, nb)
    bands = bands.cpu().numpy().T
    we, be = ostart.starting_subspace(lambda x: ohpsi.apply_h(x, kp, sy.v_r, sy.cell.grid), chi, nb)
    assert np.max(np.abs(eig - we)) < 1e-10
    # same S-orthonormal band subspace: projectors agree (bands are orthonormal in chi's metric)
    pg = bands @ bands.conj().T
    po = be @ be.conj().T
    assert np.max(np.abs(pg - po)) / np.max(np.abs(po)) < 1e-8
