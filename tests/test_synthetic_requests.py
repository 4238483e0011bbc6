"""The serving stream's requests (no GPU): a seeded stream whose first k requests do not depend on
its length, so a test may build a prefix of it and take one request; every request within the
stream's stated ranges (2-32 atoms, 4 bands an atom, ecut 20-40 Ry, grids of 24-64 that hold the
wavefunction sphere)."""
import numpy as np

from q3_b200 import synthetic


def test_requests_are_a_prefix_stable_stream():
    a = synthetic.serving_requests(3)
    b = synthetic.serving_requests(5)
    for x, y in zip(a, b[:3]):
        assert x.nbands == y.nbands and tuple(x.cell.grid) == tuple(y.cell.grid)
        assert np.array_equal(x.kpoints[0].g_to_grid, y.kpoints[0].g_to_grid)
        assert np.array_equal(x.v_r, y.v_r)
        assert np.array_equal(x.psi0[0], y.psi0[0])


def test_requests_stay_within_the_stream_ranges():
    for sy in synthetic.serving_requests(6):
        natoms = sy.cell.natoms
        assert 2 <= natoms <= 32 and sy.nbands == 4 * natoms
        assert 20.0 <= sy.cell.ecut_ry <= 40.0
        assert all(24 <= n <= 64 for n in sy.cell.grid)
        kp = sy.kpoints[0]
        assert np.all(kp.g_to_grid >= 0)          # the grid holds the sphere
        assert kp.npw >= sy.nbands
