"""The CPU oracle against the reference's own known-answer tests for this path.

The reference's tests hold no golden H|psi> or Davidson vectors for these
cells; they pin the FFT convention (test_fft_grid.cpp:13-83) and the subspace
eigensolver (test_subspace_diagonalizer.cpp:11-166).  Those are replayed here
on the oracle, plus structural checks (H Hermitian, the local term equal to
its plane-wave matrix elements V(G'-G), Davidson equal to dense
diagonalisation).
"""
import math

import numpy as np
import pytest
import scipy.fft as sfft

from oracle import davidson, hpsi
from q3_b200 import synthetic


def fftw_backward(x):
    return sfft.ifftn(x, norm="forward")


def fftw_forward(x):
    return sfft.fftn(x, norm="backward")


def test_fft_round_trip_kat():
    # test_fft_grid.cpp:13-42 -- cos(2 pi x / L) on 16^3, forward then normalised inverse
    n = 16
    i1 = np.arange(n)[None, None, :]
    data = np.broadcast_to(np.cos(2 * np.pi * i1 / n), (n, n, n)).astype(np.complex128)
    back = fftw_backward(fftw_forward(data)) / data.size
    assert np.max(np.abs(back - data)) < 1e-10


def test_fft_parseval_kat():
    # test_fft_grid.cpp:54-83 -- sum |f|^2 = (1/N) sum |F|^2 on 12^3
    n = 12
    i = np.arange(n ** 3)
    data = (np.sin(0.3 * i + 0.7) + 1j * np.cos(0.5 * i - 0.2)).reshape(n, n, n)
    sr = np.sum(np.abs(data) ** 2)
    sg = np.sum(np.abs(fftw_forward(data)) ** 2)
    assert abs(sr - sg / data.size) < 1e-6 * sr


def test_fft_sign_convention():
    # FFTW_BACKWARD is e^{+i}: a single coefficient at G=1 gives exp(+2 pi i x / n)
    n = 8
    g = np.zeros((n, n, n), complex)
    g[0, 0, 1] = 1.0
    r = fftw_backward(g)
    x = np.arange(n)
    assert np.allclose(r[0, 0, :], np.exp(2j * np.pi * x / n))


def _solve(h, s):
    w, v, info = davidson.diagonalize_subspace(np.asarray(h, complex), np.asarray(s, complex), len(h))
    return w, v, info


def test_subspace_kat_identity():
    # test_subspace_diagonalizer.cpp:11-29
    w, v, info = _solve([[2, 0], [0, 3]], np.eye(2))
    assert info == 0 and abs(w[0] - 2) < 1e-10 and abs(w[1] - 3) < 1e-10


def test_subspace_kat_generalized():
    # test_subspace_diagonalizer.cpp:31-56 -- H=diag(2,4), S=diag(1,2): both 2
    w, v, info = _solve([[2, 0], [0, 4]], [[1, 0], [0, 2]])
    assert info == 0 and abs(w[0] - 2) < 1e-10 and abs(w[1] - 2) < 1e-10


def test_subspace_kat_real_symmetric():
    # test_subspace_diagonalizer.cpp:58-86 -- [[2,1],[1,2]]: 1 and 3
    w, v, info = _solve([[2, 1], [1, 2]], np.eye(2))
    assert info == 0 and abs(w[0] - 1) < 1e-10 and abs(w[1] - 3) < 1e-10


def generalized_problem_48(n=48):
    """test_subspace_diagonalizer.cpp:88-113: the 48x48 Hermitian / HPD pair."""
    h = np.zeros((n, n), complex)
    s = np.zeros((n, n), complex)
    for col in range(n):
        for row in range(col + 1):
            re = math.sin(0.37 * (row + 1) + 0.11 * (col + 1) * (col + 1))
            im = 0.0 if row == col else math.cos(0.23 * (row + 2) * (col + 1))
            h[row, col] = re + 1j * im
            h[col, row] = re - 1j * im
            c = (2.0 + 0.01 * row) if row == col else (0.02 * re + 0.02j * im)
            s[row, col] = c
            s[col, row] = np.conj(c)
        h[col, col] += 0.5 * col
    return h, s


def test_subspace_kat_48():
    # test_subspace_diagonalizer.cpp:115-160: every eigenvector solves H c = e S c to 1e-10
    h, s = generalized_problem_48()
    w, v, info = _solve(h, s)
    assert info == 0
    assert np.all(np.diff(w) >= 0)
    res = h @ v - (s @ v) * w[None, :]
    assert np.max(np.abs(res)) < 1e-10
    # S-orthonormal
    assert np.max(np.abs(v.conj().T @ s @ v - np.eye(48))) < 1e-10


def test_config0_sizes():
    # npw of the full sphere at 30 Ry in the FCC cell, and its sticks
    sy = synthetic.config(0)
    kp = sy.kpoints[0]
    assert kp.npw == 725 and kp.nproj == 16
    cols = {(int(m[0]) % 24, int(m[1]) % 24) for m in kp.miller}
    assert len(cols) == 109
    assert np.all(kp.g_to_grid >= 0)


def test_local_term_equals_plane_wave_matrix_elements():
    # <G'|V|G> = V(G'-G) with V(G) = (1/N) sum_r V(r) e^{-iGr}: an independent
    # statement of serial.hpp:457-477
    sy = synthetic.small_system(grid=(10, 10, 10), a=6.0, ecut=6.0, nbands=4)
    kp = sy.kpoints[0]
    n = sy.cell.grid
    vg = sfft.fftn(sy.v_r.reshape(n)) / sy.cell.npoints
    m = kp.miller
    npw = kp.npw
    dm = (m[:, None, :] - m[None, :, :]) % np.array(n)[None, None, :]
    vmat = vg[dm[..., 0], dm[..., 1], dm[..., 2]]
    hmat = np.diag(kp.ke).astype(complex) + vmat
    rng = np.random.default_rng(3)
    psi = rng.standard_normal((npw, 3)) + 1j * rng.standard_normal((npw, 3))
    got = hpsi.apply_local(psi, kp.ke, kp.g_to_grid, sy.v_r, n)
    assert np.max(np.abs(got - hmat @ psi)) < 1e-11 * np.max(np.abs(got))


def test_oracle_h_hermitian_and_nonlocal():
    sy = synthetic.small_system(grid=(12, 12, 12), a=7.0, ecut=8.0, nbands=4)
    kp = sy.kpoints[0]
    hd = hpsi.dense_hamiltonian(kp, sy.v_r, sy.cell.grid)
    assert np.max(np.abs(hd - hd.conj().T)) < 1e-12 * np.max(np.abs(hd))
    # nonlocal = beta D beta^H
    nl = kp.beta @ kp.d_dense() @ kp.beta.conj().T
    eye = np.eye(kp.npw, dtype=complex)
    got = hpsi.apply_nonlocal(eye, kp.beta, kp.d_blocks, kp.atom_proj_offsets)
    assert np.max(np.abs(got - nl)) < 1e-12


def test_oracle_davidson_matches_dense():
    sy = synthetic.small_system(grid=(12, 12, 12), a=7.0, ecut=8.0, nbands=6)
    kp = sy.kpoints[0]
    hd = hpsi.dense_hamiltonian(kp, sy.v_r, sy.cell.grid)
    exact = np.linalg.eigvalsh(hd)[:6]
    res = davidson.solve(lambda x: hd @ x, kp.ke, sy.psi0[0], 6, tolerance=1e-11,
                         max_iterations=80)
    assert res.unconverged == 0
    assert np.max(np.abs(res.eigenvalues - exact)) < 1e-9


def test_oracle_davidson_seeds_from_kinetic_energy():
    # zero starting bands are replaced by the lowest-KE plane waves (davidson.hpp:1047-1101)
    sy = synthetic.small_system(grid=(12, 12, 12), a=7.0, ecut=8.0, nbands=5)
    kp = sy.kpoints[0]
    hd = hpsi.dense_hamiltonian(kp, sy.v_r, sy.cell.grid)
    exact = np.linalg.eigvalsh(hd)[:5]
    res = davidson.solve(lambda x: hd @ x, kp.ke, None, 5, tolerance=1e-11, max_iterations=80)
    assert np.max(np.abs(res.eigenvalues - exact)) < 1e-9


def test_starting_rotation_oracle_matches_reference_kat():
    """The reference's StartingSubspaceSolver test (test_starting_subspace_solver_gpu.cpp:
    61-145): diagonal H_gg = 1 + g/2, 37 plane waves, 5 vectors with its sin/cos
    formula; projections and rotation equal the direct sums.  Then the whole
    rotation: Ritz values bound the exact eigenvalues of H from above."""
    from oracle import starting as ostart
    npw, nvec, nb = 37, 5, 3
    g = np.arange(npw)[:, None]
    v = np.arange(nvec)[None, :]
    chi = np.sin(0.3 * (g + 1) * (v + 1)) + 1j * np.cos(0.7 * (g + 2) + 0.2 * v)
    diag = 1.0 + 0.5 * np.arange(npw)
    h, s = ostart.project(lambda x: diag[:, None] * x, chi)
    for i in range(nvec):
        for j in range(nvec):
            eh = sum(diag[q] * np.conj(chi[q, i]) * chi[q, j] for q in range(npw))
            es = sum(np.conj(chi[q, i]) * chi[q, j] for q in range(npw))
            assert abs(h[i, j] - eh) < 1e-11 and abs(s[i, j] - es) < 1e-11
    b = np.arange(nb)[None, :]
    vv = np.arange(nvec)[:, None]
    coef = (0.1 * (vv + 1) - 0.05 * b) + 1j * (0.03 * (b + 1) * (vv - 2))
    bands = ostart.rotate_into_bands(chi, coef, nb)
    for bb in range(nb):
        for q in range(npw):
            assert abs(bands[q, bb] - sum(chi[q, k] * coef[k, bb] for k in range(nvec))) < 1e-12
    w, bands = ostart.starting_subspace(lambda x: diag[:, None] * x, chi, nb)
    assert np.all(w >= diag[:nb] - 1e-12)
    assert np.max(np.abs(bands.conj().T @ bands - np.eye(nb))) < 1e-12


def test_density_oracle_plane_wave_and_charge():
    """One plane wave of unit coefficient has |psi(r)| = 1 at every grid point
    after the unnormalised backward transform, so rho = w everywhere; and the
    total charge of orthonormal bands is sum_b f_b (the reference's
    test_accumulator.cpp:43-99 check, at 1e-12 instead of 0.01)."""
    from oracle import density as odens
    grid = (6, 5, 4)
    n = int(np.prod(grid))
    psi = np.zeros((3, 1), dtype=np.complex128)
    psi[1, 0] = 1.0
    g2g = np.array([-1, 37, 5])
    rho = odens.accumulate(psi, g2g, grid, np.array([0.25]))
    assert np.allclose(rho, 0.25, atol=1e-14)
    rng = np.random.default_rng(2)
    q, _ = np.linalg.qr(rng.standard_normal((40, 4)) + 1j * rng.standard_normal((40, 4)))
    g2g = rng.permutation(n)[:40]
    f = np.array([2.0, 2.0, 1.0, 0.0])
    rho = odens.accumulate(q, g2g, grid, f)
    assert abs(rho.sum() / n - f.sum()) < 1e-12
    assert rho.min() >= 0.0


def test_projector_oracle_pieces_match_reference_kats():
    """The pieces of the projector builder against the reference's own tests:
    test_lagrange.cpp:10-66 (4-point Lagrange on uniform tables),
    test_harmonics.cpp:16-205, 337-362 (Y_lm closed values, order sequence,
    (l, m) index, the G = 0 convention), plus orthonormality over the sphere."""
    from oracle import projectors as op
    lin = np.array([1.0, 3.0, 5.0, 7.0, 9.0, 11.0])
    for q, v in ((0.0, 1.0), (1.0, 3.0), (2.0, 5.0), (0.5, 2.0), (1.5, 4.0), (2.3, 5.6)):
        assert abs(op.lagrange_4point(lin, q, 1.0) - v) < 1e-12
    sq = np.array([0.0, 1.0, 4.0, 9.0, 16.0, 25.0])
    for q, v in ((0.5, 0.25), (1.5, 2.25), (2.5, 6.25)):
        assert abs(op.lagrange_4point(sq, q, 1.0) - v) < 1e-12
    cu = np.array([0.0, 1.0, 8.0, 27.0, 64.0, 125.0])
    for q, v in ((0.5, 0.125), (1.5, 3.375), (2.7, 19.683)):
        assert abs(op.lagrange_4point(cu, q, 1.0) - v) < 1e-10
    assert op.lagrange_4point(np.array([1.0, 2.0, 3.0]), 1.0, 1.0) == 0.0   # too short
    assert op.order_sequence(0) == [0] and op.order_sequence(2) == [0, 1, -1, 2, -2]
    assert [op.lm_index(l, m) for l in range(3) for m in op.order_sequence(l)] == list(range(9))
    y00 = 1.0 / np.sqrt(4 * np.pi)
    c1 = np.sqrt(3.0 / (4 * np.pi))
    ex, ey, ez = np.eye(3)
    assert abs(op.real_ylm(1, ez)[op.lm_index(1, 0)] - c1) < 1e-14
    assert abs(op.real_ylm(1, -ez)[op.lm_index(1, 0)] + c1) < 1e-14
    assert abs(op.real_ylm(1, ex)[op.lm_index(1, 1)] + c1) < 1e-14      # Condon-Shortley: -x/r
    assert abs(op.real_ylm(1, ey)[op.lm_index(1, -1)] + c1) < 1e-14
    z = op.real_ylm(2, np.zeros(3))
    assert abs(z[0] - y00) < 1e-14 and abs(z[op.lm_index(1, 0)]) < 1e-14
    assert abs(z[op.lm_index(1, 1)]) < 1e-14 and z[op.lm_index(1, -1)] < -1e-3
    # orthonormal over the sphere (Gauss-Legendre in cos(theta) x uniform phi)
    lmax = 3
    x, wx = np.polynomial.legendre.leggauss(24)
    phis = np.linspace(0, 2 * np.pi, 48, endpoint=False)
    gram = np.zeros(((lmax + 1) ** 2,) * 2)
    for ct, w in zip(x, wx):
        st = np.sqrt(1 - ct * ct)
        for ph in phis:
            y = op.real_ylm(lmax, np.array([st * np.cos(ph), st * np.sin(ph), ct]))
            gram += w * (2 * np.pi / len(phis)) * np.outer(y, y)
    assert np.max(np.abs(gram - np.eye(len(gram)))) < 1e-12
    assert op.angular_phase(1) == -1j and op.angular_phase(6) == -1.0


def test_gamma_oracle_is_the_full_sphere_operator():
    """The Gamma restatement (two bands per transform, real overlaps) on states that are real in
    real space gives the full-sphere oracle's H|psi> on the half sphere, for an even and an odd
    band count."""
    from oracle import gamma as og
    sy = synthetic.small_system(nbands=5, grid=(16, 16, 16), a=8.0, ecut=10.0, natoms=3)
    kp = sy.kpoints[0]
    g = synthetic.gamma_kpoint(sy)
    assert np.array_equal(g.index, og.half_sphere(kp.miller))
    assert np.array_equal(g.minus_g_to_grid, og.minus_grid_index(kp.miller[g.index], sy.cell.grid))
    key = {tuple(m): i for i, m in enumerate(kp.miller)}
    mirror = np.array([key[tuple(-kp.miller[i])] for i in g.index])
    assert 2 * g.npw - 1 == kp.npw
    for nb in (4, 5):
        rng = np.random.default_rng(nb)
        ph = rng.standard_normal((g.npw, nb)) + 1j * rng.standard_normal((g.npw, nb))
        ph[0] = ph[0].real
        full = np.zeros((kp.npw, nb), complex)
        full[g.index] = ph
        full[mirror[1:]] = np.conj(ph[1:])
        ref = hpsi.apply_h(full, kp, sy.v_r, sy.cell.grid)[g.index]
        got = og.apply_h_gamma(ph, g.ke, g.g_to_grid, g.minus_g_to_grid, g.beta, g.d_blocks,
                               g.atom_proj_offsets, sy.v_r, sy.cell.grid)
        assert np.max(np.abs(got - ref)) < 1e-13 * np.max(np.abs(ref))


def test_gamma_overlap_oracle_is_the_full_sphere_operator():
    """The Gamma restatement of S (real overlaps) equals the full-sphere S on states that are
    real in real space, restricted to the half sphere."""
    from oracle import overlap as oov
    sy = synthetic.small_system(nbands=4, grid=(16, 16, 16), a=8.0, ecut=10.0, natoms=3)
    kp = sy.kpoints[0]
    g = synthetic.gamma_kpoint(sy)
    q = synthetic.overlap_blocks(sy)
    key = {tuple(m): i for i, m in enumerate(kp.miller)}
    mirror = np.array([key[tuple(-kp.miller[i])] for i in g.index])
    rng = np.random.default_rng(9)
    ph = rng.standard_normal((g.npw, 4)) + 1j * rng.standard_normal((g.npw, 4))
    ph[0] = ph[0].real
    full = np.zeros((kp.npw, 4), complex)
    full[g.index] = ph
    full[mirror[1:]] = np.conj(ph[1:])
    ref = oov.apply_s(full, kp.beta, q, kp.atom_proj_offsets)[g.index]
    got = oov.apply_s_gamma(ph, g.beta, q, g.atom_proj_offsets)
    assert np.max(np.abs(got - ref)) < 1e-13 * np.max(np.abs(ref))
