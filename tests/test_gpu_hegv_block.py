"""The one-block subspace eigensolver (q3_b200/csrc/dense_block.cu) on the GPU.

Problems of order up to about 110 fit one thread block; the library solves
them there alone up to order 64 (the Davidson's subspace solves of small
cells) and many per launch at any fitting order (q3b_hegv_batched).  Checked
against LAPACK (scipy's zhegv) and against the multi-kernel path of the same
library: eigenvalues within 1e-12 of the largest |eigenvalue| (times n/16 above
order 16), residuals |H z - w S z| within 1e-11, and S-orthonormal vectors.
"""
import numpy as np
import pytest
import scipy.linalg as sla

from q3_b200._lib import Q3BError

pytestmark = pytest.mark.gpu


def _problem(n, seed, nvec=None):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    h = (x + x.conj().T) / 2
    y = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    s = np.eye(n) + 1e-2 * (y @ y.conj().T) / n
    return h, s


def _check(h, s, w, z, nvec):
    n = h.shape[0]
    we = sla.eigh(h, s, eigvals_only=True)[:nvec]
    scale = max(1.0, float(np.max(np.abs(we))))
    f = max(1.0, n / 16)
    assert np.max(np.abs(w - we)) < 1e-12 * scale * f
    assert np.max(np.abs(h @ z - (s @ z) * w[None, :])) < 1e-11 * scale * f
    assert np.max(np.abs(z.conj().T @ s @ z - np.eye(nvec))) < 1e-11 * f


@pytest.fixture(scope="module")
def ap():
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    return PlanewaveHamiltonianApplicator()


@pytest.mark.parametrize("n,nvec", [(1, 1), (2, 1), (3, 3), (5, 2), (16, 8), (17, 17), (33, 16), (48, 24),
                                    (64, 32), (70, 70), (96, 48), (100, 50), (110, 16), (128, 16)])
def test_block_hegv_matches_lapack_and_the_multi_kernel_path(cuda_device, ap, n, nvec):
    from q3_b200.davidson import hegv_lowest, set_block_eigensolver_order
    h, s = _problem(n, 100 + n)
    prev = set_block_eigensolver_order(128)
    try:
        w, z = hegv_lowest(ap, h, s, nvec)
        _check(h, s, w, z, nvec)
        set_block_eigensolver_order(0)
        w2, z2 = hegv_lowest(ap, h, s, nvec)
    finally:
        set_block_eigensolver_order(prev)
    scale = max(1.0, float(np.max(np.abs(w2))))
    assert np.max(np.abs(w - w2)) < 1e-12 * scale * max(1.0, n / 16)


def test_block_hegv_degenerate(cuda_device, ap):
    # exact degeneracies (as in symmetric cells): the vectors of a multiple
    # eigenvalue come out orthonormal
    from q3_b200.davidson import hegv_lowest, set_block_eigensolver_order
    rng = np.random.default_rng(7)
    n, nvec = 60, 30
    q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    ev = np.round(rng.standard_normal(n) * 2.0)
    h = q @ np.diag(ev) @ q.conj().T
    prev = set_block_eigensolver_order(128)
    try:
        w, z = hegv_lowest(ap, h, np.eye(n), nvec)
    finally:
        set_block_eigensolver_order(prev)
    assert np.max(np.abs(w - np.sort(ev)[:nvec])) < 1e-12
    assert np.max(np.abs(z.conj().T @ z - np.eye(nvec))) < 1e-11
    assert np.max(np.abs(h @ z - z * w[None, :])) < 1e-11


def test_block_hegv_not_positive_definite(cuda_device, ap):
    from q3_b200.davidson import hegv_lowest
    with pytest.raises(Q3BError):
        hegv_lowest(ap, np.eye(4, dtype=complex), np.diag([1.0, 2.0, -1.0, 1.0]).astype(complex), 2)


def test_hegv_batched(cuda_device, ap):
    from q3_b200.davidson import hegv_batched
    sizes = [(8, 4), (16, 8), (24, 12), (40, 20), (48, 24), (64, 32), (96, 48), (100, 50)] * 4
    probs = [(*_problem(n, 500 + i), nv) for i, (n, nv) in enumerate(sizes)]
    # one problem whose S is not positive definite at order 3
    bad = np.eye(6, dtype=complex)
    bad[2, 2] = -1.0
    probs[5] = (np.eye(6, dtype=complex), bad, 3)
    out = hegv_batched(ap, probs)
    assert len(out) == len(probs)
    for i, ((h, s, nv), (w, z, info)) in enumerate(zip(probs, out)):
        if i == 5:
            assert info == 6 + 3
            continue
        assert info == 0
        _check(h, s, w, z, nv)
