"""The complex GEMMs of the path (q3b_gemm FP64, q3b_gemm_single on the tensor
cores) against numpy, over tile edges, split-K and odd leading dimensions.

Bars: FP64 within 1e-13 of sum |a||b| per entry; FP32 (TF32 split into hi+lo,
three products, FP32 accumulation) within 2e-6 of sum |a||b| per entry --
the accuracy of an FP32 GEMM.
"""
import ctypes as C

import numpy as np
import pytest

from q3_b200._lib import Cplx64, Cplx128, check

pytestmark = pytest.mark.gpu

SHAPES = [
    # (trans_a, m, n, k)
    ("C", 512, 256, 23847),   # <beta|psi> of the 64-atom cell
    ("C", 130, 70, 1000),     # tile edges on M and N
    ("C", 17, 9, 33),         # below one tile
    ("C", 256, 256, 6000),    # subspace block V^H HV
    ("N", 23847, 256, 512),   # beta (D <beta|psi>)
    ("N", 1000, 65, 129),     # edges on every axis
    ("N", 3000, 48, 96),      # corrections of config 2
    ("N", 64, 8, 7),
]


@pytest.fixture(scope="module")
def ctx(cuda_device):
    from q3_b200.applicator import Context
    return Context()


def _mats(rng, ta, m, n, k, lda_pad=1):
    ar = (k, m) if ta == "C" else (m, k)
    a = rng.standard_normal(ar) + 1j * rng.standard_normal(ar)
    b = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
    c = rng.standard_normal((m, n)) + 1j * rng.standard_normal((m, n))
    return a, b, c


def _dev(x, dtype, pad=0):
    """Column-major device copy with leading dimension rows + pad."""
    import torch
    rows, cols = x.shape
    buf = np.zeros((cols, rows + pad), dtype=dtype)
    buf[:, :rows] = x.T
    return torch.from_numpy(buf).cuda(), rows + pad


@pytest.mark.parametrize("ta,m,n,k", SHAPES)
@pytest.mark.parametrize("single", [False, True], ids=["fp64", "fp32"])
def test_gemm(ctx, ta, m, n, k, single):
    import torch
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    a, b, c = _mats(rng, ta, m, n, k)
    alpha, beta = 0.75 - 0.5j, (0.25 + 0.125j if k % 2 else 0.0)
    ref = alpha * ((a.conj().T if ta == "C" else a) @ b) + beta * c
    scale = np.abs(alpha) * ((np.abs(a).T if ta == "C" else np.abs(a)) @ np.abs(b)) + np.abs(beta) * np.abs(c)
    dt = np.complex64 if single else np.complex128
    A, lda = _dev(a, dt, pad=1)
    B, ldb = _dev(b, dt, pad=3)
    Cd, ldc = _dev(c, dt, pad=0)
    lib, h = ctx.lib, ctx.handle
    if single:
        rc = lib.q3b_gemm_single(h, ta.encode(), b"N", m, n, k, Cplx64(alpha.real, alpha.imag), A.data_ptr(),
                                 lda, B.data_ptr(), ldb, Cplx64(beta.real, beta.imag), Cd.data_ptr(), ldc)
    else:
        rc = lib.q3b_gemm(h, ta.encode(), b"N", m, n, k, Cplx128(alpha.real, alpha.imag), A.data_ptr(), lda,
                          B.data_ptr(), ldb, Cplx128(beta.real, beta.imag), Cd.data_ptr(), ldc)
    check(h, rc)
    ctx.synchronize()
    got = Cd.cpu().numpy()[:, :m].T.astype(np.complex128)
    err = np.max(np.abs(got - ref) / scale)
    assert err < (2e-6 if single else 1e-13), err


def test_gemm_rejects_unsupported(ctx):
    from q3_b200._lib import Q3BError
    lib, h = ctx.lib, ctx.handle
    rc = lib.q3b_gemm(h, b"T", b"N", 4, 4, 4, Cplx128(1, 0), None, 4, None, 4, Cplx128(0, 0), None, 4)
    with pytest.raises(Q3BError):
        check(h, rc)
