"""Host-side mirror of the reference's ``PlanewaveDavidsonDiagonalizer``.

Same knobs as ``src/layer_4_computation/diagonalizer/planewave/davidson.hpp``
(``set_tolerance`` :847, ``set_maximum_iterations`` :270,
``set_basis_expansion_factor`` :260) and the same solve contract: bands in,
eigenpairs out, at the applicator's prepared k-point.  The solve runs entirely
in libq3b.so on the GPU.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional

import numpy as np

from . import _lib
from ._lib import FP64, MIXED, DavidsonOpts, DavidsonStats, check


@dataclasses.dataclass
class SolveResult:
    eigenvalues: np.ndarray
    bands: object
    iterations: int
    fp64_iterations: int
    h_applications: int
    unconverged: int
    collapses: int
    max_residual_norm: float
    seconds: float
    stage_ms: dict
    fp64_seconds: float
    eigenvalue_history: Optional[np.ndarray] = None  # iterations x nb Ritz values (Ry), when kept


class PlanewaveDavidsonDiagonalizer:
    def __init__(self, applicator, precision: int = FP64):
        self.ap = applicator
        self.lib = applicator.lib
        self.opts = DavidsonOpts()
        self.lib.q3b_davidson_default_opts(C.byref(self.opts))
        self.opts.precision = int(precision)
        self.history_rows = 0

    def set_tolerance(self, tolerance: float) -> None:
        self.opts.tolerance = float(tolerance)

    def set_maximum_iterations(self, n: int) -> None:
        self.opts.max_iterations = max(1, int(n))

    def set_basis_expansion_factor(self, factor: int) -> None:
        if factor >= 2:
            self.opts.basis_expansion_factor = int(factor)

    def set_precision(self, precision: int, mixed_tolerance: Optional[float] = None,
                      refine_sweeps: Optional[int] = None) -> None:
        self.opts.precision = int(precision)
        if mixed_tolerance is not None:
            self.opts.mixed_tolerance = float(mixed_tolerance)
        if refine_sweeps is not None:
            self.opts.refine_sweeps = int(refine_sweeps)

    def set_mixed_expansion_factor(self, factor: int) -> None:
        """Basis expansion factor of the mixed solve's FP32 phase (0: the library's choice)."""
        self.opts.mixed_expansion_factor = int(factor)

    def set_occupied_bands(self, n: int) -> None:
        self.opts.occupied_bands = int(n)

    def set_profile_stages(self, on: bool = True) -> None:
        self.opts.profile_stages = 1 if on else 0

    def set_eigenvalue_history(self, rows: int) -> None:
        """Keep the Ritz values of up to `rows` iterations (both phases of a mixed solve) in
        SolveResult.eigenvalue_history; 0 turns it off."""
        self.history_rows = max(0, int(rows))

    def solve(self, bands, number_of_bands: int,
              stored_eigenvalues: Optional[np.ndarray] = None) -> SolveResult:
        """bands: npw x nb numpy array (host) or a torch complex128 CUDA tensor
        laid out nb x npw (band-contiguous); the eigenvectors come back in place."""
        nb = int(number_of_bands)
        eig = np.zeros(nb, dtype=np.float64) if stored_eigenvalues is None else \
            np.ascontiguousarray(stored_eigenvalues, dtype=np.float64).copy()
        st = DavidsonStats()
        h = self.ap.h
        rows = self.history_rows
        hist = np.zeros((rows, nb), dtype=np.float64) if rows else None
        self.opts.eigenvalue_history = hist.ctypes.data if rows else None
        self.opts.history_rows = rows
        if isinstance(bands, np.ndarray):
            x = np.asfortranarray(bands, dtype=np.complex128).copy(order="F")
            rc = self.lib.q3b_davidson_solve(h, x.ctypes.data, eig.ctypes.data, nb,
                                             C.byref(self.opts), C.byref(st))
            out = x
        else:
            with self.ap.ctx.ordered_with_torch():
                rc = self.lib.q3b_davidson_solve_dev(h, bands.data_ptr(), eig.ctypes.data, nb,
                                                     C.byref(self.opts), C.byref(st))
            out = bands
        check(h, rc)
        stages = dict(zip(DavidsonStats.STAGES, list(st.stage_ms)))
        if hist is not None:
            hist = hist[:min(rows, st.iterations)].copy()
        return SolveResult(eig, out, st.iterations, st.fp64_iterations, st.h_applications,
                           st.unconverged, st.collapses, st.max_residual_norm, st.seconds, stages,
                           st.fp64_seconds, hist)


def hegv(applicator, h: np.ndarray, s: np.ndarray):
    """diagonalize_subspace on the GPU: H c = w S c (upper triangles used)."""
    import torch
    n = h.shape[0]
    dev = torch.device("cuda", applicator.ctx.device)
    H = torch.from_numpy(np.ascontiguousarray(np.asarray(h, np.complex128).T)).to(dev)
    S = torch.from_numpy(np.ascontiguousarray(np.asarray(s, np.complex128).T)).to(dev)
    w = torch.empty(n, dtype=torch.float64, device=dev)
    Z = torch.empty(n, n, dtype=torch.complex128, device=dev)
    with applicator.ctx.ordered_with_torch():
        rc = applicator.lib.q3b_hegv(applicator.h, n, H.data_ptr(), S.data_ptr(), n, w.data_ptr(), Z.data_ptr())
    check(applicator.h, rc)
    return w.cpu().numpy(), Z.cpu().numpy().T


def hegv_lowest(applicator, h: np.ndarray, s: np.ndarray, nvec: int):
    """The lowest nvec eigenpairs of H c = w S c on the GPU (upper triangles used)."""
    import torch
    n = h.shape[0]
    dev = torch.device("cuda", applicator.ctx.device)
    H = torch.from_numpy(np.ascontiguousarray(np.asarray(h, np.complex128).T)).to(dev)
    S = torch.from_numpy(np.ascontiguousarray(np.asarray(s, np.complex128).T)).to(dev)
    w = torch.empty(nvec, dtype=torch.float64, device=dev)
    Z = torch.empty(nvec, n, dtype=torch.complex128, device=dev)
    with applicator.ctx.ordered_with_torch():
        rc = applicator.lib.q3b_hegv_lowest(applicator.h, n, H.data_ptr(), S.data_ptr(), n, int(nvec),
                                            w.data_ptr(), Z.data_ptr())
    check(applicator.h, rc)
    return w.cpu().numpy(), Z.cpu().numpy().T


def hegv_batched(applicator, problems):
    """Many small generalized problems in one launch: `problems` is a list of (h, s, nvec);
    returns a list of (w, Z, info) with info 0 or n + j (S not positive definite)."""
    import torch
    dev = torch.device("cuda", applicator.ctx.device)
    count = len(problems)
    keep, ns, lds, nvs, hp, sp, wp, zp = [], [], [], [], [], [], [], []
    for h, s, nvec in problems:
        n = h.shape[0]
        H = torch.from_numpy(np.ascontiguousarray(np.asarray(h, np.complex128).T)).to(dev)
        S = torch.from_numpy(np.ascontiguousarray(np.asarray(s, np.complex128).T)).to(dev)
        w = torch.empty(nvec, dtype=torch.float64, device=dev)
        Z = torch.empty(nvec, n, dtype=torch.complex128, device=dev)
        keep.append((H, S, w, Z))
        ns.append(n)
        lds.append(n)
        nvs.append(int(nvec))
        hp.append(H.data_ptr())
        sp.append(S.data_ptr())
        wp.append(w.data_ptr())
        zp.append(Z.data_ptr())
    I = C.c_int * count
    V = C.c_void_p * count
    info = I()
    with applicator.ctx.ordered_with_torch():
        rc = applicator.lib.q3b_hegv_batched(applicator.h, count, I(*ns), V(*hp), V(*sp), I(*lds), I(*nvs),
                                             V(*wp), V(*zp), info)
    check(applicator.h, rc)
    return [(w.cpu().numpy(), Z.cpu().numpy().T, int(info[i])) for i, (_H, _S, w, Z) in enumerate(keep)]


def set_block_eigensolver_order(max_order: int) -> int:
    """Largest subspace order solved in one thread block (0: none); returns the previous."""
    return int(_lib.load().q3b_set_block_eigensolver_order(int(max_order)))
