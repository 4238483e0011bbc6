"""Oracle block-Davidson (test infrastructure only; see the package docstring).

A restatement of ``PlanewaveDavidsonDiagonalizer::solve``
(``src/layer_4_computation/diagonalizer/planewave/davidson.hpp:324-841``) with
the norm-conserving (S = identity, S|V> aliased to |V>) non-Gamma branches of
``SerialPlanewaveSubspaceManager``
(``.../internal/subspace_manager/serial.hpp``) and
``SerialSubspaceDiagonalizer::solve`` (``.../subspace/serial.hpp:18-151``).
The LAPACK calls are the reference's own: zpotrf('U'), ztrsm('R','U','N','N'),
zhegv(itype=1,'V','U').
"""
from __future__ import annotations

import dataclasses
from typing import Callable, List, Optional

import numpy as np
import scipy.linalg.blas as blas
import scipy.linalg.lapack as lapack

ITERATIVE_SOLVER_NORM_THRESHOLD = 1e-14       # tolerances.hpp:39
PRECONDITIONER_DENOMINATOR_FLOOR = 1e-4       # tolerances.hpp:50
EMPTY_BAND_RELAXATION = 5.0                   # tolerances.hpp:65
EMPTY_BAND_FLOOR = 1e-5                       # tolerances.hpp:66


@dataclasses.dataclass
class DavidsonResult:
    eigenvalues: np.ndarray
    bands: np.ndarray
    iterations: int
    h_applications: int
    unconverged: int
    trace: List[np.ndarray]                   # eigenvalues at every iteration


def orthogonalize_batch(V: np.ndarray, start: int, ncand: int) -> int:
    """subspace_manager/serial.hpp:41-553 (non-Gamma, S aliased): returns accepted."""
    if ncand == 0:
        return 0
    npw = V.shape[0]
    T = V[:, start:start + ncand]
    if start > 0:
        # serial.hpp:167-204: C = V^H T ; T -= V C
        C = V[:, :start].conj().T @ T
        T -= V[:, :start] @ C
    # serial.hpp:316-367: Cholesky QR
    G = T.conj().T @ T
    U, info = lapack.zpotrf(G, lower=0, clean=1)
    if info == 0:
        V[:, start:start + ncand] = blas.ztrsm(1.0, U, np.asfortranarray(T), side=1, lower=0,
                                               trans_a=0, diag=0)
        return ncand
    # serial.hpp:370-552: modified Gram-Schmidt fallback
    accepted = 0
    for c in range(ncand):
        src = start + c
        dst = start + accepted
        if dst != src:
            V[:, dst] = V[:, src]
        nexist = dst - start
        v = V[:, dst]
        if nexist > 0:
            Bk = V[:, start:dst]
            coef = Bk.conj().T @ v
            v -= Bk @ coef
        nrm2 = float(np.vdot(v, v).real)
        if nrm2 > ITERATIVE_SOLVER_NORM_THRESHOLD:
            V[:, dst] = v / np.sqrt(nrm2)
            accepted += 1
    return accepted


def update_subspace_matrices(V, HV, Hs, Ss, start: int, new: int, total: int) -> None:
    """subspace_manager/serial.hpp:555-678 (non-Gamma): new columns of H_sub, S_sub."""
    Hs[:total, start:start + new] = V[:, :total].conj().T @ HV[:, start:start + new]
    Ss[:total, start:start + new] = V[:, :total].conj().T @ V[:, start:start + new]


def diagonalize_subspace(Hs, Ss, n: int):
    """serial.hpp:680-756 -> subspace/serial.hpp:18-151: zhegv(1,'V','U')."""
    if n == 0:
        return np.zeros(0), np.zeros((0, 0), complex), 0
    a = np.array(Hs[:n, :n], dtype=np.complex128, order="F")
    b = np.array(Ss[:n, :n], dtype=np.complex128, order="F")
    w, v, info = lapack.zhegv(a, b, itype=1, jobz="V", uplo="U")
    return w, v, info


def build_correction_vectors(V, HV, evec, evals, converged, ke, n_b: int, nb: int,
                             max_candidates: int) -> np.ndarray:
    """subspace_manager/serial.hpp:995-1156: compacted, TPA-preconditioned corrections."""
    bands = [b for b in range(nb) if not converged[b]][:max_candidates]
    if not bands:
        return np.zeros((V.shape[0], 0), dtype=np.complex128)
    c = evec[:n_b, bands]
    eps = np.asarray([evals[b] for b in bands])
    R = (V[:, :n_b] @ c) * (-eps)[None, :]
    R += HV[:, :n_b] @ c
    x = ke[:, None] - eps[None, :]
    den = 0.5 * (1.0 + x + np.sqrt(1.0 + (x - 1.0) ** 2))
    den = np.maximum(den, PRECONDITIONER_DENOMINATOR_FLOOR)
    return R / den


def collapse_subspace(V, HV, Hs, Ss, n_b: int, nb: int) -> int:
    """subspace_manager/serial.hpp:825-945: rotate V, HV onto the lowest nb Ritz vectors."""
    w, C, info = diagonalize_subspace(Hs, Ss, n_b) if Hs is not None else (None, None, -1)
    if info != 0:
        Hf = V[:, :n_b].conj().T @ HV[:, :n_b]
        Sf = V[:, :n_b].conj().T @ V[:, :n_b]
        w, C, info = diagonalize_subspace(Hf, Sf, n_b)
    V[:, :nb] = V[:, :n_b] @ C[:, :nb]
    HV[:, :nb] = HV[:, :n_b] @ C[:, :nb]
    return nb


def solve(apply_h: Callable[[np.ndarray], np.ndarray], ke: np.ndarray, psi0: np.ndarray,
          nb: int, tolerance: float, max_iterations: int = 20, expansion: int = 2,
          stored_eigenvalues: Optional[np.ndarray] = None, occupied: Optional[int] = None,
          counter: Optional[list] = None) -> DavidsonResult:
    """davidson.hpp:324-841 with the serial subspace manager (NC, non-Gamma)."""
    npw = ke.shape[0]
    maxn = max(min(expansion * nb, npw), nb)                       # :401-404
    V = np.zeros((npw, maxn), dtype=np.complex128, order="F")
    HV = np.zeros_like(V)
    Hs = np.zeros((maxn, maxn), dtype=np.complex128, order="F")
    Ss = np.zeros_like(Hs)
    napply = 0

    def H(x):
        nonlocal napply
        napply += x.shape[1]
        return apply_h(x)

    # seed from stored bands (:1000-1045)
    basis = 0
    if psi0 is not None and psi0.shape[0] == npw:
        V[:, :nb] = psi0[:, :nb]
        acc = orthogonalize_batch(V, 0, nb)
        basis = acc
        if basis > 0:
            HV[:, :basis] = H(V[:, :basis])
    # fill from lowest-KE plane waves (:1047-1101)
    if basis < nb:
        order = sorted(range(npw), key=lambda g: (ke[g], g))
        start = basis
        ncand = 0
        for band in range(start, nb):
            V[:, basis + ncand] = 0.0
            V[order[band], basis + ncand] = 1.0
            ncand += 1
        acc = orthogonalize_batch(V, basis, ncand)
        basis += acc
        if basis - start > 0:
            HV[:, start:basis] = H(V[:, start:basis])
    update_subspace_matrices(V, HV, Hs, Ss, 0, basis, basis)       # :459-469

    if stored_eigenvalues is not None and np.any(stored_eigenvalues != 0.0):
        prev = np.array(stored_eigenvalues[:nb], dtype=np.float64)
    else:
        prev = np.real(np.diag(Hs)[:nb]).copy()                   # :483-494
    occ = nb if occupied is None else occupied
    empty_tol = max(EMPTY_BAND_RELAXATION * tolerance, EMPTY_BAND_FLOOR)
    trace = []
    unconv = nb
    for it in range(max_iterations):                               # :498
        w, C, info = diagonalize_subspace(Hs, Ss, basis)
        if info != 0 and basis > nb:                               # :521-590
            basis = collapse_subspace(V, HV, None, None, basis, nb)
            Hs[:] = 0
            Ss[:] = 0
            update_subspace_matrices(V, HV, Hs, Ss, 0, basis, basis)
            w, C, info = diagonalize_subspace(Hs, Ss, basis)
            if info != 0:
                w = np.concatenate([prev, np.zeros(max(0, basis - nb))])
        evals = np.array(w, dtype=np.float64)
        trace.append(evals[:nb].copy())
        converged = [True] * nb
        all_conv = True
        for b in range(nb):                                       # :615-629
            change = abs(evals[b] - prev[b])
            tol_b = tolerance if b < occ else empty_tol
            ok = (it != 0) and change < tol_b
            if not ok:
                all_conv = False
                converged[b] = False
        unconv = sum(1 for c in converged if not c)
        if all_conv:                                               # :649-668
            psi = V[:, :basis] @ C[:, :nb]
            return DavidsonResult(evals[:nb], psi, it + 1, napply, 0, trace)
        R = build_correction_vectors(V, HV, C, evals, converged, ke, basis, nb,
                                     maxn - basis)                 # :689-703
        ncand = R.shape[1]
        V[:, basis:basis + ncand] = R
        acc = orthogonalize_batch(V, basis, ncand)                 # :705-712
        if acc > 0:
            HV[:, basis:basis + acc] = H(V[:, basis:basis + acc])  # :728-738
        old = basis
        basis += acc
        if acc > 0:
            update_subspace_matrices(V, HV, Hs, Ss, old, acc, basis)
        if basis >= maxn:                                          # :763-808
            basis = collapse_subspace(V, HV, Hs, Ss, basis, nb)
            Hs[:] = 0
            Ss[:] = 0
            update_subspace_matrices(V, HV, Hs, Ss, 0, basis, basis)
        prev = evals[:nb].copy()
    w, C, info = diagonalize_subspace(Hs, Ss, basis)               # :816-840
    evals = np.array(w, dtype=np.float64)
    trace.append(evals[:nb].copy())
    psi = V[:, :basis] @ C[:, :nb]
    return DavidsonResult(evals[:nb], psi, max_iterations, napply, unconv, trace)


def residual_norms(apply_h, psi: np.ndarray, evals: np.ndarray) -> np.ndarray:
    """||H psi_i - eps_i psi_i|| per band (an extra metric; the reference has none)."""
    r = apply_h(psi) - psi * evals[None, :]
    return np.linalg.norm(r, axis=0)
