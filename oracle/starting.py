"""Starting-subspace rotation, restated on the CPU (test infrastructure only).

``SerialStartingSubspaceSolver`` (``wavefunction/planewave/
starting_subspace_solver_serial.hpp:73-260``: H chi through the serial
applicator, H_ij = chi^H H chi and S_ij = chi^H chi by ZGEMM('C','N'), bands
= chi c by ZGEMM('N','N')) and the initializer around it
(``wavefunction/planewave/norm_conserving/initializer.hpp:250-385``: zhegv
itype 1, 'V', 'U' on the two matrices, eigenvalues and bands of the lowest
number_of_bands), non-Gamma, norm-conserving (S = I on vectors).
"""
from __future__ import annotations

from typing import Callable

import numpy as np
from scipy.linalg import lapack


def project(apply_h: Callable[[np.ndarray], np.ndarray], chi: np.ndarray):
    """initializer.hpp:250-266 / serial.hpp:96-200: (H, S) of the starting vectors."""
    hchi = apply_h(chi)
    return chi.conj().T @ hchi, chi.conj().T @ chi


def rotate_into_bands(chi: np.ndarray, coefficients: np.ndarray, nb: int) -> np.ndarray:
    """serial.hpp:242-260: band n = chi (column n of the coefficients)."""
    return chi @ coefficients[:, :nb]


def starting_subspace(apply_h, chi: np.ndarray, nb: int):
    """initializer.hpp:250-385: returns (eigenvalues[:nb], bands npw x nb)."""
    h, s = project(apply_h, chi)
    w, v, info = lapack.zhegv(h, s, itype=1, jobz="V", uplo="U")
    if info != 0:
        raise np.linalg.LinAlgError(f"zhegv info {info}")
    return w[:nb], rotate_into_bands(chi, v, nb)
