"""Host-side mirror of the reference's ``StartingSubspaceSolver``.

``wavefunction/planewave/starting_subspace_solver.hpp:29-59``: apply H to the
starting vectors, project H and S onto them, rotate them into bands; and the
initializer's whole rotation (``wavefunction/planewave/norm_conserving/
initializer.hpp:250-385``: the three steps around a zhegv itype 1 on the upper
triangles, eigenvalues and bands of the nb lowest).  FP64, on libq3b.so's
kernels at the applicator's prepared k-point.
"""
from __future__ import annotations

import numpy as np

from ._lib import check


class StartingSubspaceSolver:
    def __init__(self, applicator):
        self.ap = applicator
        self.lib = applicator.lib
        self.n = 0

    def apply_hamiltonian(self, vectors: np.ndarray, number_of_vectors: int) -> None:
        """vectors: npw x n (column-major / Fortran order) complex128 on the host."""
        chi = np.asfortranarray(vectors, dtype=np.complex128)
        check(self.ap.h, self.lib.q3b_start_apply(self.ap.h, chi.ctypes.data, int(number_of_vectors)))
        self.n = int(number_of_vectors)

    def project(self):
        """(H, S), each n x n: H_ij = chi_i^H (H chi)_j, S_ij = chi_i^H chi_j."""
        h = np.empty((self.n, self.n), dtype=np.complex128, order="F")
        s = np.empty_like(h)
        check(self.ap.h, self.lib.q3b_start_project(self.ap.h, h.ctypes.data, s.ctypes.data))
        return h, s

    def rotate_into_bands(self, coefficients: np.ndarray, number_of_bands: int):
        """Bands chi c[:, :nb] as a CUDA tensor (nb x npw, row b = band b)."""
        import torch
        c = np.asfortranarray(coefficients[:, :number_of_bands], dtype=np.complex128)
        out = torch.empty((number_of_bands, self.ap.npw), dtype=torch.complex128,
                          device=torch.device("cuda", self.ap.ctx.device))
        with self.ap.ctx.ordered_with_torch():
            rc = self.lib.q3b_start_rotate(self.ap.h, c.ctypes.data, int(number_of_bands), out.data_ptr())
        check(self.ap.h, rc)
        return out


def rotate_starting_vectors(applicator, vectors: np.ndarray, number_of_bands: int):
    """The initializer's rotation on the device.  Returns (eigenvalues (nb,),
    bands as a CUDA tensor nb x npw)."""
    import torch
    chi = np.asfortranarray(vectors, dtype=np.complex128)
    n = chi.shape[1]
    out = torch.empty((number_of_bands, applicator.npw), dtype=torch.complex128,
                      device=torch.device("cuda", applicator.ctx.device))
    eig = np.empty(number_of_bands, dtype=np.float64)
    with applicator.ctx.ordered_with_torch():
        rc = applicator.lib.q3b_starting_subspace(applicator.h, chi.ctypes.data, n, int(number_of_bands),
                                                  out.data_ptr(), eig.ctypes.data)
    check(applicator.h, rc)
    return eig, out
