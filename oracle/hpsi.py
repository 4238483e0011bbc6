"""Oracle H|psi> (test infrastructure only; see the package docstring).

Restates the non-Gamma branch of
``SerialPlanewaveHamiltonianApplicator::apply_hamiltonian_batch``
(``src/layer_4_computation/diagonalizer/planewave/internal/hamiltonian_applicator/serial.hpp``):

* ``update_potential`` (serial.hpp:64-78): V is pre-scaled by 1/N;
* per band (serial.hpp:450-477): hpsi = KE*psi; zero the grid; scatter psi by
  the G->grid map; unnormalised backward FFT (FFTW_BACKWARD, e^{+i});
  multiply by V/N; unnormalised forward FFT (e^{-i}); hpsi += grid[map];
* nonlocal (serial.hpp:567-700): B = beta^H psi (ZGEMM 'C','N'); B' = D B per
  atom block (ZGEMM per block); hpsi += beta B' (ZGEMM 'N','N', beta=1).
"""
from __future__ import annotations

import os
from typing import Optional

import numpy as np
import scipy.fft as sfft


def _workers(threads: Optional[int]) -> int:
    if threads is None:
        return 1
    return max(1, int(threads))


def restrict_potential(v_dense: np.ndarray, dense_grid, smooth_grid) -> np.ndarray:
    """V(r) on the wavefunction grid from V(r) on the larger density grid by G-space truncation
    (compute_smooth_grid_potential_from_dense, planewave_potential_utils.hpp:33-104, and
    inverse_fft_smooth_potential, :110-135): forward transform on the density grid divided by
    its point count, the coefficients of every wrapped wavefunction-grid index w taken at Miller
    index m = w (w <= n/2) or w - n (so +n/2 is the Nyquist representative), an unnormalised
    inverse transform on the wavefunction grid, the real part.  Flat (i1*N2 + i2)*N3 + i3 in and
    out."""
    d = tuple(int(x) for x in dense_grid)
    n = tuple(int(x) for x in smooth_grid)
    if d == n:
        return np.asarray(v_dense, dtype=np.float64).copy()          # serial.hpp:857-859
    vg = np.fft.fftn(np.asarray(v_dense, dtype=np.float64).reshape(d)) / float(np.prod(d))
    idx = []
    for ni, di in zip(n, d):
        w = np.arange(ni)
        m = np.where(w <= ni // 2, w, w - ni)
        idx.append(np.mod(m, di))
    vs = vg[np.ix_(*idx)]
    return np.ascontiguousarray((np.fft.ifftn(vs) * float(np.prod(n))).real.reshape(-1))


def scaled_potential(v_r: np.ndarray) -> np.ndarray:
    """serial.hpp:64-78: the cached potential is V(r) / N."""
    return np.asarray(v_r, dtype=np.float64) * (1.0 / v_r.size)


def apply_local(psi: np.ndarray, ke: np.ndarray, g_to_grid: np.ndarray, v_r: np.ndarray,
                grid, threads: Optional[int] = None) -> np.ndarray:
    """Kinetic + local potential part of H|psi> (serial.hpp:450-477).

    psi: npw x nvec complex (column = band).  Returns npw x nvec complex.
    """
    psi = np.asarray(psi, dtype=np.complex128)
    if psi.ndim == 1:
        psi = psi[:, None]
    npw, nvec = psi.shape
    n1, n2, n3 = grid
    vs = scaled_potential(v_r).reshape(n1, n2, n3)
    out = ke[:, None] * psi
    ok = g_to_grid >= 0
    idx = g_to_grid[ok]
    w = _workers(threads)
    chunk = max(1, min(nvec, 32))
    for b0 in range(0, nvec, chunk):
        b1 = min(nvec, b0 + chunk)
        g = np.zeros((b1 - b0, n1 * n2 * n3), dtype=np.complex128)
        g[:, idx] = psi[ok, b0:b1].T
        g = g.reshape(b1 - b0, n1, n2, n3)
        # FFTW_BACKWARD unnormalised == N * ifftn
        g = sfft.ifftn(g, axes=(1, 2, 3), norm="forward", workers=w)
        g *= vs[None]
        g = sfft.fftn(g, axes=(1, 2, 3), norm="backward", workers=w)
        g = g.reshape(b1 - b0, -1)
        out[ok, b0:b1] += g[:, idx].T
    return out


def apply_nonlocal(psi: np.ndarray, beta: np.ndarray, d_blocks: np.ndarray,
                   atom_proj_offsets: np.ndarray) -> np.ndarray:
    """Kleinman-Bylander term beta D beta^H psi (serial.hpp:567-700)."""
    psi = np.asarray(psi, dtype=np.complex128)
    if psi.ndim == 1:
        psi = psi[:, None]
    if beta.shape[1] == 0:
        return np.zeros_like(psi)
    b = beta.conj().T @ psi                       # P x nvec   (ZGEMM 'C','N')
    bp = np.zeros_like(b)
    off = 0
    for a in range(len(atom_proj_offsets) - 1):
        s, e = int(atom_proj_offsets[a]), int(atom_proj_offsets[a + 1])
        m = e - s
        if m == 0:
            continue
        blk = d_blocks[off:off + m * m].reshape(m, m, order="F")
        off += m * m
        blk = np.where(np.abs(blk) > 1e-15, blk, 0.0)  # d_matrix_element_threshold
        bp[s:e] = blk @ b[s:e]
    return beta @ bp                              # ZGEMM 'N','N'


def apply_h(psi: np.ndarray, kp, v_r: np.ndarray, grid, threads: Optional[int] = None) -> np.ndarray:
    """Full H|psi> for one k-point of a synthetic system."""
    out = apply_local(psi, kp.ke, kp.g_to_grid, v_r, grid, threads)
    out += apply_nonlocal(psi, kp.beta, kp.d_blocks, kp.atom_proj_offsets)
    return out


def dense_hamiltonian(kp, v_r: np.ndarray, grid) -> np.ndarray:
    """The npw x npw matrix of H (small cells only): a direct cross-check."""
    npw = kp.npw
    eye = np.eye(npw, dtype=np.complex128)
    return apply_h(eye, kp, v_r, grid)
