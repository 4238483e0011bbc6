"""Oracle Gamma-only H|psi> on half-sphere coefficient vectors (test infrastructure only).

Restates the Gamma branch of ``SerialPlanewaveHamiltonianApplicator::apply_hamiltonian_batch``
(``src/layer_4_computation/diagonalizer/planewave/internal/hamiltonian_applicator/serial.hpp``):

* local part, two bands per complex transform (serial.hpp:283-418): hpsi = KE*psi; band pair
  (2p, 2p+1) scattered as psi_1(G) + i psi_2(G) at +G and conj(psi_1(G)) + i conj(psi_2(G)) at
  -G, the origin (index 0) once as (Re psi_1(0), Re psi_2(0)); unnormalised backward FFT, times
  V/N, forward FFT; hpsi_1 += (F(+G) + conj F(-G)) / 2, hpsi_2 += -i (F(+G) - conj F(-G)) / 2, at
  the origin Re F and Im F.  A last band without a partner is scattered alone (psi at +G, its
  conjugate at -G for G != 0) and gathered from +G;
* the -G grid index of every G from its negated Miller index (serial.hpp:889-900);
* nonlocal part (serial.hpp:519-566 and the shared D and accumulate steps): the overlaps are
  real, 2 Re(beta^H psi) over the half sphere minus the origin's Re(conj(beta(0)) psi(0)); D per
  atom block; hpsi += beta B'.

The index-0 entry of the half sphere is the origin (the reference's `gamma_origin_is_local`).
"""
from __future__ import annotations

from typing import Optional, Tuple

import numpy as np
import scipy.fft as sfft

from .hpsi import scaled_potential


def half_sphere(miller: np.ndarray) -> np.ndarray:
    """Indices of a half sphere in a full-sphere Miller list: the origin first, then every G
    whose first nonzero Miller index is positive, in list order."""
    m = np.asarray(miller)
    first = np.where(m[:, 0] != 0, m[:, 0], np.where(m[:, 1] != 0, m[:, 1], m[:, 2]))
    origin = np.where(np.all(m == 0, axis=1))[0]
    if origin.size != 1:
        raise ValueError("the sphere must hold the origin once")
    pos = np.where(first > 0)[0]
    return np.concatenate([origin, pos]).astype(np.int64)


def minus_grid_index(miller: np.ndarray, grid: Tuple[int, int, int]) -> np.ndarray:
    """serial.hpp:889-900: the grid index of -G (-1 outside the grid)."""
    n = np.array(grid)
    m = -np.asarray(miller)
    out = np.full(m.shape[0], -1, dtype=np.int32)
    ok = np.all(np.abs(m) <= n[None, :] // 2, axis=1)
    w = np.where(m < 0, m + n[None, :], m)
    flat = (w[:, 0] * n[1] + w[:, 1]) * n[2] + w[:, 2]
    out[ok] = flat[ok].astype(np.int32)
    return out


def apply_local_gamma(psi: np.ndarray, ke: np.ndarray, g2g: np.ndarray, g2g_minus: np.ndarray,
                      v_r: np.ndarray, grid, threads: Optional[int] = None) -> np.ndarray:
    """serial.hpp:283-418 on npw_half x nvec vectors (column = band)."""
    psi = np.asarray(psi, dtype=np.complex128)
    npw, nvec = psi.shape
    n1, n2, n3 = grid
    N = n1 * n2 * n3
    vs = scaled_potential(v_r).reshape(n1, n2, n3)
    out = ke[:, None] * psi
    w = 1 if threads is None else max(1, int(threads))
    plus = g2g
    ok = plus >= 0
    for p in range(0, nvec, 2):
        g = np.zeros(N, dtype=np.complex128)
        p1 = psi[:, p]
        if p + 1 < nvec:
            p2 = psi[:, p + 1]
            if plus[0] >= 0:
                g[plus[0]] = p1[0].real + 1j * p2[0].real
            sel = np.arange(1, npw)[ok[1:]]
            g[plus[sel]] = p1[sel] + 1j * p2[sel]
            g[g2g_minus[sel]] = np.conj(p1[sel]) + 1j * np.conj(p2[sel])
        else:
            g[plus[ok]] = p1[ok]
            mm = np.arange(1, npw)[g2g_minus[1:] >= 0]
            g[g2g_minus[mm]] = np.conj(p1[mm])
        f = sfft.ifftn(g.reshape(n1, n2, n3), norm="forward", workers=w)
        f *= vs
        f = sfft.fftn(f, norm="backward", workers=w).reshape(-1)
        if p + 1 < nvec:
            if plus[0] >= 0:
                out[0, p] += f[plus[0]].real
                out[0, p + 1] += f[plus[0]].imag
            sel = np.arange(1, npw)[ok[1:]]
            fp = f[plus[sel]]
            fm = np.conj(f[g2g_minus[sel]])
            out[sel, p] += 0.5 * (fp + fm)
            d = 0.5 * (fp - fm)
            out[sel, p + 1] += d.imag - 1j * d.real
        else:
            out[ok, p] += f[plus[ok]]
    return out



def apply_nonlocal_gamma(psi: np.ndarray, beta: np.ndarray, d_blocks: np.ndarray,
                         atom_proj_offsets: np.ndarray) -> np.ndarray:
    """serial.hpp:519-566: real overlaps 2 Re(beta^H psi) - Re(conj beta(0) psi(0)), then D per
    atom block and hpsi += beta B'."""
    psi = np.asarray(psi, dtype=np.complex128)
    if beta.shape[1] == 0:
        return np.zeros_like(psi)
    x = 2.0 * (beta.real.T @ psi.real + beta.imag.T @ psi.imag)
    x -= (np.conj(beta[0])[:, None] * psi[0][None, :]).real
    bp = np.zeros_like(x)
    off = 0
    for a in range(len(atom_proj_offsets) - 1):
        s, e = int(atom_proj_offsets[a]), int(atom_proj_offsets[a + 1])
        m = e - s
        if m == 0:
            continue
        blk = d_blocks[off:off + m * m].reshape(m, m, order="F")
        off += m * m
        blk = np.where(np.abs(blk) > 1e-15, blk, 0.0)
        bp[s:e] = blk @ x[s:e]
    return beta @ bp.astype(np.complex128)


def apply_h_gamma(psi: np.ndarray, ke, g2g, g2g_minus, beta, d_blocks, atom_proj_offsets, v_r, grid,
                  threads: Optional[int] = None) -> np.ndarray:
    out = apply_local_gamma(psi, ke, g2g, g2g_minus, v_r, grid, threads)
    out += apply_nonlocal_gamma(psi, beta, d_blocks, atom_proj_offsets)
    return out
