"""Oracle ultrasoft overlap operator S (test infrastructure only).

Restates ``UltrasoftPseudopotentialOverlapOperator::apply_batch``
(``src/layer_4_computation/diagonalizer/planewave/internal/overlap/pseudopotential/ultrasoft/init.hpp``):

* S psi starts as a copy of psi (init.hpp:193-196);
* B = beta^H psi (ZGEMM 'C','N', init.hpp:272-289), or at a Gamma-only k-point the real
  overlaps 2 Re(beta^H psi) over the half sphere less the origin's Re(conj(beta(0)) psi(0))
  (DGEMM on interleaved parts, init.hpp:212-270);
* B' = Q B with Q block-diagonal by atom, entries |q| <= 1e-15 dropped (build_q_matrix,
  init.hpp:416-466, applied by ZGEMM at :292-323);
* S psi += beta B' (ZGEMM 'N','N', beta = 1, init.hpp:325-345).
"""
from __future__ import annotations

import numpy as np


def _apply_blocks(q_blocks: np.ndarray, offsets: np.ndarray, b: np.ndarray) -> np.ndarray:
    out = np.zeros_like(b)
    off = 0
    for a in range(len(offsets) - 1):
        s, e = int(offsets[a]), int(offsets[a + 1])
        m = e - s
        if m == 0:
            continue
        blk = q_blocks[off:off + m * m].reshape(m, m, order="F")
        off += m * m
        blk = np.where(np.abs(blk) > 1e-15, blk, 0.0)
        out[s:e] = blk @ b[s:e]
    return out


def apply_s(psi: np.ndarray, beta: np.ndarray, q_blocks: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    psi = np.asarray(psi, dtype=np.complex128)
    b = beta.conj().T @ psi
    return psi + beta @ _apply_blocks(q_blocks, offsets, b)


def apply_s_gamma(psi: np.ndarray, beta: np.ndarray, q_blocks: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    psi = np.asarray(psi, dtype=np.complex128)
    x = 2.0 * (beta.real.T @ psi.real + beta.imag.T @ psi.imag)
    x -= (np.conj(beta[0])[:, None] * psi[0][None, :]).real
    return psi + beta @ _apply_blocks(q_blocks, offsets, x).astype(np.complex128)
