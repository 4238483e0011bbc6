"""Charge-density accumulation, restated on the CPU (test infrastructure only).

``PlanewaveChargeDensityAccumulator::accumulate_on_rho_grid``
(``layer_4_computation/charge_density/planewave/internal/accumulator.hpp:375-545``),
non-Gamma branch, for a wavefunction grid equal to the density grid: for every
occupied band (occupation >= threshold, ``:520-525``), scatter the band onto the
grid by the G -> grid map (``scatter_wavefunction_to_grid``, ``:216-240``),
unnormalised backward transform (``inverse_raw``), and add
weight * |psi(r)|^2 with weight = k-point weight * occupation / cell volume
(``:536-541``).  The caller folds the three factors into one weight per band.
"""
from __future__ import annotations

import numpy as np


def accumulate(psi: np.ndarray, g_to_grid: np.ndarray, grid, weights: np.ndarray,
               rho: np.ndarray | None = None) -> np.ndarray:
    """rho (flat, natural grid order (w1*N2 + w2)*N3 + w3) += sum_b w_b |psi_b(r)|^2.

    psi: npw x nb; weights: nb (bands with weight 0 are skipped)."""
    n1, n2, n3 = (int(x) for x in grid)
    n = n1 * n2 * n3
    out = np.zeros(n) if rho is None else rho
    on_grid = g_to_grid >= 0      # G outside the grid are dropped (:222-229)
    for b in range(psi.shape[1]):
        if weights[b] == 0.0:
            continue
        g = np.zeros(n, dtype=np.complex128)
        g[g_to_grid[on_grid]] = psi[on_grid, b]
        r = np.fft.ifftn(g.reshape(n1, n2, n3)) * n      # unnormalised backward (e^{+i})
        out += weights[b] * (r.real ** 2 + r.imag ** 2).reshape(n)
    return out
