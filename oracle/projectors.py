"""Kleinman-Bylander projector set of a k-point, restated on the CPU (test
infrastructure only).

``compute_kleinman_bylander_projectors``
(``layer_3_representation/pseudopotential/planewave/internal/projector.hpp:42-199``):

  beta_{a,i,m}(G) = Omega^{-1/2} (-i)^l  f_i(|k+G|)  Y_lm(k+G)  exp(-i (k+G).r_a)

with f_i interpolated from a uniform q table by the 4-point Lagrange rule
(``math/interpolation/uniform_q_grid_table.hpp:54-63``, ``math/interpolation/lagrange.hpp:31-47``),
Y_lm the real spherical harmonics with the Condon-Shortley phase from the
normalised associated-Legendre recursion (``math/spherical/harmonics.hpp:217-330``),
the angular phase (-i)^l (``math/phase_factor.hpp:35-47``), and projectors
ordered atom by atom, beta by beta, m in the order 0, 1, -1, 2, -2, ...
(``harmonics.hpp:40-70``).  Units here are physical: k+G in bohr^-1, positions
in bohr (the reference's 2 pi (G.r) in lattice units is the same phase).
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np

ZERO_Q = 1e-10        # tolerances.hpp: zero_vector_magnitude_threshold
DEGENERATE = 1e-9     # harmonics.hpp: degenerate_direction_threshold


def lagrange_4point(table: np.ndarray, q: float, dq: float) -> float:
    """lagrange.hpp:31-47 (nodes base..base+3, evaluated at the first interval)."""
    f = q / dq
    base = int(f)
    x = f - base
    if base + 3 >= len(table):
        return 0.0
    w1, w2, w3 = 1.0 - x, 2.0 - x, 3.0 - x
    return (table[base] * w1 * w2 * w3 / 6.0 + table[base + 1] * x * w2 * w3 / 2.0
            - table[base + 2] * x * w1 * w3 / 2.0 + table[base + 3] * x * w1 * w2 / 6.0)


def interpolate(table: np.ndarray, q: float, dq: float) -> float:
    """uniform_q_grid_table.hpp:54-63."""
    if len(table) == 0:
        return 0.0
    if q < ZERO_Q:
        return float(table[0])
    return lagrange_4point(table, q, dq)


def order_sequence(l: int) -> List[int]:
    """harmonics.hpp:40-49: 0, 1, -1, 2, -2, ..."""
    out = [0]
    for m in range(1, l + 1):
        out += [m, -m]
    return out


def lm_index(l: int, m: int) -> int:
    """harmonics.hpp:61-70."""
    if m == 0:
        return l * l
    return l * l + (2 * m - 1 if m > 0 else 2 * (-m))


def real_ylm(lmax: int, v: np.ndarray) -> np.ndarray:
    """harmonics.hpp:217-330 for one vector v: values[lm_index(l, m)]."""
    n = (lmax + 1) ** 2
    out = np.zeros(n)
    g = float(np.sqrt(v @ v))
    degenerate = g < DEGENERATE
    cos_t = 0.0 if degenerate else v[2] / g
    sin_t = np.sqrt(max(0.0, 1.0 - cos_t * cos_t))
    phi = np.copysign(np.pi / 2.0, v[1]) if degenerate else np.arctan2(v[1], v[0])
    Q = {(0, 0): 1.0}
    if lmax >= 1:
        Q[(1, 0)] = cos_t
        Q[(1, 1)] = -sin_t / np.sqrt(2.0)
    for l in range(2, lmax + 1):
        for m in range(0, l - 1):
            den = np.sqrt(float(l * l - m * m))
            Q[(l, m)] = (cos_t * (2 * l - 1) / den * Q[(l - 1, m)]
                         - np.sqrt(float((l - 1) ** 2 - m * m)) / den * Q[(l - 2, m)])
        diag = np.sqrt(float(2 * l - 1))
        prev = Q[(l - 1, l - 1)]
        Q[(l, l - 1)] = cos_t * diag * prev
        Q[(l, l)] = -diag / np.sqrt(float(2 * l)) * sin_t * prev
    out[lm_index(0, 0)] = Q[(0, 0)] / np.sqrt(4 * np.pi)
    for l in range(1, lmax + 1):
        norm = np.sqrt((2 * l + 1) / (4 * np.pi))
        out[lm_index(l, 0)] = norm * Q[(l, 0)]
        off = norm * np.sqrt(2.0)
        for m in range(1, l + 1):
            out[lm_index(l, m)] = off * Q[(l, m)] * np.cos(m * phi)
            out[lm_index(l, -m)] = off * Q[(l, m)] * np.sin(m * phi)
    return out


def angular_phase(l: int) -> complex:
    """phase_factor.hpp:35-47: (-i)^l."""
    return [1.0 + 0j, -1j, -1.0 + 0j, 1j][l % 4]


def build(kpg: np.ndarray, volume: float, positions: np.ndarray, species_of_atom: Sequence[int],
          beta_l: Sequence[Sequence[int]], tables: Sequence[Sequence[np.ndarray]], dq: float) -> np.ndarray:
    """projector.hpp:42-199.  kpg: npw x 3 (bohr^-1); positions: natoms x 3 (bohr);
    beta_l[s][i], tables[s][i] per species s and beta i.  Returns npw x P."""
    npw = kpg.shape[0]
    lmax = max((l for ls in beta_l for l in ls), default=0)
    ylm = np.array([real_ylm(lmax, kpg[g]) for g in range(npw)])
    q = np.sqrt(np.sum(kpg * kpg, axis=1))
    cols = []
    for a, s in enumerate(species_of_atom):
        sf = np.exp(-1j * (kpg @ positions[a]))
        for i, l in enumerate(beta_l[s]):
            radial = np.array([interpolate(tables[s][i], q[g], dq) for g in range(npw)])
            pre = angular_phase(l) / np.sqrt(volume)
            for m in order_sequence(l):
                cols.append(radial * ylm[:, lm_index(l, m)] * sf * pre)
    return np.array(cols).T if cols else np.zeros((npw, 0), dtype=np.complex128)
