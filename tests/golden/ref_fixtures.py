"""Readers for the fixtures that tests/golden/make_ref_golden.py writes from the reference's
own CPU code: the inputs of a configuration in the reference's plane-wave order, rebuilt
from the seeded synthetic recipe plus what the fixture stores (the order, beta(q) tables, D)."""
from __future__ import annotations

import dataclasses
from pathlib import Path
from typing import Optional

import numpy as np

from q3_b200 import synthetic

HERE = Path(__file__).resolve().parent
GRAM_BANDS = 32
SKETCH_SEED = 20240601
SKETCH_COLUMNS = 8


def path(cid) -> Path:
    """cid: a configuration number, or a string such as "0_dense" for a variant fixture."""
    return HERE / f"ref_config{cid}.npz"


def load(cid):
    return np.load(path(cid))


def system(cid: int):
    """The synthetic system the fixture was made from (config 3 with its first 32 bands)."""
    return synthetic.config(cid, nbands=GRAM_BANDS) if cid == 3 else synthetic.config(cid)


def sketch_columns(npw: int) -> np.ndarray:
    rng = np.random.default_rng(SKETCH_SEED)
    return rng.choice([-1.0, 1.0], size=(npw, SKETCH_COLUMNS)).astype(np.complex128)


DENSE_GRID = (48, 36, 40)
DENSE_SEED = 20240602


def dense_potential(sy, dense_grid=DENSE_GRID) -> np.ndarray:
    """A seeded V(r) (Ry) on a density grid larger than the wavefunction grid: the smooth
    synthetic potential's Fourier content plus components that only the density grid holds,
    flat (i1*D2 + i2)*D3 + i3."""
    d = tuple(int(x) for x in dense_grid)
    rng = np.random.default_rng(DENSE_SEED)
    v = 0.25 * rng.standard_normal(d)
    x = [np.arange(di) / di for di in d]
    r = np.meshgrid(*x, indexing="ij")
    v += -1.5 * np.exp(-((np.sin(np.pi * r[0]) ** 2 + np.sin(np.pi * r[1]) ** 2
                          + np.sin(np.pi * r[2]) ** 2) / 0.15))
    return np.ascontiguousarray(v.reshape(-1))


def v_checksum(v_r: np.ndarray) -> np.ndarray:
    return np.array([np.sum(v_r), np.sum(v_r * v_r), np.sum(np.abs(v_r))])


@dataclasses.dataclass
class RefKPoint:
    """One k-point in the reference's plane-wave order (fields as q3_b200.synthetic.KPoint)."""
    k_frac: np.ndarray
    miller: np.ndarray
    ke: np.ndarray
    g_to_grid: np.ndarray
    kpg: np.ndarray
    d_blocks: np.ndarray
    atom_proj_offsets: np.ndarray
    psi0: np.ndarray
    beta: Optional[np.ndarray] = None

    @property
    def npw(self) -> int:
        return int(self.ke.shape[0])


def perm_of(g, k: int = 0) -> np.ndarray:
    p = g["perm"]
    if p.ndim == 2:
        p = p[k, :int(g["npw"][k])]
    return p.astype(np.int64)


def kpoint(sy, g, k: int = 0) -> RefKPoint:
    perm = perm_of(g, k)
    kp = sy.kpoints[k]
    mil = kp.miller[perm]
    kpg = (mil + kp.k_frac[None, :]) @ sy.cell.reciprocal
    return RefKPoint(kp.k_frac, mil, kp.ke[perm], kp.g_to_grid[perm], kpg,
                     np.asarray(g["d_blocks"]), np.asarray(g["atom_offsets"]).astype(np.int32),
                     np.asfortranarray(sy.psi0[k][perm]))


def beta_l(g):
    return [[int(x) for x in g["beta_l"]]]


def tables(g):
    return np.asarray(g["beta_tables"])


def oracle_projectors(sy, g, rk: RefKPoint) -> np.ndarray:
    """The reference's projector set, rebuilt by the oracle's restatement of its builder."""
    from oracle import projectors as oproj
    tabs = [[t for t in tables(g)]]
    return np.asfortranarray(oproj.build(rk.kpg, float(g["volume"]), np.asarray(g["positions"]),
                                         [0] * sy.cell.natoms, beta_l(g), tabs, float(g["dq"])))


def prepare_on_device(ap, sy, g, rk: RefKPoint, k: int = 0) -> None:
    """prepare_kpoint with the projector set built on the device from the fixture's tables."""
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_kpoint_build(k, rk.npw, rk.g_to_grid, rk.ke, rk.kpg, float(g["volume"]),
                            np.asarray(g["positions"]), np.zeros(sy.cell.natoms, dtype=np.int32),
                            beta_l(g), tables(g), float(g["dq"]), rk.d_blocks)
