"""Drive the reference's own CPU H|psi> and Davidson (oracle/_ref/harness) on a synthetic system.

Test infrastructure: the golden-fixture scripts under tests/golden/ and bench.py's CPU
baseline call this; nothing on the library's path does.

``write_case`` turns a :class:`q3_b200.synthetic.System` into the harness's case file (the
cell, the forced FFT grid, the species -- two s and two p beta functions
beta_l = r^l exp(-r^2/1.5^2) on a logarithmic mesh, D diagonal in Ry -- the k-points, the
potential V(r) in the reference's flat layout), ``run`` runs the harness, and ``load`` reads
what it wrote.  The reference orders each k-point's plane waves itself
(PlaneWaveSelector, basis/planewave/internal/kpoint/plane_wave_selector.hpp); ``load``
returns that order as a permutation of the synthetic system's order.
"""
from __future__ import annotations

import dataclasses
import os
import subprocess
from pathlib import Path
from typing import Dict, List, Optional, Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
HARNESS = HERE.parent / "_ref" / "harness"

# logarithmic radial mesh r_i = exp(XMIN + i DX), i < MESH (r from 9e-4 to 20 bohr)
MESH_XMIN, MESH_DX, MESH_POINTS = -7.0, 0.0125, 801
BETA_RCUT = 10.0        # bohr: beta is below 1e-19 beyond
VALENCE = 4.0


def available() -> bool:
    return HARNESS.exists()


def d_channels_of(system) -> np.ndarray:
    """The D value of each of the four beta channels (Ry), as the synthetic recipe draws them."""
    from q3_b200 import synthetic
    rng = np.random.default_rng(system.seed)
    synthetic.local_potential(system.cell, rng)
    return rng.uniform(-synthetic.D_RANGE_RY, synthetic.D_RANGE_RY, size=len(synthetic.CHANNELS))


def write_case(system, workdir: Path, mode: str = "setup", *, hpsi_vectors: int = 0,
               hpsi_repeats: int = 1, tolerance: float = 1e-10, max_iterations: int = 200,
               davidson_kpoints: Sequence[int] = (0,), dump_projectors: bool = False,
               nbands: Optional[int] = None, dense_potential: Optional[np.ndarray] = None,
               density_grid: Optional[Sequence[int]] = None) -> Path:
    from q3_b200 import synthetic
    workdir.mkdir(parents=True, exist_ok=True)
    cell = system.cell
    lat = np.asarray(cell.lattice, dtype=np.float64)
    alat = float(np.linalg.norm(lat[0])) if np.allclose(lat, np.diag(np.diag(lat))) else float(
        2.0 * abs(lat[0, 1]))
    # V(r) on the density grid when one is given (the reference restricts it), else on
    # the wavefunction grid
    v = system.v_r if dense_potential is None else dense_potential
    np.asarray(v, dtype=np.float64).tofile(workdir / "v_r.f64")
    d = d_channels_of(system)
    lines = [
        "# written by oracle/ref/run.py",
        f"alat {alat!r}",
        "lattice " + " ".join(repr(float(x)) for x in lat.reshape(-1)),
        "grid {} {} {}".format(*cell.grid),
        *(["density_grid {} {} {}".format(*density_grid)] if density_grid is not None else []),
        f"ecutwfc {float(cell.ecut_ry)!r}",
        f"valence {VALENCE!r}",
        f"mesh {MESH_XMIN!r} {MESH_DX!r} {MESH_POINTS}",
        f"beta_width {synthetic.PROJECTOR_WIDTH!r}",
        f"beta_rcut {BETA_RCUT!r}",
        "beta_l " + " ".join(str(l) for l, _ in synthetic.CHANNELS),
        "beta_d " + " ".join(repr(float(x)) for x in d),
    ]
    for p in cell.positions_frac:
        lines.append("atom " + " ".join(repr(float(x)) for x in p))
    for kp in system.kpoints:
        lines.append("kpoint " + " ".join(repr(float(x)) for x in kp.k_frac))
    lines += [
        f"nbands {int(nbands if nbands is not None else system.nbands)}",
        f"potential {workdir / 'v_r.f64'}",
        f"mode {mode}",
        f"hpsi_vectors {int(hpsi_vectors)}",
        f"hpsi_repeats {int(hpsi_repeats)}",
        f"tolerance {float(tolerance)!r}",
        f"max_iterations {int(max_iterations)}",
        "davidson_kpoints " + " ".join(str(int(k)) for k in davidson_kpoints),
        f"dump_projectors {1 if dump_projectors else 0}",
    ]
    path = workdir / "case.txt"
    path.write_text("\n".join(lines) + "\n")
    return path


def run(case: Path, outdir: Path, threads: int = 1, timeout: float = 3600.0) -> None:
    if not available():
        raise FileNotFoundError(f"{HARNESS} is not built (make -C oracle/ref)")
    outdir.mkdir(parents=True, exist_ok=True)
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads)
    env["OPENBLAS_NUM_THREADS"] = str(threads)
    r = subprocess.run([str(HARNESS), str(case), str(outdir)], capture_output=True, text=True,
                       env=env, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference harness failed ({r.returncode}): {r.stderr.strip()}")


@dataclasses.dataclass
class RefKPoint:
    npw: int
    miller: np.ndarray            # npw x 3, the reference's order
    ke: np.ndarray
    kpg: np.ndarray               # npw x 3, bohr^-1
    g_to_grid: np.ndarray
    perm: Optional[np.ndarray]    # reference order as indices into the synthetic order
    beta: Optional[np.ndarray]    # npw x P (Fortran), when dumped


@dataclasses.dataclass
class RefSetup:
    kpoints: List[RefKPoint]
    d_blocks: np.ndarray
    atom_offsets: np.ndarray
    beta_tables: np.ndarray       # nbeta x nq
    dq: float
    volume: float
    positions: np.ndarray         # natoms x 3, bohr
    v_scaled: np.ndarray


def _read(path: Path, dtype) -> np.ndarray:
    return np.fromfile(path, dtype=dtype)


def load_setup(system, outdir: Path) -> RefSetup:
    npw = _read(outdir / "npw.i32", np.int32)
    meta = _read(outdir / "beta_meta.f64", np.float64)
    nq = int(meta[1])
    tables = _read(outdir / "beta_tables.f64", np.float64).reshape(-1, nq)
    offs = _read(outdir / "atom_offsets.i32", np.int32)
    kps = []
    for k, n in enumerate(npw):
        tag = outdir / f"k{k}"
        mil = _read(Path(f"{tag}_miller.i32"), np.int32).reshape(-1, 3).astype(np.int64)
        perm = None
        if system is not None:
            ours = system.kpoints[k].miller
            key = {tuple(m): i for i, m in enumerate(ours.tolist())}
            try:
                perm = np.array([key[tuple(m)] for m in mil.tolist()], dtype=np.int64)
            except KeyError:
                perm = None
            if perm is not None and perm.size != ours.shape[0]:
                perm = None
        bpath = Path(f"{tag}_beta.c128")
        beta = None
        if bpath.exists():
            beta = np.asfortranarray(_read(bpath, np.complex128).reshape(-1, int(n)).T)
        kps.append(RefKPoint(int(n), mil, _read(Path(f"{tag}_ke.f64"), np.float64),
                             _read(Path(f"{tag}_kpg.f64"), np.float64).reshape(-1, 3),
                             _read(Path(f"{tag}_g_to_grid.i32"), np.int32), perm, beta))
    return RefSetup(kps, _read(outdir / "d_blocks.f64", np.float64), offs, tables, float(meta[0]),
                    float(meta[2]), _read(outdir / "positions.f64", np.float64).reshape(-1, 3),
                    _read(outdir / "v_scaled.f64", np.float64))


def write_vectors(outdir: Path, k: int, name: str, vectors: np.ndarray) -> None:
    np.asfortranarray(vectors.astype(np.complex128)).reshape(-1, order="F").tofile(
        outdir / f"k{k}_{name}.c128")


def read_vectors(outdir: Path, k: int, name: str, npw: int) -> np.ndarray:
    v = _read(outdir / f"k{k}_{name}.c128", np.complex128)
    return np.asfortranarray(v.reshape(-1, npw).T)


def read_davidson(outdir: Path, k: int) -> Dict[str, np.ndarray]:
    stats = _read(outdir / f"k{k}_stats.i32", np.int32)
    return {"eigenvalues": _read(outdir / f"k{k}_eig.f64", np.float64),
            "iterations": int(stats[0]), "unconverged": int(stats[1]),
            "solve_ms": float(_read(outdir / f"k{k}_solve_ms.f64", np.float64)[0])}
