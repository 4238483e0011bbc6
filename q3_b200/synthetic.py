"""Seeded synthetic plane-wave systems: the inputs of the H|psi> and Davidson path.

Builds, for a cell, a cutoff and an FFT grid, exactly the data the reference
hands its applicator and Davidson solver:

* the plane-wave list of a k-point, |k+G|^2 <= ecut (Ry), sorted by kinetic
  energy (``plane_wave_selector.hpp:78-108``), with the kinetic factor
  |k+G|^2 in Ry (``plane_wave_selector.hpp:87-91``);
* the G -> FFT-grid map ``(w1*N2 + w2)*N3 + w3`` with negative Miller indices
  wrapped, -1 outside the grid (``planewave_potential_utils.hpp:141-164``,
  ``fft_grid_serial.hpp:301-307``);
* the Kleinman-Bylander projector matrix, npw x P column-major, projector p at
  offset p*npw (``kleinman_bylander_projector_set.hpp:20-23``), with value
  (1/sqrt(Omega)) (-i)^l beta_l(|k+G|) Y_lm e^{-i(k+G).tau}
  (``projector.hpp:27-30,187-194``), and its per-atom D blocks (Ry);
* the local potential V(r) on the grid (Ry), in the reference's flat layout;
* seeded, orthonormalised starting bands.

Units are Rydberg and bohr throughout.  The synthetic recipe: Gaussian wells of
depth -4 Ry (-2 Ha) and sigma 1 bohr at every atom (a periodic sum, built in
G-space), plus a seeded Hermitian random field with Fourier components of
standard deviation 0.1 Ry (0.05 Ha) for |G| < 3 bohr^-1; two s and two p
projectors per atom with beta_l(r) = r^l exp(-r^2/1.5^2) (radial transforms in
closed form), D diagonal per species, seeded uniformly in [-2, 2] Ry.

This module is product code (input generation for the library's users, the
benchmark and the tests); it computes nothing on the H|psi> path itself.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

HA_TO_RY = 2.0
PROJECTOR_WIDTH = 1.5          # bohr, beta_l(r) = r^l exp(-r^2 / w^2)
WELL_DEPTH_RY = -4.0           # -2 Ha
WELL_SIGMA = 1.0               # bohr
RANDOM_FIELD_GMAX = 3.0        # bohr^-1
RANDOM_FIELD_STD_RY = 0.1      # 0.05 Ha
D_RANGE_RY = 2.0               # D_ii ~ U[-1, 1] Ha
# channel list per atom: (l, channel) -> two s and two p projectors
CHANNELS = ((0, 0), (0, 1), (1, 0), (1, 1))
PROJECTORS_PER_ATOM = 8        # 1 + 1 + 3 + 3


@dataclasses.dataclass
class Cell:
    lattice: np.ndarray            # 3x3, rows are a1, a2, a3 (bohr)
    positions_frac: np.ndarray     # natoms x 3
    grid: Tuple[int, int, int]
    ecut_ry: float

    @property
    def volume(self) -> float:
        return float(abs(np.linalg.det(self.lattice)))

    @property
    def reciprocal(self) -> np.ndarray:
        """Rows b1, b2, b3 with a_i . b_j = 2 pi delta_ij."""
        return 2.0 * np.pi * np.linalg.inv(self.lattice).T

    @property
    def natoms(self) -> int:
        return int(self.positions_frac.shape[0])

    @property
    def npoints(self) -> int:
        n1, n2, n3 = self.grid
        return n1 * n2 * n3


@dataclasses.dataclass
class KPoint:
    k_frac: np.ndarray             # in reciprocal-lattice coordinates
    miller: np.ndarray             # npw x 3 int
    ke: np.ndarray                 # npw, |k+G|^2 in Ry
    g_to_grid: np.ndarray          # npw int32, flat grid index or -1
    beta: np.ndarray               # npw x P complex128, Fortran order
    d_blocks: np.ndarray           # packed per-atom blocks (column-major), float64
    atom_proj_offsets: np.ndarray  # natoms+1 int32

    @property
    def npw(self) -> int:
        return int(self.ke.shape[0])

    @property
    def nproj(self) -> int:
        return int(self.beta.shape[1])

    def d_dense(self) -> np.ndarray:
        """The block-diagonal D as a dense P x P matrix (for checks only)."""
        p = self.nproj
        d = np.zeros((p, p))
        off = 0
        for a in range(len(self.atom_proj_offsets) - 1):
            s, e = int(self.atom_proj_offsets[a]), int(self.atom_proj_offsets[a + 1])
            m = e - s
            d[s:e, s:e] = self.d_blocks[off:off + m * m].reshape(m, m, order="F")
            off += m * m
        return d


@dataclasses.dataclass
class System:
    name: str
    cell: Cell
    v_r: np.ndarray                # N float64, flat index (i1*N2+i2)*N3+i3
    kpoints: List[KPoint]
    nbands: int
    psi0: List[np.ndarray]         # per k: npw x nb complex128 (Fortran order)
    seed: int


# ----------------------------------------------------------------- lattices

def fcc_lattice(a: float) -> np.ndarray:
    return 0.5 * a * np.array([[0.0, 1.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 0.0]])


def cubic_lattice(a: float) -> np.ndarray:
    return a * np.eye(3)


def random_positions(rng: np.random.Generator, lattice: np.ndarray, natoms: int,
                     min_distance: float = 2.0, max_tries: int = 200000) -> np.ndarray:
    """Uniform fractional positions with a minimum periodic distance (bohr)."""
    pos: List[np.ndarray] = []
    tries = 0
    while len(pos) < natoms:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place atoms at the minimum distance")
        f = rng.random(3)
        ok = True
        for q in pos:
            d = f - q
            d -= np.round(d)
            if np.linalg.norm(d @ lattice) < min_distance:
                ok = False
                break
        if ok:
            pos.append(f)
    return np.array(pos)


def monkhorst_pack(n: Sequence[int], shift: Sequence[int]) -> np.ndarray:
    """k_i = (2 j - n + 1 + s) / (2 n) per direction (QE convention), fractional."""
    axes = [np.array([(2 * j - ni + 1 + si) / (2.0 * ni) for j in range(ni)])
            for ni, si in zip(n, shift)]
    kk = np.array(np.meshgrid(*axes, indexing="ij")).reshape(3, -1).T
    return kk


# ----------------------------------------------------------- plane waves

def plane_waves(cell: Cell, k_frac: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Miller indices and kinetic factors of |k+G|^2 <= ecut, sorted by energy."""
    b = cell.reciprocal
    gmax = math.sqrt(cell.ecut_ry)
    lens = np.linalg.norm(cell.lattice, axis=1)
    mmax = [int(math.ceil(gmax * lens[i] / (2.0 * np.pi))) + 2 for i in range(3)]
    r = [np.arange(-m, m + 1) for m in mmax]
    mil = np.array(np.meshgrid(*r, indexing="ij")).reshape(3, -1).T
    kg = (mil + k_frac[None, :]) @ b
    ke = np.einsum("ij,ij->i", kg, kg)
    sel = ke <= cell.ecut_ry + 1e-10
    mil, ke = mil[sel], ke[sel]
    order = np.argsort(ke, kind="stable")
    return mil[order].astype(np.int64), ke[order].astype(np.float64)


def grid_map(miller: np.ndarray, grid: Tuple[int, int, int]) -> np.ndarray:
    n = np.array(grid)
    out = np.full(miller.shape[0], -1, dtype=np.int32)
    ok = np.all(np.abs(miller) <= n[None, :] // 2, axis=1)
    w = np.where(miller < 0, miller + n[None, :], miller)
    flat = (w[:, 0] * n[1] + w[:, 1]) * n[2] + w[:, 2]
    out[ok] = flat[ok].astype(np.int32)
    return out


def grid_miller(grid: Tuple[int, int, int]) -> np.ndarray:
    """Miller index of every grid point, flat order."""
    axes = []
    for n in grid:
        i = np.arange(n)
        axes.append(np.where(i <= n // 2, i, i - n))
    return np.array(np.meshgrid(*axes, indexing="ij")).reshape(3, -1).T


# ---------------------------------------------------------- projectors

def _radial_transform(l: int, q: np.ndarray) -> np.ndarray:
    """4 pi int r^2 j_l(qr) beta_l(r) dr for beta_l = r^l exp(-r^2/w^2), closed form."""
    w = PROJECTOR_WIDTH
    g = np.exp(-0.25 * (q * w) ** 2)
    if l == 0:
        return np.pi ** 1.5 * w ** 3 * g
    if l == 1:
        return 0.5 * np.pi ** 1.5 * w ** 5 * q * g
    raise ValueError(l)


def projectors(cell: Cell, k_frac: np.ndarray, miller: np.ndarray,
               d_channels: np.ndarray) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Projector matrix (npw x P, Fortran), packed D blocks and atom offsets."""
    b = cell.reciprocal
    q = (miller + k_frac[None, :]) @ b                 # npw x 3
    qn = np.linalg.norm(q, axis=1)
    inv_sqrt_omega = 1.0 / math.sqrt(cell.volume)
    tau = cell.positions_frac @ cell.lattice           # natoms x 3
    npw = miller.shape[0]
    na = cell.natoms
    P = na * PROJECTORS_PER_ATOM
    beta = np.zeros((npw, P), dtype=np.complex128, order="F")
    # angular parts (real harmonics) with the radial transforms folded in
    f0 = _radial_transform(0, qn) / math.sqrt(4.0 * np.pi)
    # F_1(q) * sqrt(3/4pi) * q_m / |q|  ->  0.5 pi^1.5 w^5 g * sqrt(3/4pi) * q_m
    w = PROJECTOR_WIDTH
    g = np.exp(-0.25 * (qn * w) ** 2)
    f1 = 0.5 * np.pi ** 1.5 * w ** 5 * g * math.sqrt(3.0 / (4.0 * np.pi))
    minus_i = -1j
    shapes = []
    for (l, _ch) in CHANNELS:
        if l == 0:
            shapes.append([f0 + 0j])
        else:
            shapes.append([minus_i * f1 * q[:, m] for m in range(3)])
    col = 0
    d_blocks = []
    offsets = [0]
    for a in range(na):
        phase = np.exp(-1j * (q @ tau[a])) * inv_sqrt_omega
        dvals = []
        for ci, (l, _ch) in enumerate(CHANNELS):
            for comp in shapes[ci]:
                beta[:, col] = comp * phase
                dvals.append(d_channels[ci])
                col += 1
        m = len(dvals)
        d_blocks.append(np.diag(np.array(dvals)).reshape(-1, order="F"))
        offsets.append(offsets[-1] + m)
    return beta, np.concatenate(d_blocks), np.array(offsets, dtype=np.int32)


# ------------------------------------------------------------ potential

def local_potential(cell: Cell, rng: np.random.Generator) -> np.ndarray:
    """V(r) on the grid (Ry): periodic Gaussian wells plus a smooth random field."""
    n1, n2, n3 = cell.grid
    mil = grid_miller(cell.grid)
    G = mil @ cell.reciprocal
    g2 = np.einsum("ij,ij->i", G, G)
    tau = cell.positions_frac @ cell.lattice
    # wells: (1/Omega) sum_a depth (2 pi s^2)^{3/2} exp(-G^2 s^2/2) e^{-i G tau_a}
    s = WELL_SIGMA
    amp = WELL_DEPTH_RY * (2.0 * np.pi * s * s) ** 1.5 / cell.volume * np.exp(-0.5 * g2 * s * s)
    sf = np.zeros(G.shape[0], dtype=np.complex128)
    for a in range(tau.shape[0]):
        sf += np.exp(-1j * (G @ tau[a]))
    vg = amp * sf
    # Hermitian random field for |G| < 3
    inball = np.nonzero(g2 < RANDOM_FIELD_GMAX ** 2)[0]
    z = (rng.standard_normal(inball.size) + 1j * rng.standard_normal(inball.size)) \
        * (RANDOM_FIELD_STD_RY / math.sqrt(2.0))
    zfull = np.zeros(G.shape[0], dtype=np.complex128)
    zfull[inball] = z
    # partner index of -G
    neg = (-mil) % np.array([n1, n2, n3])[None, :]
    negflat = (neg[:, 0] * n2 + neg[:, 1]) * n3 + neg[:, 2]
    herm = (zfull + np.conj(zfull[negflat])) / math.sqrt(2.0)
    self_partner = negflat == np.arange(G.shape[0])
    herm[self_partner] = zfull[self_partner].real * math.sqrt(2.0) + 0j
    vg = vg + herm
    vr = np.fft.ifftn(vg.reshape(n1, n2, n3)) * cell.npoints
    return np.ascontiguousarray(vr.real.reshape(-1))


def orthonormal_bands(rng: np.random.Generator, npw: int, nb: int) -> np.ndarray:
    z = rng.standard_normal((npw, nb)) + 1j * rng.standard_normal((npw, nb))
    q, r = np.linalg.qr(z)
    return np.asfortranarray(q)


# -------------------------------------------------------------- configs

def build_system(name: str, cell: Cell, kpoints_frac: np.ndarray, nbands: int,
                 seed: int) -> System:
    rng = np.random.default_rng(seed)
    v_r = local_potential(cell, rng)
    d_channels = rng.uniform(-D_RANGE_RY, D_RANGE_RY, size=len(CHANNELS))
    kps: List[KPoint] = []
    psi0 = []
    for k in kpoints_frac:
        k = np.asarray(k, dtype=np.float64)
        mil, ke = plane_waves(cell, k)
        gmap = grid_map(mil, cell.grid)
        beta, dblk, offs = projectors(cell, k, mil, d_channels)
        kps.append(KPoint(k, mil, ke, gmap, beta, dblk, offs))
        psi0.append(orthonormal_bands(rng, mil.shape[0], nbands))
    return System(name, cell, v_r, kps, nbands, psi0, seed)


def config(cid: int, nbands: Optional[int] = None, nk: Optional[int] = None) -> System:
    """The five benchmark configurations (0-3 here; 4 is a request stream).

    0: FCC a=10.26, 2 atoms, Gamma, 30 Ry, 24^3, 8 bands, 16 projectors.
    1: SC a=20.5, 64 atoms, Gamma, 30 Ry, 80^3, 256 bands, 512 projectors.
    2: SC a=10.26, 8 atoms, 30 Ry, 40^3, 48 bands, 32 k (4x4x2 shifted MP).
    3: SC a=25.8, 128 atoms, Gamma, 36 Ry, 108^3, 512 bands, 1024 projectors.
    """
    seed = 1234 + cid
    rng = np.random.default_rng(seed + 7919)
    if cid == 0:
        cell = Cell(fcc_lattice(10.26), np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]]),
                    (24, 24, 24), 15.0 * HA_TO_RY)
        ks = np.zeros((1, 3))
        nb = 8
    elif cid == 1:
        lat = cubic_lattice(20.5)
        cell = Cell(lat, random_positions(rng, lat, 64), (80, 80, 80), 15.0 * HA_TO_RY)
        ks = np.zeros((1, 3))
        nb = 256
    elif cid == 2:
        lat = cubic_lattice(10.26)
        cell = Cell(lat, random_positions(rng, lat, 8), (40, 40, 40), 15.0 * HA_TO_RY)
        ks = monkhorst_pack((4, 4, 2), (1, 1, 1))
        nb = 48
    elif cid == 3:
        lat = cubic_lattice(25.8)
        cell = Cell(lat, random_positions(rng, lat, 128), (108, 108, 108), 18.0 * HA_TO_RY)
        ks = np.zeros((1, 3))
        nb = 512
    else:
        raise ValueError(f"config {cid} is a request stream; use serving_requests()")
    if nbands is not None:
        nb = nbands
    if nk is not None:
        ks = ks[:nk]
    return build_system(f"config{cid}", cell, ks, nb, seed)


SMOOTH_SIZES = sorted({2 ** a * 3 ** b * 5 ** c for a in range(7) for b in range(5)
                       for c in range(4) if 2 ** a * 3 ** b * 5 ** c <= 128})


def smooth_grid_size(min_size: int, lo: int = 24, hi: int = 64) -> int:
    for s in SMOOTH_SIZES:
        if s >= max(min_size, lo):
            return min(s, hi) if s <= hi else hi
    return hi


def request_cell(rng: np.random.Generator) -> Tuple[Cell, int]:
    """One serving request: n ~ U{2..32} atoms, a = 5.13 n^(1/3), ecut ~ U[20, 40] Ry."""
    n = int(rng.integers(2, 33))
    a = 5.13 * n ** (1.0 / 3.0)
    ecut = float(rng.uniform(20.0, 40.0))
    lat = cubic_lattice(a)
    m = math.sqrt(ecut) * a / (2.0 * np.pi)
    size = smooth_grid_size(int(math.ceil(4.0 * m)) + 1)
    cell = Cell(lat, random_positions(rng, lat, n), (size, size, size), ecut)
    return cell, 4 * n


@dataclasses.dataclass
class RequestSpec:
    """What one serving request is built from (its cell, band count and seed)."""
    name: str
    cell: Cell
    nbands: int
    seed: int


def serving_request_specs(count: int, seed: int = 1238) -> List[RequestSpec]:
    """The cells of the serving stream's first `count` requests, drawn in order from one
    seeded stream (cheap: the inputs themselves are built by build_request)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        cell, nb = request_cell(rng)
        out.append(RequestSpec(f"request{i}", cell, nb, int(rng.integers(0, 2 ** 31))))
    return out


def build_request(spec: RequestSpec) -> System:
    """The inputs of one serving request (Gamma point)."""
    return build_system(spec.name, spec.cell, np.zeros((1, 3)), spec.nbands, spec.seed)


def serving_requests(count: int, seed: int = 1238) -> List[System]:
    """The request stream of the serving configuration (cells only; arrivals apart)."""
    return [build_request(s) for s in serving_request_specs(count, seed)]


@dataclasses.dataclass
class GammaKPoint:
    """A k = 0 point on the half sphere (the reference's Gamma-only basis): the origin first,
    then every G whose first nonzero Miller index is positive."""
    index: np.ndarray              # npw_half positions in the full-sphere list
    g_to_grid: np.ndarray          # grid index of +G
    minus_g_to_grid: np.ndarray    # grid index of -G (-1 outside the grid)
    ke: np.ndarray
    beta: np.ndarray               # npw_half x P
    d_blocks: np.ndarray
    atom_proj_offsets: np.ndarray

    @property
    def npw(self) -> int:
        return int(self.index.size)


def gamma_kpoint(system: "System", k: int = 0) -> GammaKPoint:
    kp = system.kpoints[k]
    if np.any(np.asarray(kp.k_frac) != 0.0):
        raise ValueError("a Gamma-only basis needs k = 0")
    m = kp.miller
    first = np.where(m[:, 0] != 0, m[:, 0], np.where(m[:, 1] != 0, m[:, 1], m[:, 2]))
    origin = np.flatnonzero(np.all(m == 0, axis=1))
    index = np.concatenate([origin, np.flatnonzero(first > 0)]).astype(np.int64)
    minus = grid_map(-m[index], system.cell.grid)
    return GammaKPoint(index, kp.g_to_grid[index].astype(np.int32), minus.astype(np.int32), kp.ke[index],
                       np.asfortranarray(kp.beta[index]), kp.d_blocks, kp.atom_proj_offsets)


def overlap_blocks(system: "System", seed: int = 4242, scale: float = 0.3) -> np.ndarray:
    """Ultrasoft-style q_ij blocks for the system's projector layout, packed like its D blocks:
    per atom, q couples projectors of the same l and m (the two s channels, and each m of the
    two p channels), with a seeded symmetric 2 x 2 matrix per l."""
    rng = np.random.default_rng(seed)
    def sym():
        a = rng.uniform(-scale, scale, size=(2, 2))
        return 0.5 * (a + a.T)
    qs, qp = sym(), sym()
    blk = np.zeros((PROJECTORS_PER_ATOM, PROJECTORS_PER_ATOM))
    blk[np.ix_([0, 1], [0, 1])] = qs
    for m in range(3):
        idx = [2 + m, 5 + m]
        blk[np.ix_(idx, idx)] = qp
    return np.concatenate([blk.reshape(-1, order="F")] * system.cell.natoms)


def small_system(grid=(12, 12, 12), a: float = 7.0, natoms: int = 2, ecut: float = 8.0,
                 nbands: int = 6, seed: int = 99, k_frac=(0.0, 0.0, 0.0),
                 lattice: Optional[np.ndarray] = None) -> System:
    """A small cell for fast parity tests."""
    rng = np.random.default_rng(seed)
    lat = cubic_lattice(a) if lattice is None else lattice
    cell = Cell(lat, random_positions(rng, lat, natoms, min_distance=1.5), tuple(grid), ecut)
    return build_system("small", cell, np.array([k_frac], dtype=np.float64), nbands, seed)
