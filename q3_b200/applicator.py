"""Host-side mirror of the reference's ``PlanewaveHamiltonianApplicator``.

Same method names, argument meaning and error behaviour as
``src/layer_4_computation/diagonalizer/planewave/internal/hamiltonian_applicator/init.hpp:28-153``,
over the C ABI of libq3b.so.  Device vectors are torch tensors on the
context's GPU (complex128, or complex64 for the FP32 entry); host vectors are
numpy arrays.  Nothing here computes H|psi> itself.
"""
from __future__ import annotations

import contextlib
import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import FP64, MIXED, check


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class Context:
    """Owns a q3b_context (device, stream, HBM budget, workspaces)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.q3b_context_create(int(device), int(hbm_budget), C.byref(h))
        if rc != 0:
            raise _lib.Q3BError(rc, f"cannot create a context on device {device}")
        self.handle = h.value
        self.device = device

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.q3b_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self) -> int:
        return self.lib.q3b_get_stream(self.handle) or 0

    def set_stream(self, stream_ptr: Optional[int]) -> None:
        check(self.handle, self.lib.q3b_set_stream(self.handle, stream_ptr))

    def synchronize(self) -> None:
        check(self.handle, self.lib.q3b_synchronize(self.handle))

    @contextlib.contextmanager
    def ordered_with_torch(self):
        """Order the library's stream with torch's current stream on this
        device: work issued inside the block starts after what torch has queued
        (the inputs it wrote), and torch's later work waits for it (the outputs).
        No host synchronisation."""
        import torch
        dev = torch.device("cuda", self.device)
        ours = torch.cuda.ExternalStream(self.stream, device=dev)
        theirs = torch.cuda.current_stream(dev)
        ours.wait_stream(theirs)
        try:
            yield
        finally:
            theirs.wait_stream(ours)

    def device_bytes(self) -> int:
        return int(self.lib.q3b_device_bytes(self.handle))


class PlanewaveHamiltonianApplicator:
    """update_potential / prepare_kpoint / apply_batch over libq3b."""

    def __init__(self, context: Optional[Context] = None, device: int = 0, hbm_budget: int = 0):
        self.ctx = context if context is not None else Context(device, hbm_budget)
        self.lib = self.ctx.lib
        self.h = self.ctx.handle
        self.npw = 0
        self.grid = None
        self._keep = []

    # init.hpp:40
    def update_potential(self, real_space_potential: np.ndarray, grid, density_grid=None) -> None:
        """V(r) (Ry) on the wavefunction grid `grid`, or on a larger `density_grid`, from
        which it is restricted to `grid` (the reference's dense-to-smooth step)."""
        v = np.ascontiguousarray(real_space_potential, dtype=np.float64)
        n1, n2, n3 = (int(x) for x in grid)
        if density_grid is None:
            if v.size != n1 * n2 * n3:
                raise ValueError("potential size does not match the grid")
            check(self.h, self.lib.q3b_set_potential(self.h, _ptr(v), n1, n2, n3))
        else:
            d1, d2, d3 = (int(x) for x in density_grid)
            if v.size != d1 * d2 * d3:
                raise ValueError("potential size does not match the density grid")
            check(self.h, self.lib.q3b_set_potential_dense(self.h, _ptr(v), d1, d2, d3, n1, n2, n3))
        self.grid = (n1, n2, n3)

    # init.hpp:90, :96
    def invalidate_smooth_potential_cache(self) -> None:
        check(self.h, self.lib.q3b_invalidate_potential(self.h))

    def is_smooth_potential_cache_valid(self) -> bool:
        return bool(self.lib.q3b_potential_valid(self.h))

    def is_gamma_only_current(self) -> bool:       # init.hpp:104; full sphere only
        return False

    def gamma_origin_is_local_current(self) -> bool:  # init.hpp:115; one GPU
        return True

    # init.hpp:47-50 + the projector set of the k-point
    def prepare_kpoint(self, kpoint_index: int, number_of_plane_waves: int,
                       g_vector_to_grid: np.ndarray, kinetic_energy_squared: np.ndarray,
                       projectors: Optional[np.ndarray] = None,
                       atom_proj_offsets: Optional[np.ndarray] = None,
                       d_blocks: Optional[np.ndarray] = None) -> None:
        npw = int(number_of_plane_waves)
        g2g = np.ascontiguousarray(g_vector_to_grid, dtype=np.int32)
        ke = np.ascontiguousarray(kinetic_energy_squared, dtype=np.float64)
        if g2g.size != npw or ke.size != npw:
            raise ValueError("plane-wave arrays do not match number_of_plane_waves")
        if projectors is None or projectors.shape[1] == 0:
            check(self.h, self.lib.q3b_prepare_kpoint(self.h, npw, _ptr(g2g), _ptr(ke), None, 0,
                                                      0, None, None))
        else:
            beta = np.asfortranarray(projectors, dtype=np.complex128)
            offs = np.ascontiguousarray(atom_proj_offsets, dtype=np.int32)
            dblk = np.ascontiguousarray(d_blocks, dtype=np.float64)
            if beta.shape[0] != npw:
                raise ValueError("projector rows do not match number_of_plane_waves")
            check(self.h, self.lib.q3b_prepare_kpoint(self.h, npw, _ptr(g2g), _ptr(ke),
                                                      _ptr(beta), beta.shape[1], offs.size - 1,
                                                      _ptr(offs), _ptr(dblk)))
        self.npw = npw
        self.kpoint_index = kpoint_index

    def prepare_system_kpoint(self, system, k: int = 0) -> None:
        """prepare_kpoint from a q3_b200.synthetic System."""
        kp = system.kpoints[k]
        self.prepare_kpoint(k, kp.npw, kp.g_to_grid, kp.ke, kp.beta, kp.atom_proj_offsets,
                            kp.d_blocks)

    # init.hpp:59-61 -- device vectors
    def apply_batch(self, input_wavefunctions, output_hamiltonian_wavefunctions,
                    number_of_vectors: int, precision: int = FP64) -> None:
        psi, hpsi = input_wavefunctions, output_hamiltonian_wavefunctions
        n = int(number_of_vectors)
        import torch  # device memory comes from torch; imported only for device calls
        if psi.device.type != "cuda" or hpsi.device.type != "cuda":
            raise ValueError("apply_batch takes device tensors; use apply_batch_host for host arrays")
        if psi.dtype == torch.complex64:
            if hpsi.dtype != torch.complex64:
                raise ValueError("FP32 input needs an FP32 output")
            with self.ctx.ordered_with_torch():
                rc = self.lib.q3b_apply_h_f32(self.h, psi.data_ptr(), hpsi.data_ptr(), n)
        elif psi.dtype == torch.complex128 and hpsi.dtype == torch.complex128:
            with self.ctx.ordered_with_torch():
                rc = self.lib.q3b_apply_h(self.h, psi.data_ptr(), hpsi.data_ptr(), n, int(precision))
        else:
            raise ValueError("vectors must be complex128 (or complex64 for the FP32 entry)")
        check(self.h, rc)

    # Gamma-only k-point (serial.hpp:283-418, :519-566): half-sphere vectors, two bands per transform
    def prepare_kpoint_gamma(self, number_of_plane_waves: int, g_vector_to_grid: np.ndarray,
                             minus_g_vector_to_grid: np.ndarray, kinetic_energy_squared: np.ndarray,
                             projectors: Optional[np.ndarray] = None,
                             atom_proj_offsets: Optional[np.ndarray] = None,
                             d_blocks: Optional[np.ndarray] = None) -> None:
        """Half sphere of G with the origin at index 0: +G and -G grid indices, |G|^2 (Ry) and the
        npw_half x P projectors (beta(-G) = conj(beta(G)) extends them to the full sphere)."""
        npw = int(number_of_plane_waves)
        g2g = np.ascontiguousarray(g_vector_to_grid, dtype=np.int32)
        g2m = np.ascontiguousarray(minus_g_vector_to_grid, dtype=np.int32)
        ke = np.ascontiguousarray(kinetic_energy_squared, dtype=np.float64)
        if g2g.size != npw or g2m.size != npw or ke.size != npw:
            raise ValueError("plane-wave arrays do not match number_of_plane_waves")
        if projectors is None or projectors.shape[1] == 0:
            rc = self.lib.q3b_prepare_kpoint_gamma(self.h, npw, _ptr(g2g), _ptr(g2m), _ptr(ke), None, 0, 0,
                                                   None, None)
        else:
            beta = np.asfortranarray(projectors, dtype=np.complex128)
            offs = np.ascontiguousarray(atom_proj_offsets, dtype=np.int32)
            dblk = np.ascontiguousarray(d_blocks, dtype=np.float64)
            if beta.shape[0] != npw:
                raise ValueError("projector rows do not match number_of_plane_waves")
            rc = self.lib.q3b_prepare_kpoint_gamma(self.h, npw, _ptr(g2g), _ptr(g2m), _ptr(ke), _ptr(beta),
                                                   beta.shape[1], offs.size - 1, _ptr(offs), _ptr(dblk))
        check(self.h, rc)
        self.npw = 2 * npw - 1
        self.gamma_npw = npw

    def apply_batch_gamma(self, input_wavefunctions, output_hamiltonian_wavefunctions,
                          number_of_vectors: int, precision: int = FP64) -> None:
        """H on half-sphere vectors: complex128 device tensors laid out nvec x npw_half."""
        psi, hpsi = input_wavefunctions, output_hamiltonian_wavefunctions
        import torch
        if psi.device.type != "cuda" or hpsi.device.type != "cuda":
            raise ValueError("apply_batch_gamma takes device tensors")
        if psi.dtype != torch.complex128 or hpsi.dtype != torch.complex128:
            raise ValueError("vectors must be complex128")
        with self.ctx.ordered_with_torch():
            rc = self.lib.q3b_apply_h_gamma(self.h, psi.data_ptr(), hpsi.data_ptr(), int(number_of_vectors),
                                            int(precision))
        check(self.h, rc)

    def set_d_blocks(self, d_blocks: np.ndarray) -> None:
        """The D blocks of another spin channel (set_spin_channel, init.hpp:75-80), packed like
        those given to prepare_kpoint; the projectors stay on the device."""
        d = np.ascontiguousarray(d_blocks, dtype=np.float64)
        check(self.h, self.lib.q3b_set_d_blocks(self.h, _ptr(d)))

    # UltrasoftPseudopotentialOverlapOperator (overlap/pseudopotential/ultrasoft/init.hpp)
    def set_overlap_blocks(self, q_blocks: np.ndarray) -> None:
        """Per-atom q_ij blocks, packed like the D blocks of the prepared k-point."""
        q = np.ascontiguousarray(q_blocks, dtype=np.float64)
        check(self.h, self.lib.q3b_set_overlap_blocks(self.h, _ptr(q)))

    def apply_overlap(self, input_wavefunctions, output_wavefunctions, number_of_vectors: int,
                      precision: int = FP64, gamma: bool = False) -> None:
        """S psi on complex128 device tensors (nvec x npw; half-sphere vectors with gamma=True)."""
        psi, spsi = input_wavefunctions, output_wavefunctions
        import torch
        if psi.device.type != "cuda" or spsi.device.type != "cuda":
            raise ValueError("apply_overlap takes device tensors")
        if psi.dtype != torch.complex128 or spsi.dtype != torch.complex128:
            raise ValueError("vectors must be complex128")
        fn = self.lib.q3b_apply_s_gamma if gamma else self.lib.q3b_apply_s
        with self.ctx.ordered_with_torch():
            rc = fn(self.h, psi.data_ptr(), spsi.data_ptr(), int(number_of_vectors), int(precision))
        check(self.h, rc)

    def prepare_kpoint_build(self, kpoint_index: int, number_of_plane_waves: int, g_vector_to_grid: np.ndarray,
                             kinetic_energy_squared: np.ndarray, k_plus_g: np.ndarray, cell_volume: float,
                             positions: np.ndarray, species_of_atom: np.ndarray, beta_l, beta_tables: np.ndarray,
                             dq: float, d_blocks: np.ndarray) -> None:
        """prepare_kpoint with the projector set built on the device from the
        species' beta-function tables (ProjectorSetBuilder).  k_plus_g: npw x 3
        (bohr^-1); positions: natoms x 3 (bohr); beta_l: list per species of the
        l of each beta; beta_tables: (total betas) x nq, species by species."""
        npw = int(number_of_plane_waves)
        g2g = np.ascontiguousarray(g_vector_to_grid, dtype=np.int32)
        ke = np.ascontiguousarray(kinetic_energy_squared, dtype=np.float64)
        kpg = np.ascontiguousarray(k_plus_g, dtype=np.float64)
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        spec = np.ascontiguousarray(species_of_atom, dtype=np.int32)
        nb = np.array([len(x) for x in beta_l], dtype=np.int32)
        ls = np.array([l for x in beta_l for l in x], dtype=np.int32)
        tab = np.ascontiguousarray(beta_tables, dtype=np.float64)
        dblk = np.ascontiguousarray(d_blocks, dtype=np.float64)
        nq = int(tab.shape[1]) if tab.ndim == 2 else 0
        check(self.h, self.lib.q3b_prepare_kpoint_build(
            self.h, npw, _ptr(g2g), _ptr(ke), _ptr(kpg), float(cell_volume), int(pos.shape[0]), _ptr(pos),
            _ptr(spec), int(nb.size), _ptr(nb), _ptr(ls), nq, float(dq), _ptr(tab), _ptr(dblk)))
        self.npw = npw
        self.kpoint_index = kpoint_index

    def set_local_kernel(self, choice: int, precision: int = FP64) -> None:
        """Override the autotuner's plane kernel for the prepared k-point (q3b_set_local_kernel):
        0 re-tunes, 128/256/512 the shared-memory kernel, -1/-2 the register kernel."""
        check(self.h, self.lib.q3b_set_local_kernel(self.h, int(precision), int(choice)))

    def local_kernel(self, precision: int = FP64) -> int:
        """The plane kernel in force for the prepared k-point (tuning first if needed)."""
        out = C.c_int()
        check(self.h, self.lib.q3b_get_local_kernel(self.h, int(precision), C.byref(out)))
        return out.value

    def projectors(self):
        """The prepared k-point's projector matrix as a CUDA tensor (P x npw)."""
        import ctypes as C
        import torch
        n = C.c_int()
        check(self.h, self.lib.q3b_get_projectors(self.h, None, C.byref(n)))
        out = torch.empty((n.value, self.npw), dtype=torch.complex128, device=torch.device("cuda", self.ctx.device))
        if n.value:
            with self.ctx.ordered_with_torch():
                rc = self.lib.q3b_get_projectors(self.h, out.data_ptr(), C.byref(n))
            check(self.h, rc)
        return out

    def accumulate_density(self, bands, weights: np.ndarray, rho) -> None:
        """PlanewaveChargeDensityAccumulator at this k-point: rho += sum_b w_b |psi_b(r)|^2.

        bands: complex128 CUDA tensor nb x npw (band-contiguous); weights: nb
        (k-point weight x occupation / cell volume; 0 skips a band); rho: float64
        CUDA tensor of N1*N2*N3 values, natural grid order, added to."""
        w = np.ascontiguousarray(weights, dtype=np.float64)
        with self.ctx.ordered_with_torch():
            rc = self.lib.q3b_accumulate_density(self.h, bands.data_ptr(), int(w.size), _ptr(w), rho.data_ptr())
        check(self.h, rc)

    def apply_batch_host(self, psi: np.ndarray, number_of_vectors: int,
                         precision: int = FP64) -> np.ndarray:
        x = np.asfortranarray(psi, dtype=np.complex128)
        out = np.empty_like(x, order="F")
        check(self.h, self.lib.q3b_apply_h_host(self.h, _ptr(x), _ptr(out),
                                                int(number_of_vectors), int(precision)))
        return out
