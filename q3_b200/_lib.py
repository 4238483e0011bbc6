"""ctypes binding of libq3b.so (include/q3b.h).

Loading fails loudly: there is no CPU fallback for anything this library does.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libq3b.so"

OK = 0
ERR_INVALID, ERR_CUDA, ERR_STATE, ERR_MEMORY, ERR_LINALG, ERR_INTERNAL = 1, 2, 3, 4, 5, 6
FP64, MIXED = 0, 1

STATUS_NAMES = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "STATE", 4: "MEMORY", 5: "LINALG",
                6: "INTERNAL"}


class Q3BError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"q3b error {STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


class Cplx128(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


class Cplx64(C.Structure):
    _fields_ = [("re", C.c_float), ("im", C.c_float)]


class ApplyTiming(C.Structure):
    _fields_ = [("sticks_backward_ms", C.c_double), ("planes_ms", C.c_double),
                ("sticks_forward_ms", C.c_double), ("projector_overlap_ms", C.c_double),
                ("d_apply_ms", C.c_double), ("projector_accumulate_ms", C.c_double),
                ("launches", C.c_int * 6)]

    KERNELS = ("sticks_backward", "planes", "sticks_forward", "projector_overlap", "d_apply",
               "projector_accumulate")

    def as_dict(self):
        return {k: (getattr(self, k + "_ms"), self.launches[i]) for i, k in enumerate(self.KERNELS)}


class DavidsonOpts(C.Structure):
    _fields_ = [("tolerance", C.c_double), ("max_iterations", C.c_int),
                ("basis_expansion_factor", C.c_int), ("occupied_bands", C.c_int),
                ("precision", C.c_int), ("refine_sweeps", C.c_int),
                ("mixed_tolerance", C.c_double), ("profile_stages", C.c_int),
                ("eigenvalue_history", C.c_void_p), ("history_rows", C.c_int),
                ("mixed_expansion_factor", C.c_int)]


class DavidsonStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("fp64_iterations", C.c_int),
                ("h_applications", C.c_int), ("unconverged", C.c_int), ("collapses", C.c_int),
                ("max_residual_norm", C.c_double), ("seconds", C.c_double),
                ("stage_ms", C.c_double * 8), ("fp64_seconds", C.c_double)]

    STAGES = ("seed", "diagonalize", "correction", "orthogonalize", "hamiltonian",
              "subspace_update", "collapse", "extract")


class Request(C.Structure):
    _fields_ = [("n1", C.c_int), ("n2", C.c_int), ("n3", C.c_int), ("v_r", C.c_void_p),
                ("npw", C.c_int), ("g_to_grid", C.c_void_p), ("ke", C.c_void_p),
                ("nproj", C.c_int), ("beta", C.c_void_p), ("natoms", C.c_int),
                ("atom_proj_offsets", C.c_void_p), ("d_blocks", C.c_void_p), ("nb", C.c_int),
                ("bands", C.c_void_p), ("eigenvalues", C.c_void_p),
                ("opts", C.POINTER(DavidsonOpts))]


class RequestTimes(C.Structure):
    _fields_ = [("queue_ms", C.c_double), ("solve_ms", C.c_double), ("latency_ms", C.c_double),
                ("estimated_bytes", C.c_size_t)]


_vp, _i, _d, _sz = C.c_void_p, C.c_int, C.c_double, C.c_size_t

# name -> (restype, argtypes); every symbol declared in include/q3b.h
SIGNATURES = {
    "q3b_context_create": (_i, [_i, _sz, C.POINTER(_vp)]),
    "q3b_context_destroy": (_i, [_vp]),
    "q3b_last_error": (C.c_char_p, [_vp]),
    "q3b_get_stream": (_vp, [_vp]),
    "q3b_set_stream": (_i, [_vp, _vp]),
    "q3b_synchronize": (_i, [_vp]),
    "q3b_device_bytes": (_sz, [_vp]),
    "q3b_set_potential": (_i, [_vp, _vp, _i, _i, _i]),
    "q3b_set_potential_dense": (_i, [_vp, _vp, _i, _i, _i, _i, _i, _i]),
    "q3b_invalidate_potential": (_i, [_vp]),
    "q3b_potential_valid": (_i, [_vp]),
    "q3b_prepare_kpoint": (_i, [_vp, _i, _vp, _vp, _vp, _i, _i, _vp, _vp]),
    "q3b_apply_h": (_i, [_vp, _vp, _vp, _i, _i]),
    "q3b_apply_h_f32": (_i, [_vp, _vp, _vp, _i]),
    "q3b_apply_h_host": (_i, [_vp, _vp, _vp, _i, _i]),
    "q3b_apply_h_noalloc": (_i, [_vp, _vp, _vp, _i]),
    "q3b_apply_h_timed": (_i, [_vp, _vp, _vp, _i, _i, C.POINTER(ApplyTiming)]),
    "q3b_kernel_launches": (C.c_ulonglong, []),
    "q3b_gemm": (_i, [_vp, C.c_char, C.c_char, _i, _i, _i, Cplx128, _vp, _i, _vp, _i, Cplx128, _vp, _i]),
    "q3b_gemm_single": (_i, [_vp, C.c_char, C.c_char, _i, _i, _i, Cplx64, _vp, _i, _vp, _i, Cplx64, _vp,
                             _i]),
    "q3b_davidson_default_opts": (None, [C.POINTER(DavidsonOpts)]),
    "q3b_davidson_solve": (_i, [_vp, _vp, _vp, _i, C.POINTER(DavidsonOpts), C.POINTER(DavidsonStats)]),
    "q3b_davidson_solve_dev": (_i, [_vp, _vp, _vp, _i, C.POINTER(DavidsonOpts),
                                    C.POINTER(DavidsonStats)]),
    "q3b_hegv": (_i, [_vp, _i, _vp, _vp, _i, _vp, _vp]),
    "q3b_accumulate_density": (_i, [_vp, _vp, _i, _vp, _vp]),
    "q3b_graph_stats": (_i, [_vp, C.POINTER(_i), C.POINTER(_i)]),
    "q3b_set_local_kernel": (_i, [_vp, _i, _i]),
    "q3b_measure_fp64_rate": (_i, [_vp, C.POINTER(C.c_double)]),
    "q3b_get_local_kernel": (_i, [_vp, _i, C.POINTER(_i)]),
    "q3b_prepare_kpoint_build": (_i, [_vp, _i, _vp, _vp, _vp, C.c_double, _i, _vp, _vp, _i, _vp, _vp, _i,
                                      C.c_double, _vp, _vp]),
    "q3b_get_projectors": (_i, [_vp, _vp, C.POINTER(_i)]),
    "q3b_prepare_kpoint_gamma": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp]),
    "q3b_apply_h_gamma": (_i, [_vp, _vp, _vp, _i, _i]),
    "q3b_set_overlap_blocks": (_i, [_vp, _vp]),
    "q3b_set_d_blocks": (_i, [_vp, _vp]),
    "q3b_hegv_lowest": (_i, [_vp, _i, _vp, _vp, _i, _i, _vp, _vp]),
    "q3b_server_set_batching": (_i, [_vp, _i, _i]),
    "q3b_server_batch_stats": (_i, [_vp, _vp, _vp]),
    "q3b_hegv_batched": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "q3b_set_block_eigensolver_order": (_i, [_i]),
    "q3b_apply_s": (_i, [_vp, _vp, _vp, _i, _i]),
    "q3b_apply_s_gamma": (_i, [_vp, _vp, _vp, _i, _i]),
    "q3b_start_apply": (_i, [_vp, _vp, _i]),
    "q3b_start_project": (_i, [_vp, _vp, _vp]),
    "q3b_start_rotate": (_i, [_vp, _vp, _i, _vp]),
    "q3b_starting_subspace": (_i, [_vp, _vp, _i, _i, _vp, _vp]),
    "q3b_server_create": (_i, [_i, _sz, _i, C.POINTER(_vp)]),
    "q3b_server_destroy": (_i, [_vp]),
    "q3b_server_last_error": (C.c_char_p, [_vp]),
    "q3b_server_submit": (_i, [_vp, C.POINTER(Request), C.POINTER(_i)]),
    "q3b_server_poll": (_i, [_vp, _i]),
    "q3b_server_wait": (_i, [_vp, _i, _vp, _vp, C.POINTER(DavidsonStats), C.POINTER(RequestTimes)]),
}

_lib = None


def load(path: os.PathLike | None = None) -> C.CDLL:
    """Load libq3b.so once and bind every entry point; raise if anything is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise ImportError(f"{p} is missing: build it with `python -m q3_b200.build`")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)          # AttributeError when a symbol is missing
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(ctx, rc: int) -> None:
    if rc != OK:
        msg = load().q3b_last_error(ctx)
        raise Q3BError(rc, msg.decode() if msg else "")
