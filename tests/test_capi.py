"""The C-ABI library loads and exports every symbol include/*.h declares (no GPU)."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(q3b_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_header_declares_the_applicator_entry_points():
    names = declared_symbols()
    for n in ("q3b_context_create", "q3b_set_potential", "q3b_prepare_kpoint", "q3b_apply_h"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from q3_b200 import _lib
    lib = _lib.load()
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing
    # and the binding table covers the header
    assert declared_symbols() <= set(_lib.SIGNATURES)


def test_context_create_without_gpu_fails_cleanly():
    import ctypes as C
    import torch
    from q3_b200 import _lib
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    h = C.c_void_p()
    rc = lib.q3b_context_create(0, 0, C.byref(h))
    assert rc == _lib.ERR_CUDA and not h.value


def test_davidson_default_opts_fill_every_field():
    """q3b_davidson_default_opts is host code: it fills the ctypes mirror of q3b_davidson_opts
    field by field, so a field order or size that differs from the header shows up here."""
    import ctypes as C
    from q3_b200 import _lib
    lib = _lib.load()
    o = _lib.DavidsonOpts()
    o.tolerance, o.max_iterations, o.basis_expansion_factor = -1.0, -1, -1
    o.occupied_bands, o.precision, o.refine_sweeps = -1, -1, -1
    o.mixed_tolerance, o.profile_stages = -1.0, -1
    o.eigenvalue_history, o.history_rows, o.mixed_expansion_factor = 0x1234, 77, 9
    lib.q3b_davidson_default_opts(C.byref(o))
    assert o.tolerance == 1e-2 and o.max_iterations == 20 and o.basis_expansion_factor == 2
    assert o.occupied_bands == 0 and o.precision == _lib.FP64 and o.refine_sweeps == 0
    assert o.mixed_tolerance == 1e-6 and o.profile_stages == 0
    assert not o.eigenvalue_history and o.history_rows == 0 and o.mixed_expansion_factor == 0
