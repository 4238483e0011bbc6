"""q3b_apply_h_noalloc against q3b_apply_h and the oracle, through the C ABI.

The no-allocation entry point is for callers that cannot call cudaMalloc while
they apply H (a runtime that owns all device memory through its own pool, or
one that forbids allocation after start-up).  It must give the same H|psi> as
the ordinary FP64 entry point, call after call: the second call reuses the
fixed scratch array the first one left behind.  The small case is also checked
against the CPU oracle.  This file is named to be collected last.
"""
import numpy as np
import pytest

from oracle import hpsi as ohpsi
from q3_b200 import synthetic
from q3_b200._lib import FP64, check

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


@pytest.mark.parametrize("cfg", ["small", "config1"])
def test_apply_h_noalloc_matches_apply_h(cuda_device, cfg):
    import torch
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    sy = synthetic.small_system(nbands=6) if cfg == "small" else synthetic.config(1, nbands=40)
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_system_kpoint(sy)
    lib, h = ap.lib, ap.h
    nb = sy.nbands
    x = torch.from_numpy(np.ascontiguousarray(sy.psi0[0].T)).to(cuda_device)
    # the first call resolves the scratch array's address on this device
    warm = torch.empty_like(x)
    with ap.ctx.ordered_with_torch():
        check(h, lib.q3b_apply_h_noalloc(h, x.data_ptr(), warm.data_ptr(), nb))
    torch.cuda.synchronize()
    ref = torch.empty_like(x)
    with ap.ctx.ordered_with_torch():
        check(h, lib.q3b_apply_h(h, x.data_ptr(), ref.data_ptr(), nb, FP64))
    torch.cuda.synchronize()
    scale = float(ref.abs().max())
    for call in range(2):
        out = torch.full_like(x, float("nan"))
        torch.cuda.synchronize()
        held = ap.ctx.device_bytes()
        free_before = torch.cuda.mem_get_info()[0]
        with ap.ctx.ordered_with_torch():
            check(h, lib.q3b_apply_h_noalloc(h, x.data_ptr(), out.data_ptr(), nb))
        torch.cuda.synchronize()
        assert ap.ctx.device_bytes() == held, "the call reserved context memory"
        assert torch.cuda.mem_get_info()[0] == free_before, "the call allocated device memory"
        err = float((out - ref).abs().max()) / scale
        assert err < FP64_TOL, f"call {call}: relative difference {err:.3e}"
    if cfg == "small":
        want = ohpsi.apply_h(sy.psi0[0], sy.kpoints[0], sy.v_r, sy.cell.grid)
        got = out.cpu().numpy().T
        assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < FP64_TOL
    ap.ctx.close()
