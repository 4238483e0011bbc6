"""q3b_apply_h_noalloc against q3b_apply_h, through the C ABI.

The no-allocation entry point is for callers that cannot call cudaMalloc
while they apply H (stream capture, their own memory pool).  It must give the
same H|psi> as the ordinary FP64 entry point, call after call: the second call
reuses the fixed scratch array the first one left behind.  This file is named
to be collected last.
"""
import numpy as np
import pytest

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
    npw = sy.kpoints[0].npw
    nb = sy.nbands
    x = torch.from_numpy(np.ascontiguousarray(sy.psi0[0].T)).to(cuda_device)
    ref = torch.empty_like(x)
    check(h, lib.q3b_apply_h(h, x.data_ptr(), ref.data_ptr(), nb, FP64))
    torch.cuda.synchronize()
    scale = float(ref.abs().max())
    for call in range(2):
        out = torch.full_like(x, float("nan"))
        check(h, lib.q3b_apply_h_noalloc(h, x.data_ptr(), out.data_ptr(), nb))
        torch.cuda.synchronize()
        err = float((out - ref).abs().max()) / scale
        assert err < FP64_TOL, f"call {call}: relative difference {err:.3e}"
    ap.ctx.close()
