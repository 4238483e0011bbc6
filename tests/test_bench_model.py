"""The bench's algorithmic-byte model of the local H|psi> path (no GPU).

`roofline.achieved` divides these bytes by measured kernel time, so the model is pinned here:
per application of nvec bands, B_loc = nvec (2 npw c + 4 S N3 c) + N r + npw r with c the
complex and r the real size (psi read and H psi written once; the stick buffer written by the
backward stick pass, read and written by the plane pass, read by the forward stick pass; V and
|k+G|^2 once), and the non-empty stick counts S of the configurations.
"""
import importlib.util
from pathlib import Path

import pytest

from q3_b200 import synthetic
from q3_b200.plan_info import stick_count

ROOT = Path(__file__).resolve().parents[1]


def _bench():
    spec = importlib.util.spec_from_file_location("bench_model_under_test", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("cid,sticks,mb64,mb32", [(0, 109, 1.641, 0.821), (1, 997, 1506.4, 753.2)])
def test_local_bytes_per_application(cid, sticks, mb64, mb32):
    bench = _bench()
    sy = synthetic.config(cid)
    kp = sy.kpoints[0]
    s = stick_count(kp, sy.cell.grid)
    assert s == sticks
    n3 = sy.cell.grid[2]
    n = sy.cell.grid[0] * sy.cell.grid[1] * n3
    for c, r, mb in ((16, 8, mb64), (8, 4, mb32)):
        kb = bench.kernel_bytes(kp, sy.cell.grid, s, sy.nbands, c, r)
        local = kb["sticks_backward"] + kb["planes"] + kb["planes_v"] + kb["sticks_forward"]
        assert local == sy.nbands * (2 * kp.npw * c + 4 * s * n3 * c) + n * r + kp.npw * r
        assert abs(local / 1e6 - mb) < 0.01 * mb


def test_plane_flops_of_the_bench_cell():
    # the plane pass against the FP32 pipe: 5 n log2 n per line over the 35 stick rows and all
    # 80 columns of each of the 80 planes, both ways, plus the V product: 12.17 GFLOP per
    # 256-band application of config 1
    import numpy as np
    bench = _bench()
    sy = synthetic.config(1)
    kp = sy.kpoints[0]
    n1, n2, n3 = sy.cell.grid
    rows = len(np.unique(np.asarray(kp.g_to_grid) // (n2 * n3)))
    assert rows == 35
    fl = bench.plane_flops(kp, sy.cell.grid, sy.nbands)
    line = 5.0 * 80 * np.log2(80)
    assert fl == pytest.approx(256 * 80 * (2 * 35 * line + 2 * 80 * line + 2 * 80 * 80), rel=1e-12)
    assert abs(fl / 1e9 - 12.17) < 0.01
