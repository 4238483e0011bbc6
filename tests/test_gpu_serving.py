"""The serving loop: results are the same alone and in the mix.

Requests of different sizes are submitted at once to a server with several
workers (their solves overlap on the device) and, separately, one at a time to
a one-worker server.  Each request's eigenvalues must agree to 1e-12 Ry: the
solves share no buffers and every reduction has a fixed order, so what runs
beside a request does not change it.  A budget too small for two requests at
once must still serve them all (one at a time).
"""
import numpy as np
import pytest

from q3_b200 import synthetic
from q3_b200._lib import FP64, MIXED

pytestmark = pytest.mark.gpu


def _systems():
    out = [synthetic.small_system(grid=(12, 12, 12), a=7.0, ecut=8.0, nbands=6, seed=1),
           synthetic.small_system(grid=(16, 16, 16), a=8.0, ecut=10.0, nbands=8, natoms=3, seed=2),
           synthetic.small_system(grid=(15, 15, 15), a=7.5, ecut=9.0, nbands=5, seed=3,
                                  k_frac=(0.25, 0.0, 0.125)),
           synthetic.config(0)]
    out += synthetic.serving_requests(2, seed=77)
    return out


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_alone_equals_mixed(cuda_device, precision):
    from q3_b200.serving import BandSolveServer
    systems = _systems()
    kw = dict(tolerance=1e-9, max_iterations=100, precision=precision)
    many = BandSolveServer(workers=4)
    ids = [many.submit(sy, **kw) for sy in systems]
    mixed = [many.wait(i) for i in ids]
    many.close()
    one = BandSolveServer(workers=1)
    alone = []
    for sy in systems:
        alone.append(one.wait(one.submit(sy, **kw)))
    one.close()
    for a, m in zip(alone, mixed):
        assert np.max(np.abs(a.eigenvalues - m.eigenvalues)) < 1e-12
        assert a.iterations == m.iterations


def test_budget_admission_serialises(cuda_device):
    from q3_b200.serving import BandSolveServer, run_poisson_stream
    systems = _systems()[:4]
    srv = BandSolveServer(workers=4, hbm_budget=1)     # below any request's estimate
    out = run_poisson_stream(srv, systems, rate_hz=1000.0, tolerance=1e-8)
    srv.close()
    assert out["requests"] == 4 and out["unconverged_requests"] == 0
    assert out["p99_ms"] >= out["p50_ms"] > 0
    # with one request admitted at a time, every later request waits in the queue
    assert sum(r.queue_ms > 0 for r in out["results"]) >= 3


def test_server_matches_direct_solve(cuda_device):
    from q3_b200.applicator import PlanewaveHamiltonianApplicator
    from q3_b200.davidson import PlanewaveDavidsonDiagonalizer
    from q3_b200.serving import BandSolveServer
    sy = synthetic.config(0)
    ap = PlanewaveHamiltonianApplicator()
    ap.update_potential(sy.v_r, sy.cell.grid)
    ap.prepare_system_kpoint(sy)
    dv = PlanewaveDavidsonDiagonalizer(ap)
    dv.set_tolerance(1e-9)
    dv.set_maximum_iterations(100)
    direct = dv.solve(sy.psi0[0], sy.nbands)
    srv = BandSolveServer(workers=2)
    got = srv.wait(srv.submit(sy, tolerance=1e-9, max_iterations=100))
    srv.close()
    assert np.max(np.abs(got.eigenvalues - direct.eigenvalues)) < 1e-12


@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_batched_eigensolves(cuda_device, precision):
    # workers share their subspace eigensolves' launches: the results are the same alone
    # and in the mix, batches hold several problems, and the solves agree with an
    # unbatched server to rounding (the one-block eigensolver in place of the
    # multi-kernel one above order 56)
    from q3_b200.serving import BandSolveServer
    sy2 = synthetic.config(2)
    systems = [(sy2, k) for k in range(8)] + [(s, 0) for s in _systems()[:3]]
    kw = dict(tolerance=1e-9, max_iterations=200, precision=precision)
    many = BandSolveServer(workers=8, batching=True)
    ids = [many.submit(sy, k=k, **kw) for sy, k in systems]
    mixed = [many.wait(i) for i in ids]
    batches, problems = many.batch_stats()
    many.close()
    assert problems > batches > 0
    one = BandSolveServer(workers=1, batching=True)
    alone = [one.wait(one.submit(sy, k=k, **kw)) for sy, k in systems]
    one.close()
    plain = BandSolveServer(workers=4)
    ids = [plain.submit(sy, k=k, **kw) for sy, k in systems]
    ref = [plain.wait(i) for i in ids]
    plain.close()
    for a, m, r in zip(alone, mixed, ref):
        assert m.unconverged == 0
        assert np.max(np.abs(a.eigenvalues - m.eigenvalues)) < 1e-12
        assert a.iterations == m.iterations
        assert np.max(np.abs(m.eigenvalues - r.eigenvalues)) < (4e-8 if precision == MIXED else 1e-8)
