"""Independent-unit sharding over ranks: the assignment, and the gather on
two gloo ranks (CPU processes, no GPU).  The units' "solve" is the oracle's
dense eigensolve of small seeded Hermitian matrices, so the gathered result
can be checked against a single-process run."""
import os
import socket

import numpy as np
import pytest

from q3_b200.sharding import assign_units, solve_sharded, unit_cost


def test_assignment_balanced_and_complete():
    rng = np.random.default_rng(5)
    costs = [unit_cost(int(n), 48, (40, 40, 40)) for n in rng.integers(2900, 3100, size=32)]
    for world in (1, 2, 3, 4, 8):
        parts = assign_units(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs) + 1e-9
        assert parts == assign_units(costs, world)   # deterministic


def test_assignment_edge_cases():
    assert assign_units([], 3) == [[], [], []]
    assert assign_units([1.0], 4) == [[0], [], [], []]
    with pytest.raises(ValueError):
        assign_units([1.0], 0)


def _units(count=7, n=6):
    rng = np.random.default_rng(11)
    out = []
    for _ in range(count):
        x = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        out.append((x + x.conj().T) / 2)
    return out


def _solve(h):
    import oracle.davidson as odav
    return odav.diagonalize_subspace(h, np.eye(h.shape[0]), h.shape[0])[0]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        units = _units()
        costs = [float(i % 3 + 1) for i in range(len(units))]
        got = solve_sharded(units, costs, _solve, nbands=4)
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_gather_on_two_gloo_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    units = _units()
    ref = np.stack([_solve(h)[:4] for h in units])
    for r in (0, 1):
        assert np.max(np.abs(res[r] - ref)) < 1e-12
