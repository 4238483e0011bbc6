"""Band-solve serving over libq3b's server (continuous batching on one GPU).

``BandSolveServer`` wraps ``q3b_server_*``: requests (one cell at one k-point,
built by ``q3_b200.synthetic``) are submitted as they arrive, admitted by an
HBM budget, solved concurrently on separate streams, and collected with their
queue, solve and end-to-end latencies.  ``run_poisson_stream`` drives a
seeded Poisson arrival process and reports p50/p99 latency and solves/s.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import time
from typing import Dict, Iterable, List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import FP64, MIXED, DavidsonOpts, DavidsonStats, Request, RequestTimes


@dataclasses.dataclass
class Served:
    id: int
    eigenvalues: np.ndarray
    bands: np.ndarray
    iterations: int
    fp64_iterations: int
    unconverged: int
    queue_ms: float
    solve_ms: float
    latency_ms: float
    estimated_bytes: int


class BandSolveServer:
    def __init__(self, device: int = 0, hbm_budget: int = 0, workers: int = 4, batching: bool = False,
                 batch_wait_us: int = 200):
        """batching: solve the workers' subspace eigenproblems in shared launches (one block
        each) as they reach that step together (q3b_server_set_batching)."""
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.q3b_server_create(int(device), int(hbm_budget), int(workers), C.byref(h))
        if rc != 0:
            raise _lib.Q3BError(rc, "cannot create a server")
        self.h = h.value
        self._shape: Dict[int, tuple] = {}
        if batching:
            self._check(self.lib.q3b_server_set_batching(self.h, 1, int(batch_wait_us)))

    def batch_stats(self):
        """(batches launched, problems solved in them)."""
        b, p = C.c_long(), C.c_long()
        self._check(self.lib.q3b_server_batch_stats(self.h, C.byref(b), C.byref(p)))
        return b.value, p.value

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.q3b_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != 0:
            msg = self.lib.q3b_server_last_error(self.h)
            raise _lib.Q3BError(rc, msg.decode() if msg else "")

    def submit(self, system, k: int = 0, tolerance: float = 1e-8, max_iterations: int = 100,
               precision: int = FP64, mixed_tolerance: float = 1e-6, refine_sweeps: int = 0,
               bands: Optional[np.ndarray] = None) -> int:
        """Queue one band solve of `system` at k-point `k`; returns its id.  refine_sweeps 0
        gives a mixed solve's FP64 refinement up to max_iterations iterations."""
        kp = system.kpoints[k]
        n1, n2, n3 = system.cell.grid
        v = np.ascontiguousarray(system.v_r, dtype=np.float64)
        g2g = np.ascontiguousarray(kp.g_to_grid, dtype=np.int32)
        ke = np.ascontiguousarray(kp.ke, dtype=np.float64)
        beta = np.asfortranarray(kp.beta, dtype=np.complex128)
        offs = np.ascontiguousarray(kp.atom_proj_offsets, dtype=np.int32)
        dblk = np.ascontiguousarray(kp.d_blocks, dtype=np.float64)
        psi = np.asfortranarray(system.psi0[k] if bands is None else bands, dtype=np.complex128)
        opts = DavidsonOpts()
        self.lib.q3b_davidson_default_opts(C.byref(opts))
        opts.tolerance = tolerance
        opts.max_iterations = max_iterations
        opts.precision = precision
        opts.mixed_tolerance = mixed_tolerance
        opts.refine_sweeps = refine_sweeps
        req = Request(n1, n2, n3, v.ctypes.data, kp.npw, g2g.ctypes.data, ke.ctypes.data, kp.nproj,
                      beta.ctypes.data, len(offs) - 1, offs.ctypes.data, dblk.ctypes.data,
                      system.nbands, psi.ctypes.data, None, C.pointer(opts))
        rid = C.c_int()
        self._check(self.lib.q3b_server_submit(self.h, C.byref(req), C.byref(rid)))
        self._shape[rid.value] = (kp.npw, system.nbands)
        return rid.value

    def done(self, rid: int) -> bool:
        return self.lib.q3b_server_poll(self.h, rid) == 1

    def wait(self, rid: int, keep_bands: bool = True) -> Served:
        """Block until request `rid` is done; its bands come back only with keep_bands."""
        npw, nb = self._shape.pop(rid)
        bands = np.empty((npw, nb), dtype=np.complex128, order="F") if keep_bands else None
        eig = np.empty(nb, dtype=np.float64)
        st = DavidsonStats()
        tm = RequestTimes()
        self._check(self.lib.q3b_server_wait(self.h, rid, bands.ctypes.data if keep_bands else None,
                                             eig.ctypes.data, C.byref(st), C.byref(tm)))
        return Served(rid, eig, bands, st.iterations, st.fp64_iterations, st.unconverged,
                      tm.queue_ms, tm.solve_ms, tm.latency_ms, tm.estimated_bytes)


def _summary(results, wall: float) -> Dict:
    lat = np.array([r.latency_ms for r in results])
    return {
        "requests": len(results),
        "p50_ms": float(np.percentile(lat, 50)),
        "p99_ms": float(np.percentile(lat, 99)),
        "mean_queue_ms": float(np.mean([r.queue_ms for r in results])),
        "solves_per_s": len(results) / wall,
        "wall_s": wall,
        "unconverged_requests": int(sum(1 for r in results if r.unconverged)),
        "results": results,
    }


def run_poisson_stream(server: BandSolveServer, systems: Iterable, rate_hz: float, seed: int = 1238,
                       count: Optional[int] = None, keep_bands: bool = True, **solve_kw) -> Dict:
    """Submit `systems` (a sequence, or an iterable of `count` systems built as they are
    needed) at seeded Poisson arrival times; collect every result, finished ones as the
    stream goes (without their bands unless keep_bands).

    Returns p50/p99 latency (ms), solves/s over the stream and the results in order."""
    n = len(systems) if count is None else int(count)
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, size=n)
    t0 = time.perf_counter()
    pending: List[int] = []
    done: Dict[int, Served] = {}
    order: List[int] = []
    next_t = 0.0
    for sy, gap in zip(systems, gaps):
        next_t += gap
        delay = next_t - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        rid = server.submit(sy, **solve_kw)
        order.append(rid)
        pending.append(rid)
        still = []
        for p in pending:
            if server.done(p):
                done[p] = server.wait(p, keep_bands)
            else:
                still.append(p)
        pending = still
    for p in pending:
        done[p] = server.wait(p, keep_bands)
    wall = time.perf_counter() - t0
    return _summary([done[r] for r in order], wall)


def run_closed_loop(server: BandSolveServer, systems: Iterable, window: int, keep_bands: bool = False,
                    **solve_kw) -> Dict:
    """Capacity: keep `window` requests in the server (queued or running), submitting the next
    as one finishes, over all of `systems`; solves/s over the whole run."""
    t0 = time.perf_counter()
    inflight: List[int] = []
    done: Dict[int, Served] = {}
    order: List[int] = []
    for sy in systems:
        while len(inflight) >= window:
            still = []
            for p in inflight:
                if server.done(p):
                    done[p] = server.wait(p, keep_bands)
                else:
                    still.append(p)
            inflight = still
            if len(inflight) >= window:
                time.sleep(0.0005)
        rid = server.submit(sy, **solve_kw)
        order.append(rid)
        inflight.append(rid)
    for p in inflight:
        done[p] = server.wait(p, keep_bands)
    return _summary([done[r] for r in order], time.perf_counter() - t0)
