"""Serving loop scheduling on CPU with a stand-in engine: FIFO head first,
compatible requests merged up to max_batch, admission by the memory budget,
requests arriving while batches run join later batches, per-request results
and errors delivered through futures, p50 / p99 reported."""
import threading
import time

import numpy as np
import pytest

from acoustic_isotropic_operators_b200.batch import Shot
from acoustic_isotropic_operators_b200.serving import Grid, Request, Server, batch_shared_bytes, shot_bytes


def req(op, grid, tag, vid="v0"):
    s = Shot(np.array([5 * grid.nz + 7], np.int32), np.array([6 * grid.nz + 6], np.int32))
    s.tag = tag
    return Request(op=op, grid=grid, velocity_id=vid, vel2dtw2=None, refl_scale=None, shot=s, model_id="m0")


G1 = Grid(42, 58, 20, 0.004, 2, 10.0, 10.0, 8)
G2 = Grid(74, 90, 30, 0.004, 2, 10.0, 10.0, 8)
G3 = Grid(522, 1322, 30, 0.004, 2, 10.0, 10.0, 8)


class FakeEngine:
    def __init__(self, delay=0.05):
        self.delay = delay
        self.calls = []
        self.lock = threading.Lock()
        self.active = 0
        self.max_active = 0

    def __call__(self, worker, reqs):
        with self.lock:
            self.calls.append((worker, [r.shot.tag for r in reqs], reqs[0].key()))
            self.active += 1
            self.max_active = max(self.max_active, self.active)
        time.sleep(self.delay)
        with self.lock:
            self.active -= 1
        if any(r.shot.tag == "bad" for r in reqs):
            raise RuntimeError("engine failure")
        return [("result", r.shot.tag) for r in reqs]


def test_batches_compatible_requests_and_keeps_fifo_head():
    eng = FakeEngine(delay=0.1)
    srv = Server(workers=1, max_batch=3, mem_budget_bytes=1 << 40, run_batch=eng)
    futs = [srv.submit(req("born_forward", G1, i)) for i in range(5)]
    futs.append(srv.submit(req("born_adjoint", G1, "a")))
    futs += [srv.submit(req("born_forward", G1, i)) for i in range(5, 7)]
    res = [f.result(timeout=10) for f in futs]
    srv.close()
    assert [r[1] for r in res] == list(range(5)) + ["a"] + [5, 6]
    # first batch: head 0 plus compatible 1, 2 (max 3); the adjoint is never overtaken by later forwards
    assert eng.calls[0][1] == [0, 1, 2]
    # later compatible requests may join the head's batch (5 with 3, 4), but the adjoint
    # runs as soon as it is the head: the next batch
    assert eng.calls[1][1] == [3, 4, 5] and eng.calls[2][1] == ["a"] and eng.calls[3][1] == [6]
    assert all(len(c[1]) <= 3 for c in eng.calls)


def test_memory_budget_limits_concurrency():
    eng = FakeEngine(delay=0.1)
    one = batch_shared_bytes(G2) + shot_bytes(req("born_adjoint", G2, 0))  # one single-shot batch
    srv = Server(workers=4, max_batch=1, mem_budget_bytes=2 * one, run_batch=eng)
    futs = [srv.submit(req("born_adjoint", G2, i, vid=f"v{i}")) for i in range(6)]
    [f.result(timeout=10) for f in futs]
    srv.close()
    assert eng.max_active <= 2
    with pytest.raises(ValueError):
        Server(workers=1, mem_budget_bytes=one // 2, run_batch=eng).submit(req("born_adjoint", G2, 0))


def test_late_arrivals_join_while_others_run():
    eng = FakeEngine(delay=0.2)
    srv = Server(workers=2, max_batch=8, mem_budget_bytes=1 << 40, run_batch=eng)
    f0 = srv.submit(req("nonlinear_forward", G1, "first"))
    time.sleep(0.05)                       # first batch is on the "GPU"
    late = [srv.submit(req("nonlinear_forward", G1, f"late{i}")) for i in range(3)]
    for f in [f0] + late:
        f.result(timeout=10)
    srv.close()
    # the late requests ran on the other worker while the first batch was still running
    assert eng.max_active == 2
    rep = srv.report()
    assert rep["requests"] == 4 and rep["p99_s"] >= rep["p50_s"] > 0


def test_engine_error_reaches_every_future_of_its_batch():
    eng = FakeEngine(delay=0.01)
    srv = Server(workers=1, max_batch=4, mem_budget_bytes=1 << 40, run_batch=eng)
    fa = srv.submit(req("born_forward", G1, "bad"))
    fb = srv.submit(req("born_forward", G1, "ok"))
    fc = srv.submit(req("born_adjoint", G1, "other"))
    with pytest.raises(RuntimeError):
        fa.result(timeout=10)
    with pytest.raises(RuntimeError):
        fb.result(timeout=10)
    assert fc.result(timeout=10) == ("result", "other")
    srv.close()


def test_held_buffers_are_counted_reused_and_released():
    """Memory a worker's context keeps after a batch counts against the budget while the worker
    is idle: a batch of the same grid and velocity goes to that worker and reuses it, and when the
    head of the queue would not fit otherwise, idle workers free what they hold."""
    one = batch_shared_bytes(G2) + shot_bytes(req("born_adjoint", G2, 0))
    budget = 3 * one
    released, peaks = [], []
    srv = None

    def run(worker, reqs):
        peaks.append(srv.in_use)
        time.sleep(0.02)
        return [("result", r.shot.tag) for r in reqs], one     # each worker keeps one batch's bytes

    srv = Server(workers=3, max_batch=1, mem_budget_bytes=budget, run_batch=run, reports_held=True,
                 release=lambda w: released.append(w))
    # three velocities one after the other: every worker ends up holding buffers
    for i, vid in enumerate(("v0", "v1", "v2")):
        srv.submit(req("born_adjoint", G2, i, vid=vid)).result(timeout=10)
    with srv._lock:
        assert sum(srv._held) == srv.in_use
    # same velocity as a holder: its worker reuses the buffers, nobody releases
    srv.submit(req("born_adjoint", G2, "again", vid="v1")).result(timeout=10)
    assert released == []
    # a larger request on another grid needs more than one holder's room: idle holders free theirs
    big = req("born_adjoint", G3, "big", vid="v3")
    assert one < batch_shared_bytes(G3) + shot_bytes(big) <= budget
    srv.submit(big).result(timeout=10)
    assert released
    srv.close()
    assert max(peaks) <= budget
