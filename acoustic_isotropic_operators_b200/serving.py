"""Serving loop with continuous batching for operator requests of mixed grids and lengths.

A request is one shot of one operator call — nonlinear forward, Born forward or
Born adjoint — on a given grid / time axis / velocity (and model, for Born
forward). The server keeps a FIFO of waiting requests and a set of GPU workers
(one engine context and one CUDA stream per worker and grid, so batches of
different workers overlap on the device). Whenever a worker is idle it takes
the oldest waiting request together with every other waiting request that can
share its launches — same operator, grid, velocity and model — up to
``max_batch`` shots, provided their device memory fits in what the running
batches leave of the HBM budget. Requests that arrive while others are on the
GPU therefore join the next batch that frees a slot (continuous batching).
Order: the oldest waiting request always leads the next batch (no request is
passed over while it is at the head); later compatible requests may ride in
that batch.

Each request's result does not depend on what it was batched with: every shot
of a launch is computed independently (the Born adjoint returns each shot's own
image through ``aio_born_adjoint_shots``).

Latency = completion - arrival, reported as p50 / p99 with throughput in
shots/s (``Server.report``).
"""
from __future__ import annotations

import threading
import time
from collections import deque
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

OPS = ("nonlinear_forward", "born_forward", "born_adjoint")


@dataclass(frozen=True)
class Grid:
    nz: int
    nx: int
    nts: int
    dts: float
    sub: int
    dz: float
    dx: float
    minPad: int

    @property
    def interior_points(self) -> int:
        return (self.nz - 10) * (self.nx - 10)

    @property
    def ntw(self) -> int:
        return (self.nts - 1) * self.sub + 1


@dataclass
class Request:
    op: str
    grid: Grid
    velocity_id: str                 # identity of (vel2Dtw2, reflectivityScale); equal ids share a context
    vel2dtw2: np.ndarray
    refl_scale: Optional[np.ndarray]
    shot: object                     # batch.Shot
    model_id: str = ""               # Born forward: identity of the model (equal ids share a launch)
    model: Optional[np.ndarray] = None
    arrival: float = field(default_factory=time.perf_counter)
    start: float = 0.0
    done: float = 0.0
    future: Future = field(default_factory=Future, repr=False)

    def key(self) -> Tuple:
        return (self.op, self.grid, self.velocity_id, self.model_id if self.op == "born_forward" else "")


def _slices(g: Grid):
    """(interior slice, halo slice) sizes in floats, as the engine lays them out."""
    nzi, nxi = g.nz - 10, g.nx - 10
    isz = ((nzi + 31) // 32 * 32) * nxi
    hsz = (32 + (nzi + 31) // 32 * 32 + 32) * ((nxi + 31) // 32 * 32 + 10)
    return isz, hsz


def shot_bytes(req: Request, wavefield_bytes: int = 4) -> int:
    """Device memory one shot of `req` takes in a wave of the blocked stepper: the engine's own
    per-shot figure (state and partial-sum slices, stored wavefield and, for FP16, its staging and
    scales, FP64 image, traces, halo levels), so that server and engine plan with one number."""
    g = req.grid
    isz, hsz = _slices(g)
    wavefield = req.op != "nonlinear_forward"
    b = 6 * isz * 4 + 2 * hsz * 4 + 2 * isz * 4 + (1 << 16)
    if wavefield:
        b += g.nts * isz * wavefield_bytes
        if wavefield_bytes == 2:
            b += 2 * isz * 4 + 8 * g.nts
    if req.op == "born_adjoint":
        b += isz * 8
    b += len(req.shot.src_pos) * g.ntw * 4 + 2 * len(req.shot.rec_pos) * g.nts * 4
    return b


def batch_shared_bytes(g: Grid) -> int:
    """Device memory a wave needs besides its shots (the engine's shared figure)."""
    isz, _ = _slices(g)
    return 4 * isz * 4 + (64 << 20)


def _ctx_key(req: Request) -> Tuple:
    """Requests with equal keys run on the same engine context (grid and velocity)."""
    return (req.grid, req.velocity_id)


def _engine_batch(ctx_cache: Dict, worker: int, reqs: List[Request], device: int, wavefield: str,
                  reserved: int = 0):
    """Run one batch on this worker's context for the batch's grid and velocity (created on first
    use), with the context's device-memory budget set to the bytes the server reserved for the
    batch. The worker's other contexts free their buffers first, so that a worker holds the
    buffers of one context at a time. Returns (results, device bytes the worker holds after)."""
    from .batch import Context
    r0 = reqs[0]
    g = r0.grid
    key = (worker,) + _ctx_key(r0)
    for k, c in list(ctx_cache.items()):
        if k[0] == worker and k != key:
            c.release_buffers()
    ctx = ctx_cache.get(key)
    if ctx is None:
        ctx = Context(g.nz, g.nx, g.nts, g.dts, g.sub, g.dz, g.dx, g.minPad, r0.vel2dtw2, r0.refl_scale,
                      image_fp64=True, device=device, wavefield=wavefield, mem_budget_bytes=max(reserved, 1))
        ctx_cache[key] = ctx
    if reserved > 0:
        ctx.set_budget(reserved)
    shots = [r.shot for r in reqs]
    if r0.op == "nonlinear_forward":
        out = ctx.nonlinear_forward(shots)
    elif r0.op == "born_forward":
        out = ctx.born_forward(r0.model, shots)
    else:
        out = ctx.born_adjoint_shots(shots)
    return out, ctx.device_bytes


class Server:
    """Continuous-batching request server over the engine (see module docstring).

    run_batch(worker, requests) -> list of results may replace the engine (tests of the
    scheduling logic on CPU); with reports_held it returns (results, bytes the worker holds after
    the batch), as the engine does, and release(worker) frees what a worker holds."""

    def __init__(self, *, device: int = 0, workers: int = 2, max_batch: int = 16,
                 mem_budget_bytes: Optional[int] = None, wavefield: str = "fp32",
                 run_batch: Optional[Callable] = None, release: Optional[Callable] = None,
                 reports_held: bool = False):
        self.workers = workers
        self.max_batch = max_batch
        self.wavefield = wavefield
        self.wbytes = 2 if wavefield in ("bf16", "fp16") else 4
        if mem_budget_bytes is None:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
            mem_budget_bytes = int(0.8 * free)
        self.budget = int(mem_budget_bytes)
        self.in_use = 0
        self._ctx: Dict = {}
        self._engine = run_batch is None
        self._with_held = self._engine or reports_held
        self._run = run_batch or (lambda w, reqs, reserved=0: _engine_batch(self._ctx, w, reqs, device, wavefield,
                                                                               reserved))
        # memory an idle worker's context keeps between batches (its buffers are reused by the next
        # batch of the same grid and velocity): counted in in_use, freed when the room is needed
        self._release = release or self._release_engine
        self._held = [0] * workers
        self._held_key: List[Optional[Tuple]] = [None] * workers
        self._queue: deque = deque()
        self._idle = list(range(workers))
        self._lock = threading.Condition()
        self._closing = False
        self.finished: List[Request] = []
        self._reserved: Dict[int, int] = {}    # bytes reserved per running batch (by its head request)
        self.batches: List[Tuple[int, int]] = []   # (worker, batch size)
        self._threads: List[threading.Thread] = []
        self._sched = threading.Thread(target=self._schedule, daemon=True)
        self._sched.start()

    # ------------------------------------------------------------------ client side
    def submit(self, req: Request) -> Future:
        if req.op not in OPS:
            raise ValueError(f"unknown operator {req.op!r}")
        need = batch_shared_bytes(req.grid) + shot_bytes(req, self.wbytes)
        if need > self.budget:
            raise ValueError(f"request needs {need} bytes, above the budget of {self.budget}")
        with self._lock:
            req.arrival = time.perf_counter() if not req.arrival else req.arrival
            self._queue.append(req)
            self._lock.notify_all()
        return req.future

    def close(self, wait: bool = True):
        with self._lock:
            self._closing = True
            self._lock.notify_all()
        if wait:
            self._sched.join()
            for t in self._threads:
                t.join()
        for c in self._ctx.values():
            c.close()
        self._ctx.clear()

    # ------------------------------------------------------------------ scheduling
    def _release_engine(self, w: int) -> None:
        for k, c in list(self._ctx.items()):
            if k[0] == w:
                c.release_buffers()

    def _release_idle(self, keep: int) -> None:
        """Free the buffers idle workers (other than `keep`) hold, returning their bytes."""
        for w in list(self._idle):
            if w != keep and self._held[w] > 0:
                self._release(w)
                self.in_use -= self._held[w]
                self._held[w] = 0
                self._held_key[w] = None

    def _pick_worker(self, head: Request) -> int:
        """An idle worker whose context already holds buffers for the head's grid and velocity,
        else the idle worker holding the least memory."""
        key = _ctx_key(head)
        for w in self._idle:
            if self._held_key[w] == key:
                return w
        return min(self._idle, key=lambda w: self._held[w])

    def _take_batch(self, w: int) -> Optional[List[Request]]:
        """Oldest waiting request plus compatible waiting ones that fit in free memory, for
        worker w. The memory w holds counts as free for it (reused for the same context, freed
        otherwise); idle workers' held memory is freed when the head would not fit."""
        head = self._queue[0]
        need = batch_shared_bytes(head.grid) + shot_bytes(head, self.wbytes)
        reuse = self._held_key[w] == _ctx_key(head)
        if self.in_use - self._held[w] + need > self.budget:
            self._release_idle(keep=w)
            if self.in_use - self._held[w] + need > self.budget:
                return None                               # wait for memory; no overtaking of the head
        free = self.budget - (self.in_use - self._held[w])
        batch, used = [head], need
        key = head.key()
        for r in list(self._queue)[1:]:
            if len(batch) >= self.max_batch:
                break
            if r.key() == key:
                b = shot_bytes(r, self.wbytes)
                if used + b <= free:
                    batch.append(r)
                    used += b
        for r in batch:
            self._queue.remove(r)
        reserved = max(used, self._held[w]) if reuse else used
        self.in_use += reserved - self._held[w]
        self._held[w] = 0
        self._held_key[w] = None
        self._reserved[id(batch[0])] = reserved
        return batch

    def _schedule(self):
        while True:
            with self._lock:
                while True:
                    if self._queue and self._idle:
                        w = self._pick_worker(self._queue[0])
                        batch = self._take_batch(w)
                        if batch is not None:
                            break
                    if self._closing and not self._queue:
                        return
                    self._lock.wait(timeout=0.05)
                self._idle.remove(w)
            t = threading.Thread(target=self._work, args=(w, batch), daemon=True)
            self._threads.append(t)
            t.start()

    def _work(self, w: int, batch: List[Request]):
        t0 = time.perf_counter()
        for r in batch:
            r.start = t0
        err = None
        reserved = self._reserved[id(batch[0])]
        held = 0
        try:
            if self._engine:
                results, held = self._run(w, batch, reserved)
            elif self._with_held:
                results, held = self._run(w, batch)
            else:
                results = self._run(w, batch)
        except Exception as e:  # reported through every future of the batch
            err, results = e, [None] * len(batch)
        t1 = time.perf_counter()
        with self._lock:
            self.in_use -= self._reserved.pop(id(batch[0]))
            if err is None and held > 0:
                self._held[w] = held
                self._held_key[w] = _ctx_key(batch[0])
                self.in_use += held
            self._idle.append(w)
            self.batches.append((w, len(batch)))
            for r, res in zip(batch, results):
                r.done = t1
                self.finished.append(r)
            self._lock.notify_all()
        for r, res in zip(batch, results):
            if err is not None:
                r.future.set_exception(err)
            else:
                r.future.set_result(res)

    # ------------------------------------------------------------------ report
    def report(self) -> dict:
        lat = np.array([r.done - r.arrival for r in self.finished])
        if lat.size == 0:
            return {"requests": 0}
        t0 = min(r.arrival for r in self.finished)
        t1 = max(r.done for r in self.finished)
        pts = sum(r.grid.interior_points * (r.grid.nts - 1) * r.grid.sub * (1 if r.op == "nonlinear_forward" else 2)
                  for r in self.finished)
        return {"requests": int(lat.size), "shots_per_s": lat.size / (t1 - t0), "p50_s": float(np.percentile(lat, 50)),
                "p99_s": float(np.percentile(lat, 99)), "mean_batch": float(np.mean([b for _, b in self.batches])),
                "gpts_per_s": pts / (t1 - t0) / 1e9, "makespan_s": t1 - t0}


# ---------------------------------------------------------------------------- benchmark
def _stream(n_requests: int, n_models: int, scale: float, seed: int):
    """Seeded served stream: models with grids uniform in [200x400, 1000x3000] m at 10 m (times
    `scale`), gradient + blob velocities, nts uniform in [1000, 4000] (times `scale`), operators
    one third each; every request is one shot on one of the models."""
    from . import synthetic as S
    rng = np.random.default_rng(seed)
    models = []
    for k in range(n_models):
        nzp = int(rng.uniform(200, 1000) * scale) // 16 * 16 + 16
        nxp = int(rng.uniform(400, 3000) * scale) // 16 * 16 + 16
        nts = int(rng.uniform(1000, 4000) * scale)
        d, dts = 10.0, 0.004
        p = S.padding(nzp, nxp)
        v = S.with_blobs(S.gradient(nzp, nxp), rng, d)
        vel = S.pad_model(v.astype(np.float32), p)
        sub = S.sub_for(float(v.max()), dts, d)
        shots = [S.surface_acquisition(p, p.nz, int(x)) for x in np.linspace(0, nxp - 1, 8)]
        g = Grid(p.nz, p.nx, nts, dts, sub, d, d, min(p.zPadMinus, p.zPadPlus, p.xPadMinus, p.xPadPlus))
        models.append((g, vel, shots))
    reqs = []
    for i in range(n_requests):
        k = int(rng.integers(n_models))
        op = OPS[int(rng.integers(3))]
        reqs.append((k, op, int(rng.integers(1 << 30))))
    return models, reqs


def run_stream(requests: int = 48, models: int = 4, scale: float = 1.0, plain: int = 4, workers: int = 3,
               max_batch: int = 16, load: float = 0.85, seed: int = 3, wavefield: str = "fp32") -> dict:
    """Served stream against the one-shot-per-call plain path on `requests` seeded one-shot
    requests over `models` velocity models (grids uniform in [200x400, 1000x3000] x scale, nts in
    [1000, 4000] x scale; nonlinear forward, Born forward, Born adjoint a third each).

    1. plain: the first `plain` requests, each alone through a fresh context on the per-fine-step
       stepper (the reference's schedule), FP32;
    2. capacity: every request submitted at once to a Server;
    3. served: Poisson arrivals at `load` x capacity; p50 / p99 latency and shots/s."""
    import ctypes as C
    from . import _capi
    from .batch import Context, Shot
    lib = _capi.lib()
    mods, stream = _stream(requests, models, scale, seed)
    prepared = []
    for g, vel, _ in mods:
        v2 = np.zeros(g.nz * g.nx, np.float32)
        rs = np.zeros_like(v2)
        velf = np.ascontiguousarray(vel.reshape(-1), np.float32)
        _capi.check(lib.aio_fd_precompute(g.nz, g.nx, C.c_float(g.dts), g.sub, velf.ctypes.data_as(C.c_void_p),
                                          v2.ctypes.data_as(C.c_void_p), rs.ctypes.data_as(C.c_void_p)))
        prepared.append((v2, rs))

    def make(k, op, rseed):
        g, _, shots = mods[k]
        v2, rs = prepared[k]
        rng = np.random.default_rng(rseed)
        a_ = shots[int(rng.integers(len(shots)))]
        sig = (np.sin(np.arange(g.ntw) * 0.01 * (1 + rng.random()))[None, :] * 1e-2).astype(np.float32)
        sig = np.repeat(sig, len(a_.src_pos), axis=0)
        data = (rng.standard_normal((len(a_.rec_pos), g.nts)) * 1e-3).astype(np.float32) if op == "born_adjoint" else None
        m = np.zeros((g.nx, g.nz), np.float32)
        m[5:-5, 5:-5] = 0.01
        return Request(op=op, grid=g, velocity_id=f"m{k}", vel2dtw2=v2, refl_scale=rs,
                       shot=Shot(a_.src_pos, a_.rec_pos, sig, data), model_id=f"m{k}", model=m)

    def run_alone(r):
        ctx = Context(r.grid.nz, r.grid.nx, r.grid.nts, r.grid.dts, r.grid.sub, r.grid.dz, r.grid.dx, r.grid.minPad,
                      r.vel2dtw2, r.refl_scale, image_fp64=True, stepper="fine")
        try:
            t0 = time.perf_counter()
            if r.op == "nonlinear_forward":
                ctx.nonlinear_forward([r.shot])
            elif r.op == "born_forward":
                ctx.born_forward(r.model, [r.shot])
            else:
                ctx.born_adjoint([r.shot])
            return time.perf_counter() - t0
        finally:
            ctx.close()

    plain_t = [run_alone(make(*stream[i])) for i in range(min(plain, len(stream)))]
    plain_rate = len(plain_t) / sum(plain_t)
    srv = Server(workers=workers, max_batch=max_batch, wavefield=wavefield)
    try:
        for f in [srv.submit(make(*x)) for x in stream]:
            f.result()
        cap = srv.report()["shots_per_s"]
    finally:
        srv.close()
    rate = load * cap
    gaps = np.random.default_rng(seed + 1).exponential(1.0 / rate, len(stream))
    srv = Server(workers=workers, max_batch=max_batch, wavefield=wavefield)
    try:
        futs = []
        t0 = time.perf_counter()
        for gap, x in zip(gaps, stream):
            t0 += gap
            time.sleep(max(0.0, t0 - time.perf_counter()))
            r = make(*x)
            r.arrival = time.perf_counter()
            futs.append(srv.submit(r))
        for f in futs:
            f.result()
        rep = srv.report()
    finally:
        srv.close()
    return {"shots_per_s": rep["shots_per_s"], "p50_s": rep["p50_s"], "p99_s": rep["p99_s"],
            "mean_batch": rep["mean_batch"], "gpts_per_s": rep["gpts_per_s"], "capacity_shots_per_s": cap,
            "arrival_rate": rate, "load": load, "plain_shots_per_s": plain_rate, "plain_requests": len(plain_t),
            "vs_plain": rep["shots_per_s"] / plain_rate, "capacity_vs_plain": cap / plain_rate,
            "requests": len(stream), "models": models, "scale": scale, "workers": workers,
            "max_batch": max_batch, "wavefield": wavefield,
            "grids": [[g.nz, g.nx, g.nts, g.sub] for g, _, _ in mods]}


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="served request stream vs one-shot-per-call plain path")
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--models", type=int, default=4)
    ap.add_argument("--scale", type=float, default=1.0, help="grid and nts scale of the served stream")
    ap.add_argument("--plain", type=int, default=4, help="requests timed on the plain path")
    ap.add_argument("--workers", type=int, default=3)
    ap.add_argument("--max-batch", type=int, default=16)
    ap.add_argument("--load", type=float, default=0.85, help="arrival rate as a fraction of measured capacity")
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--wavefield", default="fp32", choices=("fp32", "bf16", "fp16"))
    a = ap.parse_args(argv)
    out = run_stream(a.requests, a.models, a.scale, a.plain, a.workers, a.max_batch, a.load, a.seed, a.wavefield)
    print(json.dumps({"metric": "served shots/s (one-shot requests, mixed grids and operators)",
                      "value": out["shots_per_s"], "unit": "shots/s", **out}))


if __name__ == "__main__":
    main()
