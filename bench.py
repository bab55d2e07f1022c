#!/usr/bin/env python
"""Benchmark: batched Born forward + adjoint (400 x 1200 physical grid at 10 m,
32 shots, nts = 2000 at 4 ms, 15 Hz Ricker, 1200 receivers, smoothed-gradient
background, 20-interface reflectivity) on the B200 engine.

One step = Born forward of every shot (model -> data) followed by Born adjoint
of that data (data -> image): 4 propagation passes per shot. The metric is
grid-point updates per second: interior points x fine steps x 4 passes x shots.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

`value` is measured with inputs resident in HBM (C ABI, device pointers);
`e2e` is the same metric through the C ABI with host buffers (host<->device
copies inside the timed region). Under torchrun each rank owns its own 32
shots (weak scaling) and the images are summed with one NCCL all-reduce.
`--impl reference` times the reference scheme's CPU implementation (this
repository's CPU port of it; the reference itself has no CPU path) on a
bounded sample of the same workload, on all host threads.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gpts/s (grid-point updates per second), batched Born forward+adjoint"
UNIT = "Gpts/s"
PASSES = 4
BYTES_PER_POINT = 16  # algorithmic bytes per point update: read p_old, p_cur, v2dtw2; write p_new (FP32)


def algo_bytes_per_step(w, nshots, wbytes):
    """Algorithmic HBM bytes of one Born forward+adjoint step (implementation independent):
    4 passes x 16 B per point update, plus per coarse interval and shot: store W (b) in each
    source pass, read W and dm (b + 4) in the scattered pass, read W and read-modify-write
    the FP32 image (b + 8) in the receiver pass; b = bytes per stored wavefield sample."""
    n, t = w.n_interior, w.nts - 1
    return nshots * n * (PASSES * BYTES_PER_POINT * w.fine_steps + t * (4 * wbytes + 12))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--shots", type=int, default=32, help="shots per GPU")
    ap.add_argument("--nts", type=int, default=2000)
    ap.add_argument("--wavefield", default="fp32", choices=["fp32", "bf16", "fp16"])
    ap.add_argument("--image", default="fp32", choices=["fp64", "fp32"],
                    help="Born image accumulation: FP32 as the reference accumulates it, or FP64")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-nts", type=int, default=0, help="coarse samples of the CPU sample (0 = auto)")
    ap.add_argument("--stepper", default="auto", choices=["auto", "fine", "blocked"])
    ap.add_argument("--chunk", type=int, default=0, help="blocked-stepper chunk width (0 = automatic)")
    ap.add_argument("--ext", type=int, default=0,
                    help="instead of the Born step: time the extended (time-lag, nExt=31) Born adjoint of N "
                         "shots on the 500x1500 grid and print that line")
    ap.add_argument("--tomo", type=int, default=0,
                    help="instead of the Born step: time the extended tomo and WEMVA operators (nExt=41) of N "
                         "shots on the 800x3000 grid (912x3104 interior) and print that line")
    ap.add_argument("--tomo-nts", type=int, default=3000)
    ap.add_argument("--nl", action="store_true",
                    help="instead of the Born step: time the nonlinear forward of one shot on the 200x400 grid "
                         "(304x512 interior, nts=1000) per call and print that line")
    ap.add_argument("--variants", type=int, default=0,
                    help="N > 0: time the free-surface Born and subsurface-offset extended Born operators on N shots")
    ap.add_argument("--plain", type=int, default=0,
                    help="instead of the batched step: time N shots one per call on the per-fine-step "
                         "stepper (the reference's schedule), FP32, and print that line")
    ap.add_argument("--serve", type=int, default=0,
                    help="instead of the Born step: N > 0 one-shot requests (nonlinear forward, Born forward, "
                         "Born adjoint) on 4 models with grids in 200x400..1000x3000 and nts in 1000..4000, "
                         "served with Poisson arrivals at 85%% of measured capacity; prints that line")
    ap.add_argument("--serve-models", type=int, default=4)
    ap.add_argument("--no-configs", action="store_true",
                    help="leave out the other configurations' sub-objects of the default line")
    return ap.parse_args()


def workload(args, nshots):
    from acoustic_isotropic_operators_b200 import synthetic as S
    return S.born_workload(nshots=nshots, nts=args.nts)


def prepare_signals(w, lib):
    """Born-family source chain in the product's C++ host code (per shot)."""
    sigs = []
    velf = np.ascontiguousarray(w.vel.reshape(-1), np.float32)
    for a in w.shots:
        wav = np.repeat(w.wavelet[None, :], a.src_cidx.shape[0], axis=0).astype(np.float32)
        out = np.zeros((len(a.src_pos), w.ntw), np.float32)
        rc = lib.aio_prepare_source(1, a.src_cidx.shape[0], a.src_cidx.shape[1],
                                    a.src_cidx.ctypes.data_as(C.c_void_p), a.src_w.ctypes.data_as(C.c_void_p),
                                    len(a.src_pos), a.src_pos.ctypes.data_as(C.c_void_p), w.nts, C.c_float(w.dts),
                                    w.sub, velf.ctypes.data_as(C.c_void_p), wav.ctypes.data_as(C.c_void_p),
                                    out.ctypes.data_as(C.c_void_p))
        assert rc == 0
        sigs.append(out)
    return sigs


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            self.p.wait()

    def summary(self):
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if "Active" in v and "Not" not in v})
        load = [x for x in sm if x > 0.5 * (max(mx) if mx else 0)] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_sample(w, sigs, nts_sample, threads):
    """Time the CPU port (FP32 restatement of the reference scheme) on one shot and a
    shortened time axis of the same grid; returns Gpts/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc
    s = orc.Scheme(nz=w.nz, nx=w.nx, nts=nts_sample, dts=w.dts, sub=w.sub, dz=w.dz, dx=w.dx, minPad=w.minPad)
    a = w.shots[0]
    sig = np.ascontiguousarray(sigs[0][:, : s.ntw])
    t0 = time.perf_counter()
    d = orc.born_fwd(s, w.vel, w.model, sig, a.src_pos, a.rec_pos, dtype=np.float32)
    orc.born_adj(s, w.vel, d, sig, a.src_pos, a.rec_pos, dtype=np.float32)
    dt = time.perf_counter() - t0
    pts = w.n_interior * (nts_sample - 1) * w.sub * PASSES
    return pts / dt / 1e9, dt, pts


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    w = workload(args, 1)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import orc  # the CPU port's own source preparation: this arm loads no product code
    sigs = [orc.prepare_source(np.repeat(w.wavelet[None, :], a.src_cidx.shape[0], axis=0), a.src_cidx, a.src_w,
                               len(a.src_pos), a.src_pos, w.nts, w.dts, w.sub, w.vel) for a in w.shots]
    nts_sample = args.cpu_nts or 150
    vals = []
    for i in range(args.warmup + args.steps):
        v, dt, pts = cpu_sample(w, sigs, nts_sample, threads)
        if i >= args.warmup:
            vals.append((v, dt))
    value = statistics.mean(v for v, _ in vals)
    ms = 1000 * statistics.mean(dt for _, dt in vals)
    sample = (f"1 of {args.shots} shots, Born forward+adjoint, full {w.nz}x{w.nx} grid, "
              f"nts={nts_sample} of {args.nts} coarse samples ({(nts_sample - 1) * w.sub} fine steps)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(args, w),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def kernel_name(args, w):
    if args.stepper != "fine" and w.sub == 4:
        return "k_tile (interval-blocked stepper, one launch per coarse interval)"
    return "k_step (fused fine-step stepper)"


def config_dict(args, w):
    return {"workload": "batched Born forward+adjoint, 400x1200 at 10 m, nts=2000, 15 Hz Ricker",
            "shots_per_gpu": args.shots, "grid_padded": [w.nz, w.nx],
            "interior": [w.nz - 10, w.nx - 10], "nts": w.nts, "sub": w.sub, "fine_steps": w.fine_steps,
            "passes_per_shot": PASSES, "wavefield": args.wavefield, "image": args.image, "receivers_per_shot": 1200,
            "stepper": args.stepper, "chunk": args.chunk,
            "parallelism": f"dp{args.gpus} (shots)", "l2": "inputs larger than L2 (5.4 GB wavefield per shot)"}


def fields(w, lib):
    """v^2 dtw^2 and 2/v^3 of a workload through the product's host code (aio_fd_precompute)."""
    v2 = np.zeros(w.nz * w.nx, np.float32)
    rs = np.zeros_like(v2)
    velf = np.ascontiguousarray(w.vel.reshape(-1), np.float32)
    assert lib.aio_fd_precompute(w.nz, w.nx, C.c_float(w.dts), w.sub, velf.ctypes.data_as(C.c_void_p),
                                 v2.ctypes.data_as(C.c_void_p), rs.ctypes.data_as(C.c_void_p)) == 0
    return v2, rs


def hbm_peak():
    """(GB/s, 'measured' | 'fallback'): the measured copy bandwidth of this GPU pool."""
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        v = json.load(open(pk)).get("hbm_gbs")
        if v:
            return float(v), "measured"
    return 6650.0, "fallback"


def run_plain(args, emit=True):
    """One shot per call, per-fine-step stepper, FP32 wavefield: the plain GPU path (the
    reference's schedule on this engine), Born forward + adjoint of each shot, host buffers."""
    import torch
    from acoustic_isotropic_operators_b200 import _capi
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    w = workload(args, args.plain)
    lib = _capi.lib()
    v2, rs = fields(w, lib)
    sigs = prepare_signals(w, lib)
    model = np.ascontiguousarray(w.model, np.float32)
    times = []
    for i, (a, sg) in enumerate(zip(w.shots, sigs)):
        ctx = Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs,
                      image_fp64=getattr(args, "image", "fp32") == "fp64", stepper="fine")
        shot = Shot(a.src_pos, a.rec_pos, sg)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.born_forward(model, [shot])
        ctx.born_adjoint([shot])
        times.append(time.perf_counter() - t0)
        ctx.close()
    t = statistics.mean(times[1:] if len(times) > 1 else times)
    pts = w.n_interior * w.fine_steps * PASSES
    out = {"impl": "plain (this engine, one shot per call, per-fine-step stepper, FP32 W)",
           "metric": METRIC, "value": pts / t / 1e9, "unit": UNIT, "seconds_per_shot": t,
           "shots_per_s": 1.0 / t, "shots": len(times), "timed_shots": max(1, len(times) - 1),
           "inputs": "host buffers (copies inside the timed call)"}
    if emit:
        print(json.dumps(dict(out, config=config_dict(args, w))))
        return 0
    return out


def run_ext(args, emit=True):
    """Extended (time-lag, nExt = 31) Born adjoint of N shots on the 500x1500 physical grid
    (608x1600 interior), host buffers, one call after one warm-up call."""
    import torch
    from acoustic_isotropic_operators_b200 import _capi, synthetic as S
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    n_ext = 31
    w = S.born_workload(nz_phys=500, nx_phys=1500, nshots=args.ext, nts=args.nts)
    lib = _capi.lib()
    v2, rs = fields(w, lib)
    sigs = prepare_signals(w, lib)
    rng = np.random.default_rng(4)
    shots = [Shot(a.src_pos, a.rec_pos, sg, (rng.standard_normal((len(a.rec_pos), w.nts)) * 1e-3).astype(np.float32))
             for a, sg in zip(w.shots, sigs)]
    ctx = Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs, nExt=n_ext,
                  image_fp64=getattr(args, "image", "fp32") == "fp64", wavefield=args.wavefield)
    ctx.born_ext_adjoint(shots)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx.born_ext_adjoint(shots)
    t = time.perf_counter() - t0
    n, steps, T = w.n_interior, w.fine_steps, w.nts - 1
    pts = n * steps * 2 * len(shots)
    wb = 4 if args.wavefield == "fp32" else 2
    algo = len(shots) * n * (2 * 16 * steps + wb * w.nts + (4 + wb) * T + 8 * n_ext)
    peak, src = hbm_peak()
    out = {"impl": f"this engine, extended Born adjoint (blocked stepper, blocked lag imaging, "
                   f"{args.wavefield.upper()} stored W)", "wavefield": args.wavefield,
           "image": getattr(args, "image", "fp32"),
           "metric": "Gpts/s, extended (time-lag) Born adjoint", "value": pts / t / 1e9, "unit": UNIT,
           "seconds": t, "shots": len(shots), "shots_per_s": len(shots) / t, "nExt": n_ext,
           "interior": [w.nz - 10, w.nx - 10], "nts": w.nts,
           "roofline": {"bound": "hbm", "achieved": algo / t / 1e9, "peak": peak, "peak_source": src,
                        "unit": "GB/s", "frac": algo / t / 1e9 / peak,
                        "what": "whole call (host buffers), algorithmic bytes 16 B per update + stored / read W, "
                                "receiver samples and the FP32 extended image"},
           "inputs": "host buffers (copies inside the timed call)", "data": "synthetic (seeded)"}
    ctx.close()
    if emit:
        print(json.dumps(out))
        return 0
    return out


def run_tomo(args, emit=True):
    """Extended tomo and WEMVA forward and adjoint (time lags, nExt = 41) of N shots on the
    800x3000 physical grid (912x3104 interior, nts = 3000), host buffers; every operator is
    called twice and the second call is timed (the first one includes the stepper autotuning)."""
    import torch
    from acoustic_isotropic_operators_b200 import _capi, synthetic as S
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    w = S.tomo_workload(nshots=args.tomo, nts=args.tomo_nts)
    lib = _capi.lib()
    v2, rs = fields(w, lib)
    sigs = prepare_signals(w, lib)
    rng = np.random.default_rng(6)
    noise = lambda a: (rng.standard_normal((len(a.rec_pos), w.nts)) * 1e-3).astype(np.float32)
    shots = [Shot(a.src_pos, a.rec_pos, sg, noise(a), noise(a)) for a, sg in zip(w.shots, sigs)]
    ext = np.ascontiguousarray(w.extra["ext"], np.float32)
    m = np.ascontiguousarray(w.model, np.float32)
    ctx = Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs, nExt=w.nExt,
                  image_fp64=getattr(args, "image", "fp32") == "fp64", stepper=args.stepper, wavefield=args.wavefield)
    # (name, propagation passes, full coarse-field sweeps per shot: the source wavefield written,
    # its d2/dt2 read and written, and every later write or read of a stored field; FP32)
    ops = [("tomo_forward", 5, 9, lambda: ctx.tomo_forward(m, ext, shots)),
           ("tomo_adjoint", 4, 8, lambda: ctx.tomo_adjoint(ext, shots)),
           ("wemva_forward", 4, 8, lambda: ctx.wemva_forward(m, shots)),
           ("wemva_adjoint", 4, 8, lambda: ctx.wemva_adjoint(ext, shots))]
    n, steps = w.n_interior, w.fine_steps
    res, tot_pts, tot_t, tot_bytes = {}, 0.0, 0.0, 0.0
    for name, passes, sweeps, fn in ops:
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        t = time.perf_counter() - t0
        pts = float(n) * steps * passes * len(shots)
        nbytes = float(n) * len(shots) * (BYTES_PER_POINT * steps * passes + 4 * w.nts * sweeps)
        res[name] = {"seconds": t, "passes": passes, "Gpts_s": pts / t / 1e9, "algorithmic_GBps": nbytes / t / 1e9}
        tot_pts += pts
        tot_t += t
        tot_bytes += nbytes
    stepper = {"auto": "blocked stepper", "blocked": "blocked stepper", "fine": "per-fine-step stepper"}[args.stepper]
    peak, src = hbm_peak()
    wsrc = {"fp32": "FP32", "fp16": "FP16 + per-slice scale", "bf16": "BF16"}[args.wavefield]
    out = {"impl": f"this engine, extended tomo + WEMVA ({stepper}, source field d2/dt2 in {wsrc}, second field FP32)",
           "wavefield": args.wavefield, "image": getattr(args, "image", "fp32"),
           "metric": "Gpts/s, extended tomo + WEMVA forward and adjoint", "value": tot_pts / tot_t / 1e9,
           "unit": UNIT, "seconds": tot_t, "ops": res, "shots": len(shots), "nExt": w.nExt,
           "interior": [w.nz - 10, w.nx - 10], "nts": w.nts,
           "roofline": {"bound": "hbm", "achieved": tot_bytes / tot_t / 1e9, "peak": peak, "peak_source": src,
                        "unit": "GB/s", "frac": tot_bytes / tot_t / 1e9 / peak,
                        "what": "whole calls (host buffers), algorithmic bytes 16 B per update + coarse-field sweeps"},
           "inputs": "host buffers (copies inside the timed calls)", "data": "synthetic (seeded)"}
    ctx.close()
    if emit:
        print(json.dumps(out))
        return 0
    return out


def run_variants(args):
    """The free-surface and subsurface-offset operators on the Born benchmark grid (512x1312
    interior, nts from --nts): free-surface Born forward + adjoint and the subsurface-offset
    extended Born forward and adjoint (nExt = 31), on the blocked stepper, N shots per call through
    the C ABI with host buffers; each call is made twice and the second one timed."""
    import torch
    from acoustic_isotropic_operators_b200 import _capi, synthetic as S
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    n_ext = 31
    w = S.born_workload(nshots=args.variants, nts=args.nts)
    lib = _capi.lib()
    v2 = np.zeros(w.nz * w.nx, np.float32)
    rs = np.zeros_like(v2)
    velf = np.ascontiguousarray(w.vel.reshape(-1), np.float32)
    lib.aio_fd_precompute(w.nz, w.nx, C.c_float(w.dts), w.sub, velf.ctypes.data_as(C.c_void_p),
                          v2.ctypes.data_as(C.c_void_p), rs.ctypes.data_as(C.c_void_p))
    sigs = prepare_signals(w, lib)
    rng = np.random.default_rng(8)
    shots = [Shot(a.src_pos, a.rec_pos, sg, (rng.standard_normal((len(a.rec_pos), w.nts)) * 1e-3).astype(np.float32))
             for a, sg in zip(w.shots, sigs)]
    model = np.ascontiguousarray(w.model, np.float32)
    ext_model = np.ascontiguousarray(np.repeat(model[None], n_ext, axis=0) / n_ext, np.float32)
    n, steps = w.n_interior, w.fine_steps
    out = {}
    geo = (w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs)
    cases = [("free_surface_born_forward_adjoint", 4, dict(image_fp64=True, free_surface=1),
              lambda c: (c.born_forward(model, shots), c.born_adjoint(shots))),
             ("offset_extended_born_forward", 2, dict(nExt=n_ext, image_fp64=True, extension="offset"),
              lambda c: c.born_ext_forward(ext_model, shots)),
             ("offset_extended_born_adjoint", 2, dict(nExt=n_ext, image_fp64=True, extension="offset"),
              lambda c: c.born_ext_adjoint(shots))]
    for name, passes, kw, fn in cases:
        ctx = Context(*geo, **kw)   # one context at a time: each sizes its waves by the free memory
        fn(ctx)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn(ctx)
        t = time.perf_counter() - t0
        ctx.close()
        out[name] = {"seconds": t, "passes": passes, "Gpts_s": n * steps * passes * len(shots) / t / 1e9,
                     "seconds_per_shot": t / len(shots)}
    print(json.dumps({"impl": "this engine, free-surface Born and subsurface-offset extended Born "
                              "(blocked stepper), FP32, host buffers",
                      "metric": "Gpts/s", "unit": UNIT, "ops": out,
                      "shots": len(shots), "nExt": n_ext, "interior": [w.nz - 10, w.nx - 10], "nts": w.nts,
                      "data": "synthetic (seeded)"}))
    return 0


def run_nl(args, emit=True):
    """Nonlinear forward of one shot on the 200x400 physical grid with Gaussian blobs (304x512
    interior, nts = 1000, 400 receivers), one call per shot through the C ABI with host buffers:
    the latency-bound single-shot case (its three state slices fit in L2)."""
    import torch
    from acoustic_isotropic_operators_b200 import _capi, synthetic as S
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    w = S.nonlinear_workload()
    lib = _capi.lib()
    v2, rs = fields(w, lib)
    sig = prepare_signals(w, lib)[0]
    shot = Shot(w.shots[0].src_pos, w.shots[0].rec_pos, sig)
    out = {}
    for stepper in ("auto", "fine"):
        ctx = Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs, stepper=stepper)
        for _ in range(3):
            ctx.nonlinear_forward([shot])
        torch.cuda.synchronize()
        reps, batches = 10, 5
        ts = []
        for _ in range(batches):
            t0 = time.perf_counter()
            for _ in range(reps):
                ctx.nonlinear_forward([shot])
            ts.append((time.perf_counter() - t0) / reps)
        t = sorted(ts)[batches // 2]  # median batch
        out["blocked" if stepper == "auto" else "per_fine_step"] = {
            "seconds_per_call": t, "Gpts_s": w.n_interior * w.fine_steps / t / 1e9}
        if stepper == "auto":
            out["blocked"]["plan"] = ctx.blocked_plan(0)
        ctx.close()
    peak, src = hbm_peak()
    t = out["blocked"]["seconds_per_call"]
    algo = 16.0 * w.n_interior * w.fine_steps
    res = {"impl": "this engine, nonlinear forward, one shot per call (host buffers)",
           "metric": "Gpts/s, nonlinear forward", "unit": UNIT, "value": out["blocked"]["Gpts_s"],
           "shots_per_s": 1.0 / t, "steppers": out, "interior": [w.nz - 10, w.nx - 10], "nts": w.nts,
           "sub": w.sub, "receivers": len(w.shots[0].rec_pos),
           "roofline": {"bound": "hbm", "achieved": algo / t / 1e9, "peak": peak, "peak_source": src, "unit": "GB/s",
                        "frac": algo / t / 1e9 / peak,
                        "what": "whole call, 16 B per update; the three state slices (0.6 MB each) stay in L2"},
           "inputs": "host buffers (copies inside the timed call)", "data": "synthetic (seeded)"}
    if emit:
        print(json.dumps(res))
        return 0
    return res


def other_configs(args, batched_value):
    """The other benchmark configurations, each timed once after the headline (1 GPU): the
    single-shot nonlinear forward (200x400), the plain one-shot-per-call path on the headline's
    grid, the extended Born adjoint (500x1500, nExt = 31, 64 shots) and the extended tomo + WEMVA
    operators (800x3000, nExt = 41, 2 of 96 shots: the shots one FP32 wave holds)."""
    import copy
    out = {}
    a = copy.copy(args)
    out["nonlinear_forward_1_shot"] = run_nl(a, emit=False)
    a = copy.copy(args)
    a.plain, a.nts = 3, args.nts
    plain = run_plain(a, emit=False)
    plain["batched_over_plain"] = batched_value / plain["value"]
    out["plain_one_shot_per_call"] = plain
    for wf in ("fp32", "fp16", "bf16"):
        a = copy.copy(args)
        a.ext, a.nts, a.wavefield = 64, 2000, wf
        out[f"extended_born_adjoint_64_shots_{wf}"] = run_ext(a, emit=False)
    a = copy.copy(args)
    a.tomo, a.tomo_nts, a.stepper = 2, 3000, "auto"
    out["tomo_wemva_2_shots"] = run_tomo(a, emit=False)
    a = copy.copy(args)
    a.serve = 32
    out["served_stream"] = run_serve(a, emit=False)
    return out


def run_serve(args, emit=True):
    """Served request stream (continuous batching over the engine) against the plain
    one-shot-per-call path: seeded one-shot requests on `serve_models` velocity models with grids
    uniform in 200x400..1000x3000 and nts uniform in 1000..4000, Poisson arrivals at 85 % of the
    capacity measured on the same stream; p50 / p99 latency and shots/s."""
    from acoustic_isotropic_operators_b200.serving import run_stream
    out = run_stream(requests=args.serve, models=args.serve_models, scale=1.0, plain=4, workers=3,
                     max_batch=16, load=0.85, seed=3, wavefield="fp32")
    line = {"metric": "served shots/s (one-shot requests, mixed grids and operators)", "value": out["shots_per_s"],
            "unit": "shots/s", "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded)", **out}
    if emit:
        print(json.dumps(line))
    return line


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.plain:
        return run_plain(args)
    if args.ext:
        return run_ext(args)
    if args.tomo:
        return run_tomo(args)
    if args.variants:
        return run_variants(args)
    if args.nl:
        return run_nl(args)
    if args.serve:
        run_serve(args)
        return 0

    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    from acoustic_isotropic_operators_b200 import _capi
    from acoustic_isotropic_operators_b200.batch import Context
    from acoustic_isotropic_operators_b200 import synthetic as S

    from acoustic_isotropic_operators_b200.multigpu import max_over_ranks, reduce_image, shard
    full = workload(args, args.shots * world)
    mine = [full.shots[i] for i in shard(len(full.shots), rank, world)]
    w = full
    lib = _capi.lib()
    v2 = np.zeros(w.nz * w.nx, np.float32)
    rs = np.zeros(w.nz * w.nx, np.float32)
    velf = np.ascontiguousarray(w.vel.reshape(-1), np.float32)
    assert lib.aio_fd_precompute(w.nz, w.nx, C.c_float(w.dts), w.sub, velf.ctypes.data_as(C.c_void_p),
                                 v2.ctypes.data_as(C.c_void_p), rs.ctypes.data_as(C.c_void_p)) == 0
    w_mine = S.Workload(w.name, w.pad, w.nts, w.dts, w.sub, w.dz, w.dx, w.vel, w.wavelet, mine, model=w.model)
    sigs = prepare_signals(w_mine, lib)

    ctx = Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs, wavefield=args.wavefield,
                  image_fp64=args.image == "fp64", device=local, stepper=args.stepper, chunk_columns=args.chunk)
    dev = torch.device("cuda", local)
    model_d = torch.from_numpy(np.ascontiguousarray(w.model, np.float32)).to(dev)
    image_d = torch.zeros((w.nx, w.nz), dtype=torch.float32, device=dev)
    sig_d = [torch.from_numpy(s).to(dev) for s in sigs]
    dat_d = [torch.zeros((len(a.rec_pos), w.nts), dtype=torch.float32, device=dev) for a in mine]
    torch.cuda.synchronize()
    shots = [(a.src_pos, a.rec_pos, s.data_ptr(), d.data_ptr(), 0, 0) for a, s, d in zip(mine, sig_d, dat_d)]

    def step():
        ctx.device_call("born_forward", C.c_void_p(model_d.data_ptr()), shots=shots)
        ctx.device_call("born_adjoint", C.c_void_p(image_d.data_ptr()), C.c_int(0), shots=shots)

    stream = torch.cuda.ExternalStream(ctx.stream_ptr, device=dev)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    ctx.reset_stats()
    ctx.profile(16)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        barrier()
    ctx.profile(0)
    kernels, step_ms, n_timed, step_pts = ctx.stats()
    ms = max_over_ranks(e0.elapsed_time(e1), device=dev)
    reduce_image(image_d)  # the images of all ranks' shots (the one collective of the path)
    ms_per_step = ms / args.steps
    pts_per_step = w.n_interior * w.fine_steps * PASSES * args.shots * world
    value = pts_per_step / (ms_per_step / 1e3) / 1e9

    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    hbm_peak = peaks.get("hbm_gbs")
    peak_src = "measured" if hbm_peak else "fallback"
    hbm_peak = hbm_peak or 6650.0
    # Dominant kernel: the stepper. Every 16th stepper launch is bracketed by CUDA events on
    # the context stream; achieved = algorithmic bytes of those launches / their device time.
    wbytes = 2 if args.wavefield in ("bf16", "fp16") else 4
    algo_step = algo_bytes_per_step(w, args.shots, wbytes)
    pts_step_rank = w.n_interior * w.fine_steps * PASSES * args.shots
    bytes_per_update = algo_step / pts_step_rank  # launches of all passes are sampled alike
    achieved = (bytes_per_update * step_pts / 1e9) / (step_ms / 1e3) if step_ms > 0 else None
    launch_pts = args.shots * w.n_interior * w.sub  # point updates of one stepper launch (one interval, all shots)
    traffic = None
    tr = os.path.join(ROOT, "profiles", "stepper_traffic.json")
    if os.path.exists(tr):
        try:
            byp = json.load(open(tr))["bytes_per_point_update"]
            key = args.wavefield if args.image == "fp32" else args.wavefield + "_fp64_image"
            traffic = byp[key] * launch_pts if key in byp else None
        except Exception:
            traffic = None

    try:  # plan of the timed region's last launch (a receiver pass of the last wave)
        plan = ctx.blocked_plan(0) if kernel_name(args, w).startswith("k_tile") else None
    except Exception:
        plan = None

    # ------------------------------------------------ e2e through the C ABI (host buffers)
    e2e = None
    if not args.no_e2e:
        from acoustic_isotropic_operators_b200.batch import Shot
        host_shots = [Shot(a.src_pos, a.rec_pos, s) for a, s in zip(mine, sigs)]
        model_h = np.ascontiguousarray(w.model, np.float32)
        ctx.born_forward(model_h, host_shots)
        barrier()
        t0 = time.perf_counter()
        for _ in range(max(1, args.steps)):
            ctx.born_forward(model_h, host_shots)
            img = ctx.born_adjoint(host_shots)
        barrier()
        e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / max(1, args.steps), device=dev)
        h2d = model_h.nbytes + 2 * sum(s.nbytes for s in sigs) + sum(len(a.rec_pos) * w.nts * 4 for a in mine)
        d2h = sum(len(a.rec_pos) * w.nts * 4 for a in mine) + img.nbytes
        e2e = {"value": pts_per_step / (e_ms / 1e3) / 1e9, "unit": UNIT, "ms_per_step": e_ms,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        nts_sample = args.cpu_nts or 150
        v, dt, _ = cpu_sample(w_mine, sigs, nts_sample, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"1 shot, Born forward+adjoint, full grid, nts={nts_sample} ({dt:.1f} s)"}

    ctx.close()
    configs = None
    if world == 1 and not args.no_configs:
        configs = other_configs(args, value)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded, the workload's shapes)",
                "config": dict(config_dict(args, w), plan=plan),
                "roofline": {"bound": "hbm", "kernel": kernel_name(args, w),
                             "achieved": achieved, "peak": hbm_peak, "peak_source": peak_src, "unit": "GB/s",
                             "frac": (achieved / hbm_peak) if achieved else None,
                             "traffic": traffic, "traffic_unit": "bytes per launch (ncu dram read+write)",
                             "algorithmic_bytes_per_step": algo_step, "timed_launches": n_timed,
                             "stepper_ms_share": (step_ms * 16 / ms) if ms > 0 else None},
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": kernels, "clocks": clk.summary()}
        if configs is not None:
            line["configs"] = configs
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
