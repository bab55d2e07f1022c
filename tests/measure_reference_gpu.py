"""Times the reference's own GPU drivers (oracle/_ref: the reference's FP32
BornShotsGpuFunctions.cu compiled unmodified for sm_100a) on one shot of the
Born benchmark workload (512x1312 interior, nts=2000, sub=4): Born forward then
Born adjoint through its free functions, one shot per call as the reference's
shot loop does. Prints one JSON line (Gpts/s over the 4 propagation passes and
shots/s). Run on a GPU machine with oracle/_ref built:

    python tests/measure_reference_gpu.py [--nts 2000] [--repeats 2]
    python tests/measure_reference_gpu.py --nl     # nonlinear forward, 1 shot, 304x512 interior, nts=1000
    python tests/measure_reference_gpu.py --variants   # free-surface Born forward + adjoint and the
                                                        # subsurface-offset extended Born forward and
                                                        # adjoint (nExt = 31)
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nts", type=int, default=2000)
    ap.add_argument("--repeats", type=int, default=2)
    ap.add_argument("--nl", action="store_true")
    ap.add_argument("--variants", action="store_true")
    a = ap.parse_args()
    import orc
    import refgpu
    import bench
    from acoustic_isotropic_operators_b200 import _capi, synthetic as S
    if a.nl:
        w = S.nonlinear_workload()
        sig = bench.prepare_signals(w, _capi.lib())[0]
        sh = w.shots[0]
        s = orc.Scheme(nz=w.nz, nx=w.nx, nts=w.nts, dts=w.dts, sub=w.sub, dz=w.dz, dx=w.dx, minPad=w.minPad)
        # init + allocate once (per operator, as the reference's shot loop does), then time the
        # per-shot driver call, which allocates, copies and frees its own shot buffers
        import ctypes as C
        L = refgpu._lib("nl", np.float32)
        k = orc.constants(s, w.vel, dtype=np.float32)
        v2 = np.ascontiguousarray(k["v2"], np.float32)
        assert L.ref_init(s.dz, s.dx, s.nz, s.nx, s.nts, s.dts, s.sub, s.minPad, s.alphaCos, 1, 1, 1, 0) == 0
        assert L.ref_allocate(v2.ctypes.data_as(C.c_void_p), None, 0) == 0
        sp = np.ascontiguousarray(sh.src_pos, np.int32)
        rp = np.ascontiguousarray(sh.rec_pos, np.int32)
        m = np.ascontiguousarray(sig, np.float32)
        d = np.zeros((len(rp), s.nts), np.float32)
        P = lambda x: x.ctypes.data_as(C.c_void_p)
        times = []
        for _ in range(a.repeats + 3):
            t0 = time.perf_counter()
            assert L.ref_nl_fwd(P(m), P(d), P(sp), len(sp), P(rp), len(rp), None, 0) == 0
            times.append(time.perf_counter() - t0)
        L.ref_deallocate(0)
        t = float(np.mean(times[3:]))
        print(json.dumps({"impl": "reference-gpu (own sm_100a build, one shot per call)",
                          "workload": "nonlinear forward, 1 shot, %dx%d interior, nts=%d" % (w.nz - 10, w.nx - 10,
                                                                                             w.nts),
                          "seconds_per_shot": t, "gpts_per_s": w.n_interior * w.fine_steps / t / 1e9}))
        return
    w = S.born_workload(nshots=1, nts=a.nts)
    sig = bench.prepare_signals(w, _capi.lib())[0]
    sh = w.shots[0]
    s = orc.Scheme(nz=w.nz, nx=w.nx, nts=w.nts, dts=w.dts, sub=w.sub, dz=w.dz, dx=w.dx, minPad=w.minPad)
    if a.variants:
        import dataclasses
        out = {}
        sfs = dataclasses.replace(s, freeSurface=1)
        soff = dataclasses.replace(s, extension=1, nExt=31)
        d0 = (np.random.default_rng(8).standard_normal((len(sh.rec_pos), s.nts)) * 1e-3).astype(np.float32)
        ext_model = np.ascontiguousarray(np.repeat(w.model[None], 31, axis=0) / 31, np.float32)
        cases = [("free_surface_born_forward_adjoint", 4,
                  lambda: refgpu.born_adj(sfs, w.vel, refgpu.born_fwd(sfs, w.vel, w.model, sig, sh.src_pos, sh.rec_pos),
                                          sig, sh.src_pos, sh.rec_pos)),
                 ("offset_extended_born_forward", 2,
                  lambda: refgpu.bornext_fwd(soff, w.vel, ext_model, sig, sh.src_pos, sh.rec_pos)),
                 ("offset_extended_born_adjoint", 2,
                  lambda: refgpu.bornext_adj(soff, w.vel, d0, sig, sh.src_pos, sh.rec_pos))]
        for name, passes, fn in cases:
            times = []
            for _ in range(a.repeats + 1):
                t0 = time.perf_counter()
                fn()
                times.append(time.perf_counter() - t0)
            t = float(np.mean(times[1:]))
            out[name] = {"seconds_per_shot": t, "passes": passes,
                         "Gpts_s": w.n_interior * w.fine_steps * passes / t / 1e9}
        print(json.dumps({"impl": "reference-gpu (own sm_100a build, one shot per call)",
                          "workload": "512x1312 interior, nts=%d, nExt=31 for offsets" % w.nts, "ops": out}))
        return
    times = []
    for _ in range(a.repeats + 1):
        t0 = time.perf_counter()
        d = refgpu.born_fwd(s, w.vel, w.model, sig, sh.src_pos, sh.rec_pos)
        refgpu.born_adj(s, w.vel, d, sig, sh.src_pos, sh.rec_pos)
        times.append(time.perf_counter() - t0)
    t = float(np.mean(times[1:]))
    pts = w.n_interior * w.fine_steps * 4
    print(json.dumps({"impl": "reference-gpu (own sm_100a build, one shot per call)",
                      "workload": "Born forward+adjoint, 1 shot, 512x1312 interior, nts=%d" % w.nts,
                      "seconds_per_shot": t, "gpts_per_s": pts / t / 1e9, "shots_per_s": 1.0 / t}))


if __name__ == "__main__":
    main()
