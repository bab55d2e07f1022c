"""Speed of this engine against the reference's own GPU drivers (oracle/_ref: the reference's FP32
*ShotsGpuFunctions.cu compiled unmodified for sm_100a) on the same workloads, on the same GPU.

The reference runs one shot per call through its free functions, as its shot loop does
(F/src/BornShotsGpu.cpp:103-135): init and allocate once per operator, then per shot a driver call
that allocates, copies and frees its own shot buffers. This engine runs the same shots as one
batched call through the C ABI with host buffers (copies included). The reference is timed on
its second call, this engine on its third: the first runs its interval loops as direct launches,
the second captures them into CUDA graphs (a one-time host cost), later calls replay them.
Printed: Gpts/s of both (interior points x fine steps x propagation passes / time);
asserted: the batched engine is at least 5x the reference's per-shot rate for Born forward +
adjoint, and at least 2x for the single-shot nonlinear forward and the free-surface Born pair.

Workloads: the Born benchmark grid (400x1200 physical, 512x1312 interior) at nts = 500 (the
per-interval cost does not depend on nts), 8 shots; the 200x400 nonlinear forward at its full
size (nts = 1000, one shot); the extended Born adjoint grid (500x1500, 608x1600 interior, nExt =
31) at nts = 300, 4 shots; the tomo / WEMVA grid (800x3000, 912x3104 interior, nExt = 41) at
nts = 150, one shot through the four operators (asserted: >= 3x and >= 2x the reference's
drivers). The CPU oracle's rates (FP32 and FP64, every host thread) on each configuration's grid
over 20 fine steps are printed beside them.
"""
import ctypes as C
import json
import time

import numpy as np
import pytest

import orc
import refgpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refgpu.available(), reason="oracle/_ref not built (make -C oracle ref)")]


def _prep(w, second):
    from test_gpu_configs import _prep as prep
    return prep(w, second)


def _ref_time(family, s, vel, nExt, call):
    """Seconds of one per-shot driver call after init + allocate (second of two calls)."""
    L = refgpu._lib(family, np.float32)
    k = orc.constants(s, vel, dtype=np.float32)
    v2 = np.ascontiguousarray(k["v2"], np.float32)
    rs = np.ascontiguousarray(k["rs"], np.float32)
    assert L.ref_init(s.dz, s.dx, s.nz, s.nx, s.nts, s.dts, s.sub, s.minPad, s.alphaCos, nExt, 1, 1, 0) == 0
    assert L.ref_allocate(v2.ctypes.data_as(C.c_void_p), rs.ctypes.data_as(C.c_void_p), 0) == 0
    try:
        call(L)
        t0 = time.perf_counter()
        call(L)
        return time.perf_counter() - t0
    finally:
        L.ref_deallocate(0)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _scheme(w, **kw):
    return orc.Scheme(nz=w.nz, nx=w.nx, nts=w.nts, dts=w.dts, sub=w.sub, dz=w.dz, dx=w.dx, minPad=w.minPad, **kw)


@pytest.mark.parametrize("free_surface", [0, 1])
def test_born_batched_vs_reference_drivers(free_surface):
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    from acoustic_isotropic_operators_b200 import synthetic as S
    w = S.born_workload(nshots=8, nts=500)
    v2, rs, sigs = _prep(w, 1)
    s = _scheme(w, freeSurface=free_surface)
    model = np.ascontiguousarray(w.model, np.float32)
    a = w.shots[0]
    sp, rp = np.ascontiguousarray(a.src_pos, np.int32), np.ascontiguousarray(a.rec_pos, np.int32)
    d = np.zeros((len(rp), w.nts), np.float32)
    img = np.zeros((w.nx, w.nz), np.float32)
    fwd = "ref_born_fwd_fs" if free_surface else "ref_born_fwd"
    adj = "ref_born_adj_fs" if free_surface else "ref_born_adj"

    def one_shot(L):
        getattr(L, fwd)(_p(model), _p(d), _p(sigs[0]), _p(sp), len(sp), _p(rp), len(rp), 0)
        getattr(L, adj)(_p(img), _p(d), _p(sigs[0]), _p(sp), len(sp), _p(rp), len(rp), 0)

    t_ref = _ref_time("born", s, w.vel, 1, one_shot)
    pts = float(w.n_interior) * w.fine_steps * 4
    ref_rate = pts / t_ref / 1e9
    ctx = Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs, image_fp64=True,
                  free_surface=free_surface)
    try:
        shots = [Shot(x.src_pos, x.rec_pos, g) for x, g in zip(w.shots, sigs)]
        for rep in range(3):  # direct launches, graph capture, replay (timed: the steady state)
            t0 = time.perf_counter()
            ctx.born_forward(model, shots)
            ctx.born_adjoint(shots)
            t = time.perf_counter() - t0
    finally:
        ctx.close()
    rate = pts * len(shots) / t / 1e9
    print(json.dumps({"born_fwd_adj": {"free_surface": free_surface, "engine_Gpts_s": rate,
                                       "reference_driver_Gpts_s": ref_rate, "ratio": rate / ref_rate}}))
    assert rate >= (5.0 if not free_surface else 2.0) * ref_rate


def test_nonlinear_single_shot_vs_reference_driver():
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    from acoustic_isotropic_operators_b200 import synthetic as S
    w = S.nonlinear_workload()
    v2, rs, sigs = _prep(w, 0)
    s = _scheme(w)
    a = w.shots[0]
    sp, rp = np.ascontiguousarray(a.src_pos, np.int32), np.ascontiguousarray(a.rec_pos, np.int32)
    d = np.zeros((len(rp), w.nts), np.float32)
    t_ref = _ref_time("nl", s, w.vel, 1,
                      lambda L: L.ref_nl_fwd(_p(sigs[0]), _p(d), _p(sp), len(sp), _p(rp), len(rp), None, 0))
    pts = float(w.n_interior) * w.fine_steps
    ctx = Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs)
    try:
        shot = [Shot(a.src_pos, a.rec_pos, sigs[0])]
        for _ in range(3):  # direct launches, graph capture, replay
            ctx.nonlinear_forward(shot)
        t0 = time.perf_counter()
        ctx.nonlinear_forward(shot)
        t = time.perf_counter() - t0
    finally:
        ctx.close()
    rate, ref_rate = pts / t / 1e9, pts / t_ref / 1e9
    print(json.dumps({"nonlinear_1_shot": {"engine_Gpts_s": rate, "reference_driver_Gpts_s": ref_rate,
                                           "ratio": rate / ref_rate}}))
    assert rate >= 2.0 * ref_rate


def test_ext_born_adjoint_vs_reference_driver():
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    from acoustic_isotropic_operators_b200 import synthetic as S
    n_ext = 31
    w = S.born_workload(nz_phys=500, nx_phys=1500, nshots=4, nts=300)
    v2, rs, sigs = _prep(w, 1)
    s = _scheme(w, nExt=n_ext)
    rng = np.random.default_rng(4)
    data = [(rng.standard_normal((len(a.rec_pos), w.nts)) * 1e-3).astype(np.float32) for a in w.shots]
    a = w.shots[0]
    sp, rp = np.ascontiguousarray(a.src_pos, np.int32), np.ascontiguousarray(a.rec_pos, np.int32)
    img = np.zeros((n_ext, w.nx, w.nz), np.float32)
    t_ref = _ref_time("bornext", s, w.vel, n_ext,
                      lambda L: L.ref_bornext_adj(_p(img), _p(data[0]), _p(sigs[0]), _p(sp), len(sp), _p(rp),
                                                  len(rp), 0, 0))
    pts = float(w.n_interior) * w.fine_steps * 2
    ctx = Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs, nExt=n_ext, image_fp64=True)
    try:
        shots = [Shot(x.src_pos, x.rec_pos, g, d) for x, g, d in zip(w.shots, sigs, data)]
        for _ in range(3):  # direct launches, graph capture, replay (timed: the steady state)
            t0 = time.perf_counter()
            ctx.born_ext_adjoint(shots)
            t = time.perf_counter() - t0
    finally:
        ctx.close()
    rate, ref_rate = pts * len(shots) / t / 1e9, pts / t_ref / 1e9
    print(json.dumps({"extended_born_adjoint": {"nExt": n_ext, "shots": len(shots), "engine_Gpts_s": rate,
                                                "reference_driver_Gpts_s": ref_rate, "ratio": rate / ref_rate}}))
    assert rate >= 3.0 * ref_rate


def test_tomo_wemva_vs_reference_drivers():
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    from acoustic_isotropic_operators_b200 import synthetic as S
    w = S.tomo_workload(nshots=1, nts=150)
    v2, rs, sigs = _prep(w, 1)
    s = _scheme(w, nExt=w.nExt)
    rng = np.random.default_rng(6)
    a = w.shots[0]
    sp, rp = np.ascontiguousarray(a.src_pos, np.int32), np.ascontiguousarray(a.rec_pos, np.int32)
    d = (rng.standard_normal((len(rp), w.nts)) * 1e-3).astype(np.float32)
    wd = (rng.standard_normal((len(rp), w.nts)) * 1e-3).astype(np.float32)
    ext = np.ascontiguousarray(w.extra["ext"], np.float32)
    m = np.ascontiguousarray(w.model, np.float32)
    out_d = np.zeros_like(d)
    out_m = np.zeros((w.nx, w.nz), np.float32)
    out_i = np.zeros((w.nExt, w.nx, w.nz), np.float32)
    g = sigs[0]

    def tomo(L):
        L.ref_tomo_fwd(_p(m), _p(out_d), _p(ext), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0, 0)
        L.ref_tomo_adj(_p(out_m), _p(d), _p(ext), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0, 0)

    def wemva(L):
        L.ref_wemva_fwd(_p(m), _p(out_i), _p(g), _p(sp), len(sp), _p(wd), _p(rp), len(rp), 0)
        L.ref_wemva_adj(_p(out_m), _p(ext), _p(g), _p(sp), len(sp), _p(wd), _p(rp), len(rp), 0)

    t_ref = _ref_time("tomo", s, w.vel, w.nExt, tomo) + _ref_time("wemva", s, w.vel, w.nExt, wemva)
    ctx = Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs, nExt=w.nExt, image_fp64=True)
    try:
        shots = [Shot(a.src_pos, a.rec_pos, g, d, wd)]
        for _ in range(3):  # direct launches, graph capture, replay (timed: the steady state)
            t0 = time.perf_counter()
            ctx.tomo_forward(m, ext, shots)
            ctx.tomo_adjoint(ext, shots)
            ctx.wemva_forward(m, shots)
            ctx.wemva_adjoint(ext, shots)
            t = time.perf_counter() - t0
    finally:
        ctx.close()
    pts = float(w.n_interior) * w.fine_steps * (5 + 4 + 4 + 4)
    rate, ref_rate = pts / t / 1e9, pts / t_ref / 1e9
    print(json.dumps({"tomo_wemva_1_shot": {"nExt": w.nExt, "engine_Gpts_s": rate, "reference_drivers_Gpts_s": ref_rate,
                                            "ratio": rate / ref_rate}}))
    assert rate >= 2.0 * ref_rate


def test_cpu_oracle_rates():
    """The CPU restatement of the scheme (every host thread, FP32 and FP64) on each configuration's
    grid over 20 fine steps (6 coarse samples), per propagation pass."""
    import os
    from acoustic_isotropic_operators_b200 import synthetic as S
    nts = 6
    cases = [("nonlinear 304x512", S.nonlinear_workload(nts=nts), 1, "nl"),
             ("born 512x1312", S.born_workload(nshots=1, nts=nts), 1, "born"),
             ("extended born 608x1600 nExt=31", S.born_workload(nz_phys=500, nx_phys=1500, nshots=1, nts=nts), 31,
              "ext"),
             ("tomo 912x3104 nExt=41", S.tomo_workload(nshots=1, nts=nts), 41, "tomo")]
    w0 = cases[0][1]
    orc.nl_fwd(_scheme(w0), w0.vel, np.zeros((len(w0.shots[0].src_pos), w0.ntw), np.float32), w0.shots[0].src_pos,
               w0.shots[0].rec_pos, dtype=np.float32)  # warm-up: library load, thread pool
    for label, w, n_ext, kind in cases:
        s = _scheme(w, nExt=n_ext)
        a = w.shots[0]
        rng = np.random.default_rng(0)
        sig = (rng.standard_normal((len(a.src_pos), w.ntw)) * 1e-2).astype(np.float32)
        d = (rng.standard_normal((len(a.rec_pos), w.nts)) * 1e-3).astype(np.float32)
        m = np.ascontiguousarray(w.model, np.float32)
        line = {"cpu_oracle": label, "threads": os.cpu_count(), "fine_steps": w.fine_steps}
        for dt in (np.float32, np.float64):
            t0 = time.perf_counter()
            if kind == "nl":
                orc.nl_fwd(s, w.vel, sig, a.src_pos, a.rec_pos, dtype=dt)
                passes = 1
            elif kind == "born":
                orc.born_fwd(s, w.vel, m, sig, a.src_pos, a.rec_pos, dtype=dt)
                orc.born_adj(s, w.vel, d, sig, a.src_pos, a.rec_pos, dtype=dt)
                passes = 4
            elif kind == "ext":
                orc.bornext_adj(s, w.vel, d, sig, a.src_pos, a.rec_pos, dtype=dt)
                passes = 2
            else:
                ext = np.ascontiguousarray(w.extra["ext"], np.float32)
                orc.tomo_fwd(s, w.vel, m, ext, sig, a.src_pos, a.rec_pos, dtype=dt)
                passes = 5
            el = time.perf_counter() - t0
            line[np.dtype(dt).name + "_Gpts_s"] = float(w.n_interior) * w.fine_steps * passes / el / 1e9
        print(json.dumps(line))
        assert line["float32_Gpts_s"] > 0 and line["float64_Gpts_s"] > 0
