"""Speed of this engine against the reference's own GPU drivers (oracle/_ref: the reference's FP32
*ShotsGpuFunctions.cu compiled unmodified for sm_100a) on the same workloads, on the same GPU.

The reference runs one shot per call through its free functions, as its shot loop does
(F/src/BornShotsGpu.cpp:103-135): init and allocate once per operator, then per shot a driver call
that allocates, copies and frees its own shot buffers. This engine runs the same shots as one
batched call through the C ABI with host buffers (copies included). Each side is timed on its
second call. Printed: Gpts/s of both (interior points x fine steps x propagation passes / time);
asserted: the batched engine is at least 5x the reference's per-shot rate for Born forward +
adjoint, and at least 2x for the single-shot nonlinear forward and the free-surface Born pair.

Workloads: the Born benchmark grid (400x1200 physical, 512x1312 interior) at nts = 500 (the
per-interval cost does not depend on nts), 8 shots; the 200x400 nonlinear forward at its full
size (nts = 1000, one shot).
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
        for rep in range(2):
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
