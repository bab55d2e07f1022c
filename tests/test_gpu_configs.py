"""Parity at the benchmark configurations, on the code paths the benchmark times.

* Nonlinear forward at its full size: 200x400 physical grid with Gaussian blobs (304x512
  interior, 314x522 padded), nts = 1000, sub = 4, one source at x = 2000 m, 400 receivers.
  Host preparation through the product's own C ABI (aio_fd_precompute, aio_prepare_source), the
  blocked stepper through the batched API. Gates (relative L2 over the recorded data): <= 1e-5
  against the FP32 oracle, <= 1e-4 against the FP64 oracle (the scheme of acoustic_iso_double),
  <= 1e-5 against the reference's own FP32 driver built for sm_100a (propShotsFwdGpu,
  F/src/nonlinearShotsGpuFunctions.cu:227-309).
* Born forward and adjoint on the 400x1200 grid (512x1312 interior, 522x1322 padded) with the
  benchmark's plan: 32 shots in one wave, no forced chunk width (the autotuned strip / chunk
  plan the benchmark runs), FP32 stored wavefield, FP64 image, nts shortened to 60 so that the
  oracle finishes in seconds. The perturbation adds 200 seeded point scatterers in the top 25
  rows to the benchmark's interfaces, so that every shot records backscattered energy within the
  window: the interfaces alone lie deeper than the 0.24 s of this window reaches, which leaves
  some shots' data zero or a faint onset, and a smooth dense perturbation scatters mostly
  forward, leaving a small residual at the receivers; a relative error of such data measures
  its conditioning, not the code. Gates: forward data of 8 of the 32
  shots and the adjoint image of a wave whose data is non-zero on those 8 shots, <= 1e-5 against
  the FP32 oracle; the dot-product test of the 32-shot pair with FP64 inner products reduced on
  the GPU (aio_dot_f64) <= 1e-5.
"""
import ctypes as C

import numpy as np
import pytest

import orc
import refgpu
from cases import rel_l2

pytestmark = pytest.mark.gpu


def _prep(w, second_derivative):
    """v^2 dtw^2, 2/v^3 and every shot's fine source traces from the product's host code."""
    from acoustic_isotropic_operators_b200 import _capi as A
    lib = A.lib()
    velf = np.ascontiguousarray(w.vel.reshape(-1), np.float32)
    v2 = np.zeros(w.nz * w.nx, np.float32)
    rs = np.zeros_like(v2)
    A.check(lib.aio_fd_precompute(w.nz, w.nx, C.c_float(w.dts), w.sub, A.fptr(velf), A.fptr(v2), A.fptr(rs)))
    sigs = []
    for a in w.shots:
        wav = np.ascontiguousarray(np.repeat(w.wavelet[None, :], a.src_cidx.shape[0], axis=0), np.float32)
        out = np.zeros((len(a.src_pos), w.ntw), np.float32)
        A.check(lib.aio_prepare_source(second_derivative, a.src_cidx.shape[0], a.src_cidx.shape[1],
                                       A.iptr(a.src_cidx), A.fptr(a.src_w), len(a.src_pos), A.iptr(a.src_pos),
                                       w.nts, C.c_float(w.dts), w.sub, A.fptr(velf), A.fptr(wav), A.fptr(out)))
        sigs.append(out)
    return v2, rs, sigs


def _scheme(w):
    return orc.Scheme(nz=w.nz, nx=w.nx, nts=w.nts, dts=w.dts, sub=w.sub, dz=w.dz, dx=w.dx, minPad=w.minPad)


def test_nonlinear_forward_full_size():
    from acoustic_isotropic_operators_b200 import synthetic as S
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    w = S.nonlinear_workload()
    assert (w.nz, w.nx, w.nts, w.sub) == (314, 522, 1000, 4)
    v2, rs, sigs = _prep(w, 0)
    a = w.shots[0]
    assert a.rec_cidx.shape[0] == 400  # 400 receivers (their 4 corners give the regular traces)
    ctx = Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs)
    try:
        got = ctx.nonlinear_forward([Shot(a.src_pos, a.rec_pos, sigs[0])])[0].copy()
        launches = ctx.last_launches
    finally:
        ctx.close()
    assert launches == w.nts - 1  # one blocked launch per coarse interval
    s = _scheme(w)
    r32 = orc.nl_fwd(s, w.vel, sigs[0], a.src_pos, a.rec_pos, dtype=np.float32)
    r64 = orc.nl_fwd(s, w.vel.astype(np.float64), sigs[0].astype(np.float64), a.src_pos, a.rec_pos,
                     dtype=np.float64)
    e32, e64 = rel_l2(got, r32), rel_l2(got, r64)
    msg = f"vs FP32 oracle {e32:.2e}, vs FP64 oracle {e64:.2e}"
    if refgpu.available("nl"):
        eref = rel_l2(got, refgpu.nl_fwd(s, w.vel, sigs[0], a.src_pos, a.rec_pos))
        msg += f", vs reference FP32 driver {eref:.2e}"
        assert eref < 1e-5, msg
    print("nonlinear forward 314x522 nts=1000:", msg)
    assert e32 < 1e-5, msg
    assert e64 < 1e-4, msg


CHECKED = [0, 5, 10, 15, 16, 21, 26, 31]  # shots compared with the oracle (strip / chunk positions vary)


@pytest.fixture(scope="module")
def born32():
    from acoustic_isotropic_operators_b200 import synthetic as S
    w = S.born_workload(nshots=32, nts=60)
    assert (w.nz, w.nx, w.sub) == (522, 1322, 4)
    v2, rs, sigs = _prep(w, 1)
    return w, v2, rs, sigs


def _ctx(w, v2, rs, image_fp64=True):
    from acoustic_isotropic_operators_b200.batch import Context
    return Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, v2, rs, image_fp64=image_fp64)


def test_born_benchmark_plan(born32):
    from acoustic_isotropic_operators_b200 import _capi as A
    from acoustic_isotropic_operators_b200.batch import Shot
    w, v2, rs, sigs = born32
    ctx = _ctx(w, v2, rs)
    try:
        assert ctx.capacity(A.AIO_BORN) >= 32  # one wave
        # the benchmark's interfaces plus 200 point scatterers in the top 25 rows of the physical
        # area, which send energy back to the receivers within the shortened window
        rng = np.random.default_rng(20)
        model = np.array(w.model, np.float32)
        z0, x0 = 5 + w.pad.zPadMinus, 5 + w.pad.xPadMinus
        for _ in range(200):
            model[x0 + rng.integers(0, w.pad.nx_phys), z0 + rng.integers(0, 25)] += rng.uniform(-1, 1)
        shots = [Shot(a.src_pos, a.rec_pos, g) for a, g in zip(w.shots, sigs)]
        data = [d.copy() for d in ctx.born_forward(model, shots)]
        plan = ctx.blocked_plan(32)
        assert ctx.last_launches == 2 * (w.nts - 1)  # source + scattered pass, one launch per interval
        s = _scheme(w)
        errs = []
        for i in CHECKED:
            a = w.shots[i]
            r = orc.born_fwd(s, w.vel, model, sigs[i], a.src_pos, a.rec_pos, dtype=np.float32)
            errs.append(rel_l2(data[i], r))
        print("Born forward 522x1322 nts=60, 32 shots, plan", plan, "max rel err", max(errs))
        assert max(errs) < 1e-5, errs
        rng = np.random.default_rng(21)
        adj_data = [np.zeros((len(a.rec_pos), w.nts), np.float32) for a in w.shots]
        for i in CHECKED:
            adj_data[i] = (rng.standard_normal(adj_data[i].shape) * 1e-3).astype(np.float32)
        img = ctx.born_adjoint([Shot(a.src_pos, a.rec_pos, g, d) for a, g, d in zip(w.shots, sigs, adj_data)])
        ref = np.zeros((w.nx, w.nz), np.float64)
        for i in CHECKED:
            a = w.shots[i]
            ref += orc.born_adj(s, w.vel, adj_data[i], sigs[i], a.src_pos, a.rec_pos, dtype=np.float32)
        e = rel_l2(img, ref)
        print("Born adjoint 522x1322 nts=60, 32-shot wave, rel err", e)
        assert e < 1e-5
    finally:
        ctx.close()


@pytest.mark.parametrize("image_fp64", [True, False])
def test_born_benchmark_dot(born32, image_fp64):
    """Dot-product test of the benchmark's Born pair, with the image accumulated in FP64 and in
    FP32 (the reference's accumulation)."""
    from acoustic_isotropic_operators_b200 import _capi as A
    from acoustic_isotropic_operators_b200.batch import Shot
    w, v2, rs, sigs = born32
    ctx = _ctx(w, v2, rs, image_fp64)
    try:
        rng = np.random.default_rng(22)
        m = np.zeros((w.nx, w.nz), np.float32)
        m[5:-5, 5:-5] = rng.standard_normal((w.nx - 10, w.nz - 10))
        d = [rng.standard_normal((len(a.rec_pos), w.nts)).astype(np.float32) for a in w.shots]
        fm = ctx.born_forward(m, [Shot(a.src_pos, a.rec_pos, g) for a, g in zip(w.shots, sigs)])
        fm = np.concatenate([x.reshape(-1) for x in fm])
        ad = ctx.born_adjoint([Shot(a.src_pos, a.rec_pos, g, x) for a, g, x in zip(w.shots, sigs, d)])
        lhs = A.dot_f64(fm, np.concatenate([x.reshape(-1) for x in d]))
        rhs = A.dot_f64(m, ad)
        err = abs(lhs - rhs) / abs(rhs)
        print(f"Born dot test 522x1322 nts=60, 32 shots, FP{64 if image_fp64 else 32} image: "
              f"<Fm,d>={lhs:.10e} <m,F*d>={rhs:.10e} rel {err:.2e}")
        assert err < 1e-5
    finally:
        ctx.close()
