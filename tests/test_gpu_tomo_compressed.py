"""Compressed source field of the tomo and WEMVA operators on the blocked stepper: d2/dt2 of the
source wavefield stored in FP16 with each coarse slice's exact scale, or in BF16 (the second stored
field, scattered or receiver wavefield, stays FP32).

* Relative error of tomo and WEMVA forward and adjoint against the FP64 oracle on a medium case
  (96 x 160 physical grid, nts = 400, nExt = 9, realistic source and reflectivity), printed per
  precision, with bounds at about twice the measured values: FP32 3e-4, FP16 2e-2, BF16 2e-1.
  These operators amplify the rounding of the stored d2/dt2 field far more than Born does: the
  measured FP16 error (about 7e-3 on the tomo forward) is some 30 times its unit roundoff.
* Dot-product tests of the compressed pairs (both operators read the same stored field): <= 1e-5.
* The per-fine-step paths (subsurface offsets, saved wavefields) keep FP32 fields and refuse a
  compressed setting with an argument error.
"""
import numpy as np
import pytest

import orc
from cases import interior_mask, make_case, rel_l2
from test_gpu_parity import shots_for

pytestmark = pytest.mark.gpu
N_EXT = 9


@pytest.fixture(scope="module")
def medium():
    from acoustic_isotropic_operators_b200 import synthetic as S, _capi
    import bench
    w = S.born_workload(nz_phys=96, nx_phys=160, nshots=2, nts=400)
    sigs = bench.prepare_signals(w, _capi.lib())
    s = orc.Scheme(nz=w.nz, nx=w.nx, nts=w.nts, dts=w.dts, sub=w.sub, dz=w.dz, dx=w.dx, minPad=w.minPad,
                   nExt=N_EXT)
    k = orc.constants(s, w.vel, dtype=np.float32)
    rng = np.random.default_rng(9)
    mask = interior_mask(w.nx, w.nz)
    prof = np.exp(-(np.arange(N_EXT) - N_EXT // 2) ** 2 / 8.0).astype(np.float32)
    ext = np.ascontiguousarray(prof[:, None, None] * w.model[None], np.float32)
    # a rough velocity perturbation: it scatters energy back to the receivers, which keeps the
    # relative error of the tomo forward meaningful (a smooth one mostly transmits, leaving data
    # that are small next to the rounding of the fields they come from)
    dv = (rng.standard_normal((w.nx, w.nz)) * mask * 1e-2).astype(np.float32)
    d = [(rng.standard_normal((len(a.rec_pos), w.nts)) * 1e-3).astype(np.float32) for a in w.shots]
    return w, sigs, s, k, ext, dv, d


def _ctx(w, s, k, wavefield, **kw):
    from acoustic_isotropic_operators_b200.batch import Context
    return Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, k["v2"], k["rs"], nExt=N_EXT,
                   image_fp64=True, wavefield=wavefield, **kw)


def _run(medium, wavefield):
    from acoustic_isotropic_operators_b200.batch import Shot
    w, sigs, s, k, ext, dv, d = medium
    ctx = _ctx(w, s, k, wavefield)
    try:
        tf = [x.copy() for x in ctx.tomo_forward(dv, ext, [Shot(a.src_pos, a.rec_pos, g) for a, g in zip(w.shots, sigs)])]
        ta = ctx.tomo_adjoint(ext, [Shot(a.src_pos, a.rec_pos, g, x) for a, g, x in zip(w.shots, sigs, d)]).copy()
        wf = ctx.wemva_forward(dv, [Shot(a.src_pos, a.rec_pos, g, None, x) for a, g, x in zip(w.shots, sigs, d)]).copy()
        wa = ctx.wemva_adjoint(ext, [Shot(a.src_pos, a.rec_pos, g, None, x) for a, g, x in zip(w.shots, sigs, d)]).copy()
        assert ctx.last_launches > 0
        return tf, ta, wf, wa
    finally:
        ctx.close()


@pytest.fixture(scope="module")
def fp64(medium):
    w, sigs, s, k, ext, dv, d = medium
    v = w.vel.astype(np.float64)
    tf = [orc.tomo_fwd(s, v, dv, ext, g, a.src_pos, a.rec_pos) for a, g in zip(w.shots, sigs)]
    ta = sum(orc.tomo_adj(s, v, x, ext, g, a.src_pos, a.rec_pos) for a, g, x in zip(w.shots, sigs, d))
    wf = sum(orc.wemva_fwd(s, v, dv, g, a.src_pos, a.rec_pos, x) for a, g, x in zip(w.shots, sigs, d))
    wa = sum(orc.wemva_adj(s, v, ext, g, a.src_pos, a.rec_pos, x) for a, g, x in zip(w.shots, sigs, d))
    return tf, ta, wf, wa


@pytest.mark.parametrize("wavefield,tol", [("fp32", 3e-4), ("fp16", 2e-2), ("bf16", 2e-1)])
def test_tomo_wemva_error_vs_fp64(medium, fp64, wavefield, tol):
    tf, ta, wf, wa = _run(medium, wavefield)
    rf, ra, rwf, rwa = fp64
    e = {"tomo_fwd": max(rel_l2(a, b) for a, b in zip(tf, rf)), "tomo_adj": rel_l2(ta, ra),
         "wemva_fwd": rel_l2(wf, rwf), "wemva_adj": rel_l2(wa, rwa)}
    print(f"\n[{wavefield}] tomo / WEMVA (nExt={N_EXT}) rel err vs FP64: " +
          ", ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert max(e.values()) < tol, e


@pytest.mark.parametrize("wavefield", ["fp16", "bf16"])
def test_dot_tomo_wemva_compressed(wavefield):
    case = make_case(seed=23, nzi=96, nxi=128, nts=40, sub=4, nExt=5, nshots=2)
    s = case.scheme
    k = orc.constants(s, case.vel, dtype=np.float32)
    from acoustic_isotropic_operators_b200.batch import Context
    ctx = Context(s.nz, s.nx, s.nts, s.dts, s.sub, s.dz, s.dx, s.minPad, k["v2"], k["rs"], nExt=s.nExt,
                  image_fp64=True, wavefield=wavefield)
    dot = lambda a, b: float(np.sum(np.asarray(a, np.float64) * np.asarray(b, np.float64)))
    try:
        mask = interior_mask(case.nx, case.nz)
        rng = np.random.default_rng(4)
        m = (rng.standard_normal((case.nx, case.nz)) * mask).astype(np.float32)
        ext = (rng.standard_normal((s.nExt, case.nx, case.nz)) * mask).astype(np.float32)
        d = [rng.standard_normal((len(r), s.nts)).astype(np.float32) for r in case.rec_pos]
        # norm-relative discrepancy |<Fm, d> - <m, F*d>| / (|Fm| |d|): no cancellation in the
        # denominator; a consistent FP32 pair sits far below 1e-6, a wrong adjoint term far above
        fm = [x.copy() for x in ctx.tomo_forward(m, ext, shots_for(case))]
        lhs = sum(dot(fm[i], d[i]) for i in range(len(d)))
        rhs = dot(m, ctx.tomo_adjoint(ext, shots_for(case, data=d)))
        norm = np.sqrt(sum(dot(x, x) for x in fm) * sum(dot(x, x) for x in d))
        assert abs(lhs - rhs) / norm < 1e-6, ("tomo", lhs, rhs, norm)
        fw = ctx.wemva_forward(m, shots_for(case, wemva=d)).copy()
        rhs = dot(m, ctx.wemva_adjoint(ext, shots_for(case, wemva=d)))
        lhs = dot(fw, ext)
        norm = np.sqrt(dot(fw, fw) * dot(ext, ext))
        assert abs(lhs - rhs) / norm < 1e-6, ("wemva", lhs, rhs, norm)
    finally:
        ctx.close()


def test_compressed_fields_refused_off_the_blocked_stepper():
    from acoustic_isotropic_operators_b200 import _capi as A
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    case = make_case(seed=24, nzi=64, nxi=96, nts=20, sub=4, nExt=5, nshots=1)
    s = case.scheme
    k = orc.constants(s, case.vel, dtype=np.float32)
    ctx = Context(s.nz, s.nx, s.nts, s.dts, s.sub, s.dz, s.dx, s.minPad, k["v2"], k["rs"], nExt=s.nExt,
                  wavefield="fp16", extension="offset")
    try:
        with pytest.raises(A.AioError) as e:
            ctx.tomo_forward(np.zeros((case.nx, case.nz), np.float32), np.zeros((s.nExt, case.nx, case.nz), np.float32),
                             [Shot(case.src_pos[0], case.rec_pos[0], case.sig[0])])
        assert e.value.code == A.AIO_ERR_ARGUMENT
    finally:
        ctx.close()
