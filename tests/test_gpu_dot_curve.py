"""Dot-product test error of the FP32 operators as a function of problem size, beside the
reference's own FP32 drivers on the same draws.

The north-star gate for the dot-product test is 1e-6. Here the inner products are exact FP64
products summed on the GPU (aio_dot_f64) and the Born image accumulates in FP64, so what is left
is the round-off of the FP32 propagation itself: forward and adjoint each carry an independent
relative error that grows with the number of fine steps. The reference's definition
(F/include/operator.h:50-88) divides the discrepancy by <m, F* d>, which for random vectors is
itself a random quantity of either sign: the ratio of the two is heavy-tailed, so single draws
range over orders of magnitude. Every size therefore runs 5 draws and reports, per draw,

* rel  = |<F m, d> - <m, F* d>| / |<m, F* d>|           (the reference's measure)
* nrel = |<F m, d> - <m, F* d>| / (||F m|| ||d||)        (norm-relative: no cancellation)

for this engine and, where the reference's FP32 driver of the operator exists (oracle/_ref), for
that driver on the same m and d. One JSON line per size is printed (the committed curve is
assembled from these lines). Gates: nrel <= 1e-6 on every draw (a consistent FP32 adjoint pair
sits near 1e-8 there; a wrong adjoint term would show at 1e-3 or more), and the median rel of
this engine within the reach of the FP32 round-off the reference's own drivers show on the same
draws: at most 5 times their median, or 1e-5.
"""
import json

import numpy as np
import pytest

import orc
import refgpu
from cases import interior_mask, make_case

pytestmark = pytest.mark.gpu
DRAWS = 5


def _errs(lhs, rhs, nfm, nd):
    return abs(lhs - rhs) / abs(rhs), abs(lhs - rhs) / (nfm * nd)


def _cat(xs):
    return np.concatenate([np.asarray(x, np.float32).reshape(-1) for x in xs])


def _born_draw(ctx, s, vel, shots, rng, ref):
    from acoustic_isotropic_operators_b200 import _capi as A
    from acoustic_isotropic_operators_b200.batch import Shot
    m = (rng.standard_normal((s.nx, s.nz)) * interior_mask(s.nx, s.nz)).astype(np.float32)
    d = [rng.standard_normal((len(rp), s.nts)).astype(np.float32) for _, rp, _ in shots]
    fm = _cat(ctx.born_forward(m, [Shot(sp, rp, g) for sp, rp, g in shots]))
    ad = ctx.born_adjoint([Shot(sp, rp, g, x) for (sp, rp, g), x in zip(shots, d)])
    dd = _cat(d)
    ours = _errs(A.dot_f64(fm, dd), A.dot_f64(m, ad), np.linalg.norm(fm.astype(np.float64)),
                 np.linalg.norm(dd.astype(np.float64)))
    theirs = None
    if ref:
        rfm = _cat([refgpu.born_fwd(s, vel, m, g, sp, rp) for sp, rp, g in shots])
        rad = sum(refgpu.born_adj(s, vel, x, g, sp, rp).astype(np.float64) for (sp, rp, g), x in zip(shots, d))
        theirs = _errs(A.dot_f64(rfm, dd), A.dot_f64(m, rad.astype(np.float32)),
                       np.linalg.norm(rfm.astype(np.float64)), np.linalg.norm(dd.astype(np.float64)))
    return ours, theirs


def _nl_draw(ctx, s, vel, shots, rng, ref):
    from acoustic_isotropic_operators_b200 import _capi as A
    from acoustic_isotropic_operators_b200.batch import Shot
    m = [rng.standard_normal((len(sp), s.ntw)).astype(np.float32) for sp, _, _ in shots]
    d = [rng.standard_normal((len(rp), s.nts)).astype(np.float32) for _, rp, _ in shots]
    fm = _cat(ctx.nonlinear_forward([Shot(sp, rp, x) for (sp, rp, _), x in zip(shots, m)]))
    ad = _cat(ctx.nonlinear_adjoint([Shot(sp, rp, None, x) for (sp, rp, _), x in zip(shots, d)]))
    mm, dd = _cat(m), _cat(d)
    ours = _errs(A.dot_f64(fm, dd), A.dot_f64(mm, ad), np.linalg.norm(fm.astype(np.float64)),
                 np.linalg.norm(dd.astype(np.float64)))
    theirs = None
    if ref:
        rfm = _cat([refgpu.nl_fwd(s, vel, x, sp, rp) for (sp, rp, _), x in zip(shots, m)])
        rad = _cat([refgpu.nl_adj(s, vel, x, sp, rp) for (sp, rp, _), x in zip(shots, d)])
        theirs = _errs(A.dot_f64(rfm, dd), A.dot_f64(mm, rad), np.linalg.norm(rfm.astype(np.float64)),
                       np.linalg.norm(dd.astype(np.float64)))
    return ours, theirs


def _small(nts, sub):
    c = make_case(seed=31, nts=nts, sub=sub, nshots=1)
    return c.scheme, c.vel, list(zip(c.src_pos, c.rec_pos, c.sig))


def _born_grid(nts):
    from acoustic_isotropic_operators_b200 import synthetic as S
    w = S.born_workload(nshots=1, nts=nts)
    s = orc.Scheme(nz=w.nz, nx=w.nx, nts=w.nts, dts=w.dts, sub=w.sub, dz=w.dz, dx=w.dx, minPad=w.minPad)
    rng = np.random.default_rng(3)
    a = w.shots[0]
    sig = (rng.standard_normal((len(a.src_pos), s.ntw)) * 1e-2).astype(np.float32)
    return s, w.vel, [(a.src_pos, a.rec_pos, sig)]


def _nl_grid():
    from acoustic_isotropic_operators_b200 import synthetic as S
    w = S.nonlinear_workload()
    s = orc.Scheme(nz=w.nz, nx=w.nx, nts=w.nts, dts=w.dts, sub=w.sub, dz=w.dz, dx=w.dx, minPad=w.minPad)
    a = w.shots[0]
    return s, w.vel, [(a.src_pos, a.rec_pos, None)]


# (label, operator, problem)
SIZES = [
    ("born 48x64 nts=40 sub=3", "born", lambda: _small(40, 3)),
    ("born 48x64 nts=40 sub=4", "born", lambda: _small(40, 4)),
    ("born 48x64 nts=200 sub=4", "born", lambda: _small(200, 4)),
    ("born 512x1312 nts=60", "born", lambda: _born_grid(60)),
    ("born 512x1312 nts=500", "born", lambda: _born_grid(500)),
    ("born 512x1312 nts=2000", "born", lambda: _born_grid(2000)),
    ("nonlinear 48x64 nts=40 sub=4", "nl", lambda: _small(40, 4)),
    ("nonlinear 304x512 nts=1000", "nl", _nl_grid),
]


@pytest.mark.parametrize("label,op,problem", SIZES, ids=[s[0] for s in SIZES])
def test_dot_curve(label, op, problem):
    from acoustic_isotropic_operators_b200.batch import Context
    s, vel, shots = problem()
    k = orc.constants(s, vel, dtype=np.float32)
    ref = refgpu.available("born" if op == "born" else "nl")
    ctx = Context(s.nz, s.nx, s.nts, s.dts, s.sub, s.dz, s.dx, s.minPad, k["v2"], k["rs"], image_fp64=True)
    try:
        rng = np.random.default_rng(17)
        draws = [(_born_draw if op == "born" else _nl_draw)(ctx, s, vel, shots, rng, ref) for _ in range(DRAWS)]
    finally:
        ctx.close()
    ours = np.array([d[0] for d in draws])
    line = {"dot_curve": label, "fine_steps": (s.nts - 1) * s.sub, "interior": [s.nz - 10, s.nx - 10],
            "rel": ours[:, 0].tolist(), "rel_median": float(np.median(ours[:, 0])),
            "nrel_max": float(ours[:, 1].max())}
    if ref:
        theirs = np.array([d[1] for d in draws])
        line.update(ref_rel=theirs[:, 0].tolist(), ref_rel_median=float(np.median(theirs[:, 0])),
                    ref_nrel_max=float(theirs[:, 1].max()))
    print(json.dumps(line))
    assert ours[:, 1].max() <= 1e-6
    bound = max(5 * line["ref_rel_median"], 1e-5) if ref else 1e-5
    assert line["rel_median"] <= bound
