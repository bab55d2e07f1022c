"""Interval-blocked stepper (one launch per coarse interval, sub = 4, 2-D
register tiles) vs the CPU oracle and vs the per-fine-step stepper.

The grid is chosen so the blocked kernel runs several z-strips and x-chunks,
with sources on strip / chunk boundaries (the recomputed halo regions must
inject too). Tolerances: relative L2 1e-5 vs the FP32 oracle for FP32 storage;
BF16 storage of the source wavefield is checked against the FP64 oracle at
1e-2 (8-bit significand) and reported.
"""
import numpy as np
import pytest

import orc
import refgpu
from cases import Case, interior_mask, rel_l2

pytestmark = pytest.mark.gpu


def blocked_case(seed=4, nzi=320, nxi=288, nts=30, nshots=2):
    rng = np.random.default_rng(seed)
    nz, nx = nzi + 10, nxi + 10
    s = orc.Scheme(nz=nz, nx=nx, nts=nts, dts=0.004, sub=4, dz=10.0, dx=10.0, minPad=20)
    zz = np.linspace(0, 1, nz)[None, :]
    vel = (2000.0 + 800.0 * zz + 100.0 * rng.random((nx, nz))).astype(np.float32)
    src_pos, rec_pos, sig = [], [], []
    # strip boundary at interior z = 160, chunk boundaries at multiples of 64 (chunk_columns=64)
    src_pts = [[(5 + 63, 5 + 159), (5 + 64, 5 + 160), (5 + 140, 5 + 12)],
               [(5 + 127, 5 + 161), (5 + 200, 5 + 158), (5 + 30, 5 + 300)]]
    for k in range(nshots):
        sp = np.array([ix * nz + iz for ix, iz in src_pts[k % 2]], np.int32)
        rp = np.array([ix * nz + 5 + 9 for ix in range(5, nx - 5)] +
                      [ix * nz + 5 + 165 for ix in range(5, nx - 5, 3)], np.int32)
        src_pos.append(sp)
        rec_pos.append(rp)
        sig.append((rng.standard_normal((len(sp), s.ntw)) * 1e-2).astype(np.float32))
    return Case(s, vel, src_pos, rec_pos, sig, rng)


@pytest.fixture(scope="module")
def case():
    return blocked_case()


def ctx(case, **kw):
    from acoustic_isotropic_operators_b200.batch import Context
    s = case.scheme
    k = orc.constants(s, case.vel, dtype=np.float32)
    return Context(s.nz, s.nx, s.nts, s.dts, s.sub, s.dz, s.dx, s.minPad, k["v2"], k["rs"], chunk_columns=64, **kw)


def shots(case, data=None):
    from acoustic_isotropic_operators_b200.batch import Shot
    return [Shot(case.src_pos[i], case.rec_pos[i], case.sig[i], None if data is None else data[i])
            for i in range(len(case.src_pos))]


STEPPERS = ["blocked"]


@pytest.mark.parametrize("stepper", STEPPERS)
def test_nonlinear_forward_blocked(case, stepper):
    got = ctx(case, stepper=stepper).nonlinear_forward(shots(case))
    fine = ctx(case, stepper="fine").nonlinear_forward(shots(case))
    for i in range(len(got)):
        r32 = orc.nl_fwd(case.scheme, case.vel, case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32)
        assert rel_l2(got[i], r32) < 1e-5
        assert rel_l2(got[i], fine[i]) < 1e-5


@pytest.mark.parametrize("stepper", STEPPERS)
def test_born_forward_blocked(case, stepper):
    m = case.rng.standard_normal((case.nx, case.nz)).astype(np.float32) * interior_mask(case.nx, case.nz)
    c = ctx(case, stepper=stepper)
    got = c.born_forward(m, shots(case))
    assert c.last_launches == 2 * (case.scheme.nts - 1)
    for i in range(len(got)):
        r32 = orc.born_fwd(case.scheme, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32)
        assert rel_l2(got[i], r32) < 1e-5


@pytest.mark.parametrize("stepper", STEPPERS)
def test_born_adjoint_blocked(case, stepper):
    d = [case.rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
    got = ctx(case, stepper=stepper).born_adjoint(shots(case, d))
    r32 = sum(orc.born_adj(case.scheme, case.vel, d[i], case.sig[i], case.src_pos[i], case.rec_pos[i],
                           dtype=np.float32) for i in range(len(d)))
    assert rel_l2(got, r32) < 1e-5
    assert np.all(got[~interior_mask(case.nx, case.nz)] == 0)


@pytest.mark.parametrize("stepper", STEPPERS)
def test_born_dot_blocked(case, stepper):
    c = ctx(case, stepper=stepper)
    m = case.rng.standard_normal((case.nx, case.nz)).astype(np.float32) * interior_mask(case.nx, case.nz)
    d = [case.rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
    fm = c.born_forward(m, shots(case))
    ad = c.born_adjoint(shots(case, d))
    a = sum(float(np.sum(fm[i].astype(np.float64) * d[i])) for i in range(len(d)))
    b = float(np.sum(m.astype(np.float64) * ad))
    assert abs(a - b) / abs(b) < 1e-5


@pytest.mark.parametrize("stepper", STEPPERS)
def test_born_bf16_error(case, stepper):
    m = case.rng.standard_normal((case.nx, case.nz)).astype(np.float32) * interior_mask(case.nx, case.nz)
    got = ctx(case, stepper=stepper, wavefield="bf16").born_forward(m, shots(case))
    v64 = case.vel.astype(np.float64)
    for i in range(len(got)):
        r64 = orc.born_fwd(case.scheme, v64, m, case.sig[i], case.src_pos[i], case.rec_pos[i])
        assert rel_l2(got[i], r64) < 1e-2
    d = [case.rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
    ga = ctx(case, stepper=stepper, wavefield="bf16").born_adjoint(shots(case, d))
    r64 = sum(orc.born_adj(case.scheme, v64, d[i], case.sig[i], case.src_pos[i], case.rec_pos[i])
              for i in range(len(d)))
    assert rel_l2(ga, r64) < 1e-2


@pytest.mark.parametrize("stepper", STEPPERS)
def test_ragged_grid(stepper):
    """Interior extents that are not multiples of 4, 16 or 32 (last strip / chunk / quad partial)."""
    c = blocked_case(seed=9, nzi=250, nxi=203, nts=24, nshots=1)
    got = ctx(c, stepper=stepper).nonlinear_forward(shots(c))[0]
    r32 = orc.nl_fwd(c.scheme, c.vel, c.sig[0], c.src_pos[0], c.rec_pos[0], dtype=np.float32)
    assert rel_l2(got, r32) < 1e-5
    m = c.rng.standard_normal((c.nx, c.nz)).astype(np.float32) * interior_mask(c.nx, c.nz)
    d = [c.rng.standard_normal((len(c.rec_pos[0]), c.scheme.nts)).astype(np.float32)]
    ga = ctx(c, stepper=stepper).born_adjoint(shots(c, d))
    ra = orc.born_adj(c.scheme, c.vel, d[0], c.sig[0], c.src_pos[0], c.rec_pos[0], dtype=np.float32)
    assert rel_l2(ga, ra) < 1e-5
    gf = ctx(c, stepper=stepper).born_forward(m, shots(c))[0]
    rf = orc.born_fwd(c.scheme, c.vel, m, c.sig[0], c.src_pos[0], c.rec_pos[0], dtype=np.float32)
    assert rel_l2(gf, rf) < 1e-5


def test_born_fp16_dot_and_error(case):
    """FP16 stored wavefield with per-slice scales: the operator stays linear in the model
    (dot test at the FP32 bound) and close to the FP64 oracle."""
    c = ctx(case, stepper="blocked", wavefield="fp16")
    m = case.rng.standard_normal((case.nx, case.nz)).astype(np.float32) * interior_mask(case.nx, case.nz)
    d = [case.rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
    fm = c.born_forward(m, shots(case))
    fm = [x.copy() for x in fm]
    ad = c.born_adjoint(shots(case, d))
    a = sum(float(np.sum(fm[i].astype(np.float64) * d[i])) for i in range(len(d)))
    b = float(np.sum(m.astype(np.float64) * ad))
    assert abs(a - b) / abs(b) < 1e-5
    v64 = case.vel.astype(np.float64)
    for i in range(len(fm)):
        r64 = orc.born_fwd(case.scheme, v64, m, case.sig[i], case.src_pos[i], case.rec_pos[i])
        assert rel_l2(fm[i], r64) < 1e-3


@pytest.mark.parametrize("sloth", [0, 1])
def test_born_ext_adjoint_blocked(case, sloth):
    """Extended (time-lag) Born adjoint with the receiver pass on the blocked stepper: vs the
    FP32 oracle, and the dot test against the extended forward (per-fine-step stepper)."""
    import dataclasses
    s5 = dataclasses.replace(case.scheme, nExt=5)
    from acoustic_isotropic_operators_b200.batch import Context
    k = orc.constants(s5, case.vel, dtype=np.float32)
    c = Context(s5.nz, s5.nx, s5.nts, s5.dts, s5.sub, s5.dz, s5.dx, s5.minPad, k["v2"], k["rs"], nExt=5,
                sloth=sloth, chunk_columns=64)
    d = [case.rng.standard_normal((len(r), s5.nts)).astype(np.float32) for r in case.rec_pos]
    got = c.born_ext_adjoint(shots(case, d))
    assert c.last_launches == 2 * (s5.nts - 1)          # both passes on the blocked stepper (+ the autotuner's)
    ref = sum(orc.bornext_adj(s5, case.vel, d[i], case.sig[i], case.src_pos[i], case.rec_pos[i],
                              dtype=np.float32, sloth=sloth) for i in range(len(d)))
    assert rel_l2(got, ref) < 1e-5
    m = case.rng.standard_normal((5, case.nx, case.nz)).astype(np.float32) * interior_mask(case.nx, case.nz)
    fm = c.born_ext_forward(m, shots(case))
    assert c.last_launches == 2 * (s5.nts - 1)          # forward also on the blocked stepper
    fm = [x.copy() for x in fm]
    for i in range(len(fm)):
        r32 = orc.bornext_fwd(s5, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32,
                              sloth=sloth)
        assert rel_l2(fm[i], r32) < 1e-5
    a = sum(float(np.sum(fm[i].astype(np.float64) * d[i])) for i in range(len(d)))
    b = float(np.sum(m.astype(np.float64) * got))
    assert abs(a - b) / abs(b) < 1e-5


def _ext_ctx(case, n_ext=5, **kw):
    import dataclasses
    from acoustic_isotropic_operators_b200.batch import Context
    s5 = dataclasses.replace(case.scheme, nExt=n_ext)
    k = orc.constants(s5, case.vel, dtype=np.float32)
    return s5, Context(s5.nz, s5.nx, s5.nts, s5.dts, s5.sub, s5.dz, s5.dx, s5.minPad, k["v2"], k["rs"], nExt=n_ext,
                       chunk_columns=64, image_fp64=True, **kw)


def _wshots(case, rdata):
    from acoustic_isotropic_operators_b200.batch import Shot
    return [Shot(case.src_pos[i], case.rec_pos[i], case.sig[i], None, rdata[i]) for i in range(len(case.src_pos))]


@pytest.mark.parametrize("legs,sloth", [((1, 0), 0), ((0, 1), 0), ((1, 1), 0), ((1, 1), 1)])
def test_tomo_blocked(case, legs, sloth):
    """Extended tomo forward / adjoint with every leg on the blocked stepper: vs the FP32 oracle
    (relative L2 1e-5) and the dot test (1e-5). The inputs come from their own seeded generator:
    the relative dot-test error |<Fm,d> - <m,F'd>| / |<m,F'd>| of an FP32 operator depends on the
    draw through the cancellation in <Fm,d>; on this draw the FP32 oracle itself gives 1.4e-6 -
    4.5e-6 and the per-fine-step stepper 1.4e-6 - 2.0e-6."""
    l1, l2 = legs
    s5, c = _ext_ctx(case, leg1=l1, leg2=l2, sloth=sloth)
    rng = np.random.default_rng(3)
    mask = interior_mask(case.nx, case.nz)
    m = rng.standard_normal((case.nx, case.nz)).astype(np.float32) * mask
    ext = rng.standard_normal((5, case.nx, case.nz)).astype(np.float32) * mask
    fm = [x.copy() for x in c.tomo_forward(m, ext, shots(case))]
    assert c.last_launches == (1 + 2 * (l1 + l2)) * (s5.nts - 1)   # source pass + two passes per leg
    for i in range(len(fm)):
        r32 = orc.tomo_fwd(s5, case.vel, m, ext, case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32,
                           sloth=sloth, leg1=l1, leg2=l2)
        assert rel_l2(fm[i], r32) < 1e-5
    d = [rng.standard_normal((len(r), s5.nts)).astype(np.float32) for r in case.rec_pos]
    got = c.tomo_adjoint(ext, shots(case, d))
    assert c.last_launches == (2 + l1 + l2) * (s5.nts - 1)         # source, receiver, one pass per leg
    ref = sum(orc.tomo_adj(s5, case.vel, d[i], ext, case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32,
                           sloth=sloth, leg1=l1, leg2=l2) for i in range(len(d)))
    assert rel_l2(got, ref) < 1e-5
    a = sum(float(np.sum(fm[i].astype(np.float64) * d[i])) for i in range(len(d)))
    b = float(np.sum(m.astype(np.float64) * got))
    assert abs(a - b) / abs(b) < 1e-5


@pytest.mark.parametrize("legs", [(1, 0), (0, 1), (1, 1)])
def test_wemva_blocked(case, legs):
    """Extended WEMVA forward / adjoint with every leg on the blocked stepper: vs the FP32 oracle
    (relative L2 1e-5) and the dot test (1e-5), on inputs from their own seeded generator."""
    l1, l2 = legs
    s5, c = _ext_ctx(case, leg1=l1, leg2=l2)
    rng = np.random.default_rng(3)
    mask = interior_mask(case.nx, case.nz)
    m = rng.standard_normal((case.nx, case.nz)).astype(np.float32) * mask
    img = rng.standard_normal((5, case.nx, case.nz)).astype(np.float32) * mask
    rd = [rng.standard_normal((len(r), s5.nts)).astype(np.float32) for r in case.rec_pos]
    fimg = c.wemva_forward(m, _wshots(case, rd)).copy()
    assert c.last_launches == (2 + l1 + l2) * (s5.nts - 1)
    ref = sum(orc.wemva_fwd(s5, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i], rd[i], dtype=np.float32,
                            leg1=l1, leg2=l2) for i in range(len(rd)))
    assert rel_l2(fimg, ref) < 1e-5
    got = c.wemva_adjoint(img, _wshots(case, rd))
    assert c.last_launches == (2 + l1 + l2) * (s5.nts - 1)
    ref = sum(orc.wemva_adj(s5, case.vel, img, case.sig[i], case.src_pos[i], case.rec_pos[i], rd[i],
                            dtype=np.float32, leg1=l1, leg2=l2) for i in range(len(rd)))
    assert rel_l2(got, ref) < 1e-5
    a = float(np.sum(fimg.astype(np.float64) * img))
    b = float(np.sum(m.astype(np.float64) * got))
    assert abs(a - b) / abs(b) < 1e-5


def test_short_strip_variant():
    """Interiors of at most 64 rows run the short-strip kernel variant (narrower rings, two CTAs
    per SM): nonlinear forward and Born forward / adjoint against the FP32 oracle."""
    c = blocked_case(seed=12, nzi=56, nxi=150, nts=26, nshots=1)
    c.src_pos[0] = np.array([(5 + 40) * c.nz + 5 + 20, (5 + 90) * c.nz + 5 + 50], np.int32)
    c.sig[0] = (c.rng.standard_normal((2, c.scheme.ntw)) * 1e-2).astype(np.float32)
    c.rec_pos[0] = np.array([ix * c.nz + 5 + 9 for ix in range(5, c.nx - 5)], np.int32)
    got = ctx(c, stepper="blocked").nonlinear_forward(shots(c))[0]
    r32 = orc.nl_fwd(c.scheme, c.vel, c.sig[0], c.src_pos[0], c.rec_pos[0], dtype=np.float32)
    assert rel_l2(got, r32) < 1e-5
    m = c.rng.standard_normal((c.nx, c.nz)).astype(np.float32) * interior_mask(c.nx, c.nz)
    gf = ctx(c, stepper="blocked").born_forward(m, shots(c))[0]
    assert rel_l2(gf, orc.born_fwd(c.scheme, c.vel, m, c.sig[0], c.src_pos[0], c.rec_pos[0], dtype=np.float32)) < 1e-5
    d = [c.rng.standard_normal((len(c.rec_pos[0]), c.scheme.nts)).astype(np.float32)]
    ga = ctx(c, stepper="blocked").born_adjoint(shots(c, d))
    assert rel_l2(ga, orc.born_adj(c.scheme, c.vel, d[0], c.sig[0], c.src_pos[0], c.rec_pos[0], dtype=np.float32)) < 1e-5


def _strip_case(nzi, seed):
    c = blocked_case(seed=seed, nzi=nzi, nxi=150, nts=26, nshots=2)
    c.src_pos[0] = np.array([(5 + 40) * c.nz + 5 + 20, (5 + 90) * c.nz + 5 + nzi - 8], np.int32)
    c.src_pos[1] = np.array([(5 + 70) * c.nz + 5 + nzi // 2], np.int32)
    for i in range(2):
        c.sig[i] = (c.rng.standard_normal((len(c.src_pos[i]), c.scheme.ntw)) * 1e-2).astype(np.float32)
        c.rec_pos[i] = np.array([ix * c.nz + 5 + 9 for ix in range(5, c.nx - 5)], np.int32)
    return c


@pytest.mark.parametrize("nzi", [72, 80])
def test_mid_strip_variant(nzi):
    """Interiors of 65 to 80 rows run the mid-strip kernel variant (two CTAs per SM, v^2 of the
    first level read through L1): every kind of blocked pass — nonlinear, Born forward / adjoint,
    extended Born forward / adjoint, tomo and WEMVA with both legs — against the FP32 oracle
    (relative L2 1e-5)."""
    c = _strip_case(nzi, seed=13)
    s = c.scheme
    got = ctx(c, stepper="blocked").nonlinear_forward(shots(c))
    for i in range(2):
        r32 = orc.nl_fwd(s, c.vel, c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)
        assert rel_l2(got[i], r32) < 1e-5
    mask = interior_mask(c.nx, c.nz)
    rng = np.random.default_rng(5)
    m = (rng.standard_normal((c.nx, c.nz)) * mask).astype(np.float32)
    gf = [x.copy() for x in ctx(c, stepper="blocked").born_forward(m, shots(c))]
    for i in range(2):
        assert rel_l2(gf[i], orc.born_fwd(s, c.vel, m, c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)) < 1e-5
    d = [rng.standard_normal((len(r), s.nts)).astype(np.float32) for r in c.rec_pos]
    ga = ctx(c, stepper="blocked").born_adjoint(shots(c, d))
    ref = sum(orc.born_adj(s, c.vel, d[i], c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32) for i in range(2))
    assert rel_l2(ga, ref) < 1e-5
    s5, e = _ext_ctx(c)
    ext = (rng.standard_normal((5, c.nx, c.nz)) * mask).astype(np.float32)
    fe = [x.copy() for x in e.born_ext_forward(ext, shots(c))]
    assert e.last_launches == 2 * (s5.nts - 1)
    for i in range(2):
        r32 = orc.bornext_fwd(s5, c.vel, ext, c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)
        assert rel_l2(fe[i], r32) < 1e-5
    ae = e.born_ext_adjoint(shots(c, d))
    ref = sum(orc.bornext_adj(s5, c.vel, d[i], c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)
              for i in range(2))
    assert rel_l2(ae, ref) < 1e-5
    s5, t = _ext_ctx(c, leg1=1, leg2=1)
    ft = [x.copy() for x in t.tomo_forward(m, ext, shots(c))]
    assert t.last_launches == 5 * (s5.nts - 1)
    for i in range(2):
        r32 = orc.tomo_fwd(s5, c.vel, m, ext, c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)
        assert rel_l2(ft[i], r32) < 1e-5
    at = t.tomo_adjoint(ext, shots(c, d))
    ref = sum(orc.tomo_adj(s5, c.vel, d[i], ext, c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)
              for i in range(2))
    assert rel_l2(at, ref) < 1e-5
    fw = t.wemva_forward(m, _wshots(c, d)).copy()
    ref = sum(orc.wemva_fwd(s5, c.vel, m, c.sig[i], c.src_pos[i], c.rec_pos[i], d[i], dtype=np.float32)
              for i in range(2))
    assert rel_l2(fw, ref) < 1e-5
    aw = t.wemva_adjoint(ext, _wshots(c, d))
    ref = sum(orc.wemva_adj(s5, c.vel, ext, c.sig[i], c.src_pos[i], c.rec_pos[i], d[i], dtype=np.float32)
              for i in range(2))
    assert rel_l2(aw, ref) < 1e-5


@pytest.mark.parametrize("n_ext", [5, 31])
def test_born_ext_offset_adjoint_blocked(case, n_ext):
    """Extended Born forward and adjoint with subsurface offsets on the blocked stepper (SCATX pass
    fed by per-sample offset sources; ADJR receiver pass with offset imaging in blocks of 32 coarse
    samples): vs the FP32 oracle (1e-5), and the dot test."""
    import dataclasses
    from acoustic_isotropic_operators_b200.batch import Context
    s = dataclasses.replace(case.scheme, nExt=n_ext, extension=1)
    k = orc.constants(s, case.vel, dtype=np.float32)
    c = Context(s.nz, s.nx, s.nts, s.dts, s.sub, s.dz, s.dx, s.minPad, k["v2"], k["rs"], nExt=n_ext,
                extension="offset", image_fp64=True, chunk_columns=64)
    rng = np.random.default_rng(31)
    d = [rng.standard_normal((len(r), s.nts)).astype(np.float32) for r in case.rec_pos]
    got = c.born_ext_adjoint(shots(case, d))
    assert c.last_launches == 2 * (s.nts - 1)          # both passes on the blocked stepper
    ref = sum(orc.bornext_adj(s, case.vel, d[i], case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32)
              for i in range(len(d)))
    assert rel_l2(got, ref) < 1e-5
    m = (rng.standard_normal((n_ext, case.nx, case.nz)) * interior_mask(case.nx, case.nz)).astype(np.float32)
    fm = [x.copy() for x in c.born_ext_forward(m, shots(case))]
    assert c.last_launches == 2 * (s.nts - 1)          # forward on the blocked stepper too
    r32 = [orc.bornext_fwd(s, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32)
           for i in range(len(fm))]
    for i in range(len(fm)):
        assert rel_l2(fm[i], r32[i]) < 1e-5
    a = sum(float(np.sum(fm[i].astype(np.float64) * d[i])) for i in range(len(d)))
    b = float(np.sum(m.astype(np.float64) * got))
    a32 = sum(float(np.sum(r32[i].astype(np.float64) * d[i])) for i in range(len(d)))
    b32 = float(np.sum(m.astype(np.float64) * ref))
    assert abs(a - b) / abs(b) < max(1e-5, 2 * abs(a32 - b32) / abs(b32))


def _fs_case():
    import dataclasses
    c = blocked_case(seed=21, nts=40)
    c.scheme = dataclasses.replace(c.scheme, freeSurface=1)
    # a source 3 rows below the surface in each shot: the surface reflection reaches the receivers
    for i in range(len(c.src_pos)):
        c.src_pos[i] = np.concatenate([c.src_pos[i], np.array([(5 + 100 + 50 * i) * c.nz + 5 + 3], np.int32)])
        c.sig[i] = (c.rng.standard_normal((len(c.src_pos[i]), c.scheme.ntw)) * 1e-2).astype(np.float32)
    return c


def test_free_surface_blocked():
    """Free surface on the blocked stepper (forward modes: the top row zeroed and the rows above it
    mirrored; adjoint modes: stepAdjFsGpu's corrections, in U-form): nonlinear forward / adjoint,
    Born forward / adjoint, extended (time-lag) Born forward / adjoint and tomo with both legs
    against the FP32 oracle with the free surface (relative L2 1e-5), one launch per interval and
    pass, and the Born dot test."""
    from acoustic_isotropic_operators_b200.batch import Shot
    c = _fs_case()
    s = c.scheme
    k = lambda **kw: ctx(c, free_surface=1, **kw)  # noqa: E731
    nl = k().nonlinear_forward(shots(c))
    for i in range(2):
        r32 = orc.nl_fwd(s, c.vel, c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)
        assert rel_l2(nl[i], r32) < 1e-5
    plain = ctx(c).nonlinear_forward(shots(c))[0]
    assert rel_l2(plain, nl[0]) > 1e-3                   # the surface changes the answer
    rng = np.random.default_rng(22)
    d = [rng.standard_normal((len(r), s.nts)).astype(np.float32) for r in c.rec_pos]
    na = k().nonlinear_adjoint([Shot(c.src_pos[i], c.rec_pos[i], None, d[i]) for i in range(2)])
    for i in range(2):
        assert rel_l2(na[i], orc.nl_adj(s, c.vel, d[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)) < 1e-5
    mask = interior_mask(c.nx, c.nz)
    m = (rng.standard_normal((c.nx, c.nz)) * mask).astype(np.float32)
    b = k(image_fp64=True)
    fm = [x.copy() for x in b.born_forward(m, shots(c))]
    assert b.last_launches == 2 * (s.nts - 1)
    for i in range(2):
        assert rel_l2(fm[i], orc.born_fwd(s, c.vel, m, c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)) < 1e-5
    ad = b.born_adjoint(shots(c, d))
    assert b.last_launches == 2 * (s.nts - 1)
    ref = sum(orc.born_adj(s, c.vel, d[i], c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32) for i in range(2))
    assert rel_l2(ad, ref) < 1e-5
    a_ = sum(float(np.sum(fm[i].astype(np.float64) * d[i])) for i in range(2))
    b_ = float(np.sum(m.astype(np.float64) * ad))
    assert abs(a_ - b_) / abs(b_) < 1e-5
    s5, e = _ext_ctx(c, free_surface=1)
    ext = (rng.standard_normal((5, c.nx, c.nz)) * mask).astype(np.float32)
    fe = [x.copy() for x in e.born_ext_forward(ext, shots(c))]
    assert e.last_launches == 2 * (s5.nts - 1)
    for i in range(2):
        assert rel_l2(fe[i], orc.bornext_fwd(s5, c.vel, ext, c.sig[i], c.src_pos[i], c.rec_pos[i],
                                             dtype=np.float32)) < 1e-5
    ae = e.born_ext_adjoint(shots(c, d))
    ref = sum(orc.bornext_adj(s5, c.vel, d[i], c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)
              for i in range(2))
    assert rel_l2(ae, ref) < 1e-5
    s5, t = _ext_ctx(c, free_surface=1, leg1=1, leg2=1)
    ft = [x.copy() for x in t.tomo_forward(m, ext, shots(c))]
    assert t.last_launches == 5 * (s5.nts - 1)
    for i in range(2):
        assert rel_l2(ft[i], orc.tomo_fwd(s5, c.vel, m, ext, c.sig[i], c.src_pos[i], c.rec_pos[i],
                                          dtype=np.float32)) < 1e-5
    at = t.tomo_adjoint(ext, shots(c, d))
    ref = sum(orc.tomo_adj(s5, c.vel, d[i], ext, c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)
              for i in range(2))
    assert rel_l2(at, ref) < 1e-5


@pytest.mark.skipif(not refgpu.available("born"), reason="oracle/_ref not built (make -C oracle ref)")
def test_free_surface_blocked_vs_reference_drivers():
    """Blocked stepper with the free surface against the reference's own free-surface drivers
    (nonlinear forward, Born forward / adjoint; one shot)."""
    from acoustic_isotropic_operators_b200.batch import Shot
    c = _fs_case()
    s = c.scheme
    sp, rp, sig = c.src_pos[0], c.rec_pos[0], c.sig[0]
    one = [Shot(sp, rp, sig)]
    b = ctx(c, free_surface=1, image_fp64=True)
    assert rel_l2(b.nonlinear_forward(one)[0], refgpu.nl_fwd(s, c.vel, sig, sp, rp)) < 1e-5
    m = (np.random.default_rng(23).standard_normal((c.nx, c.nz)) * interior_mask(c.nx, c.nz)).astype(np.float32)
    assert rel_l2(b.born_forward(m, one)[0], refgpu.born_fwd(s, c.vel, m, sig, sp, rp)) < 1e-5
    d = (np.random.default_rng(24).standard_normal((len(rp), s.nts)) * 1e-2).astype(np.float32)
    assert rel_l2(b.born_adjoint([Shot(sp, rp, sig, d)]), refgpu.born_adj(s, c.vel, d, sig, sp, rp)) < 1e-5
