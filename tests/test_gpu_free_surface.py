"""Free surface (the reference's freeSurface = 1 drivers, *FsGpu) on the CUDA path.

The top interior row is a pressure-free surface: forward steps see the current
level with that row zeroed and the rows above it mirrored with opposite sign
(setFsConditionFwdGpu), adjoint steps use stepAdjFsGpu, the taper ignores the
top edge (dampCosineEdgeFs). Gates (relative L2): CUDA vs the FP32 oracle with
the free surface 1e-5, vs the FP64 oracle 1e-4, vs the reference's own
free-surface drivers (oracle/_ref) 1e-5; dot tests 1e-5.
"""
import dataclasses

import numpy as np
import pytest

import orc
import refgpu
from cases import interior_mask, make_case, rel_l2
from test_gpu_parity import ctx_for, shots_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    c = make_case(seed=5, nts=40)
    c.scheme = dataclasses.replace(c.scheme, freeSurface=1)
    return c


def _dot(a, b):
    return float(np.sum(np.asarray(a, np.float64) * np.asarray(b, np.float64)))


def _data(case, rng):
    return [rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]


def test_nonlinear_fs(case):
    ctx = ctx_for(case, free_surface=1)
    s = case.scheme
    got = [x.copy() for x in ctx.nonlinear_forward(shots_for(case))]
    for i in range(len(got)):
        assert rel_l2(got[i], orc.nl_fwd(s, case.vel, case.sig[i], case.src_pos[i], case.rec_pos[i],
                                         dtype=np.float32)) < 1e-5
        assert rel_l2(got[i], orc.nl_fwd(s, case.vel.astype(np.float64), case.sig[i], case.src_pos[i],
                                         case.rec_pos[i], dtype=np.float64)) < 1e-4
    # the surface changes the answer: the plain operator differs
    plain = ctx_for(case).nonlinear_forward(shots_for(case))[0]
    assert rel_l2(plain, got[0]) > 1e-3
    rng = np.random.default_rng(2)
    d = _data(case, rng)
    from acoustic_isotropic_operators_b200.batch import Shot
    ad = ctx.nonlinear_adjoint([Shot(case.src_pos[i], case.rec_pos[i], None, d[i]) for i in range(len(d))])
    for i in range(len(d)):
        assert rel_l2(ad[i], orc.nl_adj(s, case.vel, d[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32)) < 1e-5
    m = [rng.standard_normal(x.shape).astype(np.float32) for x in case.sig]
    fm = ctx.nonlinear_forward([Shot(case.src_pos[i], case.rec_pos[i], m[i]) for i in range(len(m))])
    a = sum(_dot(fm[i], d[i]) for i in range(len(d)))
    b = sum(_dot(m[i], ad[i]) for i in range(len(d)))
    assert abs(a - b) / abs(b) < 1e-5


def test_born_fs(case):
    ctx = ctx_for(case, free_surface=1, image_fp64=True)
    s = case.scheme
    rng = np.random.default_rng(3)
    m = (rng.standard_normal((case.nx, case.nz)) * interior_mask(case.nx, case.nz)).astype(np.float32)
    fm = [x.copy() for x in ctx.born_forward(m, shots_for(case))]
    for i in range(len(fm)):
        assert rel_l2(fm[i], orc.born_fwd(s, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i],
                                          dtype=np.float32)) < 1e-5
    d = _data(case, rng)
    ad = ctx.born_adjoint(shots_for(case, data=d))
    ref = sum(orc.born_adj(s, case.vel, d[i], case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32)
              for i in range(len(d)))
    assert rel_l2(ad, ref) < 1e-5
    a = sum(_dot(fm[i], d[i]) for i in range(len(d)))
    assert abs(a - _dot(m, ad)) / abs(_dot(m, ad)) < 1e-5


def test_born_fs_sub4_runs_blocked():
    """With sub = 4 the free surface runs on the interval-blocked stepper (one launch per coarse
    interval and pass) and matches the oracle."""
    c = make_case(seed=8, nts=30, sub=4)
    c.scheme = dataclasses.replace(c.scheme, freeSurface=1)
    ctx = ctx_for(c, free_surface=1)
    m = (np.random.default_rng(4).standard_normal((c.nx, c.nz)) * interior_mask(c.nx, c.nz)).astype(np.float32)
    got = ctx.born_forward(m, shots_for(c))
    assert ctx.last_launches == 2 * (c.scheme.nts - 1)
    for i in range(len(got)):
        assert rel_l2(got[i], orc.born_fwd(c.scheme, c.vel, m, c.sig[i], c.src_pos[i], c.rec_pos[i],
                                           dtype=np.float32)) < 1e-5


def test_born_ext_fs(case):
    ctx = ctx_for(case, free_surface=1, image_fp64=True)
    s = case.scheme
    rng = np.random.default_rng(5)
    m = (rng.standard_normal((s.nExt, case.nx, case.nz)) * interior_mask(case.nx, case.nz)).astype(np.float32)
    fm = [x.copy() for x in ctx.born_ext_forward(m, shots_for(case))]
    for i in range(len(fm)):
        assert rel_l2(fm[i], orc.bornext_fwd(s, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i],
                                             dtype=np.float32)) < 1e-5
    d = _data(case, rng)
    ad = ctx.born_ext_adjoint(shots_for(case, data=d))
    ref = sum(orc.bornext_adj(s, case.vel, d[i], case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32)
              for i in range(len(d)))
    assert rel_l2(ad, ref) < 1e-5
    a = sum(_dot(fm[i], d[i]) for i in range(len(d)))
    assert abs(a - _dot(m, ad)) / abs(_dot(m, ad)) < 1e-5


@pytest.mark.parametrize("legs", [(1, 0), (0, 1), (1, 1)])
def test_tomo_fs(case, legs):
    l1, l2 = legs
    ctx = ctx_for(case, free_surface=1, leg1=l1, leg2=l2, image_fp64=True)
    s = case.scheme
    rng = np.random.default_rng(6)
    mask = interior_mask(case.nx, case.nz)
    m = (rng.standard_normal((case.nx, case.nz)) * mask).astype(np.float32)
    ext = (rng.standard_normal((s.nExt, case.nx, case.nz)) * mask).astype(np.float32)
    fm = [x.copy() for x in ctx.tomo_forward(m, ext, shots_for(case))]
    r32 = [orc.tomo_fwd(s, case.vel, m, ext, case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32,
                        leg1=l1, leg2=l2) for i in range(len(fm))]
    for i in range(len(fm)):
        assert rel_l2(fm[i], r32[i]) < 1e-5
    d = _data(case, rng)
    ad = ctx.tomo_adjoint(ext, shots_for(case, data=d))
    ref = sum(orc.tomo_adj(s, case.vel, d[i], ext, case.sig[i], case.src_pos[i], case.rec_pos[i],
                           dtype=np.float32, leg1=l1, leg2=l2) for i in range(len(d)))
    assert rel_l2(ad, ref) < 1e-5
    # Dot test: 1e-5, or twice the FP32 oracle's own error on the same draw where that is larger
    # (FP32 round-off of the second leg exceeds 1e-5 on this draw: 3.7e-5 for the oracle, while
    # the FP64 oracle pair is adjoint to 7e-15).
    a = sum(_dot(fm[i], d[i]) for i in range(len(d)))
    a32 = sum(_dot(r32[i], d[i]) for i in range(len(d)))
    oracle_err = abs(a32 - _dot(m, ref)) / abs(_dot(m, ref))
    assert abs(a - _dot(m, ad)) / abs(_dot(m, ad)) < max(1e-5, 2 * oracle_err)


@pytest.mark.skipif(not refgpu.available("tomo"), reason="oracle/_ref not built (make -C oracle ref)")
def test_vs_reference_fs_drivers(case):
    """CUDA path vs the reference's own free-surface drivers compiled for sm_100a (one shot)."""
    s, i = case.scheme, 0
    rng = np.random.default_rng(7)
    mask = interior_mask(case.nx, case.nz)
    sp, rp, sig = case.src_pos[i], case.rec_pos[i], case.sig[i]
    from acoustic_isotropic_operators_b200.batch import Shot
    one = [Shot(sp, rp, sig)]
    d = (rng.standard_normal((len(rp), s.nts)) * 1e-2).astype(np.float32)
    ctx = ctx_for(case, free_surface=1, image_fp64=True)
    assert rel_l2(ctx.nonlinear_forward(one)[0], refgpu.nl_fwd(s, case.vel, sig, sp, rp)) < 1e-5
    m = (rng.standard_normal((case.nx, case.nz)) * mask).astype(np.float32)
    assert rel_l2(ctx.born_forward(m, one)[0], refgpu.born_fwd(s, case.vel, m, sig, sp, rp)) < 1e-5
    assert rel_l2(ctx.born_adjoint([Shot(sp, rp, sig, d)]), refgpu.born_adj(s, case.vel, d, sig, sp, rp)) < 1e-5
    ext = (rng.standard_normal((s.nExt, case.nx, case.nz)) * mask).astype(np.float32)
    assert rel_l2(ctx.born_ext_forward(ext, one)[0], refgpu.bornext_fwd(s, case.vel, ext, sig, sp, rp)) < 1e-5
    assert rel_l2(ctx.born_ext_adjoint([Shot(sp, rp, sig, d)]),
                  refgpu.bornext_adj(s, case.vel, d, sig, sp, rp)) < 1e-5
    assert rel_l2(ctx.tomo_forward(m, ext, one)[0], refgpu.tomo_fwd(s, case.vel, m, ext, sig, sp, rp)) < 1e-5
    assert rel_l2(ctx.tomo_adjoint(ext, [Shot(sp, rp, sig, d)]),
                  refgpu.tomo_adj(s, case.vel, d, ext, sig, sp, rp)) < 1e-5
