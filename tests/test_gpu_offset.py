"""Subsurface-offset extension (the reference's extension = "offset" drivers, *OffsetShots*) on
the CUDA path: extended Born, tomo and WEMVA, forward and adjoint, on the per-fine-step stepper.

Gates (relative L2): CUDA vs the FP32 oracle with the offset axis 1e-5, vs the FP64 oracle 1e-4,
vs the reference's own offset drivers (oracle/_ref) 1e-5; dot tests 1e-5, or twice the FP32
oracle's own error on the same draw where that is larger (the FP64 oracle pairs are adjoint to
~1e-15, tests/test_oracle.py and the CPU check below).
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
    c = make_case(seed=9, nts=40)
    c.scheme = dataclasses.replace(c.scheme, extension=1)
    return c


def _dot(a, b):
    return float(np.sum(np.asarray(a, np.float64) * np.asarray(b, np.float64)))


def _dot_err(fm, d, m, ad):
    a = sum(_dot(fm[i], d[i]) for i in range(len(d))) if isinstance(fm, list) else _dot(fm, d)
    b = _dot(m, ad)
    return abs(a - b) / abs(b)


def test_born_offset(case):
    s = case.scheme
    ctx = ctx_for(case, extension="offset", image_fp64=True)
    rng = np.random.default_rng(11)
    mask = interior_mask(case.nx, case.nz)
    m = (rng.standard_normal((s.nExt, case.nx, case.nz)) * mask).astype(np.float32)
    fm = [x.copy() for x in ctx.born_ext_forward(m, shots_for(case))]
    r32 = [orc.bornext_fwd(s, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32)
           for i in range(len(fm))]
    for i in range(len(fm)):
        assert rel_l2(fm[i], r32[i]) < 1e-5
        r64 = orc.bornext_fwd(s, case.vel.astype(np.float64), m, case.sig[i], case.src_pos[i], case.rec_pos[i],
                              dtype=np.float64)
        assert rel_l2(fm[i], r64) < 1e-4
    # the offset axis changes the answer: the time-lag operator differs
    lag = ctx_for(case, image_fp64=True).born_ext_forward(m, shots_for(case))[0]
    assert rel_l2(lag, fm[0]) > 1e-2
    d = [rng.standard_normal((len(r), s.nts)).astype(np.float32) for r in case.rec_pos]
    ad = ctx.born_ext_adjoint(shots_for(case, data=d))
    ref = sum(orc.bornext_adj(s, case.vel, d[i], case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32)
              for i in range(len(d)))
    assert rel_l2(ad, ref) < 1e-5
    assert _dot_err(fm, d, m, ad) < max(1e-5, 2 * _dot_err(r32, d, m, ref))


@pytest.mark.parametrize("legs", [(1, 0), (0, 1), (1, 1)])
def test_tomo_offset(case, legs):
    l1, l2 = legs
    s = case.scheme
    ctx = ctx_for(case, extension="offset", leg1=l1, leg2=l2, image_fp64=True)
    rng = np.random.default_rng(12)
    mask = interior_mask(case.nx, case.nz)
    m = (rng.standard_normal((case.nx, case.nz)) * mask).astype(np.float32)
    ext = (rng.standard_normal((s.nExt, case.nx, case.nz)) * mask).astype(np.float32)
    fm = [x.copy() for x in ctx.tomo_forward(m, ext, shots_for(case))]
    r32 = [orc.tomo_fwd(s, case.vel, m, ext, case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32,
                        leg1=l1, leg2=l2) for i in range(len(fm))]
    for i in range(len(fm)):
        assert rel_l2(fm[i], r32[i]) < 1e-5
    d = [rng.standard_normal((len(r), s.nts)).astype(np.float32) for r in case.rec_pos]
    ad = ctx.tomo_adjoint(ext, shots_for(case, data=d))
    ref = sum(orc.tomo_adj(s, case.vel, d[i], ext, case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32,
                           leg1=l1, leg2=l2) for i in range(len(d)))
    assert rel_l2(ad, ref) < 1e-5
    assert _dot_err(fm, d, m, ad) < max(1e-5, 2 * _dot_err(r32, d, m, ref))


@pytest.mark.parametrize("legs", [(1, 0), (0, 1), (1, 1)])
def test_wemva_offset(case, legs):
    l1, l2 = legs
    s = case.scheme
    ctx = ctx_for(case, extension="offset", leg1=l1, leg2=l2, image_fp64=True)
    rng = np.random.default_rng(13)
    mask = interior_mask(case.nx, case.nz)
    m = (rng.standard_normal((case.nx, case.nz)) * mask).astype(np.float32)
    img = (rng.standard_normal((s.nExt, case.nx, case.nz)) * mask).astype(np.float32)
    rd = [rng.standard_normal((len(r), s.nts)).astype(np.float32) for r in case.rec_pos]
    fimg = ctx.wemva_forward(m, shots_for(case, wemva=rd)).copy()
    ref_f = sum(orc.wemva_fwd(s, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i], rd[i],
                              dtype=np.float32, leg1=l1, leg2=l2) for i in range(len(rd)))
    assert rel_l2(fimg, ref_f) < 1e-5
    ad = ctx.wemva_adjoint(img, shots_for(case, wemva=rd))
    ref_a = sum(orc.wemva_adj(s, case.vel, img, case.sig[i], case.src_pos[i], case.rec_pos[i], rd[i],
                              dtype=np.float32, leg1=l1, leg2=l2) for i in range(len(rd)))
    assert rel_l2(ad, ref_a) < 1e-5
    assert _dot_err(fimg, img, m, ad) < max(1e-5, 2 * _dot_err(ref_f, img, m, ref_a))


def test_offset_free_surface_sub4():
    """Offsets with the free surface, sub = 4 (blocked stepper), vs the FP32 oracle."""
    c = make_case(seed=10, nts=30, sub=4)
    s = dataclasses.replace(c.scheme, extension=1, freeSurface=1)
    c.scheme = s
    ctx = ctx_for(c, extension="offset", free_surface=1, image_fp64=True)
    rng = np.random.default_rng(14)
    m = (rng.standard_normal((s.nExt, c.nx, c.nz)) * interior_mask(c.nx, c.nz)).astype(np.float32)
    got = ctx.born_ext_forward(m, shots_for(c))
    assert ctx.last_launches == 2 * (s.nts - 1)
    for i in range(len(got)):
        assert rel_l2(got[i], orc.bornext_fwd(s, c.vel, m, c.sig[i], c.src_pos[i], c.rec_pos[i],
                                              dtype=np.float32)) < 1e-5
    d = [rng.standard_normal((len(r), s.nts)).astype(np.float32) for r in c.rec_pos]
    ad = ctx.born_ext_adjoint(shots_for(c, data=d))
    ref = sum(orc.bornext_adj(s, c.vel, d[i], c.sig[i], c.src_pos[i], c.rec_pos[i], dtype=np.float32)
              for i in range(len(d)))
    assert rel_l2(ad, ref) < 1e-5


@pytest.mark.skipif(not refgpu.available("wemva"), reason="oracle/_ref not built (make -C oracle ref)")
def test_vs_reference_offset_drivers(case):
    """CUDA path vs the reference's own subsurface-offset drivers compiled for sm_100a (one shot)."""
    s, i = case.scheme, 0
    rng = np.random.default_rng(15)
    mask = interior_mask(case.nx, case.nz)
    sp, rp, sig = case.src_pos[i], case.rec_pos[i], case.sig[i]
    from acoustic_isotropic_operators_b200.batch import Shot
    d = (rng.standard_normal((len(rp), s.nts)) * 1e-2).astype(np.float32)
    ctx = ctx_for(case, extension="offset", image_fp64=True)
    ext = (rng.standard_normal((s.nExt, case.nx, case.nz)) * mask).astype(np.float32)
    m = (rng.standard_normal((case.nx, case.nz)) * mask).astype(np.float32)
    assert rel_l2(ctx.born_ext_forward(ext, [Shot(sp, rp, sig)])[0],
                  refgpu.bornext_fwd(s, case.vel, ext, sig, sp, rp)) < 1e-5
    assert rel_l2(ctx.born_ext_adjoint([Shot(sp, rp, sig, d)]), refgpu.bornext_adj(s, case.vel, d, sig, sp, rp)) < 1e-5
    assert rel_l2(ctx.tomo_forward(m, ext, [Shot(sp, rp, sig)])[0],
                  refgpu.tomo_fwd(s, case.vel, m, ext, sig, sp, rp)) < 1e-5
    assert rel_l2(ctx.tomo_adjoint(ext, [Shot(sp, rp, sig, d)]),
                  refgpu.tomo_adj(s, case.vel, d, ext, sig, sp, rp)) < 1e-5
    assert rel_l2(ctx.wemva_forward(m, [Shot(sp, rp, sig, None, d)]),
                  refgpu.wemva_fwd(s, case.vel, m, sig, sp, rp, d)) < 1e-5
    assert rel_l2(ctx.wemva_adjoint(ext, [Shot(sp, rp, sig, None, d)]),
                  refgpu.wemva_adj(s, case.vel, ext, sig, sp, rp, d)) < 1e-5


@pytest.mark.parametrize("n_ext", [33, 35])
def test_wide_offsets(n_ext):
    """Wide offset ranges (hExt = 16, 17) through the blocked offset imaging: extended Born adjoint
    and WEMVA forward (the two imaging forms, in passes running backward and forward in time)
    against the FP32 oracle; nts = 70 spans three blocks of 32 coarse samples, the last one partial."""
    c = make_case(seed=19, nxi=80, nts=70, nExt=n_ext, nshots=1)
    s = dataclasses.replace(c.scheme, extension=1)
    c.scheme = s
    ctx = ctx_for(c, extension="offset", image_fp64=True)
    rng = np.random.default_rng(20)
    d = [rng.standard_normal((len(r), s.nts)).astype(np.float32) for r in c.rec_pos]
    ad = ctx.born_ext_adjoint(shots_for(c, data=d))
    ref = orc.bornext_adj(s, c.vel, d[0], c.sig[0], c.src_pos[0], c.rec_pos[0], dtype=np.float32)
    assert rel_l2(ad, ref) < 1e-5
    m = (rng.standard_normal((c.nx, c.nz)) * interior_mask(c.nx, c.nz)).astype(np.float32)
    fimg = ctx.wemva_forward(m, shots_for(c, wemva=d))
    ref_f = orc.wemva_fwd(s, c.vel, m, c.sig[0], c.src_pos[0], c.rec_pos[0], d[0], dtype=np.float32)
    assert rel_l2(fimg, ref_f) < 1e-5
