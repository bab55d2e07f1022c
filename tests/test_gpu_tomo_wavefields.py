"""Saved wavefields of the tomo and WEMVA operators (the reference's saveWavefield = 1 drivers:
F/src/tomoExtShotsGpuFunctions.cu:355-465, :797-910 and F/src/wemvaExtShotsGpuFunctions.cu:344-456,
:575-688, with their offset and free-surface variants): d2/dt2 of the source wavefield and two
secondary wavefields [nts][nx][nz] per call of one shot.

Checked against the reference's own drivers (oracle/_ref) and the FP32 oracle, relative L2 <= 1e-5
for the operator's output and each wavefield: through the batched C ABI
(aio_{tomo,wemva}_ext_{forward,adjoint}_wavefield) and through the reference-named seam with
saveWavefield = 1.
"""
import dataclasses

import numpy as np
import pytest

import orc
import refgpu
from cases import interior_mask, make_case, rel_l2
from test_gpu_parity import ctx_for

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refgpu.available("tomo"), reason="oracle/_ref not built (make -C oracle ref)")]

TOL = 1e-5
SCHEMES = [("time", {}), ("offset", dict(extension=1)), ("time-fs", dict(freeSurface=1)),
           ("offset-fs", dict(extension=1, freeSurface=1))]


@pytest.fixture(scope="module")
def base():
    return make_case(seed=21, nts=30, nshots=1, nExt=5)


def _inputs(case, s):
    rng = np.random.default_rng(3)
    mask = interior_mask(case.nx, case.nz)
    dv = (rng.standard_normal((case.nx, case.nz)) * mask).astype(np.float32)
    ext = (rng.standard_normal((s.nExt, case.nx, case.nz)) * mask).astype(np.float32)
    d = rng.standard_normal((len(case.rec_pos[0]), s.nts)).astype(np.float32)
    return dv, ext, d


def _ctx(case, s):
    return ctx_for(dataclasses.replace(case, scheme=s), image_fp64=True, free_surface=s.freeSurface,
                   extension="offset" if s.extension else "time")


def _check(got, ref, orc32, what):
    for i, (a, b, c) in enumerate(zip(got, ref, orc32)):
        assert rel_l2(a, b) < TOL, (what, i, rel_l2(a, b))
        assert rel_l2(a, c) < TOL, (what, i, rel_l2(a, c))


@pytest.mark.parametrize("name,kw", SCHEMES, ids=[x[0] for x in SCHEMES])
def test_tomo_wavefields(base, name, kw):
    from acoustic_isotropic_operators_b200.batch import Shot
    s = dataclasses.replace(base.scheme, **kw)
    sp, rp, sig = base.src_pos[0], base.rec_pos[0], base.sig[0]
    dv, ext, d = _inputs(base, s)
    ctx = _ctx(base, s)
    try:
        got_f = [x.copy() for x in ctx.tomo_forward_wavefield(dv, ext, Shot(sp, rp, sig))]
        got_a = ctx.tomo_adjoint_wavefield(ext, Shot(sp, rp, sig, d))
    finally:
        ctx.close()
    ref_f = refgpu.tomo_fwd_wavefields(s, base.vel, dv, ext, sig, sp, rp)
    orc_f = orc.tomo_fwd(s, base.vel, dv, ext, sig, sp, rp, dtype=np.float32, wavefields=True)
    _check(got_f, ref_f, orc_f, "tomo forward")
    ref_a = refgpu.tomo_adj_wavefields(s, base.vel, d, ext, sig, sp, rp)
    orc_a = orc.tomo_adj(s, base.vel, d, ext, sig, sp, rp, dtype=np.float32, wavefields=True)
    _check(got_a, ref_a, orc_a, "tomo adjoint")
    assert all(np.abs(x).max() > 0 for x in list(got_f[1:]) + list(got_a[1:]))


@pytest.mark.parametrize("name,kw", SCHEMES[:2], ids=[x[0] for x in SCHEMES[:2]])
def test_wemva_wavefields(base, name, kw):
    from acoustic_isotropic_operators_b200.batch import Shot
    s = dataclasses.replace(base.scheme, **kw)
    sp, rp, sig = base.src_pos[0], base.rec_pos[0], base.sig[0]
    dv, img, rdata = _inputs(base, s)
    ctx = _ctx(base, s)
    try:
        got_f = [x.copy() for x in ctx.wemva_forward_wavefield(dv, Shot(sp, rp, sig, None, rdata))]
        got_a = ctx.wemva_adjoint_wavefield(img, Shot(sp, rp, sig, None, rdata))
    finally:
        ctx.close()
    ref_f = refgpu.wemva_fwd_wavefields(s, base.vel, dv, sig, sp, rp, rdata)
    orc_f = orc.wemva_fwd(s, base.vel, dv, sig, sp, rp, rdata, dtype=np.float32, wavefields=True)
    _check(got_f, ref_f, orc_f, "wemva forward")
    ref_a = refgpu.wemva_adj_wavefields(s, base.vel, img, sig, sp, rp, rdata)
    orc_a = orc.wemva_adj(s, base.vel, img, sig, sp, rp, rdata, dtype=np.float32, wavefields=True)
    _check(got_a, ref_a, orc_a, "wemva adjoint")


def test_batched_calls_unchanged_after_saving(base):
    """A saving call leaves the batched (blocked or fine) path of the same context as it was."""
    from acoustic_isotropic_operators_b200.batch import Shot
    s = base.scheme
    sp, rp, sig = base.src_pos[0], base.rec_pos[0], base.sig[0]
    dv, ext, _ = _inputs(base, s)
    ctx = _ctx(base, s)
    try:
        before = ctx.tomo_forward(dv, ext, [Shot(sp, rp, sig)])[0].copy()
        ctx.tomo_forward_wavefield(dv, ext, Shot(sp, rp, sig))
        after = ctx.tomo_forward(dv, ext, [Shot(sp, rp, sig)])[0].copy()
    finally:
        ctx.close()
    np.testing.assert_array_equal(before, after)


def test_seam_save_wavefield(base):
    """The seam's tomo and WEMVA calls with saveWavefield = 1 fill the three arrays as the
    reference's drivers do."""
    from test_gpu_seam import seam, _geo, _consts
    s = base.scheme
    sp, rp, sig = base.src_pos[0], base.rec_pos[0], base.sig[0]
    dv, ext, d = _inputs(base, s)
    v2, rs = _consts(base)
    z = lambda: np.zeros((s.nts, s.nx, s.nz), np.float32)
    seam("initTomoExtGpu", *_geo(s), s.nExt, 1, 1, 1, 0, 0)
    seam("allocateTomoExtShotsGpu", v2, rs, 0, 0)
    try:
        data = np.zeros((len(rp), s.nts), np.float32)
        W = [z(), z(), z()]
        seam("tomoTimeShotsFwdGpu", dv, data, ext, sig, sp, len(sp), rp, len(rp), *W, 0, 0, 0, 1)
        ref = refgpu.tomo_fwd_wavefields(s, base.vel, dv, ext, sig, sp, rp)
        for a, b in zip([data] + W, ref):
            assert rel_l2(a, b) < TOL
        m = np.zeros((s.nx, s.nz), np.float32)
        W = [z(), z(), z()]
        seam("tomoTimeShotsAdjGpu", m, d, ext, sig, sp, len(sp), rp, len(rp), *W, 0, 0, 0, 1)
        ref = refgpu.tomo_adj_wavefields(s, base.vel, d, ext, sig, sp, rp)
        for a, b in zip([m] + W, ref):
            assert rel_l2(a, b) < TOL
    finally:
        seam("deallocateTomoExtShotsGpu", 0, 0)
    seam("initWemvaExtGpu", *_geo(s), s.nExt, 1, 1, 1, 0, 0)
    seam("allocateWemvaExtShotsGpu", v2, rs, 0, 0)
    try:
        img = np.zeros((s.nExt, s.nx, s.nz), np.float32)
        W = [z(), z(), z()]
        seam("wemvaTimeShotsFwdGpu", dv, img, sig, sp, len(sp), d, rp, len(rp), *W, 0, 0, 1)
        ref = refgpu.wemva_fwd_wavefields(s, base.vel, dv, sig, sp, rp, d)
        for a, b in zip([img] + W, ref):
            assert rel_l2(a, b) < TOL
    finally:
        seam("deallocateWemvaExtShotsGpu", 0, 0)
