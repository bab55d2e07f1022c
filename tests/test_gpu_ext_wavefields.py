"""Saved extended-Born wavefields (the reference's BornExtShotsGpu forwardWavefield /
adjointWavefield and its *Wavefield drivers): the coarse source and scattered wavefields of an
extended Born forward, the coarse source and receiver wavefields of an extended Born adjoint,
[nts][nx][nz] with a zero FAT ring, for time lags and subsurface offsets, with and without the
free surface.

Gates (relative L2): vs the FP32 oracle 1e-5 (data or image, and each wavefield), vs the
reference's own wavefield drivers (oracle/_ref) 1e-5.
"""
import contextlib
import dataclasses

import numpy as np
import pytest

import orc
import refgpu
from cases import interior_mask, make_case, rel_l2
from test_gpu_parity import ctx_for

pytestmark = pytest.mark.gpu

KINDS = [("time", 0), ("offset", 0), ("time", 1), ("offset", 1)]


def _case(ext, fs):
    c = make_case(seed=31, nts=40, nshots=1, nExt=5)
    c.scheme = dataclasses.replace(c.scheme, extension=int(ext == "offset"), freeSurface=fs)
    return c


def _shot(c, data=None):
    from acoustic_isotropic_operators_b200.batch import Shot
    return Shot(c.src_pos[0], c.rec_pos[0], c.sig[0], data)


@contextlib.contextmanager
def _ctx(c, ext, fs):
    ctx = ctx_for(c, extension=ext, free_surface=fs, image_fp64=True)
    try:
        yield ctx
    finally:
        ctx.close()


def _ring_zero(c, *fields):
    """Every returned wavefield is zero on the whole FAT ring (all four edges, every sample)."""
    outside = ~interior_mask(c.nx, c.nz)
    for f in fields:
        assert not f[:, outside].any()


@pytest.mark.parametrize("ext,fs", KINDS)
def test_ext_forward_wavefields(ext, fs):
    c = _case(ext, fs)
    s = c.scheme
    m = (np.random.default_rng(1).standard_normal((s.nExt, c.nx, c.nz)) * interior_mask(c.nx, c.nz)).astype(
        np.float32)
    with _ctx(c, ext, fs) as ctx:
        d, W, S = ctx.born_ext_forward_wavefield(m, _shot(c))
        d = d.copy()
        # the batched operator gives the same data (non-sloth scaling)
        batched = ctx.born_ext_forward(m, [_shot(c)])[0].copy()
    rd, rW, rS = orc.bornext_fwd(s, c.vel, m, c.sig[0], c.src_pos[0], c.rec_pos[0], dtype=np.float32,
                                 secondary=True)
    assert W.shape == (s.nts, c.nx, c.nz)
    assert rel_l2(d, rd) < 1e-5 and rel_l2(W, rW) < 1e-5 and rel_l2(S, rS) < 1e-5
    _ring_zero(c, W, S)
    assert rel_l2(batched, d) < 1e-5


@pytest.mark.parametrize("ext,fs", KINDS)
def test_ext_adjoint_wavefields(ext, fs):
    c = _case(ext, fs)
    s = c.scheme
    d = np.random.default_rng(2).standard_normal((len(c.rec_pos[0]), s.nts)).astype(np.float32)
    with _ctx(c, ext, fs) as ctx:
        img, W, R = ctx.born_ext_adjoint_wavefield(_shot(c, d))
        batched = ctx.born_ext_adjoint([_shot(c, d)]).copy()
    ri, rW, rR = orc.bornext_adj(s, c.vel, d, c.sig[0], c.src_pos[0], c.rec_pos[0], dtype=np.float32,
                                 secondary=True)
    assert rel_l2(img, ri) < 1e-5 and rel_l2(W, rW) < 1e-5 and rel_l2(R, rR) < 1e-5
    _ring_zero(c, W, R)
    assert rel_l2(batched, img) < 1e-5


@pytest.mark.skipif(not refgpu.available("bornext"), reason="oracle/_ref not built (make -C oracle ref)")
@pytest.mark.parametrize("ext,fs", KINDS)
def test_vs_reference_ext_wavefield_drivers(ext, fs):
    c = _case(ext, fs)
    s = c.scheme
    rng = np.random.default_rng(3)
    m = (rng.standard_normal((s.nExt, c.nx, c.nz)) * interior_mask(c.nx, c.nz)).astype(np.float32)
    with _ctx(c, ext, fs) as ctx:
        got = [x.copy() for x in ctx.born_ext_forward_wavefield(m, _shot(c))]
    ref = refgpu.bornext_fwd_wavefields(s, c.vel, m, c.sig[0], c.src_pos[0], c.rec_pos[0])
    for a, b in zip(got, ref):
        assert rel_l2(a, b) < 1e-5
    d = (rng.standard_normal((len(c.rec_pos[0]), s.nts)) * 1e-2).astype(np.float32)
    with _ctx(c, ext, fs) as ctx:
        got = ctx.born_ext_adjoint_wavefield(_shot(c, d))
    ref = refgpu.bornext_adj_wavefields(s, c.vel, d, c.sig[0], c.src_pos[0], c.rec_pos[0])
    for a, b in zip(got, ref):
        assert rel_l2(a, b) < 1e-5
