"""Saved Born wavefields (the reference's forwardWavefield / adjointWavefield, getSrcWfld /
getSecWfld): the coarse source and scattered wavefields of a Born forward and the source and
scaled receiver wavefields of a Born adjoint, [nts][nx][nz] with a zero FAT ring.

Gates (relative L2): vs the FP32 oracle 1e-5 (data, image and each wavefield), vs the reference's
own wavefield drivers (oracle/_ref, BornShots{Fwd,Adj}GpuWavefield) 1e-5.
"""
import numpy as np
import pytest

import orc
import refgpu
from cases import interior_mask, make_case, rel_l2
from test_gpu_parity import ctx_for

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    return make_case(seed=21, nts=40, nshots=1)


def _shot(case, data=None):
    from acoustic_isotropic_operators_b200.batch import Shot
    return Shot(case.src_pos[0], case.rec_pos[0], case.sig[0], data)


def test_born_forward_wavefields(case):
    s = case.scheme
    m = (np.random.default_rng(1).standard_normal((case.nx, case.nz)) * interior_mask(case.nx, case.nz)).astype(
        np.float32)
    d, W, S = ctx_for(case).born_forward_wavefield(m, _shot(case))
    rd, rW, rS = orc.born_fwd(s, case.vel, m, case.sig[0], case.src_pos[0], case.rec_pos[0], dtype=np.float32,
                              secondary=True)
    assert W.shape == (s.nts, case.nx, case.nz)
    assert rel_l2(d, rd) < 1e-5 and rel_l2(W, rW) < 1e-5 and rel_l2(S, rS) < 1e-5
    assert not W[:, :5].any() and not W[:, :, :5].any()  # zero FAT ring
    # the batched call gives the same data
    assert rel_l2(ctx_for(case).born_forward(m, [_shot(case)])[0], d) < 1e-6


def test_born_adjoint_wavefields(case):
    s = case.scheme
    d = np.random.default_rng(2).standard_normal((len(case.rec_pos[0]), s.nts)).astype(np.float32)
    img, W, R = ctx_for(case).born_adjoint_wavefield(_shot(case, d))
    ri, rW, rR = orc.born_adj(s, case.vel, d, case.sig[0], case.src_pos[0], case.rec_pos[0], dtype=np.float32,
                              secondary=True)
    assert rel_l2(img, ri) < 1e-5 and rel_l2(W, rW) < 1e-5 and rel_l2(R, rR) < 1e-5


@pytest.mark.skipif(not refgpu.available("born"), reason="oracle/_ref not built (make -C oracle ref)")
def test_vs_reference_wavefield_drivers(case):
    s = case.scheme
    rng = np.random.default_rng(3)
    m = (rng.standard_normal((case.nx, case.nz)) * interior_mask(case.nx, case.nz)).astype(np.float32)
    got = ctx_for(case).born_forward_wavefield(m, _shot(case))
    ref = refgpu.born_fwd_wavefields(s, case.vel, m, case.sig[0], case.src_pos[0], case.rec_pos[0])
    for a, b in zip(got, ref):
        assert rel_l2(a, b) < 1e-5
    d = rng.standard_normal((len(case.rec_pos[0]), s.nts)).astype(np.float32)
    img, _, rec = ctx_for(case).born_adjoint_wavefield(_shot(case, d))
    rimg, rsrc, rrec = refgpu.born_adj_wavefields(s, case.vel, d, case.sig[0], case.src_pos[0], case.rec_pos[0])
    assert rel_l2(img, rimg) < 1e-5 and rel_l2(rec, rrec) < 1e-5
    assert not rsrc.any()  # the reference's adjoint wavefield driver does not return the source wavefield
