"""The reference's own GPU drivers (oracle/_ref, compiled from the reference
sources for sm_100a) vs this build's CUDA path and vs the CPU oracle.

* CUDA path vs reference FP32: relative L2 <= 1e-5 (north-star FP32 parity).
* CPU FP32 oracle vs reference FP32: <= 1e-5 (pins the restatement).
* CPU FP64 oracle vs reference FP64: <= 1e-10 (pins the FP64 scheme).
"""
import numpy as np
import pytest

import orc
import refgpu
from cases import interior_mask, make_case, rel_l2
from test_gpu_parity import ctx_for, shots_for

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refgpu.available(), reason="oracle/_ref not built (make -C oracle ref)")]


@pytest.fixture(scope="module")
def case():
    return make_case(seed=3, nts=45, nshots=1)


def test_nonlinear(case):
    s, i = case.scheme, 0
    ref32 = refgpu.nl_fwd(s, case.vel, case.sig[i], case.src_pos[i], case.rec_pos[i])
    got = ctx_for(case).nonlinear_forward(shots_for(case))[0]
    assert rel_l2(got, ref32) < 1e-5
    assert rel_l2(orc.nl_fwd(s, case.vel, case.sig[i], case.src_pos[i], case.rec_pos[i], dtype=np.float32),
                  ref32) < 1e-5
    ref64 = refgpu.nl_fwd(s, case.vel.astype(np.float64), case.sig[i], case.src_pos[i], case.rec_pos[i],
                          dtype=np.float64)
    o64 = orc.nl_fwd(s, case.vel.astype(np.float64), case.sig[i], case.src_pos[i], case.rec_pos[i])
    assert rel_l2(o64, ref64) < 1e-10
    d = case.rng.standard_normal((len(case.rec_pos[i]), s.nts)).astype(np.float32)
    ra = refgpu.nl_adj(s, case.vel, d, case.src_pos[i], case.rec_pos[i])
    from acoustic_isotropic_operators_b200.batch import Shot
    ga = ctx_for(case).nonlinear_adjoint([Shot(case.src_pos[i], case.rec_pos[i], None, d)])[0]
    assert rel_l2(ga, ra) < 1e-5


def test_born(case):
    s, i = case.scheme, 0
    m = case.rng.standard_normal((case.nx, case.nz)).astype(np.float32) * interior_mask(case.nx, case.nz)
    ref = refgpu.born_fwd(s, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i])
    got = ctx_for(case).born_forward(m, shots_for(case))[0]
    assert rel_l2(got, ref) < 1e-5
    d = case.rng.standard_normal((len(case.rec_pos[i]), s.nts)).astype(np.float32)
    ra = refgpu.born_adj(s, case.vel, d, case.sig[i], case.src_pos[i], case.rec_pos[i])
    ga = ctx_for(case).born_adjoint(shots_for(case, data=[d]))
    assert rel_l2(ga, ra) < 1e-5
    o64 = orc.born_adj(s, case.vel.astype(np.float64), d, case.sig[i], case.src_pos[i], case.rec_pos[i])
    r64 = refgpu.born_adj(s, case.vel.astype(np.float64), d, case.sig[i], case.src_pos[i], case.rec_pos[i],
                          dtype=np.float64)
    assert rel_l2(o64, r64) < 1e-10


@pytest.mark.parametrize("sloth", [0, 1])
def test_born_ext(case, sloth):
    s, i = case.scheme, 0
    m = case.rng.standard_normal((s.nExt, case.nx, case.nz)).astype(np.float32) * interior_mask(case.nx, case.nz)
    ref = refgpu.bornext_fwd(s, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i], sloth=sloth)
    got = ctx_for(case, sloth=sloth).born_ext_forward(m, shots_for(case))[0]
    assert rel_l2(got, ref) < 1e-5
    d = case.rng.standard_normal((len(case.rec_pos[i]), s.nts)).astype(np.float32)
    ra = refgpu.bornext_adj(s, case.vel, d, case.sig[i], case.src_pos[i], case.rec_pos[i], sloth=sloth)
    ga = ctx_for(case, sloth=sloth).born_ext_adjoint(shots_for(case, data=[d]))
    assert rel_l2(ga, ra) < 1e-5


@pytest.mark.parametrize("legs", [(1, 0), (0, 1)])
def test_tomo(case, legs):
    s, i = case.scheme, 0
    mask = interior_mask(case.nx, case.nz)
    m = case.rng.standard_normal((case.nx, case.nz)).astype(np.float32) * mask
    ext = case.rng.standard_normal((s.nExt, case.nx, case.nz)).astype(np.float32) * mask
    ref = refgpu.tomo_fwd(s, case.vel, m, ext, case.sig[i], case.src_pos[i], case.rec_pos[i], leg1=legs[0],
                          leg2=legs[1])
    got = ctx_for(case, leg1=legs[0], leg2=legs[1]).tomo_forward(m, ext, shots_for(case))[0]
    assert rel_l2(got, ref) < 1e-5
    d = case.rng.standard_normal((len(case.rec_pos[i]), s.nts)).astype(np.float32)
    ra = refgpu.tomo_adj(s, case.vel, d, ext, case.sig[i], case.src_pos[i], case.rec_pos[i], leg1=legs[0],
                         leg2=legs[1])
    ga = ctx_for(case, leg1=legs[0], leg2=legs[1]).tomo_adjoint(ext, shots_for(case, data=[d]))
    assert rel_l2(ga, ra) < 1e-5


@pytest.mark.parametrize("legs", [(1, 0), (0, 1)])
def test_wemva(case, legs):
    s, i = case.scheme, 0
    mask = interior_mask(case.nx, case.nz)
    m = case.rng.standard_normal((case.nx, case.nz)).astype(np.float32) * mask
    rd = case.rng.standard_normal((len(case.rec_pos[i]), s.nts)).astype(np.float32)
    ref = refgpu.wemva_fwd(s, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i], rd, leg1=legs[0],
                           leg2=legs[1])
    got = ctx_for(case, leg1=legs[0], leg2=legs[1]).wemva_forward(m, shots_for(case, wemva=[rd]))
    assert rel_l2(got, ref) < 1e-5
    img = case.rng.standard_normal((s.nExt, case.nx, case.nz)).astype(np.float32) * mask
    ra = refgpu.wemva_adj(s, case.vel, img, case.sig[i], case.src_pos[i], case.rec_pos[i], rd, leg1=legs[0],
                          leg2=legs[1])
    ga = ctx_for(case, leg1=legs[0], leg2=legs[1]).wemva_adjoint(img, shots_for(case, wemva=[rd]))
    assert rel_l2(ga, ra) < 1e-5
