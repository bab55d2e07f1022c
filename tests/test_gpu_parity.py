"""CUDA path (C ABI, batched) vs the CPU oracle (FP32 restatement and FP64 scheme).

Tolerances (relative L2 over the whole output):
  * vs the FP32 oracle: 1e-5 (the north-star FP32 parity bar; the residual is
    summation order / FMA contraction only),
  * vs the FP64 oracle: 1e-4 (the north-star error budget vs FP64).
"""
import numpy as np
import pytest

import orc
from cases import interior_mask, make_case, rel_l2

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-5
TOL_F64 = 1e-4


def ctx_for(case, **kw):
    from acoustic_isotropic_operators_b200.batch import Context
    s = case.scheme
    k = orc.constants(s, case.vel, dtype=np.float32)
    return Context(s.nz, s.nx, s.nts, s.dts, s.sub, s.dz, s.dx, s.minPad, k["v2"], k["rs"], nExt=s.nExt, **kw)


def shots_for(case, data=None, wemva=None):
    from acoustic_isotropic_operators_b200.batch import Shot
    out = []
    for i in range(len(case.src_pos)):
        out.append(Shot(case.src_pos[i], case.rec_pos[i], case.sig[i],
                        None if data is None else data[i], None if wemva is None else wemva[i]))
    return out


@pytest.fixture(scope="module")
def case():
    return make_case(seed=1)


def _both(fn, case, *args, **kw):
    return fn(case.scheme, case.vel, *args, dtype=np.float32, **kw), fn(case.scheme, case.vel.astype(np.float64),
                                                                           *args, dtype=np.float64, **kw)


def test_nonlinear_forward(case):
    ctx = ctx_for(case)
    shots = shots_for(case)
    got = ctx.nonlinear_forward(shots)
    assert ctx.last_launches == (case.scheme.nts - 1) * case.scheme.sub
    for i in range(len(shots)):
        r32, r64 = _both(orc.nl_fwd, case, case.sig[i], case.src_pos[i], case.rec_pos[i])
        assert rel_l2(got[i], r32) < TOL_F32
        assert rel_l2(got[i], r64) < TOL_F64


def test_nonlinear_adjoint(case):
    ctx = ctx_for(case)
    data = [case.rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
    shots = shots_for(case, data=data)
    got = ctx.nonlinear_adjoint(shots)
    for i in range(len(shots)):
        r32, r64 = _both(orc.nl_adj, case, data[i], case.src_pos[i], case.rec_pos[i])
        assert rel_l2(got[i], r32) < TOL_F32
        assert rel_l2(got[i], r64) < TOL_F64


def _model(case, slices=None):
    shape = (case.nx, case.nz) if slices is None else (slices, case.nx, case.nz)
    m = case.rng.standard_normal(shape).astype(np.float32)
    return m * interior_mask(case.nx, case.nz)


def test_born_forward(case):
    ctx = ctx_for(case)
    m = _model(case)
    got = ctx.born_forward(m, shots_for(case))
    for i in range(len(got)):
        r32, r64 = _both(orc.born_fwd, case, m, case.sig[i], case.src_pos[i], case.rec_pos[i])
        assert rel_l2(got[i], r32) < TOL_F32
        assert rel_l2(got[i], r64) < TOL_F64


@pytest.mark.parametrize("fp64", [False, True])
def test_born_adjoint(case, fp64):
    ctx = ctx_for(case, image_fp64=fp64)
    data = [case.rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
    got = ctx.born_adjoint(shots_for(case, data=data))
    r32 = sum(orc.born_adj(case.scheme, case.vel, data[i], case.sig[i], case.src_pos[i], case.rec_pos[i],
                           dtype=np.float32) for i in range(len(data)))
    r64 = sum(orc.born_adj(case.scheme, case.vel.astype(np.float64), data[i], case.sig[i], case.src_pos[i],
                           case.rec_pos[i], dtype=np.float64) for i in range(len(data)))
    assert rel_l2(got, r32) < TOL_F32
    assert rel_l2(got, r64) < TOL_F64
    assert np.all(got[~interior_mask(case.nx, case.nz)] == 0)


@pytest.mark.parametrize("sloth", [0, 1])
def test_born_ext(case, sloth):
    ctx = ctx_for(case, sloth=sloth)
    m = _model(case, case.scheme.nExt)
    got = ctx.born_ext_forward(m, shots_for(case))
    for i in range(len(got)):
        r32, r64 = _both(orc.bornext_fwd, case, m, case.sig[i], case.src_pos[i], case.rec_pos[i], sloth=sloth)
        assert rel_l2(got[i], r32) < TOL_F32
        assert rel_l2(got[i], r64) < TOL_F64
    data = [case.rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
    got = ctx.born_ext_adjoint(shots_for(case, data=data))
    r32 = sum(orc.bornext_adj(case.scheme, case.vel, data[i], case.sig[i], case.src_pos[i], case.rec_pos[i],
                              dtype=np.float32, sloth=sloth) for i in range(len(data)))
    assert rel_l2(got, r32) < TOL_F32


@pytest.mark.parametrize("legs", [(1, 0), (0, 1), (1, 1)])
def test_tomo(case, legs):
    l1, l2 = legs
    ctx = ctx_for(case, leg1=l1, leg2=l2)
    m = _model(case)
    ext = _model(case, case.scheme.nExt)
    got = ctx.tomo_forward(m, ext, shots_for(case))
    for i in range(len(got)):
        r32 = orc.tomo_fwd(case.scheme, case.vel, m, ext, case.sig[i], case.src_pos[i], case.rec_pos[i],
                           dtype=np.float32, leg1=l1, leg2=l2)
        assert rel_l2(got[i], r32) < TOL_F32
    data = [case.rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
    got = ctx.tomo_adjoint(ext, shots_for(case, data=data))
    r32 = sum(orc.tomo_adj(case.scheme, case.vel, data[i], ext, case.sig[i], case.src_pos[i], case.rec_pos[i],
                           dtype=np.float32, leg1=l1, leg2=l2) for i in range(len(data)))
    assert rel_l2(got, r32) < TOL_F32


@pytest.mark.parametrize("legs", [(1, 0), (0, 1), (1, 1)])
def test_wemva(case, legs):
    l1, l2 = legs
    ctx = ctx_for(case, leg1=l1, leg2=l2)
    m = _model(case)
    rdata = [case.rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
    got = ctx.wemva_forward(m, shots_for(case, wemva=rdata))
    r32 = sum(orc.wemva_fwd(case.scheme, case.vel, m, case.sig[i], case.src_pos[i], case.rec_pos[i], rdata[i],
                            dtype=np.float32, leg1=l1, leg2=l2) for i in range(len(rdata)))
    assert rel_l2(got, r32) < TOL_F32
    img = _model(case, case.scheme.nExt)
    got = ctx.wemva_adjoint(img, shots_for(case, wemva=rdata))
    r32 = sum(orc.wemva_adj(case.scheme, case.vel, img, case.sig[i], case.src_pos[i], case.rec_pos[i], rdata[i],
                            dtype=np.float32, leg1=l1, leg2=l2) for i in range(len(rdata)))
    assert rel_l2(got, r32) < TOL_F32


def test_batch_equals_single(case):
    """A shot's result is the same alone and inside a batch (forward: bitwise)."""
    ctx = ctx_for(case)
    m = _model(case)
    batch = ctx.born_forward(m, shots_for(case))
    for i in range(len(batch)):
        from acoustic_isotropic_operators_b200.batch import Shot
        single = ctx.born_forward(m, [Shot(case.src_pos[i], case.rec_pos[i], case.sig[i])])[0]
        assert np.array_equal(single, batch[i])


def test_wave_splitting(case):
    """A memory budget that forces one shot per wave gives the same results."""
    full = ctx_for(case)
    s = case.scheme
    small = ctx_for(case, mem_budget_bytes=int(3.2 * (s.nts * (s.nz + 40) * (s.nx + 40) * 4) + (8 << 20)))
    assert small.capacity(1) >= 1
    m = _model(case)
    a = full.born_forward(m, shots_for(case))
    b = small.born_forward(m, shots_for(case))
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
