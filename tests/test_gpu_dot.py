"""Dot-product tests of every forward/adjoint pair on the CUDA path.

|<F m, d> - <m, F^T d>| / |<m, F^T d>| <= 1e-5, dot products in FP64 on the
host (the reference's Operator::dotTest, F/include/operator.h:50-88, uses
1e-5 with FP32 dot products).
"""
import numpy as np
import pytest

from cases import interior_mask, make_case
from test_gpu_parity import ctx_for, shots_for

pytestmark = pytest.mark.gpu
TOL = 1e-5  # Operator::dotTest default, F/include/operator.h:50


def dot(a, b):
    return float(np.sum(np.asarray(a, np.float64) * np.asarray(b, np.float64)))


def rel(a, b):
    return abs(a - b) / abs(b)


@pytest.fixture(scope="module")
def case():
    return make_case(seed=7, nts=40)


def _data(case):
    return [case.rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]


def test_dot_nonlinear(case):
    ctx = ctx_for(case)
    m = [case.rng.standard_normal(s.shape).astype(np.float32) for s in case.sig]
    d = _data(case)
    from acoustic_isotropic_operators_b200.batch import Shot
    fm = ctx.nonlinear_forward([Shot(case.src_pos[i], case.rec_pos[i], m[i]) for i in range(len(m))])
    ad = ctx.nonlinear_adjoint([Shot(case.src_pos[i], case.rec_pos[i], None, d[i]) for i in range(len(m))])
    assert rel(sum(dot(fm[i], d[i]) for i in range(len(m))), sum(dot(m[i], ad[i]) for i in range(len(m)))) < TOL


@pytest.mark.parametrize("fp64", [False, True])
def test_dot_born(case, fp64):
    ctx = ctx_for(case, image_fp64=fp64)
    m = case.rng.standard_normal((case.nx, case.nz)).astype(np.float32) * interior_mask(case.nx, case.nz)
    d = _data(case)
    fm = ctx.born_forward(m, shots_for(case))
    ad = ctx.born_adjoint(shots_for(case, data=d))
    assert rel(sum(dot(fm[i], d[i]) for i in range(len(d))), dot(m, ad)) < TOL


@pytest.mark.parametrize("sloth", [0, 1])
def test_dot_born_ext(case, sloth):
    ctx = ctx_for(case, sloth=sloth, image_fp64=True)
    m = case.rng.standard_normal((case.scheme.nExt, case.nx, case.nz)).astype(np.float32)
    m *= interior_mask(case.nx, case.nz)
    d = _data(case)
    fm = ctx.born_ext_forward(m, shots_for(case))
    ad = ctx.born_ext_adjoint(shots_for(case, data=d))
    assert rel(sum(dot(fm[i], d[i]) for i in range(len(d))), dot(m, ad)) < TOL


@pytest.mark.parametrize("legs", [(1, 0), (0, 1), (1, 1)])
def test_dot_tomo(case, legs):
    ctx = ctx_for(case, leg1=legs[0], leg2=legs[1], image_fp64=True)
    mask = interior_mask(case.nx, case.nz)
    m = case.rng.standard_normal((case.nx, case.nz)).astype(np.float32) * mask
    ext = case.rng.standard_normal((case.scheme.nExt, case.nx, case.nz)).astype(np.float32) * mask
    d = _data(case)
    fm = ctx.tomo_forward(m, ext, shots_for(case))
    ad = ctx.tomo_adjoint(ext, shots_for(case, data=d))
    assert rel(sum(dot(fm[i], d[i]) for i in range(len(d))), dot(m, ad)) < TOL


@pytest.mark.parametrize("legs", [(1, 0), (0, 1), (1, 1)])
def test_dot_wemva(case, legs):
    ctx = ctx_for(case, leg1=legs[0], leg2=legs[1], image_fp64=True)
    mask = interior_mask(case.nx, case.nz)
    m = case.rng.standard_normal((case.nx, case.nz)).astype(np.float32) * mask
    img = case.rng.standard_normal((case.scheme.nExt, case.nx, case.nz)).astype(np.float32) * mask
    rd = _data(case)
    fm = ctx.wemva_forward(m, shots_for(case, wemva=rd))
    ad = ctx.wemva_adjoint(img, shots_for(case, wemva=rd))
    assert rel(dot(fm, img), dot(m, ad)) < TOL
