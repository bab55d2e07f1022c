"""CUDA-graph-captured time loops: a blocked pass's per-interval launches run directly the first
time their key (plan, buffers) is seen, are captured into a graph the second time and replayed
afterwards. Replayed calls must give bitwise the results of direct launches (same kernels, same
arguments), for the nonlinear forward, Born forward and Born adjoint on the blocked stepper, with
new inputs between calls (the graphs read their inputs at replay)."""
import os

import numpy as np
import pytest

import orc
from cases import interior_mask
from test_gpu_blocked import blocked_case

pytestmark = pytest.mark.gpu


def _ctx(case, graphs):
    from acoustic_isotropic_operators_b200.batch import Context
    s = case.scheme
    k = orc.constants(s, case.vel, dtype=np.float32)
    old = os.environ.get("AIO_GRAPHS")
    os.environ["AIO_GRAPHS"] = "1" if graphs else "0"
    try:
        return Context(s.nz, s.nx, s.nts, s.dts, s.sub, s.dz, s.dx, s.minPad, k["v2"], k["rs"], image_fp64=True)
    finally:
        if old is None:
            del os.environ["AIO_GRAPHS"]
        else:
            os.environ["AIO_GRAPHS"] = old


def test_graph_replays_match_direct_launches():
    from acoustic_isotropic_operators_b200.batch import Shot
    case = blocked_case(seed=12, nts=24)
    rng = np.random.default_rng(5)
    models = [(rng.standard_normal((case.nx, case.nz)) * interior_mask(case.nx, case.nz)).astype(np.float32)
              for _ in range(3)]
    datas = [[rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
             for _ in range(3)]
    sigs = [[(rng.standard_normal(g.shape) * 1e-2).astype(np.float32) for g in case.sig] for _ in range(3)]
    results = {}
    for graphs in (False, True):
        ctx = _ctx(case, graphs)
        try:
            out = []
            for i in range(3):  # eager, captured, replayed
                nl = [x.copy() for x in ctx.nonlinear_forward(
                    [Shot(case.src_pos[j], case.rec_pos[j], sigs[i][j]) for j in range(len(case.src_pos))])]
                bf = [x.copy() for x in ctx.born_forward(models[i], [Shot(case.src_pos[j], case.rec_pos[j], case.sig[j])
                                                                      for j in range(len(case.src_pos))])]
                ba = ctx.born_adjoint([Shot(case.src_pos[j], case.rec_pos[j], case.sig[j], datas[i][j])
                                       for j in range(len(case.src_pos))]).copy()
                out.append((nl, bf, ba))
            results[graphs] = (out, ctx.graph_replays)
        finally:
            ctx.close()
    assert results[False][1] == 0
    assert results[True][1] >= 4  # calls 2 and 3 of each pass ran from graphs
    for (nl0, bf0, ba0), (nl1, bf1, ba1) in zip(results[False][0], results[True][0]):
        for a, b in zip(nl0 + bf0, nl1 + bf1):
            assert np.array_equal(a, b)
        assert np.array_equal(ba0, ba1)


def test_graph_keys_separate_free_surface():
    """A call with the free surface (another kernel variant) after two plain calls of the same
    plan and buffers must not replay the plain calls' graph."""
    from acoustic_isotropic_operators_b200.batch import Shot
    case = blocked_case(seed=13, nts=20)
    shots = [Shot(case.src_pos[j], case.rec_pos[j], case.sig[j]) for j in range(len(case.src_pos))]
    ctx = _ctx(case, True)
    try:
        for _ in range(3):
            plain = [x.copy() for x in ctx.nonlinear_forward(shots)]
    finally:
        ctx.close()
    from acoustic_isotropic_operators_b200.batch import Context
    s = case.scheme
    k = orc.constants(s, case.vel, dtype=np.float32)
    fs = Context(s.nz, s.nx, s.nts, s.dts, s.sub, s.dz, s.dx, s.minPad, k["v2"], k["rs"], free_surface=1)
    try:
        want = [x.copy() for x in fs.nonlinear_forward(shots)]
    finally:
        fs.close()
    # the seam switches the free surface on an existing context: drive it that way
    from test_gpu_seam import seam, _geo
    v2 = np.ascontiguousarray(k["v2"], np.float32)
    seam("initNonlinearGpu", *_geo(s), 1, 0, 0)
    seam("allocateNonlinearGpu", v2, 0, 0)
    try:
        for i in range(3):
            d = np.zeros((len(case.rec_pos[0]), s.nts), np.float32)
            seam("propShotsFwdGpu", case.sig[0], d, case.src_pos[0], len(case.src_pos[0]), case.rec_pos[0],
                 len(case.rec_pos[0]), None, 0, 0)
            assert np.array_equal(d, plain[0])
        d = np.zeros((len(case.rec_pos[0]), s.nts), np.float32)
        seam("propShotsFwdFsGpu", case.sig[0], d, case.src_pos[0], len(case.src_pos[0]), case.rec_pos[0],
             len(case.rec_pos[0]), None, 0, 0)
        assert np.array_equal(d, want[0])
        assert not np.array_equal(d, plain[0])
    finally:
        seam("deallocateNonlinearGpu", 0, 0)
