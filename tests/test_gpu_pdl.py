"""Programmatic dependent launches of the blocked stepper: a launch may run its prologue (ring
zeroing, column tables, sparse entries) while the previous launch of its stream still runs, and
waits for that launch before it reads the state, partial sums, stored slices or their scales.
The overlap changes scheduling only: every mode (off, release after the dependency wait, release
at the last iteration) must give bitwise the same results, for direct launches and for graph
replays, with FP32 and FP16 stored wavefields (the FP16 slice scales are read after the wait), and
with a second context alive on the device (which moves the automatic release point)."""
import os

import numpy as np
import pytest

import orc
from cases import interior_mask
from test_gpu_blocked import blocked_case

pytestmark = pytest.mark.gpu


def _ctx(case, mode, wavefield="fp32"):
    from acoustic_isotropic_operators_b200.batch import Context
    s = case.scheme
    k = orc.constants(s, case.vel, dtype=np.float32)
    old = os.environ.get("AIO_PDL")
    if mode is None:
        os.environ.pop("AIO_PDL", None)
    else:
        os.environ["AIO_PDL"] = mode
    try:
        return Context(s.nz, s.nx, s.nts, s.dts, s.sub, s.dz, s.dx, s.minPad, k["v2"], k["rs"], image_fp64=True,
                       wavefield=wavefield)
    finally:
        if old is None:
            os.environ.pop("AIO_PDL", None)
        else:
            os.environ["AIO_PDL"] = old


def _run(ctx, case, model, data):
    from acoustic_isotropic_operators_b200.batch import Shot
    n = len(case.src_pos)
    out = []
    for _ in range(3):  # direct launches, captured, replayed
        nl = [x.copy() for x in ctx.nonlinear_forward([Shot(case.src_pos[j], case.rec_pos[j], case.sig[j])
                                                       for j in range(n)])]
        bf = [x.copy() for x in ctx.born_forward(model, [Shot(case.src_pos[j], case.rec_pos[j], case.sig[j])
                                                         for j in range(n)])]
        ba = ctx.born_adjoint([Shot(case.src_pos[j], case.rec_pos[j], case.sig[j], data[j])
                               for j in range(n)]).copy()
        out.append(nl + bf + [ba])
    return out


@pytest.mark.parametrize("wavefield", ["fp32", "fp16"])
def test_overlap_modes_bitwise_equal(wavefield):
    case = blocked_case(seed=21, nts=26)
    rng = np.random.default_rng(8)
    model = (rng.standard_normal((case.nx, case.nz)) * interior_mask(case.nx, case.nz)).astype(np.float32)
    data = [rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
    results = {}
    for mode in ("0", "1", "2", None):
        ctx = _ctx(case, mode, wavefield)
        try:
            results[mode] = _run(ctx, case, model, data)
        finally:
            ctx.close()
    ref = results["0"]
    for mode in ("1", "2", None):
        for call_ref, call in zip(ref, results[mode]):
            for a, b in zip(call_ref, call):
                assert np.array_equal(a, b), f"AIO_PDL={mode} differs from launches without overlap"


def test_overlap_with_two_live_contexts():
    """Two contexts alive on the device: the automatic mode releases at the last iteration; both
    contexts give the one-context results bitwise."""
    case = blocked_case(seed=22, nts=22)
    rng = np.random.default_rng(9)
    model = (rng.standard_normal((case.nx, case.nz)) * interior_mask(case.nx, case.nz)).astype(np.float32)
    data = [rng.standard_normal((len(r), case.scheme.nts)).astype(np.float32) for r in case.rec_pos]
    ctx = _ctx(case, "0")
    try:
        ref = _run(ctx, case, model, data)
    finally:
        ctx.close()
    a, b = _ctx(case, None), _ctx(case, None)
    try:
        for ctx in (a, b):
            for call_ref, call in zip(ref, _run(ctx, case, model, data)):
                for x, y in zip(call_ref, call):
                    assert np.array_equal(x, y)
    finally:
        a.close()
        b.close()
