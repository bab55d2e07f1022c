"""Serving loop on the GPU: a mix of nonlinear-forward, Born-forward and
Born-adjoint requests on two grids and three velocity models (two of them on the
same grid), arriving while earlier batches run, gives for every request the same
result as that request run alone (relative L2 <= 1e-6; shots of a launch are
computed independently, so the results agree to round-off of identical
arithmetic). A context's per-call buffers are counted and can be released
between calls without changing its results."""
import time

import numpy as np
import pytest

import orc
from cases import rel_l2

pytestmark = pytest.mark.gpu


def grid_case(seed, nzi, nxi, nts):
    from acoustic_isotropic_operators_b200.serving import Grid
    rng = np.random.default_rng(seed)
    g = Grid(nzi + 10, nxi + 10, nts, 0.004, 4, 10.0, 10.0, 10)
    zz = np.linspace(0, 1, g.nz)[None, :]
    vel = (2000.0 + 500.0 * zz + 50.0 * rng.random((g.nx, g.nz))).astype(np.float32)
    s = orc.Scheme(nz=g.nz, nx=g.nx, nts=nts, dts=0.004, sub=4, dz=10.0, dx=10.0, minPad=10)
    k = orc.constants(s, vel, dtype=np.float32)
    m = np.zeros((g.nx, g.nz), np.float32)
    m[5:-5, 5:-5] = rng.standard_normal((nxi, nzi))
    return g, k["v2"], k["rs"], m, rng


def make_shot(g, rng, with_data):
    from acoustic_isotropic_operators_b200.batch import Shot
    ix = 5 + int(rng.integers(3, g.nx - 13))
    sp = np.array([ix * g.nz + 8], np.int32)
    rp = np.array([x * g.nz + 7 for x in range(5, g.nx - 5)], np.int32)
    sig = (rng.standard_normal((1, g.ntw)) * 1e-2).astype(np.float32)
    d = (rng.standard_normal((len(rp), g.nts)) * 1e-3).astype(np.float32) if with_data else None
    return Shot(sp, rp, sig, d)


def test_results_alone_equal_results_in_the_mix():
    from acoustic_isotropic_operators_b200.batch import Context
    from acoustic_isotropic_operators_b200.serving import Request, Server
    # velocity models v0 and v2 share a grid: they run on separate contexts, overlapping on the device
    cases = [grid_case(1, 64, 96, 36), grid_case(2, 96, 128, 28), grid_case(3, 64, 96, 36)]
    reqs = []
    for gi, (g, v2, rs, m, rng) in enumerate(cases):
        for op in ("nonlinear_forward", "born_forward", "born_adjoint"):
            for _ in range(3):
                reqs.append(Request(op=op, grid=g, velocity_id=f"v{gi}", vel2dtw2=v2, refl_scale=rs,
                                    shot=make_shot(g, rng, op == "born_adjoint"), model_id=f"m{gi}", model=m))
    order = np.random.default_rng(0).permutation(len(reqs))
    srv = Server(workers=2, max_batch=4)
    futs = {}
    for j, i in enumerate(order):
        r = reqs[i]
        r.arrival = 0.0
        futs[i] = srv.submit(r)
        if j % 4 == 3:
            time.sleep(0.02)          # later requests arrive while batches are on the GPU
    got = {i: f.result(timeout=600) for i, f in futs.items()}
    srv.close()
    assert max(b for _, b in srv.batches) > 1          # requests were merged
    assert len({w for w, _ in srv.batches}) == 2       # both workers (streams) were used
    for i, r in enumerate(reqs):
        ctx = Context(r.grid.nz, r.grid.nx, r.grid.nts, r.grid.dts, r.grid.sub, r.grid.dz, r.grid.dx,
                      r.grid.minPad, r.vel2dtw2, r.refl_scale, image_fp64=True)
        from acoustic_isotropic_operators_b200.batch import Shot
        s = Shot(r.shot.src_pos, r.shot.rec_pos, r.shot.src_sig, None if r.op != "born_adjoint" else r.shot.data)
        if r.op == "nonlinear_forward":
            alone = ctx.nonlinear_forward([s])[0]
        elif r.op == "born_forward":
            alone = ctx.born_forward(r.model, [s])[0]
        else:
            alone = ctx.born_adjoint([s])
        ctx.close()
        assert rel_l2(got[i], alone) <= 1e-6, (r.op, rel_l2(got[i], alone))
    rep = srv.report()
    assert rep["requests"] == len(reqs) and rep["p99_s"] >= rep["p50_s"]


def test_context_buffers_counted_and_released():
    from acoustic_isotropic_operators_b200.batch import Context
    g, v2, rs, m, rng = grid_case(4, 64, 96, 36)
    shots = [make_shot(g, rng, False) for _ in range(3)]
    ctx = Context(g.nz, g.nx, g.nts, g.dts, g.sub, g.dz, g.dx, g.minPad, v2, rs, image_fp64=True)
    try:
        base = ctx.device_bytes
        first = [d.copy() for d in ctx.born_forward(m, shots)]
        held = ctx.device_bytes
        assert held > base + g.nts * (g.nz - 10) * (g.nx - 10) * 4 * len(shots)  # stored wavefields
        ctx.release_buffers()
        assert ctx.device_bytes == base
        again = ctx.born_forward(m, shots)
        for a, b in zip(first, again):
            assert rel_l2(a, b) <= 1e-6
    finally:
        ctx.close()
