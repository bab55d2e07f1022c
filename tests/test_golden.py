"""CPU oracle vs committed outputs of the reference's own GPU drivers.

tests/golden/reference_small.npz holds, for one small seeded case, the outputs
of the reference's *ShotsGpuFunctions.cu (compiled unmodified for sm_100a and
run on a B200 by tests/golden/make_golden.py) for every operator family in
FP32 and FP64. This pins the CPU oracle without a GPU:

* FP64 oracle vs reference FP64 (acoustic_iso_double): relative L2 <= 1e-10,
* FP32 oracle vs reference FP32 (acoustic_iso_float):  relative L2 <= 1e-5.
"""
import os

import numpy as np
import pytest

import orc
from cases import rel_l2

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_small.npz")
TOL = {"f64": 1e-10, "f32": 1e-5}
DT = {"f64": np.float64, "f32": np.float32}

pytestmark = pytest.mark.skipif(not os.path.exists(GOLD), reason="golden fixtures not generated")


@pytest.fixture(scope="module")
def g():
    z = np.load(GOLD)
    f = {k: z[k] for k in z.files}
    nz, nx, nts, sub, minPad, nExt = (int(v) for v in f["scheme"])
    dz, dx, dts, alpha = (float(v) for v in f["scheme_f"])
    f["s"] = orc.Scheme(nz=nz, nx=nx, nts=nts, dts=dts, sub=sub, dz=dz, dx=dx, minPad=minPad, nExt=nExt,
                        alphaCos=alpha)
    return f


def _vel(g, tag):
    return g["vel"].astype(DT[tag])


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_nonlinear(g, tag):
    s, v, dt = g["s"], _vel(g, tag), DT[tag]
    assert rel_l2(orc.nl_fwd(s, v, g["sig"], g["src_pos"], g["rec_pos"], dtype=dt), g[f"nl_fwd_{tag}"]) < TOL[tag]
    assert rel_l2(orc.nl_adj(s, v, g["data_in"], g["src_pos"], g["rec_pos"], dtype=dt), g[f"nl_adj_{tag}"]) < TOL[tag]


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_born(g, tag):
    s, v, dt = g["s"], _vel(g, tag), DT[tag]
    got = orc.born_fwd(s, v, g["dm"], g["sig"], g["src_pos"], g["rec_pos"], dtype=dt)
    assert rel_l2(got, g[f"born_fwd_{tag}"]) < TOL[tag]
    got = orc.born_adj(s, v, g["data_in"], g["sig"], g["src_pos"], g["rec_pos"], dtype=dt)
    assert rel_l2(got, g[f"born_adj_{tag}"]) < TOL[tag]


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("sloth", [0, 1])
def test_born_ext(g, tag, sloth):
    s, v, dt = g["s"], _vel(g, tag), DT[tag]
    got = orc.bornext_fwd(s, v, g["ext"], g["sig"], g["src_pos"], g["rec_pos"], dtype=dt, sloth=sloth)
    assert rel_l2(got, g[f"bornext_fwd_s{sloth}_{tag}"]) < TOL[tag]
    got = orc.bornext_adj(s, v, g["data_in"], g["sig"], g["src_pos"], g["rec_pos"], dtype=dt, sloth=sloth)
    assert rel_l2(got, g[f"bornext_adj_s{sloth}_{tag}"]) < TOL[tag]


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("sloth", [0, 1])
@pytest.mark.parametrize("legs", [(1, 1), (1, 0), (0, 1)])
def test_tomo(g, tag, sloth, legs):
    s, v, dt = g["s"], _vel(g, tag), DT[tag]
    k = f"s{sloth}_l{legs[0]}{legs[1]}_{tag}"
    got = orc.tomo_fwd(s, v, g["dm"], g["ext"], g["sig"], g["src_pos"], g["rec_pos"], dtype=dt, sloth=sloth,
                       leg1=legs[0], leg2=legs[1])
    assert rel_l2(got, g["tomo_fwd_" + k]) < TOL[tag]
    got = orc.tomo_adj(s, v, g["data_in"], g["ext"], g["sig"], g["src_pos"], g["rec_pos"], dtype=dt, sloth=sloth,
                       leg1=legs[0], leg2=legs[1])
    assert rel_l2(got, g["tomo_adj_" + k]) < TOL[tag]


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("legs", [(1, 1), (1, 0), (0, 1)])
def test_wemva(g, tag, legs):
    s, v, dt = g["s"], _vel(g, tag), DT[tag]
    k = f"l{legs[0]}{legs[1]}_{tag}"
    got = orc.wemva_fwd(s, v, g["dm"], g["sig"], g["src_pos"], g["rec_pos"], g["rdata"], dtype=dt, leg1=legs[0],
                        leg2=legs[1])
    assert rel_l2(got, g["wemva_fwd_" + k]) < TOL[tag]
    got = orc.wemva_adj(s, v, g["image_in"], g["sig"], g["src_pos"], g["rec_pos"], g["rdata"], dtype=dt,
                        leg1=legs[0], leg2=legs[1])
    assert rel_l2(got, g["wemva_adj_" + k]) < TOL[tag]


def test_fixture_is_nontrivial(g):
    # every stored reference output carries signal (a silent all-zero output would pin nothing)
    for k, a in g.items():
        if k.endswith(("_f32", "_f64")):
            assert np.abs(a).max() > 0, k
