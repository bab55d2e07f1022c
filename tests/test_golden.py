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
    return _load(GOLD)


def _load(path):
    z = np.load(path)
    f = {k: z[k] for k in z.files}
    nz, nx, nts, sub, minPad, nExt = (int(v) for v in f["scheme"][:6])
    fs = int(f["scheme"][6]) if len(f["scheme"]) > 6 else 0
    ext_axis = int(f["scheme"][7]) if len(f["scheme"]) > 7 else 0
    dz, dx, dts, alpha = (float(v) for v in f["scheme_f"])
    f["s"] = orc.Scheme(nz=nz, nx=nx, nts=nts, dts=dts, sub=sub, dz=dz, dx=dx, minPad=minPad, nExt=nExt,
                        alphaCos=alpha, freeSurface=fs, extension=ext_axis)
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


GOLD_FS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_small_fs.npz")


@pytest.mark.skipif(not os.path.exists(GOLD_FS), reason="free-surface fixtures not generated")
@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_free_surface(tag):
    """Oracle with freeSurface = 1 vs the reference's free-surface drivers (*FsGpu) run on a B200:
    nonlinear, Born, extended Born and tomo (all legs), forward and adjoint."""
    g = _load(GOLD_FS)
    s, v, dt = g["s"], g["vel"].astype(DT[tag]), DT[tag]
    assert s.freeSurface == 1
    sp, rp, sig = g["src_pos"], g["rec_pos"], g["sig"]
    checks = [
        (orc.nl_fwd(s, v, sig, sp, rp, dtype=dt), "nl_fwd"),
        (orc.nl_adj(s, v, g["data_in"], sp, rp, dtype=dt), "nl_adj"),
        (orc.born_fwd(s, v, g["dm"], sig, sp, rp, dtype=dt), "born_fwd"),
        (orc.born_adj(s, v, g["data_in"], sig, sp, rp, dtype=dt), "born_adj"),
        (orc.bornext_fwd(s, v, g["ext"], sig, sp, rp, dtype=dt), "bornext_fwd"),
        (orc.bornext_adj(s, v, g["data_in"], sig, sp, rp, dtype=dt), "bornext_adj"),
    ]
    for l1, l2 in ((1, 1), (1, 0), (0, 1)):
        checks.append((orc.tomo_fwd(s, v, g["dm"], g["ext"], sig, sp, rp, dtype=dt, leg1=l1, leg2=l2),
                       f"tomo_fwd_l{l1}{l2}"))
        checks.append((orc.tomo_adj(s, v, g["data_in"], g["ext"], sig, sp, rp, dtype=dt, leg1=l1, leg2=l2),
                       f"tomo_adj_l{l1}{l2}"))
    for got, key in checks:
        assert rel_l2(got, g[f"{key}_{tag}"]) < TOL[tag], key


GOLD_OFF = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_small_offset.npz")


@pytest.mark.skipif(not os.path.exists(GOLD_OFF), reason="subsurface-offset fixtures not generated")
@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_subsurface_offset(tag):
    """Oracle with extension = 1 vs the reference's subsurface-offset drivers run on a B200:
    extended Born, tomo and WEMVA (all legs), forward and adjoint."""
    g = _load(GOLD_OFF)
    s, v, dt = g["s"], g["vel"].astype(DT[tag]), DT[tag]
    assert s.extension == 1
    sp, rp, sig = g["src_pos"], g["rec_pos"], g["sig"]
    checks = [(orc.bornext_fwd(s, v, g["ext"], sig, sp, rp, dtype=dt), "bornext_fwd"),
              (orc.bornext_adj(s, v, g["data_in"], sig, sp, rp, dtype=dt), "bornext_adj")]
    for l1, l2 in ((1, 1), (1, 0), (0, 1)):
        k = f"l{l1}{l2}"
        checks += [(orc.tomo_fwd(s, v, g["dm"], g["ext"], sig, sp, rp, dtype=dt, leg1=l1, leg2=l2), "tomo_fwd_" + k),
                   (orc.tomo_adj(s, v, g["data_in"], g["ext"], sig, sp, rp, dtype=dt, leg1=l1, leg2=l2),
                    "tomo_adj_" + k),
                   (orc.wemva_fwd(s, v, g["dm"], sig, sp, rp, g["rdata"], dtype=dt, leg1=l1, leg2=l2),
                    "wemva_fwd_" + k),
                   (orc.wemva_adj(s, v, g["image_in"], sig, sp, rp, g["rdata"], dtype=dt, leg1=l1, leg2=l2),
                    "wemva_adj_" + k)]
    for got, key in checks:
        assert rel_l2(got, g[f"{key}_{tag}"]) < TOL[tag], key
