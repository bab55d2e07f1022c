"""CPU-only checks of the oracle (FP64 dot tests, FP32 vs FP64 agreement)."""
import numpy as np
import pytest

import orc
from cases import interior_mask, make_case, rel_l2


@pytest.fixture(scope="module")
def case():
    return make_case(seed=11, nzi=32, nxi=48, nts=30)


def dot(a, b):
    return float(np.sum(np.asarray(a, np.float64) * np.asarray(b, np.float64)))


def _mask(case, m):
    return m * interior_mask(case.nx, case.nz)


def test_fp64_dot_all_operators(case):
    s, v = case.scheme, case.vel.astype(np.float64)
    rng = np.random.default_rng(5)
    sp, rp, sig = case.src_pos[0], case.rec_pos[0], case.sig[0].astype(np.float64)
    d = rng.standard_normal((len(rp), s.nts))
    m = rng.standard_normal(sig.shape)
    assert abs(dot(orc.nl_fwd(s, v, m, sp, rp), d) - dot(m, orc.nl_adj(s, v, d, sp, rp))) < 1e-12 * abs(dot(d, d))
    pairs = []
    mb = _mask(case, rng.standard_normal((case.nx, case.nz)))
    pairs.append((dot(orc.born_fwd(s, v, mb, sig, sp, rp), d), dot(mb, orc.born_adj(s, v, d, sig, sp, rp))))
    me = _mask(case, rng.standard_normal((s.nExt, case.nx, case.nz)))
    for sl in (0, 1):
        pairs.append((dot(orc.bornext_fwd(s, v, me, sig, sp, rp, sloth=sl), d),
                      dot(me, orc.bornext_adj(s, v, d, sig, sp, rp, sloth=sl))))
    for l1, l2 in ((1, 0), (0, 1)):
        pairs.append((dot(orc.tomo_fwd(s, v, mb, me, sig, sp, rp, leg1=l1, leg2=l2), d),
                      dot(mb, orc.tomo_adj(s, v, d, me, sig, sp, rp, leg1=l1, leg2=l2))))
        pairs.append((dot(orc.wemva_fwd(s, v, mb, sig, sp, rp, d, leg1=l1, leg2=l2), me),
                      dot(mb, orc.wemva_adj(s, v, me, sig, sp, rp, d, leg1=l1, leg2=l2))))
    for a, b in pairs:
        assert abs(a - b) <= 1e-12 * abs(b)


def test_fp32_close_to_fp64(case):
    s = case.scheme
    d32 = orc.nl_fwd(s, case.vel, case.sig[0], case.src_pos[0], case.rec_pos[0], dtype=np.float32)
    d64 = orc.nl_fwd(s, case.vel.astype(np.float64), case.sig[0], case.src_pos[0], case.rec_pos[0])
    assert rel_l2(d32, d64) < 1e-5


def test_host_prep_adjoints():
    rng = np.random.default_rng(0)
    nts, dts, sub = 37, 0.004, 4
    m = rng.standard_normal((3, nts))
    d = rng.standard_normal((3, (nts - 1) * sub + 1))
    assert abs(dot(orc.time_interp_fwd(nts, dts, sub, m), d) -
               dot(m, orc.time_interp_adj(nts, dts, sub, d))) < 1e-12 * abs(dot(d, d))
    a = rng.standard_normal((3, nts))
    b = rng.standard_normal((3, nts))
    assert abs(dot(orc.second_deriv(nts, dts, a), b) - dot(a, orc.second_deriv(nts, dts, b))) < 1e-9 * abs(
        dot(a, a)) / dts ** 2
