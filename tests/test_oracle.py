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


def test_tomo_wemva_saved_wavefields_leave_outputs_unchanged():
    """Asking the oracle for the saved wavefields changes none of the operators' outputs; the
    source d2/dt2 and the receiver wavefield are shared by the calls that compute them, and the
    secondary fields are non-zero."""
    import numpy as np
    from cases import interior_mask, make_case
    c = make_case(seed=22, nts=16, nshots=1, nExt=3, nzi=24, nxi=32)
    s, sp, rp, sig = c.scheme, c.src_pos[0], c.rec_pos[0], c.sig[0]
    rng = np.random.default_rng(1)
    mask = interior_mask(c.nx, c.nz)
    dv = rng.standard_normal((c.nx, c.nz)) * mask
    ext = rng.standard_normal((s.nExt, c.nx, c.nz)) * mask
    d = rng.standard_normal((len(rp), s.nts))
    v = c.vel.astype(np.float64)
    f = orc.tomo_fwd(s, v, dv, ext, sig, sp, rp, wavefields=True)
    assert np.array_equal(f[0], orc.tomo_fwd(s, v, dv, ext, sig, sp, rp))
    a = orc.tomo_adj(s, v, d, ext, sig, sp, rp, wavefields=True)
    assert np.array_equal(a[0], orc.tomo_adj(s, v, d, ext, sig, sp, rp))
    np.testing.assert_array_equal(f[1], a[1])
    wf = orc.wemva_fwd(s, v, dv, sig, sp, rp, d, wavefields=True)
    assert np.array_equal(wf[0], orc.wemva_fwd(s, v, dv, sig, sp, rp, d))
    wa = orc.wemva_adj(s, v, ext, sig, sp, rp, d, wavefields=True)
    assert np.array_equal(wa[0], orc.wemva_adj(s, v, ext, sig, sp, rp, d))
    np.testing.assert_array_equal(wf[2], wa[2])
    np.testing.assert_array_equal(a[2], wa[2])
    for x in (f[2], f[3], a[3], wf[3], wa[3]):
        assert np.abs(x).max() > 0
