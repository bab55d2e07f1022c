"""Reference-named operator classes (pybind11 modules pyAcoustic_iso_float_*) on
the GPU: results against the CPU oracle fed by the oracle's own host chain
(spread to the grid, d2/dt2, dtw^2 v^2, fine-time interpolation), and the
reference's dot-product test through Operator::dotTest for every family.

Tolerances: relative L2 1e-5 against the FP32 oracle (the FP32 parity bar);
dot tests at the reference's default maxError 1e-5.
"""
import numpy as np
import pytest

import orc
from cases import rel_l2

pytestmark = pytest.mark.gpu

NZI, NXI, NTS, DTS, SUB, PAD = 32, 48, 40, 0.004, 3, 8
NZ, NX = NZI + 10, NXI + 10


@pytest.fixture(scope="module")
def api():
    from acoustic_isotropic_operators_b200 import reference_api
    return reference_api


@pytest.fixture(scope="module")
def setup(api):
    rng = np.random.default_rng(5)
    zz = np.linspace(0, 1, NZ)[None, :]
    vel = (2000.0 + 400.0 * zz + 50.0 * rng.random((NX, NZ))).astype(np.float32)
    par = api.params(nts=NTS, dts=DTS, sub=SUB, nz=NZ, nx=NX, zPadMinus=PAD, zPadPlus=PAD, xPadMinus=PAD,
                     xPadPlus=PAD, dz=10.0, dx=10.0, fMax=20.0, blockSize=16, fat=5, nShot=2, iGpu=[0], nExt=5,
                     leg1=1, leg2=1, extension="time")
    v = api.vector(vel, [(NZ, 0.0, 10.0), (NX, 0.0, 10.0)])
    nl = api.pyAcoustic_iso_float_nl
    srcs = [nl.deviceGpu([9], [15], v, NTS, 0, 0, 0), nl.deviceGpu([10], [40], v, NTS, 0, 0, 0)]
    rec = nl.deviceGpu([8] * 40, list(range(8, 48)), v, NTS, 0, 0, 0)
    t = np.arange(NTS) * DTS - 0.05
    wav = ((1 - 2 * (np.pi * 15 * t) ** 2) * np.exp(-(np.pi * 15 * t) ** 2)).astype(np.float32)
    sig = api.vector(wav[None, :], [(NTS, 0.0, DTS), (1, 0.0, 1.0)])
    s = orc.Scheme(nz=NZ, nx=NX, nts=NTS, dts=DTS, sub=SUB, dz=10.0, dx=10.0, minPad=PAD, nExt=5)
    par_off = api.params(nts=NTS, dts=DTS, sub=SUB, nz=NZ, nx=NX, zPadMinus=PAD, zPadPlus=PAD, xPadMinus=PAD,
                         xPadPlus=PAD, dz=10.0, dx=10.0, fMax=20.0, blockSize=16, fat=5, nShot=2, iGpu=[0], nExt=5,
                         leg1=1, leg2=1, extension="offset")
    return dict(vel=vel, v=v, par=par, par_off=par_off, srcs=srcs, rec=rec, wav=wav, sig=sig, scheme=s, rng=rng)


def oracle_source(st, dev, d2):
    """Regular fine source traces of a grid-point device via the oracle's host chain."""
    pos = np.array(dev.getRegPosUnique(), np.int32)
    reg = np.zeros((len(pos), NTS))
    reg[0] = st["wav"]                    # corner 0 carries weight 1, the other corners 0
    if d2:
        reg = orc.second_deriv(NTS, DTS, reg, dtype=np.float32)
    dtw = np.float32(DTS / SUB)
    vflat = st["vel"].reshape(-1)
    reg = (reg * (dtw * dtw * vflat[pos] * vflat[pos])[:, None]).astype(np.float32)
    return pos, orc.time_interp_fwd(NTS, DTS, SUB, reg, dtype=np.float32)


def rec_gather(st, dreg):
    """Irregular receiver traces from regular ones: each receiver is corner 0 of its 4."""
    pos = st["rec"].getRegPosUnique()
    index = {p: i for i, p in enumerate(pos)}
    return np.stack([dreg[index[(8 + r) * NZ + 8]] for r in range(40)])


def data_vec(api, values=None):
    return api.vector(values, [(NTS, 0.0, DTS), (40, 0.0, 1.0), (2, 0.0, 1.0)])


def test_born_forward_matches_oracle(api, setup):
    st = setup
    rng = np.random.default_rng(1)
    m = np.zeros((NX, NZ), np.float32)
    m[5:-5, 5:-5] = rng.standard_normal((NXI, NZI))
    op = api.pyAcoustic_iso_float_born.BornShotsGpu(st["v"], st["par"], st["srcs"], [st["sig"]], [st["rec"]])
    model = api.vector(m, [(NZ, 0.0, 10.0), (NX, 0.0, 10.0)])
    data = data_vec(api)
    op.forward(False, model, data)
    got = data.getNdArray().copy()
    rpos = np.array(st["rec"].getRegPosUnique(), np.int32)
    for i, src in enumerate(st["srcs"]):
        spos, sig = oracle_source(st, src, True)
        dreg = orc.born_fwd(st["scheme"], st["vel"], m, sig, spos, rpos, dtype=np.float32)
        assert rel_l2(got[i], rec_gather(st, dreg)) < 1e-5
    # add=True accumulates
    op.forward(True, model, data)
    assert rel_l2(data.getNdArray(), 2 * got) < 1e-6


def test_nonlinear_forward_matches_oracle(api, setup):
    st = setup
    op = api.pyAcoustic_iso_float_nl.nonlinearPropShotsGpu(st["v"], st["par"], st["srcs"], [st["rec"]])
    model = api.vector(st["wav"][None, None, :], [(NTS, 0.0, DTS), (1, 0.0, 1.0), (1, 0.0, 1.0)])
    data = data_vec(api)
    op.forward(False, model, data)
    rpos = np.array(st["rec"].getRegPosUnique(), np.int32)
    for i, src in enumerate(st["srcs"]):
        spos, sig = oracle_source(st, src, False)
        dreg = orc.nl_fwd(st["scheme"], st["vel"], sig, spos, rpos, dtype=np.float32)
        assert rel_l2(data.getNdArray()[i], rec_gather(st, dreg)) < 1e-5


@pytest.mark.parametrize("family", ["nl", "born", "born_ext", "tomo", "wemva", "born_ext_offset", "tomo_offset",
                                    "wemva_offset"])
def test_dot_product(api, setup, family):
    st = dict(setup)
    if family.endswith("_offset"):  # the same classes with extension = "offset"
        st["par"] = st["par_off"]
        family = family[:-len("_offset")]
    rng = np.random.default_rng(7)
    img2 = [(NZ, 0.0, 10.0), (NX, 0.0, 10.0)]
    ext3 = [(NZ, 0.0, 10.0), (NX, 0.0, 10.0), (5, -2 * DTS, DTS)]
    if family == "nl":
        op = api.pyAcoustic_iso_float_nl.nonlinearPropShotsGpu(st["v"], st["par"], st["srcs"], [st["rec"]])
        m1 = api.vector(None, [(NTS, 0.0, DTS), (1, 0.0, 1.0), (2, 0.0, 1.0)])
        d1 = data_vec(api)
    elif family == "born":
        op = api.pyAcoustic_iso_float_born.BornShotsGpu(st["v"], st["par"], st["srcs"], [st["sig"]], [st["rec"]])
        m1, d1 = api.vector(None, img2), data_vec(api)
    elif family == "born_ext":
        op = api.pyAcoustic_iso_float_born_ext.BornExtShotsGpu(st["v"], st["par"], st["srcs"], [st["sig"]], [st["rec"]])
        m1, d1 = api.vector(None, ext3), data_vec(api)
    elif family == "tomo":
        refl = np.zeros((5, NX, NZ), np.float32)
        refl[:, 5:-5, 5:-5] = rng.standard_normal((5, NXI, NZI))
        op = api.pyAcoustic_iso_float_tomo.tomoExtShotsGpu(st["v"], st["par"], st["srcs"], [st["sig"]], [st["rec"]],
                                                            api.vector(refl, ext3))
        m1, d1 = api.vector(None, img2), data_vec(api)
    else:
        rd = [api.vector(rng.standard_normal((40, NTS)).astype(np.float32) * 1e-2, [(NTS, 0.0, DTS), (40, 0.0, 1.0)])
              for _ in range(2)]
        op = api.pyAcoustic_iso_float_wemva.wemvaExtShotsGpu(st["v"], st["par"], st["srcs"], [st["sig"]], [st["rec"]],
                                                              rd)
        m1, d1 = api.vector(None, img2), api.vector(None, ext3)
    op.setDomainRange(m1, d1)
    assert op.dotTest(False, 1e-5)


def test_extension_must_be_named(api, setup):
    """The extended classes refuse an extension other than "time" / "offset" (the reference runs no
    driver for it in tomo, WEMVA and the extended Born adjoint)."""
    st = setup
    par = api.params(nts=NTS, dts=DTS, sub=SUB, nz=NZ, nx=NX, zPadMinus=PAD, zPadPlus=PAD, xPadMinus=PAD,
                     xPadPlus=PAD, dz=10.0, dx=10.0, fMax=20.0, blockSize=16, fat=5, nShot=2, iGpu=[0], nExt=5)
    with pytest.raises(Exception):
        api.pyAcoustic_iso_float_born_ext.BornExtShotsGpu(st["v"], par, st["srcs"], [st["sig"]], [st["rec"]])


def test_born_saved_wavefields(api, setup):
    """BornShotsGpu.forwardWavefield with saveWavefield = 1 keeps the coarse source and scattered
    wavefields of shot wavefieldShotNumber (getSrcWfld / getSecWfld), equal to the oracle's."""
    st = setup
    par = api.params(nts=NTS, dts=DTS, sub=SUB, nz=NZ, nx=NX, zPadMinus=PAD, zPadPlus=PAD, xPadMinus=PAD,
                     xPadPlus=PAD, dz=10.0, dx=10.0, fMax=20.0, blockSize=16, fat=5, nShot=2, iGpu=[0],
                     saveWavefield=1, wavefieldShotNumber=1)
    rng = np.random.default_rng(4)
    m = np.zeros((NX, NZ), np.float32)
    m[5:-5, 5:-5] = rng.standard_normal((NXI, NZI))
    op = api.pyAcoustic_iso_float_born.BornShotsGpu(st["v"], par, st["srcs"], [st["sig"]], [st["rec"]])
    model = api.vector(m, [(NZ, 0.0, 10.0), (NX, 0.0, 10.0)])
    data = data_vec(api)
    op.forwardWavefield(False, model, data)
    src, sec = op.getSrcWfld().getNdArray(), op.getSecWfld().getNdArray()
    spos, sig = oracle_source(st, st["srcs"][1], True)
    rpos = np.array(st["rec"].getRegPosUnique(), np.int32)
    _, rW, rS = orc.born_fwd(st["scheme"], st["vel"], m, sig, spos, rpos, dtype=np.float32, secondary=True)
    assert src.shape == (NTS, NX, NZ)
    assert rel_l2(src, rW) < 1e-5 and rel_l2(sec, rS) < 1e-5


def test_born_ext_saved_wavefields(api, setup):
    """BornExtShotsGpu.forwardWavefield / adjointWavefield with saveWavefield = 1 keep the coarse
    wavefields of shot wavefieldShotNumber (getSrcWfld / getSecWfld), equal to the oracle's."""
    st = setup
    par = api.params(nts=NTS, dts=DTS, sub=SUB, nz=NZ, nx=NX, zPadMinus=PAD, zPadPlus=PAD, xPadMinus=PAD,
                     xPadPlus=PAD, dz=10.0, dx=10.0, fMax=20.0, blockSize=16, fat=5, nShot=2, iGpu=[0], nExt=5,
                     extension="time", saveWavefield=1, wavefieldShotNumber=1)
    rng = np.random.default_rng(6)
    m = np.zeros((5, NX, NZ), np.float32)
    m[:, 5:-5, 5:-5] = rng.standard_normal((5, NXI, NZI))
    op = api.pyAcoustic_iso_float_born_ext.BornExtShotsGpu(st["v"], par, st["srcs"], [st["sig"]], [st["rec"]])
    model = api.vector(m, [(NZ, 0.0, 10.0), (NX, 0.0, 10.0), (5, -2 * DTS, DTS)])
    data = data_vec(api)
    op.forwardWavefield(False, model, data)
    spos, sig = oracle_source(st, st["srcs"][1], True)
    rpos = np.array(st["rec"].getRegPosUnique(), np.int32)
    _, rW, rS = orc.bornext_fwd(st["scheme"], st["vel"], m, sig, spos, rpos, dtype=np.float32, secondary=True)
    assert rel_l2(op.getSrcWfld().getNdArray(), rW) < 1e-5 and rel_l2(op.getSecWfld().getNdArray(), rS) < 1e-5
    d = (rng.standard_normal((2, 40, NTS)) * 1e-2).astype(np.float32)
    op.adjointWavefield(False, model, data_vec(api, d))
    dreg = np.zeros((len(rpos), NTS), np.float32)
    index = {p: i for i, p in enumerate(rpos)}
    for r in range(40):
        dreg[index[(8 + r) * NZ + 8]] = d[1, r]
    _, rW, rR = orc.bornext_adj(st["scheme"], st["vel"], dreg, sig, spos, rpos, dtype=np.float32, secondary=True)
    assert rel_l2(op.getSrcWfld().getNdArray(), rW) < 1e-5 and rel_l2(op.getSecWfld().getNdArray(), rR) < 1e-5
