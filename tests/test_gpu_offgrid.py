"""Off-grid devices on the GPU: sources and receivers at physical coordinates between grid
nodes (bilinear, F/src/deviceGpu.cpp:8-81), receivers as dipoles, through the
reference-named shot classes. The oracle chain is the oracle's own device geometry
(orc.device_bilinear, bit-exact with the C++ class, tests/test_devices_cpu.py) -> spread ->
d2/dt2 -> dtw^2 v^2 -> fine-time interpolation -> propagation at the unique grid points ->
gather. Kaiser-windowed sinc devices (deviceGpu.windowedSinc, 64 grid points per device) go
through the same chain with the oracle's sinc weights (orc.device_sinc). Gates: relative L2
1e-5 against the FP32 oracle; dot tests 1e-5.
"""
import numpy as np
import pytest

import orc
from cases import rel_l2
from test_gpu_operators import DTS, NTS, NX, NXI, NZ, NZI, SUB

pytestmark = pytest.mark.gpu

D = 10.0
NREC = 30


@pytest.fixture(scope="module")
def api():
    from acoustic_isotropic_operators_b200 import reference_api
    return reference_api


@pytest.fixture(scope="module")
def geo(api):
    rng = np.random.default_rng(21)
    zz = np.linspace(0, 1, NZ)[None, :]
    vel = (2000.0 + 400.0 * zz + 50.0 * rng.random((NX, NZ))).astype(np.float32)
    v = api.vector(vel, [(NZ, 0.0, D), (NX, 0.0, D)])
    nl = api.pyAcoustic_iso_float_nl
    # two shots, each one off-grid source; receivers off-grid along a line, as dipoles
    sz = [np.float32(93.7), np.float32(121.2)]
    sx = [np.float32(152.4), np.float32(388.9)]
    srcs = [nl.deviceGpu(api.vector([sz[i]], [(1, 0, 1)]), api.vector([sx[i]], [(1, 0, 1)]), v, NTS, 0, 0.0, 0.0)
            for i in range(2)]
    rz = np.full(NREC, 81.5, np.float32)
    rx = np.linspace(85.0, 470.0, NREC).astype(np.float32) + 0.37
    rec = nl.deviceGpu(api.vector(rz, [(NREC, 0, 1)]), api.vector(rx, [(NREC, 0, 1)]), v, NTS, 1, 10.0, 0.0)
    t = np.arange(NTS) * DTS - 0.05
    wav = ((1 - 2 * (np.pi * 15 * t) ** 2) * np.exp(-(np.pi * 15 * t) ** 2)).astype(np.float32)
    par = api.params(nts=NTS, dts=DTS, sub=SUB, nz=NZ, nx=NX, zPadMinus=8, zPadPlus=8, xPadMinus=8, xPadPlus=8,
                     dz=D, dx=D, fMax=20.0, blockSize=16, fat=5, nShot=2, iGpu=[0], nExt=5, leg1=1, leg2=1,
                     extension="time")
    s = orc.Scheme(nz=NZ, nx=NX, nts=NTS, dts=DTS, sub=SUB, dz=D, dx=D, minPad=8, nExt=5)
    src_geo = [orc.device_bilinear([sz[i]], [sx[i]], NZ, 0.0, D, 0.0, D) for i in range(2)]
    rec_geo = orc.device_bilinear(rz, rx, NZ, 0.0, D, 0.0, D, 1, 10.0, 0.0)
    return dict(vel=vel, v=v, srcs=srcs, rec=rec, wav=wav, par=par, scheme=s, src_geo=src_geo, rec_geo=rec_geo,
                sig=api.vector(wav[None, :], [(NTS, 0.0, DTS), (1, 0.0, 1.0)]))


def _source(g, i, d2):
    """Regular fine source traces of shot i through the oracle's host chain."""
    idx, w = g["src_geo"][i]
    pos, reg = orc.device_spread(idx, w, 4, g["wav"][None, :])
    if d2:
        reg = orc.second_deriv(NTS, DTS, reg, dtype=np.float32)
    dtw = np.float32(DTS / SUB)
    vflat = g["vel"].reshape(-1)
    reg = (reg * (dtw * dtw * vflat[pos] * vflat[pos])[:, None]).astype(np.float32)
    return pos, orc.time_interp_fwd(NTS, DTS, SUB, reg, dtype=np.float32)


def _rec_pos(g):
    return orc.device_unique(g["rec_geo"][0])[0]


def _gather(g, dreg):
    idx, w = g["rec_geo"]
    return orc.device_gather(idx, w, 8, dreg)


def _data(api, values=None):
    return api.vector(values, [(NTS, 0.0, DTS), (NREC, 0.0, 1.0), (2, 0.0, 1.0)])


def test_geometry_is_off_grid(geo):
    assert len(geo["src_geo"][0][0]) == 4 and np.all(geo["src_geo"][0][1] > 0)   # four live corners
    assert len(_rec_pos(geo)) > 2 * NREC                                           # dipole corners add points
    assert np.array_equal(np.array(geo["rec"].getRegPosUnique(), np.int32), _rec_pos(geo))


def test_nonlinear_off_grid(api, geo):
    op = api.pyAcoustic_iso_float_nl.nonlinearPropShotsGpu(geo["v"], geo["par"], geo["srcs"], [geo["rec"]])
    model = api.vector(geo["wav"][None, None, :], [(NTS, 0.0, DTS), (1, 0.0, 1.0), (1, 0.0, 1.0)])
    data = _data(api)
    op.forward(False, model, data)
    for i in range(2):
        spos, sig = _source(geo, i, False)
        want = _gather(geo, orc.nl_fwd(geo["scheme"], geo["vel"], sig, spos, _rec_pos(geo), dtype=np.float32))
        assert rel_l2(data.getNdArray()[i], want) < 1e-5
    m1 = api.vector(None, [(NTS, 0.0, DTS), (1, 0.0, 1.0), (2, 0.0, 1.0)])
    op.setDomainRange(m1, _data(api))
    assert op.dotTest(False, 1e-5)


def test_born_off_grid(api, geo):
    rng = np.random.default_rng(2)
    m = np.zeros((NX, NZ), np.float32)
    m[5:-5, 5:-5] = rng.standard_normal((NXI, NZI))
    op = api.pyAcoustic_iso_float_born.BornShotsGpu(geo["v"], geo["par"], geo["srcs"], [geo["sig"]], [geo["rec"]])
    model = api.vector(m, [(NZ, 0.0, D), (NX, 0.0, D)])
    data = _data(api)
    op.forward(False, model, data)
    got = data.getNdArray().copy()
    rpos = _rec_pos(geo)
    sigs = [_source(geo, i, True) for i in range(2)]
    for i in range(2):
        spos, sig = sigs[i]
        want = _gather(geo, orc.born_fwd(geo["scheme"], geo["vel"], m, sig, spos, rpos, dtype=np.float32))
        assert rel_l2(got[i], want) < 1e-5
    # adjoint: spread the data to the receiver corners (deviceGpu::adjoint), image, sum over shots
    d = (rng.standard_normal((2, NREC, NTS)) * 1e-2).astype(np.float32)
    img = api.vector(None, [(NZ, 0.0, D), (NX, 0.0, D)])
    op.adjoint(False, img, _data(api, d))
    idx, w = geo["rec_geo"]
    want = sum(orc.born_adj(geo["scheme"], geo["vel"], orc.device_spread(idx, w, 8, d[i])[1], sigs[i][1],
                            sigs[i][0], rpos, dtype=np.float32) for i in range(2))
    interior = np.zeros((NX, NZ), bool)
    interior[5:-5, 5:-5] = True
    assert rel_l2(img.getNdArray()[interior], want[interior]) < 1e-5
    op.setDomainRange(model, _data(api))
    assert op.dotTest(False, 1e-5)


def _sinc_devices(api, geo, r=4):
    nl = api.pyAcoustic_iso_float_nl
    sz, sx = [np.float32(93.7), np.float32(121.2)], [np.float32(152.4), np.float32(388.9)]
    srcs = [nl.deviceGpu.windowedSinc(api.vector([sz[i]], [(1, 0, 1)]), api.vector([sx[i]], [(1, 0, 1)]), geo["v"],
                                      NTS, r) for i in range(2)]
    rz = np.full(NREC, 81.5, np.float32)
    rx = np.linspace(85.0, 470.0, NREC).astype(np.float32) + 0.37
    rec = nl.deviceGpu.windowedSinc(api.vector(rz, [(NREC, 0, 1)]), api.vector(rx, [(NREC, 0, 1)]), geo["v"], NTS, r)
    sgeo = [orc.device_sinc([sz[i]], [sx[i]], NZ, NX, 0.0, D, 0.0, D, r) for i in range(2)]
    rgeo = orc.device_sinc(rz, rx, NZ, NX, 0.0, D, 0.0, D, r)
    return srcs, rec, sgeo, rgeo


def test_nonlinear_windowed_sinc(api, geo):
    """Kaiser-windowed sinc sources and receivers (64 grid points each) through the nonlinear
    shot class, against the oracle chain with the oracle's sinc weights; dot test."""
    srcs, rec, sgeo, rgeo = _sinc_devices(api, geo)
    op = api.pyAcoustic_iso_float_nl.nonlinearPropShotsGpu(geo["v"], geo["par"], srcs, [rec])
    model = api.vector(geo["wav"][None, None, :], [(NTS, 0.0, DTS), (1, 0.0, 1.0), (1, 0.0, 1.0)])
    data = _data(api)
    op.forward(False, model, data)
    nc_s, nc_r = len(sgeo[0][0]), len(rgeo[0]) // NREC
    rpos = orc.device_unique(rgeo[0])[0]
    dtw = np.float32(DTS / SUB)
    vflat = geo["vel"].reshape(-1)
    for i in range(2):
        pos, reg = orc.device_spread(sgeo[i][0], sgeo[i][1], nc_s, geo["wav"][None, :])
        reg = (reg * (dtw * dtw * vflat[pos] * vflat[pos])[:, None]).astype(np.float32)
        sig = orc.time_interp_fwd(NTS, DTS, SUB, reg, dtype=np.float32)
        dreg = orc.nl_fwd(geo["scheme"], geo["vel"], sig, pos, rpos, dtype=np.float32)
        want = orc.device_gather(rgeo[0], rgeo[1], nc_r, dreg)
        assert rel_l2(data.getNdArray()[i], want) < 1e-5
    m1 = api.vector(None, [(NTS, 0.0, DTS), (1, 0.0, 1.0), (2, 0.0, 1.0)])
    op.setDomainRange(m1, _data(api))
    assert op.dotTest(False, 1e-5)


def test_windowed_sinc_on_node_equals_grid_device(api, geo):
    """On grid nodes the windowed sinc is a delta: the same data as grid-point devices."""
    nl = api.pyAcoustic_iso_float_nl
    v = geo["v"]
    rz, rx = [8] * 20, list(range(10, 30))
    grid_src = [nl.deviceGpu([9], [15], v, NTS, 0, 0, 0), nl.deviceGpu([11], [40], v, NTS, 0, 0, 0)]
    grid_rec = nl.deviceGpu(rz, rx, v, NTS, 0, 0, 0)
    f = lambda a: api.vector(np.asarray(a, np.float32) * D, [(len(a), 0, 1)])  # noqa: E731
    sinc_src = [nl.deviceGpu.windowedSinc(f([9]), f([15]), v, NTS), nl.deviceGpu.windowedSinc(f([11]), f([40]), v, NTS)]
    sinc_rec = nl.deviceGpu.windowedSinc(f(rz), f(rx), v, NTS)
    model = api.vector(geo["wav"][None, None, :], [(NTS, 0.0, DTS), (1, 0.0, 1.0), (1, 0.0, 1.0)])
    out = []
    for s, r in ((grid_src, grid_rec), (sinc_src, sinc_rec)):
        op = api.pyAcoustic_iso_float_nl.nonlinearPropShotsGpu(v, geo["par"], s, [r])
        d = api.vector(None, [(NTS, 0.0, DTS), (20, 0.0, 1.0), (2, 0.0, 1.0)])
        op.forward(False, model, d)
        out.append(d.getNdArray().copy())
    assert rel_l2(out[1], out[0]) < 1e-6
