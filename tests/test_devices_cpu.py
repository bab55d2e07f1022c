"""Off-grid devices (deviceGpu, F/src/deviceGpu.cpp): the C++ class against the oracle's
restatement of the reference's geometry. Corner indices, weights and the unique grid
points are integer / float work done with the reference's expression sequence, so the
bar is bit-exact; spread and gather accumulate in the reference's device-corner order
and are bit-exact too. The Kaiser-windowed sinc devices (an addition: the reference's
devices are bilinear) match the oracle's restatement to FP32 rounding. CPU only."""
import numpy as np
import pytest

import orc

NZ, NX, D = 42, 58, 10.0


@pytest.fixture(scope="module")
def api():
    from acoustic_isotropic_operators_b200 import reference_api
    return reference_api


def _vel(api, oz=0.0, ox=0.0):
    return api.vector(np.full((NX, NZ), 2000.0, np.float32), [(NZ, oz, D), (NX, ox, D)])


@pytest.mark.parametrize("dipole,zsh,xsh", [(0, 0.0, 0.0), (1, 30.0, 0.0), (1, 7.3, 12.9), (1, 0.0, 4.1)])
@pytest.mark.parametrize("origin", [(0.0, 0.0), (-25.0, 113.0)])
def test_bilinear_weights_bit_exact(api, dipole, zsh, xsh, origin):
    oz, ox = origin
    rng = np.random.default_rng(3 + dipole)
    n = 25
    z = (oz + rng.uniform(60.0, 300.0, n)).astype(np.float32)
    x = (ox + rng.uniform(60.0, 450.0, n)).astype(np.float32)
    z[:3] = oz + np.array([100.0, 150.0, 95.0], np.float32)   # on-node and half-cell coordinates
    x[:3] = ox + np.array([200.0, 205.0, 203.0], np.float32)
    nl = api.pyAcoustic_iso_float_nl
    dev = nl.deviceGpu(api.vector(z, [(n, 0, 1)]), api.vector(x, [(n, 0, 1)]), _vel(api, oz, ox), 16, dipole,
                       zsh, xsh)
    idx, w = orc.device_bilinear(z, x, NZ, oz, D, ox, D, dipole, zsh, xsh)
    assert np.array_equal(np.array(dev.getRegPos(), np.int32), idx)
    assert np.array_equal(np.array(dev.getWeights(), np.float32), w)   # bit-exact
    uniq, _ = orc.device_unique(idx)
    assert np.array_equal(np.array(dev.getRegPosUnique(), np.int32), uniq)
    assert dev.getNDeviceReg() == len(uniq) and dev.getNDeviceIrreg() == n
    # weights of every device (and of its dipole point) sum to 1 (-1)
    nc = 8 if dipole else 4
    assert np.allclose(w.reshape(n, nc)[:, :4].sum(1), 1.0, atol=1e-6)
    if dipole:
        assert np.allclose(w.reshape(n, nc)[:, 4:].sum(1), -1.0, atol=1e-6)


@pytest.mark.parametrize("dipole", [0, 1])
def test_grid_constructors_match_oracle(api, dipole):
    nl = api.pyAcoustic_iso_float_nl
    vel = _vel(api)
    iz, ix = [9, 9, 20, 33], [20, 21, 40, 7]
    d2 = nl.deviceGpu(iz, ix, vel, 16, dipole, 2, -1)
    idx, w = orc.device_on_grid(iz, ix, NZ, dipole, 2, -1)
    assert np.array_equal(np.array(d2.getRegPos(), np.int32), idx)
    assert np.array_equal(np.array(d2.getWeights(), np.float32), w)
    assert np.array_equal(np.array(d2.getRegPosUnique(), np.int32), orc.device_unique(idx)[0])
    # constructor #3: regular array, z fastest inside x
    d3 = nl.deviceGpu(3, 9, 2, 4, 10, 3, vel, 16, dipole, 1, 1)
    zz = [9 + 2 * k for _ in range(4) for k in range(3)]
    xx = [10 + 3 * j for j in range(4) for _ in range(3)]
    idx3, w3 = orc.device_on_grid(zz, xx, NZ, dipole, 1, 1)
    assert np.array_equal(np.array(d3.getRegPos(), np.int32), idx3)
    assert np.array_equal(np.array(d3.getWeights(), np.float32), w3)


@pytest.mark.parametrize("dipole", [0, 1])
def test_spread_gather_bit_exact(api, dipole):
    nl = api.pyAcoustic_iso_float_nl
    rng = np.random.default_rng(8)
    n, nt = 6, 24
    z = rng.uniform(50.0, 200.0, n).astype(np.float32)
    x = rng.uniform(50.0, 300.0, n).astype(np.float32)
    z[1], x[1] = z[0] + 4.0, x[0] + 3.0      # devices sharing corners: accumulation order matters
    dev = nl.deviceGpu(api.vector(z, [(n, 0, 1)]), api.vector(x, [(n, 0, 1)]), _vel(api), nt, dipole, 10.0, 10.0)
    idx, w = orc.device_bilinear(z, x, NZ, 0.0, D, 0.0, D, dipole, 10.0, 10.0)
    nc = 8 if dipole else 4
    sig = rng.standard_normal((n, nt)).astype(np.float32)
    irr = api.vector(sig, [(nt, 0, 1), (n, 0, 1)])
    reg = api.vector(None, [(nt, 0, 1), (dev.getNDeviceReg(), 0, 1)])
    dev.adjoint(False, reg, irr)
    _, want = orc.device_spread(idx, w, nc, sig)
    assert np.array_equal(reg.getNdArray(), want)
    back = api.vector(None, [(nt, 0, 1), (n, 0, 1)])
    dev.forward(False, reg, back)
    assert np.array_equal(back.getNdArray(), orc.device_gather(idx, w, nc, want))


def test_device_on_last_node_is_out_of_bounds(api):
    """A coordinate on the last node (or beyond) is rejected (F/src/deviceGpu.cpp:248-261)."""
    nl = api.pyAcoustic_iso_float_nl
    vel = _vel(api)
    zmax = (NZ - 1) * D
    with pytest.raises(RuntimeError, match="out of bounds"):
        nl.deviceGpu(api.vector([zmax], [(1, 0, 1)]), api.vector([100.0], [(1, 0, 1)]), vel, 16, 0, 0.0, 0.0)
    nl.deviceGpu(api.vector([zmax - 0.5], [(1, 0, 1)]), api.vector([100.0], [(1, 0, 1)]), vel, 16, 0, 0.0, 0.0)


@pytest.mark.parametrize("r,dipole", [(4, 0), (3, 1), (2, 0)])
def test_windowed_sinc_devices(api, r, dipole):
    """Kaiser-windowed sinc devices (Hicks 2002) against the oracle's restatement: same grid
    points, weights to FP32 rounding (both evaluate the window in double)."""
    nl = api.pyAcoustic_iso_float_nl
    rng = np.random.default_rng(10 + r)
    n = 7
    z = rng.uniform(80.0, 300.0, n).astype(np.float32)
    x = rng.uniform(80.0, 450.0, n).astype(np.float32)
    dev = nl.deviceGpu.windowedSinc(api.vector(z, [(n, 0, 1)]), api.vector(x, [(n, 0, 1)]), _vel(api), 16, r, 4.14,
                                    dipole, 13.0, 0.0)
    idx, w = orc.device_sinc(z, x, NZ, NX, 0.0, D, 0.0, D, r, 4.14, dipole, 13.0, 0.0)
    assert np.array_equal(np.array(dev.getRegPos(), np.int32), idx)
    assert np.allclose(np.array(dev.getWeights(), np.float32), w, rtol=1e-6, atol=1e-7)
    assert np.array_equal(np.array(dev.getRegPosUnique(), np.int32), orc.device_unique(idx)[0])
    npt = (2 * r) ** 2
    # a windowed sinc interpolates a constant to within a few per cent
    assert np.allclose(w.reshape(n, -1)[:, :npt].sum(1), 1.0, atol=0.05)
    reg = api.vector(None, [(16, 0, 1), (dev.getNDeviceReg(), 0, 1)])
    irr = api.vector(None, [(16, 0, 1), (n, 0, 1)])
    dev.setDomainRange(reg, irr)
    assert dev.dotTest(False, 1e-5)


def test_windowed_sinc_on_node_is_a_delta(api):
    nl = api.pyAcoustic_iso_float_nl
    z = np.array([100.0, 210.0], np.float32)
    x = np.array([200.0, 330.0], np.float32)
    dev = nl.deviceGpu.windowedSinc(api.vector(z, [(2, 0, 1)]), api.vector(x, [(2, 0, 1)]), _vel(api), 16)
    w = np.array(dev.getWeights(), np.float32).reshape(2, -1)
    pos = np.array(dev.getRegPos(), np.int32).reshape(2, -1)
    for i in range(2):
        k = int(np.argmax(np.abs(w[i])))
        assert w[i, k] == 1.0 and pos[i, k] == int(x[i] / D) * NZ + int(z[i] / D)
        assert np.max(np.abs(np.delete(w[i], k))) < 1e-7
    with pytest.raises(RuntimeError, match="out of bounds"):
        nl.deviceGpu.windowedSinc(api.vector([15.0], [(1, 0, 1)]), api.vector([200.0], [(1, 0, 1)]), _vel(api), 16)
