"""Reference-named operator layer on CPU: SEP containers, parameter objects,
deviceGpu geometry (all three constructors) and the fdParam checks. No GPU
work: constructing a shot-loop operator on a machine without a GPU must raise
a clean RuntimeError."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def api():
    from acoustic_isotropic_operators_b200 import reference_api
    return reference_api


def vel_vec(api, nz=42, nx=58, d=10.0, v=2000.0):
    return api.vector(np.full((nx, nz), v, np.float32), [(nz, 0.0, d), (nx, 0.0, d)])


def test_sep_vectors(api):
    a = api.vector(np.arange(12, dtype=np.float32).reshape(3, 4), [(4, 0, 1), (3, 0, 1)])
    b = a.clone()
    assert a.dot(b) == pytest.approx(float(np.sum(np.arange(12.0) ** 2)))
    b.scaleAdd(a, 2.0, -1.0)          # b = 2b - a = a
    assert np.array_equal(b.getNdArray(), a.getNdArray())
    c = a.cloneSpace()
    assert c.getNdArray().shape == (3, 4) and not c.getNdArray().any()
    assert a.getHyper().getAxis(1).n == 4 and a.getHyper().getAxis(2).n == 3
    assert a.max() == 11 and a.min() == 0


def test_device_constructors(api):
    nl = api.pyAcoustic_iso_float_nl
    vel = vel_vec(api)
    nt = 30
    # grid points: one device -> its 4 corners are the unique regular points
    d2 = nl.deviceGpu([9, 9], [20, 21], vel, nt, 0, 0, 0)
    assert d2.getNDeviceIrreg() == 2
    pos = d2.getRegPosUnique()
    nz = 42
    assert pos[:4] == [20 * nz + 9, 20 * nz + 10, 21 * nz + 9, 21 * nz + 10]
    assert d2.getNDeviceReg() == 6          # shared corners counted once
    # regular array constructor
    d3 = nl.deviceGpu(1, 9, 1, 3, 10, 2, vel, nt, 0, 0, 0)
    assert d3.getNDeviceIrreg() == 3
    # coordinates (bilinear), with a dipole
    z = api.vector([95.0], [(1, 0, 1)])
    x = api.vector([203.0], [(1, 0, 1)])
    d1 = nl.deviceGpu(z, x, vel, nt, 1, 30.0, 0.0)   # dipole 3 cells below: no shared corners
    assert d1.getNDeviceIrreg() == 1 and d1.getNDeviceReg() == 8


def test_device_out_of_bounds(api):
    nl = api.pyAcoustic_iso_float_nl
    vel = vel_vec(api)
    with pytest.raises(RuntimeError):
        nl.deviceGpu([42], [5], vel, 30, 0, 0, 0)   # z index == nz


def test_spread_gather_adjoint(api):
    """deviceGpu forward (grid -> devices) and adjoint are transposes (dot test)."""
    nl = api.pyAcoustic_iso_float_nl
    vel = vel_vec(api)
    z = api.vector([95.0, 133.3], [(2, 0, 1)])
    x = api.vector([203.7, 211.1], [(2, 0, 1)])
    d = nl.deviceGpu(z, x, vel, 16, 0, 0.0, 0.0)
    reg = api.vector(None, [(16, 0, 1), (d.getNDeviceReg(), 0, 1)])
    irr = api.vector(None, [(16, 0, 1), (2, 0, 1)])
    d.setDomainRange(reg, irr)
    assert d.dotTest(False, 1e-5)


def _par(api, **over):
    p = dict(nts=40, dts=0.004, sub=3, nz=42, nx=58, zPadMinus=8, zPadPlus=8, xPadMinus=8, xPadPlus=8, dz=10.0,
             dx=10.0, fMax=20.0, blockSize=16, fat=5, nShot=1, iGpu=[0])
    p.update(over)
    return api.params(**p)


def test_shot_operator_without_gpu_raises(api):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    born = api.pyAcoustic_iso_float_born
    nl = api.pyAcoustic_iso_float_nl
    vel = vel_vec(api, nz=42, nx=58)
    src = nl.deviceGpu([9], [20], vel, 40, 0, 0, 0)
    rec = nl.deviceGpu([8] * 10, list(range(10, 20)), vel, 40, 0, 0, 0)
    sig = api.vector(np.zeros((1, 40), np.float32), [(40, 0, 0.004), (1, 0, 1)])
    with pytest.raises(RuntimeError):
        born.BornShotsGpu(vel, _par(api), [src], [sig], [rec])


def test_gpu_list_rules(api):
    """Duplicate GPU ids and a missing GPU list are rejected before any device call."""
    born = api.pyAcoustic_iso_float_born
    nl = api.pyAcoustic_iso_float_nl
    vel = vel_vec(api)
    src = nl.deviceGpu([9], [20], vel, 40, 0, 0, 0)
    sig = api.vector(np.zeros((1, 40), np.float32), [(40, 0, 0.004), (1, 0, 1)])
    with pytest.raises(RuntimeError, match="duplicates"):
        born.BornShotsGpu(vel, _par(api, iGpu=[0, 0]), [src], [sig], [src])
    p = _par(api)
    with pytest.raises(RuntimeError, match="list of GPUs"):
        born.BornShotsGpu(vel, api.params(nShot=1), [src], [sig], [src])


def test_cpp_headers_compile():
    """The C++ operator layer and the reference-named seam shims compile as a program would use them."""
    import os
    import subprocess
    import tempfile
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = ('#include "aio_reference_seam.hpp"\n#include "aio_shots.hpp"\n'
           'int main() { std::vector<int> g{0}; (void)getGpuInfo(g, 0, 0); return 0; }\n')
    with tempfile.TemporaryDirectory() as d:
        f = os.path.join(d, "t.cpp")
        open(f, "w").write(src)
        subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(root, "include"), "-I",
                        os.path.join(root, "acoustic_isotropic_operators_b200", "cpp"), f], check=True)
