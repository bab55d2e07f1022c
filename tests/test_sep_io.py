"""SEP .H datasets and command-line parameters (the genericIO calls the reference's programs
and Python scripts make: getRegFile / getHyper / readFloatStream / writeDescription /
writeFloatStream, genericIO.defaultIO.getVector / writeVector, genericIO.io(params=argv)).
CPU only."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def api():
    from acoustic_isotropic_operators_b200 import reference_api
    return reference_api


def _keys(text):
    import shlex
    out = {}
    for tok in shlex.split(text):
        if "=" in tok:
            k, v = tok.split("=", 1)
            out[k] = v
    return out


@pytest.mark.parametrize("fmt,dt", [("xdr_float", ">f4"), ("native_float", "<f4")])
def test_write_read_round_trip(api, tmp_path, fmt, dt):
    rng = np.random.default_rng(0)
    vals = rng.standard_normal((3, 5, 7)).astype(np.float32)
    v = api.vector(vals, [(7, 0.0, 10.0), (5, -20.0, 12.5), (3, 0.0, 0.004)])
    h = str(tmp_path / "data.H")
    api.writeVector(h, v, fmt)
    k = _keys(open(h).read())
    assert (k["n1"], k["n2"], k["n3"]) == ("7", "5", "3")
    assert float(k["o2"]) == -20.0 and float(k["d2"]) == 12.5 and float(k["d3"]) == pytest.approx(0.004)
    assert k["esize"] == "4" and k["data_format"] == fmt and k["in"] == h + "@"
    raw = np.fromfile(h + "@", dtype=dt)
    assert np.array_equal(raw.astype(np.float32), vals.ravel())      # byte order of the format
    r = api.getVector(h)
    assert r.getHyper().getNdim() == 3
    assert np.array_equal(r.getNdArray(), vals)
    ax = r.getHyper().getAxis(2)
    assert (ax.n, ax.o, ax.d) == (5, -20.0, 12.5)


def test_hand_written_header(api, tmp_path):
    """A header as SEP tools write it: history lines, quoted values, a later n2 overriding an
    earlier one, trailing n3=1 (trimmed: a 2-D dataset), no data_format (xdr_float)."""
    vals = np.arange(12, dtype=np.float32).reshape(4, 3)
    (tmp_path / "vel.H@").write_bytes(vals.astype(">f4").tobytes())
    (tmp_path / "vel.H").write_text(
        '\nMakevel: version 1.0\n\t\tn1=3 o1=0 d1=10 label1="z [m]"\n\t\tn2=9 o2=0 d2=10\n'
        '\nWindow: \n\t\tn2=4 n3=1\n\t\tesize=4 in="' + str(tmp_path / "vel.H@") + '"\n')
    r = api.getVector(str(tmp_path / "vel.H"))
    assert r.getHyper().getNdim() == 2
    assert np.array_equal(r.getNdArray(), vals)
    r3 = api.getVector(str(tmp_path / "vel.H"), 3)      # padded to 3 axes
    assert r3.getHyper().getNdim() == 3 and r3.getNdArray().shape == (1, 4, 3)


def test_datapath(api, tmp_path, monkeypatch):
    dp = tmp_path / "dp"
    dp.mkdir()
    monkeypatch.setenv("DATAPATH", str(dp) + "/")
    v = api.vector(np.ones((2, 3), np.float32), [(3, 0, 1), (2, 0, 1)])
    api.writeVector(str(tmp_path / "m.H"), v)
    assert (dp / "m.H@").exists()
    assert np.array_equal(api.getVector(str(tmp_path / "m.H")).getNdArray(), np.ones((2, 3), np.float32))


def test_errors(api, tmp_path):
    (tmp_path / "a.H").write_text("n1=4 esize=8 in=a.H@\n")
    with pytest.raises(RuntimeError, match="esize"):
        api.getVector(str(tmp_path / "a.H"))
    (tmp_path / "b.H").write_text("n1=4\n")
    with pytest.raises(RuntimeError, match="in="):
        api.getVector(str(tmp_path / "b.H"))
    (tmp_path / "c.H@").write_bytes(np.zeros(3, ">f4").tobytes())
    (tmp_path / "c.H").write_text(f'n1=4 in="{tmp_path / "c.H@"}"\n')
    with pytest.raises(RuntimeError, match="fewer samples"):
        api.getVector(str(tmp_path / "c.H"))
    with pytest.raises(RuntimeError, match="cannot open"):
        api.getVector(str(tmp_path / "missing.H"))


def test_command_line_params(api, tmp_path):
    (tmp_path / "p.par").write_text("# propagation\nnts=100 dts=0.004 # coarse\nsub=4\niGpu=0,1,2\n")
    p = api.io(["prog", f"par={tmp_path / 'p.par'}", "nts=2000", "vel=vel.H"])
    assert p.getInt("nts", 0) == 2000           # later argument overrides the par file
    assert p.getFloat("dts", 0.0) == pytest.approx(0.004)
    assert p.getInt("sub", 0) == 4 and p.getInts("iGpu") == [0, 1, 2]
    assert p.getString("vel", "") == "vel.H" and p.getInt("missing", 7) == 7


def test_cpp_program_reads_and_writes(api, tmp_path):
    """A C++ program written the way the reference's mains use genericIO (ioModes ->
    getDefaultIO -> getParamObj / getRegFile(tag, usage) -> readFloatStream; setHyper ->
    writeDescription -> writeFloatStream) reads a dataset this module wrote and writes one
    it reads back."""
    src = r'''
#include "aio_sepio.hpp"
using namespace SEP;
int main(int argc, char** argv) {
    ioModes modes(argc, argv);
    std::shared_ptr<genericIO> io = modes.getDefaultIO();
    std::shared_ptr<paramObj> par = io->getParamObj();
    const float scale = par->getFloat("scale");
    std::shared_ptr<genericRegFile> velFile = io->getRegFile("vel", usageIn);
    std::shared_ptr<hypercube> velHyper = velFile->getHyper();
    std::shared_ptr<float2DReg> vel(new float2DReg(velHyper));
    velFile->readFloatStream(vel);
    vel->scale(scale);
    std::shared_ptr<genericRegFile> outFile = io->getRegFile(std::string("out"), usageOut);
    outFile->setHyper(velHyper);
    outFile->writeDescription();
    outFile->writeFloatStream(vel);
    return (*vel->_mat)[1][2] == scale * 5.f ? 0 : 3;
}
'''
    f = tmp_path / "prog.cpp"
    f.write_text(src)
    exe = tmp_path / "prog"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "acoustic_isotropic_operators_b200", "cpp"),
                    str(f), "-o", str(exe)], check=True)
    vals = np.arange(12, dtype=np.float32).reshape(4, 3)
    api.writeVector(str(tmp_path / "vel.H"), api.vector(vals, [(3, 0.0, 10.0), (4, 0.0, 10.0)]))
    subprocess.run([str(exe), f"vel={tmp_path / 'vel.H'}", f"out={tmp_path / 'out.H'}", "scale=2.5"], check=True)
    out = api.getVector(str(tmp_path / "out.H"))
    assert np.array_equal(out.getNdArray(), 2.5 * vals)
