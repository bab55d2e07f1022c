"""The reference-named C seam of libaio_b200.so, driven the way the reference's per-shot
operators drive their GPU functions: init -> allocate -> shot calls -> deallocate
(F/src/nonlinearPropGpu.cpp:30-72, F/src/BornGpu.cpp:29-89, and the same sequence in
BornExtGpu.cpp, tomoExtGpu.cpp, wemvaExtGpu.cpp), through ctypes with the reference's own
argument lists (F/include/*ShotsGpuFunctions.h).

Every seam entry point of include/aio_b200.h is called here and its outputs are compared with
the reference's own drivers (oracle/_ref, compiled from the reference sources for sm_100a) given
the same arguments: relative L2 <= 1e-5 (the FP32 parity bar). Where the reference harness has
no counterpart of a driver (the free-surface subsurface-offset calls without wavefields, the
free-surface nonlinear wavefield calls), the FP32 oracle stands in, at the same bar.

Two slots (iGpu 0 and 1, both on device 0) and two families are alive at once, as in a
multi-GPU shot loop of the reference where every slot holds its own state.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

import orc
import refgpu
from cases import interior_mask, make_case, rel_l2

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refgpu.available(), reason="oracle/_ref not built (make -C oracle ref)")]

TOL = 1e-5
NEXT = 5


def _arg(a):
    if isinstance(a, float):
        return C.c_float(a)
    if isinstance(a, (bool, int, np.integer)):
        return C.c_int(int(a))
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous and a.dtype in (np.float32, np.int32)
        return a.ctypes.data_as(C.c_void_p)
    raise TypeError(type(a))


def seam(name, *args):
    """Call aio_<name>(*args) with C argument types; raise on a non-zero status."""
    from acoustic_isotropic_operators_b200 import _capi as A
    fn = getattr(A.lib(), "aio_" + name)
    rc = fn(*[_arg(a) for a in args])
    if rc != 0:
        raise A.AioError(rc, A.lib().aio_last_error().decode())


CASES = {
    # per-fine-step stepper (sub = 3)
    "fine": dict(seed=13, nts=40, nshots=1, nExt=NEXT),
    # interval-blocked stepper (sub = 4): two z-strips
    "blocked": dict(seed=14, nzi=160, nxi=192, nts=30, sub=4, nshots=1, nExt=NEXT, minPad=12),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    return make_case(**CASES[request.param])


def _geo(s):
    return (float(s.dz), float(s.dx), s.nz, s.nx, s.nts, float(s.dts), s.sub, s.minPad, 16, float(s.alphaCos))


def _consts(case):
    k = orc.constants(case.scheme, case.vel, dtype=np.float32)
    return np.ascontiguousarray(k["v2"], np.float32), np.ascontiguousarray(k["rs"], np.float32)


def _shot(case):
    return case.sig[0], case.src_pos[0], len(case.src_pos[0]), case.rec_pos[0], len(case.rec_pos[0])


def _zeros(*shape):
    return np.zeros(shape, np.float32)


def _rand(case, *shape, mask=False):
    a = case.rng.standard_normal(shape).astype(np.float32)
    if mask:
        a *= interior_mask(case.nx, case.nz)
    return np.ascontiguousarray(a)


def test_gpu_info():
    seam("getGpuInfo", np.array([0], np.int32), 1, 0, 0)
    with pytest.raises(Exception):
        seam("getGpuInfo", np.array([4096], np.int32), 1, 0, 0)


def test_nonlinear_two_slots_and_born_alive(case):
    s = case.scheme
    v2, rs = _consts(case)
    sig, sp, ns, rp, nr = _shot(case)
    seam("initNonlinearGpu", *_geo(s), 2, 0, 0)
    seam("allocateNonlinearGpu", v2, 0, 0)
    seam("allocateNonlinearGpu", v2, 1, 0)
    seam("initBornGpu", *_geo(s), 1, 0, 0)
    seam("allocateBornShotsGpu", v2, rs, 0, 0)
    try:
        ref = refgpu.nl_fwd(s, case.vel, sig, sp, rp)
        for slot in (0, 1):
            d = _zeros(nr, s.nts)
            seam("propShotsFwdGpu", sig, d, sp, ns, rp, nr, None, slot, 0)
            assert rel_l2(d, ref) < TOL
        # a Born call between two nonlinear calls: the families keep separate state
        m = _rand(case, case.nx, case.nz, mask=True)
        db = _zeros(nr, s.nts)
        seam("BornShotsFwdGpu", m, db, sig, sp, ns, rp, nr, None, None, 0, 0)
        assert rel_l2(db, refgpu.born_fwd(s, case.vel, m, sig, sp, rp)) < TOL
        rd, rW = refgpu.nl_fwd_wavefield(s, case.vel, sig, sp, rp)
        d, W = _zeros(nr, s.nts), _zeros(s.nts, s.nx, s.nz)
        seam("propShotsFwdGpuWavefield", sig, d, sp, ns, rp, nr, W, 1, 0)
        assert rel_l2(d, rd) < TOL and rel_l2(W, rW) < TOL
        data = _rand(case, nr, s.nts)
        ra = refgpu.nl_adj(s, case.vel, data, sp, rp)
        for slot in (0, 1):
            out = _zeros(ns, s.ntw)
            seam("propShotsAdjGpu", out, data, sp, ns, rp, nr, None, slot, 0)
            assert rel_l2(out, ra) < TOL
        ra, rW = refgpu.nl_adj_wavefield(s, case.vel, data, sp, rp)
        out, W = _zeros(ns, s.ntw), _zeros(s.nts, s.nx, s.nz)
        seam("propShotsAdjGpuWavefield", out, data, sp, ns, rp, nr, W, 0, 0)
        assert rel_l2(out, ra) < TOL and rel_l2(W, rW) < TOL
    finally:
        seam("deallocateNonlinearGpu", 0, 0)
        seam("deallocateNonlinearGpu", 1, 0)
        seam("deallocateBornShotsGpu", 0, 0)
    # a call after deallocate is a state error, not a crash
    with pytest.raises(Exception):
        seam("propShotsFwdGpu", sig, _zeros(nr, s.nts), sp, ns, rp, nr, None, 0, 0)


def test_nonlinear_free_surface(case):
    s = dataclasses.replace(case.scheme, freeSurface=1)
    v2, _ = _consts(case)
    sig, sp, ns, rp, nr = _shot(case)
    seam("initNonlinearGpu", *_geo(s), 1, 0, 0)
    seam("allocateNonlinearGpu", v2, 0, 0)
    try:
        d = _zeros(nr, s.nts)
        seam("propShotsFwdFsGpu", sig, d, sp, ns, rp, nr, None, 0, 0)
        assert rel_l2(d, refgpu.nl_fwd(s, case.vel, sig, sp, rp)) < TOL
        od, oW = orc.nl_fwd(s, case.vel, sig, sp, rp, dtype=np.float32, wavefield=True)
        d2, W = _zeros(nr, s.nts), _zeros(s.nts, s.nx, s.nz)
        seam("propShotsFwdFsGpuWavefield", sig, d2, sp, ns, rp, nr, W, 0, 0)
        assert rel_l2(d2, d) < TOL and rel_l2(W, oW) < TOL
        data = _rand(case, nr, s.nts)
        out = _zeros(ns, s.ntw)
        seam("propShotsAdjFsGpu", out, data, sp, ns, rp, nr, None, 0, 0)
        assert rel_l2(out, refgpu.nl_adj(s, case.vel, data, sp, rp)) < TOL
        om, oW = orc.nl_adj(s, case.vel, data, sp, rp, dtype=np.float32, wavefield=True)
        out2, W = _zeros(ns, s.ntw), _zeros(s.nts, s.nx, s.nz)
        seam("propShotsAdjFsGpuWavefield", out2, data, sp, ns, rp, nr, W, 0, 0)
        assert rel_l2(out2, out) < TOL and rel_l2(W, oW) < TOL
    finally:
        seam("deallocateNonlinearGpu", 0, 0)


def test_born(case):
    s = case.scheme
    v2, rs = _consts(case)
    sig, sp, ns, rp, nr = _shot(case)
    m = _rand(case, case.nx, case.nz, mask=True)
    data = _rand(case, nr, s.nts)
    seam("initBornGpu", *_geo(s), 1, 0, 0)
    seam("allocateBornShotsGpu", v2, rs, 0, 0)
    try:
        d = _zeros(nr, s.nts)
        seam("BornShotsFwdGpu", m, d, sig, sp, ns, rp, nr, None, None, 0, 0)
        assert rel_l2(d, refgpu.born_fwd(s, case.vel, m, sig, sp, rp)) < TOL
        img = _zeros(case.nx, case.nz)
        seam("BornShotsAdjGpu", img, data, sig, sp, ns, rp, nr, None, None, 0, 0)
        assert rel_l2(img, refgpu.born_adj(s, case.vel, data, sig, sp, rp)) < TOL
        rd, rW, rS = refgpu.born_fwd_wavefields(s, case.vel, m, sig, sp, rp)
        d, W, S = _zeros(nr, s.nts), _zeros(s.nts, s.nx, s.nz), _zeros(s.nts, s.nx, s.nz)
        seam("BornShotsFwdGpuWavefield", m, d, sig, sp, ns, rp, nr, W, S, 0, 0)
        assert rel_l2(d, rd) < TOL and rel_l2(W, rW) < TOL and rel_l2(S, rS) < TOL
        rm, _, rR = refgpu.born_adj_wavefields(s, case.vel, data, sig, sp, rp)
        img, W, R = _zeros(case.nx, case.nz), _zeros(s.nts, s.nx, s.nz), _zeros(s.nts, s.nx, s.nz)
        seam("BornShotsAdjGpuWavefield", img, data, sig, sp, ns, rp, nr, W, R, 0, 0)
        assert rel_l2(img, rm) < TOL and rel_l2(R, rR) < TOL
    finally:
        seam("deallocateBornShotsGpu", 0, 0)
    sf = dataclasses.replace(s, freeSurface=1)
    seam("initBornGpu", *_geo(sf), 1, 0, 0)
    seam("allocateBornShotsGpu", v2, rs, 0, 0)
    try:
        d = _zeros(nr, s.nts)
        seam("BornShotsFwdFsGpu", m, d, sig, sp, ns, rp, nr, None, None, 0, 0)
        assert rel_l2(d, refgpu.born_fwd(sf, case.vel, m, sig, sp, rp)) < TOL
        img = _zeros(case.nx, case.nz)
        seam("BornShotsAdjFsGpu", img, data, sig, sp, ns, rp, nr, None, None, 0, 0)
        assert rel_l2(img, refgpu.born_adj(sf, case.vel, data, sig, sp, rp)) < TOL
    finally:
        seam("deallocateBornShotsGpu", 0, 0)


def _ext_init(s, v2, rs):
    seam("initBornExtGpu", *_geo(s), s.nExt, 1, 0, 0)
    seam("allocateBornExtShotsGpu", v2, rs, 0, 0)


def test_born_ext_time(case):
    s = case.scheme
    v2, rs = _consts(case)
    sig, sp, ns, rp, nr = _shot(case)
    m = _rand(case, s.nExt, case.nx, case.nz, mask=True)
    data = _rand(case, nr, s.nts)
    _ext_init(s, v2, rs)
    try:
        for sloth in (0, 1):
            d = _zeros(nr, s.nts)
            seam("BornTimeShotsFwdGpu", m, d, sig, sp, ns, rp, nr, None, None, sloth, 0, 0)
            assert rel_l2(d, refgpu.bornext_fwd(s, case.vel, m, sig, sp, rp, sloth=sloth)) < TOL
            img = _zeros(s.nExt, case.nx, case.nz)
            seam("BornTimeShotsAdjGpu", img, data, sig, sp, ns, rp, nr, None, None, sloth, 0, 0)
            assert rel_l2(img, refgpu.bornext_adj(s, case.vel, data, sig, sp, rp, sloth=sloth)) < TOL
        sf = dataclasses.replace(s, freeSurface=1)
        d = _zeros(nr, s.nts)
        seam("BornTimeShotsFwdFsGpu", m, d, sig, sp, ns, rp, nr, None, None, 0, 0)
        assert rel_l2(d, refgpu.bornext_fwd(sf, case.vel, m, sig, sp, rp)) < TOL
        img = _zeros(s.nExt, case.nx, case.nz)
        seam("BornTimeShotsAdjFsGpu", img, data, sig, sp, ns, rp, nr, None, None, 0, 0)
        assert rel_l2(img, refgpu.bornext_adj(sf, case.vel, data, sig, sp, rp)) < TOL
    finally:
        seam("deallocateBornExtShotsGpu", 0, 0)


def test_born_ext_offset(case):
    s = case.scheme
    so = dataclasses.replace(s, extension=1)
    sof = dataclasses.replace(so, freeSurface=1)
    v2, rs = _consts(case)
    sig, sp, ns, rp, nr = _shot(case)
    m = _rand(case, s.nExt, case.nx, case.nz, mask=True)
    data = _rand(case, nr, s.nts)
    _ext_init(s, v2, rs)
    try:
        d = _zeros(nr, s.nts)
        seam("BornOffsetShotsFwdGpu", m, d, sig, sp, ns, rp, nr, None, None, 0, 0)
        assert rel_l2(d, refgpu.bornext_fwd(so, case.vel, m, sig, sp, rp)) < TOL
        img = _zeros(s.nExt, case.nx, case.nz)
        seam("BornOffsetShotsAdjGpu", img, data, sig, sp, ns, rp, nr, None, None, 0, 0)
        assert rel_l2(img, refgpu.bornext_adj(so, case.vel, data, sig, sp, rp)) < TOL
        d = _zeros(nr, s.nts)
        seam("BornOffsetShotsFwdFsGpu", m, d, sig, sp, ns, rp, nr, None, None, 0, 0)
        assert rel_l2(d, orc.bornext_fwd(sof, case.vel, m, sig, sp, rp, dtype=np.float32)) < TOL
        assert rel_l2(d, refgpu.bornext_fwd_wavefields(sof, case.vel, m, sig, sp, rp)[0]) < TOL
        img = _zeros(s.nExt, case.nx, case.nz)
        seam("BornOffsetShotsAdjFsGpu", img, data, sig, sp, ns, rp, nr, None, None, 0, 0)
        assert rel_l2(img, orc.bornext_adj(sof, case.vel, data, sig, sp, rp, dtype=np.float32)) < TOL
        assert rel_l2(img, refgpu.bornext_adj_wavefields(sof, case.vel, data, sig, sp, rp)[0]) < TOL
    finally:
        seam("deallocateBornExtShotsGpu", 0, 0)


WFLD = [("Time", False, False), ("Offset", True, False), ("TimeFs", False, True), ("OffsetFs", True, True)]


@pytest.mark.parametrize("kind,offset,fs", WFLD)
def test_born_ext_wavefields(case, kind, offset, fs):
    s = dataclasses.replace(case.scheme, extension=int(offset), freeSurface=int(fs))
    v2, rs = _consts(case)
    sig, sp, ns, rp, nr = _shot(case)
    m = _rand(case, s.nExt, case.nx, case.nz, mask=True)
    data = _rand(case, nr, s.nts)
    name = {"Time": "Time", "Offset": "Offset", "TimeFs": "Time", "OffsetFs": "Offset"}[kind]
    fsn = "Fs" if fs else ""
    _ext_init(case.scheme, v2, rs)
    try:
        rd, rW, rS = refgpu.bornext_fwd_wavefields(s, case.vel, m, sig, sp, rp)
        d, W, S = _zeros(nr, s.nts), _zeros(s.nts, s.nx, s.nz), _zeros(s.nts, s.nx, s.nz)
        seam(f"Born{name}ShotsFwd{fsn}GpuWavefield", m, d, sig, sp, ns, rp, nr, W, S, 0, 0)
        assert rel_l2(d, rd) < TOL and rel_l2(W, rW) < TOL and rel_l2(S, rS) < TOL
        rm, rW, rR = refgpu.bornext_adj_wavefields(s, case.vel, data, sig, sp, rp)
        img, W, R = _zeros(s.nExt, s.nx, s.nz), _zeros(s.nts, s.nx, s.nz), _zeros(s.nts, s.nx, s.nz)
        seam(f"Born{name}ShotsAdj{fsn}GpuWavefield", img, data, sig, sp, ns, rp, nr, W, R, 0, 0)
        assert rel_l2(img, rm) < TOL and rel_l2(W, rW) < TOL and rel_l2(R, rR) < TOL
    finally:
        seam("deallocateBornExtShotsGpu", 0, 0)


def test_tomo(case):
    s = case.scheme
    v2, rs = _consts(case)
    sig, sp, ns, rp, nr = _shot(case)
    dv = _rand(case, case.nx, case.nz, mask=True)
    ext = _rand(case, s.nExt, case.nx, case.nz, mask=True)
    data = _rand(case, nr, s.nts)
    seam("initTomoExtGpu", *_geo(s), s.nExt, 1, 1, 1, 0, 0)
    seam("allocateTomoExtShotsGpu", v2, rs, 0, 0)
    try:
        for sloth in (0, 1):
            d = _zeros(nr, s.nts)
            seam("tomoTimeShotsFwdGpu", dv, d, ext, sig, sp, ns, rp, nr, None, None, None, sloth, 0, 0, 0)
            assert rel_l2(d, refgpu.tomo_fwd(s, case.vel, dv, ext, sig, sp, rp, sloth=sloth)) < TOL
            out = _zeros(case.nx, case.nz)
            seam("tomoTimeShotsAdjGpu", out, data, ext, sig, sp, ns, rp, nr, None, None, None, sloth, 0, 0, 0)
            assert rel_l2(out, refgpu.tomo_adj(s, case.vel, data, ext, sig, sp, rp, sloth=sloth)) < TOL
        variants = [("tomoTimeShotsFwdFsGpu", "tomoTimeShotsAdjFsGpu", dict(freeSurface=1), True),
                    ("tomoOffsetShotsFwdGpu", "tomoOffsetShotsAdjGpu", dict(extension=1), True),
                    ("tomoOffsetShotsFwdFsGpu", "tomoOffsetShotsAdjFsGpu", dict(extension=1, freeSurface=1), False)]
        for fwd, adj, kw, has_ref in variants:
            sv = dataclasses.replace(s, **kw)
            d = _zeros(nr, s.nts)
            seam(fwd, dv, d, ext, sig, sp, ns, rp, nr, None, None, None, 0, 0, 0)
            want = (refgpu.tomo_fwd(sv, case.vel, dv, ext, sig, sp, rp) if has_ref else
                    orc.tomo_fwd(sv, case.vel, dv, ext, sig, sp, rp, dtype=np.float32))
            assert rel_l2(d, want) < TOL, fwd
            out = _zeros(case.nx, case.nz)
            seam(adj, out, data, ext, sig, sp, ns, rp, nr, None, None, None, 0, 0, 0)
            want = (refgpu.tomo_adj(sv, case.vel, data, ext, sig, sp, rp) if has_ref else
                    orc.tomo_adj(sv, case.vel, data, ext, sig, sp, rp, dtype=np.float32))
            assert rel_l2(out, want) < TOL, adj
    finally:
        seam("deallocateTomoExtShotsGpu", 0, 0)


def test_wemva(case):
    s = case.scheme
    v2, rs = _consts(case)
    sig, sp, ns, rp, nr = _shot(case)
    dv = _rand(case, case.nx, case.nz, mask=True)
    image = _rand(case, s.nExt, case.nx, case.nz, mask=True)
    rdata = _rand(case, nr, s.nts)
    seam("initWemvaExtGpu", *_geo(s), s.nExt, 1, 1, 1, 0, 0)
    seam("allocateWemvaExtShotsGpu", v2, rs, 0, 0)
    try:
        for kind, kw in (("Time", {}), ("Offset", dict(extension=1))):
            sv = dataclasses.replace(s, **kw)
            img = _zeros(s.nExt, case.nx, case.nz)
            seam(f"wemva{kind}ShotsFwdGpu", dv, img, sig, sp, ns, rdata, rp, nr, None, None, None, 0, 0, 0)
            assert rel_l2(img, refgpu.wemva_fwd(sv, case.vel, dv, sig, sp, rp, rdata)) < TOL
            out = _zeros(case.nx, case.nz)
            seam(f"wemva{kind}ShotsAdjGpu", out, image, sig, sp, ns, rdata, rp, nr, None, None, None, 0, 0, 0)
            assert rel_l2(out, refgpu.wemva_adj(sv, case.vel, image, sig, sp, rp, rdata)) < TOL
    finally:
        seam("deallocateWemvaExtShotsGpu", 0, 0)


def test_every_seam_entry_point_is_called():
    """The list of seam names above covers every reference-seam declaration of the header."""
    import os
    import re
    import inspect
    src = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                            "aio_b200.h")).read()
    block = src.split("-- reference seam")[1].split("aio_propShotsFwdGpu_noalloc")[0]
    block = re.sub(r"/\*.*?\*/", "", block, flags=re.S)
    declared = set(re.findall(r"\baio_([A-Za-z0-9_]+)\s*\(", block)) - {"dot_f64"}
    here = inspect.getsource(inspect.getmodule(test_every_seam_entry_point_is_called))
    called = set(re.findall(r'"([A-Za-z0-9_{}]+)"', here))
    expanded = set()
    for c in called:
        if "{" in c:
            for name in ("Time", "Offset"):
                for fsn in ("", "Fs"):
                    expanded.add(c.replace("{name}", name).replace("{fsn}", fsn).replace("{kind}", name))
        else:
            expanded.add(c)
    missing = sorted(declared - expanded)
    assert not missing, missing
