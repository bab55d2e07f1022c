"""ctypes binding of oracle/_ref: the reference's own GPU drivers compiled for
sm_100a (built by ``make -C oracle ref`` from the reference sources).

TEST INFRASTRUCTURE ONLY (parity checker). Each operator family is a separate
shared library because the reference keeps its state in per-translation-unit
globals. Every call here runs one shot through the reference's own free
functions: init -> allocate -> fwd/adj -> deallocate. A scheme with freeSurface = 1 runs the
reference's free-surface drivers (*FsGpu; the time-lag ones take no sloth flag); one with
extension = 1 runs its subsurface-offset drivers (*OffsetShots*Gpu).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")
_libs = {}


def available(family="born", dtype=np.float32) -> bool:
    return os.path.exists(_path(family, dtype))


def _path(family, dtype):
    suf = "f64" if np.dtype(dtype) == np.float64 else "f32"
    return os.path.join(REF_DIR, f"libref_{family}_{suf}.so")


def _lib(family, dtype):
    key = (family, np.dtype(dtype).name)
    if key not in _libs:
        L = C.CDLL(_path(family, dtype), mode=os.RTLD_LOCAL)
        R = C.c_double if np.dtype(dtype) == np.float64 else C.c_float
        L.ref_init.argtypes = [R, R, C.c_int, C.c_int, C.c_int, R, C.c_int, C.c_int, R, C.c_int, C.c_int, C.c_int,
                               C.c_int]
        _libs[key] = L
    return _libs[key]


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _run(family, s, vel, dtype, call, nExt=1, leg1=1, leg2=1, device=0):
    import orc
    L = _lib(family, dtype)
    k = orc.constants(s, vel, dtype=dtype)
    v2 = np.ascontiguousarray(k["v2"], dtype)
    rs = np.ascontiguousarray(k["rs"], dtype)
    rc = L.ref_init(s.dz, s.dx, s.nz, s.nx, s.nts, s.dts, s.sub, s.minPad, s.alphaCos, nExt, leg1, leg2, device)
    assert rc == 0, "reference init failed"
    assert L.ref_allocate(_p(v2), _p(rs), device) == 0
    try:
        out = call(L)
    finally:
        L.ref_deallocate(device)
    return out


def _fs(s):
    return bool(getattr(s, "freeSurface", 0))


def _off(s):
    return bool(getattr(s, "extension", 0))


def _i(a):
    return np.ascontiguousarray(a, np.int32)


def _a(a, dtype):
    return np.ascontiguousarray(a, dtype)


def nl_fwd(s, vel, model_dtw, sp, rp, dtype=np.float32):
    sp, rp = _i(sp), _i(rp)
    m = _a(model_dtw, dtype)
    d = np.zeros((len(rp), s.nts), dtype)
    _run("nl", s, vel, dtype, lambda L: (L.ref_nl_fwd_fs if _fs(s) else L.ref_nl_fwd)(
        _p(m), _p(d), _p(sp), len(sp), _p(rp), len(rp), None, 0))
    return d


def nl_adj(s, vel, data, sp, rp, dtype=np.float32):
    sp, rp = _i(sp), _i(rp)
    d = _a(data, dtype)
    m = np.zeros((len(sp), s.ntw), dtype)
    _run("nl", s, vel, dtype, lambda L: (L.ref_nl_adj_fs if _fs(s) else L.ref_nl_adj)(
        _p(m), _p(d), _p(sp), len(sp), _p(rp), len(rp), None, 0))
    return m


def nl_fwd_wavefield(s, vel, model_dtw, sp, rp, dtype=np.float32):
    """(data, coarse wavefield [nts][nx][nz]) from propShotsFwdGpuWavefield."""
    sp, rp = _i(sp), _i(rp)
    m = _a(model_dtw, dtype)
    d = np.zeros((len(rp), s.nts), dtype)
    W = np.zeros((s.nts, s.nx, s.nz), dtype)
    _run("nl", s, vel, dtype, lambda L: L.ref_nl_fwd(_p(m), _p(d), _p(sp), len(sp), _p(rp), len(rp), _p(W), 0))
    return d, W


def nl_adj_wavefield(s, vel, data, sp, rp, dtype=np.float32):
    """(fine source traces, coarse adjoint wavefield) from propShotsAdjGpuWavefield."""
    sp, rp = _i(sp), _i(rp)
    d = _a(data, dtype)
    m = np.zeros((len(sp), s.ntw), dtype)
    W = np.zeros((s.nts, s.nx, s.nz), dtype)
    _run("nl", s, vel, dtype, lambda L: L.ref_nl_adj(_p(m), _p(d), _p(sp), len(sp), _p(rp), len(rp), _p(W), 0))
    return m, W


def born_fwd(s, vel, model, sig, sp, rp, dtype=np.float32):
    sp, rp = _i(sp), _i(rp)
    m, g = _a(model, dtype), _a(sig, dtype)
    d = np.zeros((len(rp), s.nts), dtype)
    _run("born", s, vel, dtype, lambda L: (L.ref_born_fwd_fs if _fs(s) else L.ref_born_fwd)(
        _p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0))
    return d


def born_adj(s, vel, data, sig, sp, rp, dtype=np.float32):
    sp, rp = _i(sp), _i(rp)
    d, g = _a(data, dtype), _a(sig, dtype)
    m = np.zeros((s.nx, s.nz), dtype)
    _run("born", s, vel, dtype, lambda L: (L.ref_born_adj_fs if _fs(s) else L.ref_born_adj)(
        _p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0))
    return m


def born_fwd_wavefields(s, vel, model, sig, sp, rp, dtype=np.float32):
    """(data, source wavefield, scattered wavefield) from BornShotsFwdGpuWavefield."""
    sp, rp = _i(sp), _i(rp)
    m, g = _a(model, dtype), _a(sig, dtype)
    d = np.zeros((len(rp), s.nts), dtype)
    W = np.zeros((s.nts, s.nx, s.nz), dtype)
    S = np.zeros_like(W)
    _run("born", s, vel, dtype, lambda L: L.ref_born_fwd_wfld(_p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp),
                                                              _p(W), _p(S), 0))
    return d, W, S


def born_adj_wavefields(s, vel, data, sig, sp, rp, dtype=np.float32):
    """(image, source wavefield, scaled receiver wavefield) from BornShotsAdjGpuWavefield."""
    sp, rp = _i(sp), _i(rp)
    d, g = _a(data, dtype), _a(sig, dtype)
    m = np.zeros((s.nx, s.nz), dtype)
    W = np.zeros((s.nts, s.nx, s.nz), dtype)
    R = np.zeros_like(W)
    _run("born", s, vel, dtype, lambda L: L.ref_born_adj_wfld(_p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp),
                                                              _p(W), _p(R), 0))
    return m, W, R


def bornext_fwd(s, vel, model, sig, sp, rp, sloth=0, dtype=np.float32):
    sp, rp = _i(sp), _i(rp)
    m, g = _a(model, dtype), _a(sig, dtype)
    d = np.zeros((len(rp), s.nts), dtype)
    _run("bornext", s, vel, dtype,
         lambda L: L.ref_bornext_fwd_off(_p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0) if _off(s) else
         L.ref_bornext_fwd_fs(_p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0) if _fs(s) else
         L.ref_bornext_fwd(_p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp), sloth, 0), nExt=s.nExt)
    return d


def bornext_adj(s, vel, data, sig, sp, rp, sloth=0, dtype=np.float32):
    sp, rp = _i(sp), _i(rp)
    d, g = _a(data, dtype), _a(sig, dtype)
    m = np.zeros((s.nExt, s.nx, s.nz), dtype)
    _run("bornext", s, vel, dtype,
         lambda L: L.ref_bornext_adj_off(_p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0) if _off(s) else
         L.ref_bornext_adj_fs(_p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0) if _fs(s) else
         L.ref_bornext_adj(_p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp), sloth, 0), nExt=s.nExt)
    return m


def bornext_fwd_wavefields(s, vel, model, sig, sp, rp, dtype=np.float32):
    """(data, source wavefield, scattered wavefield) from the extended Born forward wavefield drivers
    (time lags or offsets, with or without the free surface, by the scheme)."""
    sp, rp = _i(sp), _i(rp)
    m, g = _a(model, dtype), _a(sig, dtype)
    d = np.zeros((len(rp), s.nts), dtype)
    W = np.zeros((s.nts, s.nx, s.nz), dtype)
    S = np.zeros_like(W)
    _run("bornext", s, vel, dtype,
         lambda L: L.ref_bornext_fwd_wfld(_p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp), _p(W), _p(S),
                                          int(_off(s)), int(_fs(s)), 0), nExt=s.nExt)
    return d, W, S


def bornext_adj_wavefields(s, vel, data, sig, sp, rp, dtype=np.float32):
    """(image, source wavefield, receiver wavefield) from the extended Born adjoint wavefield drivers."""
    sp, rp = _i(sp), _i(rp)
    d, g = _a(data, dtype), _a(sig, dtype)
    m = np.zeros((s.nExt, s.nx, s.nz), dtype)
    W = np.zeros((s.nts, s.nx, s.nz), dtype)
    R = np.zeros_like(W)
    _run("bornext", s, vel, dtype,
         lambda L: L.ref_bornext_adj_wfld(_p(m), _p(d), _p(g), _p(sp), len(sp), _p(rp), len(rp), _p(W), _p(R),
                                          int(_off(s)), int(_fs(s)), 0), nExt=s.nExt)
    return m, W, R


def tomo_fwd(s, vel, model, ext, sig, sp, rp, sloth=0, leg1=1, leg2=1, dtype=np.float32):
    sp, rp = _i(sp), _i(rp)
    m, e, g = _a(model, dtype), _a(ext, dtype), _a(sig, dtype)
    d = np.zeros((len(rp), s.nts), dtype)
    _run("tomo", s, vel, dtype,
         lambda L: L.ref_tomo_fwd_off(_p(m), _p(d), _p(e), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0) if _off(s) else
         L.ref_tomo_fwd_fs(_p(m), _p(d), _p(e), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0) if _fs(s) else
         L.ref_tomo_fwd(_p(m), _p(d), _p(e), _p(g), _p(sp), len(sp), _p(rp), len(rp), sloth, 0),
         nExt=s.nExt, leg1=leg1, leg2=leg2)
    return d


def tomo_adj(s, vel, data, ext, sig, sp, rp, sloth=0, leg1=1, leg2=1, dtype=np.float32):
    sp, rp = _i(sp), _i(rp)
    d, e, g = _a(data, dtype), _a(ext, dtype), _a(sig, dtype)
    m = np.zeros((s.nx, s.nz), dtype)
    _run("tomo", s, vel, dtype,
         lambda L: L.ref_tomo_adj_off(_p(m), _p(d), _p(e), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0) if _off(s) else
         L.ref_tomo_adj_fs(_p(m), _p(d), _p(e), _p(g), _p(sp), len(sp), _p(rp), len(rp), 0) if _fs(s) else
         L.ref_tomo_adj(_p(m), _p(d), _p(e), _p(g), _p(sp), len(sp), _p(rp), len(rp), sloth, 0),
         nExt=s.nExt, leg1=leg1, leg2=leg2)
    return m


def wemva_fwd(s, vel, model, sig, sp, rp, rdata, leg1=1, leg2=1, dtype=np.float32):
    sp, rp = _i(sp), _i(rp)
    m, g, r = _a(model, dtype), _a(sig, dtype), _a(rdata, dtype)
    img = np.zeros((s.nExt, s.nx, s.nz), dtype)
    _run("wemva", s, vel, dtype,
         lambda L: (L.ref_wemva_fwd_off if _off(s) else L.ref_wemva_fwd)(
             _p(m), _p(img), _p(g), _p(sp), len(sp), _p(r), _p(rp), len(rp), 0),
         nExt=s.nExt, leg1=leg1, leg2=leg2)
    return img


def wemva_adj(s, vel, image, sig, sp, rp, rdata, leg1=1, leg2=1, dtype=np.float32):
    sp, rp = _i(sp), _i(rp)
    img, g, r = _a(image, dtype), _a(sig, dtype), _a(rdata, dtype)
    m = np.zeros((s.nx, s.nz), dtype)
    _run("wemva", s, vel, dtype,
         lambda L: (L.ref_wemva_adj_off if _off(s) else L.ref_wemva_adj)(
             _p(m), _p(img), _p(g), _p(sp), len(sp), _p(r), _p(rp), len(rp), 0),
         nExt=s.nExt, leg1=leg1, leg2=leg2)
    return m


def _w3(s, dtype):
    return [np.zeros((s.nts, s.nx, s.nz), dtype) for _ in range(3)]


def tomo_fwd_wavefields(s, vel, model, ext, sig, sp, rp, sloth=0, leg1=1, leg2=1, dtype=np.float32):
    """(data, source d2/dt2, secondary 1, secondary 2) from the tomo forward drivers with
    saveWavefield = 1 (time lags or offsets, with or without the free surface, by the scheme)."""
    sp, rp = _i(sp), _i(rp)
    m, e, g = _a(model, dtype), _a(ext, dtype), _a(sig, dtype)
    d = np.zeros((len(rp), s.nts), dtype)
    W = _w3(s, dtype)
    _run("tomo", s, vel, dtype, lambda L: L.ref_tomo_fwd_wfld(_p(m), _p(d), _p(e), _p(g), _p(sp), len(sp), _p(rp),
                                                              len(rp), *[_p(x) for x in W], int(_off(s)),
                                                              int(_fs(s)), sloth, 0),
         nExt=s.nExt, leg1=leg1, leg2=leg2)
    return (d, *W)


def tomo_adj_wavefields(s, vel, data, ext, sig, sp, rp, sloth=0, leg1=1, leg2=1, dtype=np.float32):
    """(model, source d2/dt2, receiver wavefield, the last leg's scattered coarse samples) from
    the tomo adjoint drivers with saveWavefield = 1."""
    sp, rp = _i(sp), _i(rp)
    d, e, g = _a(data, dtype), _a(ext, dtype), _a(sig, dtype)
    m = np.zeros((s.nx, s.nz), dtype)
    W = _w3(s, dtype)
    _run("tomo", s, vel, dtype, lambda L: L.ref_tomo_adj_wfld(_p(m), _p(d), _p(e), _p(g), _p(sp), len(sp), _p(rp),
                                                              len(rp), *[_p(x) for x in W], int(_off(s)),
                                                              int(_fs(s)), sloth, 0),
         nExt=s.nExt, leg1=leg1, leg2=leg2)
    return (m, *W)


def wemva_fwd_wavefields(s, vel, model, sig, sp, rp, rdata, leg1=1, leg2=1, dtype=np.float32):
    """(image, source d2/dt2, receiver wavefield, the last leg's scattered coarse samples) from
    the WEMVA forward drivers with saveWavefield = 1."""
    sp, rp = _i(sp), _i(rp)
    m, g, r = _a(model, dtype), _a(sig, dtype), _a(rdata, dtype)
    img = np.zeros((s.nExt, s.nx, s.nz), dtype)
    W = _w3(s, dtype)
    _run("wemva", s, vel, dtype, lambda L: L.ref_wemva_fwd_wfld(_p(m), _p(img), _p(g), _p(sp), len(sp), _p(r), _p(rp),
                                                                len(rp), *[_p(x) for x in W], int(_off(s)), 0),
         nExt=s.nExt, leg1=leg1, leg2=leg2)
    return (img, *W)


def wemva_adj_wavefields(s, vel, image, sig, sp, rp, rdata, leg1=1, leg2=1, dtype=np.float32):
    """(model, source d2/dt2, receiver wavefield, the last leg's scattered coarse samples) from
    the WEMVA adjoint drivers with saveWavefield = 1."""
    sp, rp = _i(sp), _i(rp)
    img, g, r = _a(image, dtype), _a(sig, dtype), _a(rdata, dtype)
    m = np.zeros((s.nx, s.nz), dtype)
    W = _w3(s, dtype)
    _run("wemva", s, vel, dtype, lambda L: L.ref_wemva_adj_wfld(_p(m), _p(img), _p(g), _p(sp), len(sp), _p(r), _p(rp),
                                                                len(rp), *[_p(x) for x in W], int(_off(s)), 0),
         nExt=s.nExt, leg1=leg1, leg2=leg2)
    return (m, *W)
