"""ctypes binding of the CPU oracle (oracle/aio_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker. The product path never uses it.

Every function works at the reference's regular-grid seam: slices are
(nx, nz) float arrays with z fastest (the reference's ``index = ix*nz + iz``),
traces are (nDevice, nt) with time fastest, device positions are linear grid
indices. ``dtype`` selects the FP32 restatement (float32) or the FP64 one
(float64, the reference's acoustic_iso_double scheme).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


class OrcParams(C.Structure):
    _fields_ = [("nz", C.c_int), ("nx", C.c_int), ("nts", C.c_int), ("sub", C.c_int),
                ("minPad", C.c_int), ("nExt", C.c_int), ("dz", C.c_double), ("dx", C.c_double),
                ("dts", C.c_double), ("alphaCos", C.c_double), ("freeSurface", C.c_int), ("extension", C.c_int)]


def build() -> str:
    """Compile liboracle.so with g++ (no GPU needed)."""
    subprocess.check_call(["make", "-s", "-C", _HERE, "liboracle.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
    return _lib


@dataclass
class Scheme:
    """Grid and time parameters of one operator instance (reference par keys)."""
    nz: int
    nx: int
    nts: int
    dts: float
    sub: int
    dz: float
    dx: float
    minPad: int
    alphaCos: float = 0.99
    nExt: int = 1
    freeSurface: int = 0
    extension: int = 0  # 0 time lags, 1 subsurface offsets

    @property
    def ntw(self) -> int:
        return (self.nts - 1) * self.sub + 1

    def c(self) -> OrcParams:
        return OrcParams(self.nz, self.nx, self.nts, self.sub, self.minPad, self.nExt,
                         self.dz, self.dx, self.dts, self.alphaCos, self.freeSurface, self.extension)


def _suf(dtype) -> str:
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _ip(a):
    return np.ascontiguousarray(a, dtype=np.int32).ctypes.data_as(C.c_void_p)


def _arr(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


def constants(s: Scheme, vel, dtype=np.float64):
    vel = _arr(vel, dtype)
    zc = np.zeros(6, dtype); xc = np.zeros(6, dtype)
    h = np.zeros(2 * (s.sub + 1), dtype); taper = np.zeros(max(s.minPad, 1), dtype)
    v2 = np.zeros_like(vel); rs = np.zeros_like(vel)
    getattr(lib(), "orc_constants_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(zc), _p(xc), _p(h), _p(taper),
                                                   _p(v2), _p(rs))
    return dict(zc=zc, xc=xc, h=h, taper=taper[: s.minPad], v2=v2, rs=rs)


def nl_fwd(s, vel, model_dtw, src_pos, rec_pos, dtype=np.float64, wavefield=False):
    vel = _arr(vel, dtype); m = _arr(model_dtw, dtype)
    nr = len(rec_pos)
    d = np.zeros((nr, s.nts), dtype)
    W = np.zeros((s.nts, s.nx, s.nz), dtype) if wavefield else None
    getattr(lib(), "orc_nl_fwd_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _ip(src_pos), len(src_pos),
                                                _ip(rec_pos), nr, _p(d), _p(W) if W is not None else None)
    return (d, W) if wavefield else d


def nl_adj(s, vel, data, src_pos, rec_pos, dtype=np.float64, wavefield=False):
    vel = _arr(vel, dtype); d = _arr(data, dtype)
    m = np.zeros((len(src_pos), s.ntw), dtype)
    W = np.zeros((s.nts, s.nx, s.nz), dtype) if wavefield else None
    getattr(lib(), "orc_nl_adj_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _ip(src_pos), len(src_pos),
                                                _ip(rec_pos), len(rec_pos), _p(d), _p(W) if W is not None else None)
    return (m, W) if wavefield else m


def born_fwd(s, vel, model, sig_dtw, src_pos, rec_pos, dtype=np.float64, wavefield=False, secondary=False):
    """Born forward data; wavefield=True also returns the coarse source wavefield, secondary=True
    also the coarse scattered wavefield ((nts, nx, nz) each)."""
    vel = _arr(vel, dtype); m = _arr(model, dtype); sig = _arr(sig_dtw, dtype)
    d = np.zeros((len(rec_pos), s.nts), dtype)
    W = np.zeros((s.nts, s.nx, s.nz), dtype) if (wavefield or secondary) else None
    S = np.zeros((s.nts, s.nx, s.nz), dtype) if secondary else None
    getattr(lib(), "orc_born_fwd_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _p(sig), _ip(src_pos),
                                                  len(src_pos), _ip(rec_pos), len(rec_pos), _p(d),
                                                  _p(W) if W is not None else None, _p(S) if S is not None else None)
    if secondary:
        return d, W, S
    return (d, W) if wavefield else d


def born_adj(s, vel, data, sig_dtw, src_pos, rec_pos, dtype=np.float64, wavefield=False, secondary=False):
    """Born adjoint image; wavefield=True also returns the coarse source wavefield, secondary=True
    also the scaled coarse receiver wavefield ((nts, nx, nz) each)."""
    vel = _arr(vel, dtype); d = _arr(data, dtype); sig = _arr(sig_dtw, dtype)
    m = np.zeros((s.nx, s.nz), dtype)
    W = np.zeros((s.nts, s.nx, s.nz), dtype) if (wavefield or secondary) else None
    R = np.zeros((s.nts, s.nx, s.nz), dtype) if secondary else None
    getattr(lib(), "orc_born_adj_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _p(sig), _ip(src_pos),
                                                  len(src_pos), _ip(rec_pos), len(rec_pos), _p(d),
                                                  _p(W) if W is not None else None, _p(R) if R is not None else None)
    if secondary:
        return m, W, R
    return (m, W) if wavefield else m


def bornext_fwd(s, vel, model_ext, sig_dtw, src_pos, rec_pos, dtype=np.float64, sloth=0, secondary=False):
    """Extended Born forward data; secondary=True (non-sloth scaling, as the reference's wavefield
    drivers) returns (data, coarse source wavefield, coarse scattered wavefield)."""
    vel = _arr(vel, dtype); m = _arr(model_ext, dtype); sig = _arr(sig_dtw, dtype)
    d = np.zeros((len(rec_pos), s.nts), dtype)
    if secondary:
        W = np.zeros((s.nts, s.nx, s.nz), dtype)
        S = np.zeros_like(W)
        getattr(lib(), "orc_bornext_fwd_wfld_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _p(sig),
                                                              _ip(src_pos), len(src_pos), _ip(rec_pos),
                                                              len(rec_pos), _p(d), _p(W), _p(S))
        return d, W, S
    getattr(lib(), "orc_bornext_fwd_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _p(sig), _ip(src_pos),
                                                     len(src_pos), _ip(rec_pos), len(rec_pos), _p(d), sloth)
    return d


def bornext_adj(s, vel, data, sig_dtw, src_pos, rec_pos, dtype=np.float64, sloth=0, secondary=False):
    """Extended Born adjoint image; secondary=True (non-sloth scaling) returns (image, coarse source
    wavefield, receiver wavefield: scaled by 2/v^3 v^2 dtw^2 for time lags, by v^2 dtw^2 for offsets)."""
    vel = _arr(vel, dtype); d = _arr(data, dtype); sig = _arr(sig_dtw, dtype)
    m = np.zeros((s.nExt, s.nx, s.nz), dtype)
    if secondary:
        W = np.zeros((s.nts, s.nx, s.nz), dtype)
        R = np.zeros_like(W)
        getattr(lib(), "orc_bornext_adj_wfld_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _p(sig),
                                                              _ip(src_pos), len(src_pos), _ip(rec_pos),
                                                              len(rec_pos), _p(d), _p(W), _p(R))
        return m, W, R
    getattr(lib(), "orc_bornext_adj_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _p(sig), _ip(src_pos),
                                                     len(src_pos), _ip(rec_pos), len(rec_pos), _p(d), sloth)
    return m


def _wfld(s, dtype, on):
    """Three [nts][nx][nz] arrays for saved wavefields (and their pointers), or null pointers."""
    if not on:
        return [], [None, None, None]
    W = [np.zeros((s.nts, s.nx, s.nz), dtype) for _ in range(3)]
    return W, [_p(x) for x in W]


def tomo_fwd(s, vel, model, ext_refl, sig_dtw, src_pos, rec_pos, dtype=np.float64, sloth=0, leg1=1, leg2=1,
             wavefields=False):
    """Tomo forward data; with wavefields=True (data, source d2/dt2, the last leg's first
    scattered wavefield, its recorded scattered wavefield)."""
    vel = _arr(vel, dtype); m = _arr(model, dtype); e = _arr(ext_refl, dtype); sig = _arr(sig_dtw, dtype)
    d = np.zeros((len(rec_pos), s.nts), dtype)
    W, wp = _wfld(s, dtype, wavefields)
    getattr(lib(), "orc_tomo_fwd_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _p(e), _p(sig), _ip(src_pos),
                                                  len(src_pos), _ip(rec_pos), len(rec_pos), _p(d), sloth, leg1, leg2,
                                                  *wp)
    return (d, *W) if wavefields else d


def tomo_adj(s, vel, data, ext_refl, sig_dtw, src_pos, rec_pos, dtype=np.float64, sloth=0, leg1=1, leg2=1,
             wavefields=False):
    """Tomo adjoint model; with wavefields=True (model, source d2/dt2, receiver wavefield, the
    last leg's scattered coarse samples)."""
    vel = _arr(vel, dtype); d = _arr(data, dtype); e = _arr(ext_refl, dtype); sig = _arr(sig_dtw, dtype)
    m = np.zeros((s.nx, s.nz), dtype)
    W, wp = _wfld(s, dtype, wavefields)
    getattr(lib(), "orc_tomo_adj_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _p(e), _p(sig), _ip(src_pos),
                                                  len(src_pos), _ip(rec_pos), len(rec_pos), _p(d), sloth, leg1, leg2,
                                                  *wp)
    return (m, *W) if wavefields else m


def wemva_fwd(s, vel, model, sig_dtw, src_pos, rec_pos, rdata, dtype=np.float64, leg1=1, leg2=1, wavefields=False):
    """WEMVA forward extended image; with wavefields=True (image, source d2/dt2, receiver
    wavefield, the last leg's scattered coarse samples)."""
    vel = _arr(vel, dtype); m = _arr(model, dtype); sig = _arr(sig_dtw, dtype); r = _arr(rdata, dtype)
    img = np.zeros((s.nExt, s.nx, s.nz), dtype)
    W, wp = _wfld(s, dtype, wavefields)
    getattr(lib(), "orc_wemva_fwd_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _p(sig), _ip(src_pos),
                                                   len(src_pos), _ip(rec_pos), len(rec_pos), _p(r), _p(img),
                                                   leg1, leg2, *wp)
    return (img, *W) if wavefields else img


def wemva_adj(s, vel, image, sig_dtw, src_pos, rec_pos, rdata, dtype=np.float64, leg1=1, leg2=1, wavefields=False):
    """WEMVA adjoint model; with wavefields=True (model, source d2/dt2, receiver wavefield, the
    last leg's scattered coarse samples)."""
    vel = _arr(vel, dtype); img = _arr(image, dtype); sig = _arr(sig_dtw, dtype); r = _arr(rdata, dtype)
    m = np.zeros((s.nx, s.nz), dtype)
    W, wp = _wfld(s, dtype, wavefields)
    getattr(lib(), "orc_wemva_adj_" + _suf(dtype))(C.byref(s.c()), _p(vel), _p(m), _p(sig), _ip(src_pos),
                                                   len(src_pos), _ip(rec_pos), len(rec_pos), _p(r), _p(img),
                                                   leg1, leg2, *wp)
    return (m, *W) if wavefields else m


def time_interp_fwd(nts, dts, sub, m, ots=0.0, dtype=np.float64):
    m = _arr(m, dtype)
    ntw = (nts - 1) * sub + 1
    d = np.zeros((m.shape[0], ntw), dtype)
    getattr(lib(), "orc_time_interp_fwd_" + _suf(dtype))(nts, C.c_double(dts), C.c_double(ots), sub, m.shape[0], _p(m), _p(d))
    return d


def time_interp_adj(nts, dts, sub, d, ots=0.0, dtype=np.float64):
    d = _arr(d, dtype)
    m = np.zeros((d.shape[0], nts), dtype)
    getattr(lib(), "orc_time_interp_adj_" + _suf(dtype))(nts, C.c_double(dts), C.c_double(ots), sub, d.shape[0], _p(m), _p(d))
    return m


def second_deriv(nt, dt, m, dtype=np.float64):
    m = _arr(m, dtype)
    d = np.zeros_like(m)
    getattr(lib(), "orc_second_deriv_" + _suf(dtype))(nt, C.c_double(dt), m.shape[0], _p(m), _p(d))
    return d


# ------------------------------------------------------------------ devices (deviceGpu)
# Restatement of the reference's device geometry (F/src/deviceGpu.cpp) in numpy, with
# float32 where the reference computes in float and float64 where a double literal
# promotes the expression, so corner indices and weights are bit-identical.

def device_bilinear(zc, xc, nz, oz, dz, ox, dx, dipole=0, zshift=0.0, xshift=0.0):
    """Corner indices and weights of devices at physical coordinates (constructor #1,
    F/src/deviceGpu.cpp:8-81): 4 corners per device (8 with a dipole, whose corners
    carry the negated weights of the shifted point). Returns (idx int32, w float32),
    both of length nCorner * nDevice, device-major."""
    f32 = np.float32
    nc = 8 if dipole == 1 else 4
    n = len(zc)
    idx = np.zeros(nc * n, np.int32)
    w = np.zeros(nc * n, np.float32)

    def corners(i1, z, x, sign):
        wz = f32(f32(f32(z) - f32(oz)) / f32(dz))
        wx = f32(f32(f32(x) - f32(ox)) / f32(dx))
        zr, xr = int(wz), int(wx)                    # truncation toward zero (int zReg = wz)
        wz = f32(1.0 - float(f32(wz - f32(zr))))     # wz = wz - zReg; wz = 1.0 - wz
        wx = f32(1.0 - float(f32(wx - f32(xr))))
        base = xr * nz + zr
        idx[i1:i1 + 4] = [base, base + 1, base + nz, base + nz + 1]
        if sign > 0:
            w[i1] = f32(wz * wx)
            w[i1 + 1] = f32((1.0 - float(wz)) * float(wx))
            w[i1 + 2] = f32(float(wz) * (1.0 - float(wx)))
            w[i1 + 3] = f32((1.0 - float(wz)) * (1.0 - float(wx)))
        else:
            w[i1] = f32((-1.0 * float(wz)) * float(wx))
            w[i1 + 1] = f32((-1.0 * (1.0 - float(wz))) * float(wx))
            w[i1 + 2] = f32((-1.0 * float(wz)) * (1.0 - float(wx)))
            w[i1 + 3] = f32((-1.0 * (1.0 - float(wz))) * (1.0 - float(wx)))

    for i in range(n):
        corners(i * nc, zc[i], xc[i], 1)
        if nc == 8:
            corners(i * nc + 4, f32(f32(zc[i]) + f32(zshift)), f32(f32(xc[i]) + f32(xshift)), -1)
    return idx, w


def device_on_grid(iz, ix, nz, dipole=0, zshift=0, xshift=0):
    """Corner indices and weights of devices on grid points (constructors #2 and #3,
    F/src/deviceGpu.cpp:84-190): weight 1 on the point (-1 on the dipole point), 0 on
    the other three corners."""
    nc = 8 if dipole == 1 else 4
    idx = np.zeros(nc * len(iz), np.int32)
    w = np.zeros(nc * len(iz), np.float32)
    for i in range(len(iz)):
        b = ix[i] * nz + iz[i]
        idx[i * nc:i * nc + 4] = [b, b + 1, b + nz, b + nz + 1]
        w[i * nc] = 1.0
        if nc == 8:
            b2 = (ix[i] + xshift) * nz + iz[i] + zshift
            idx[i * nc + 4:i * nc + 8] = [b2, b2 + 1, b2 + nz, b2 + nz + 1]
            w[i * nc + 4] = -1.0
    return idx, w


def device_unique(idx):
    """Unique grid indices in order of first appearance and the trace of every corner
    (convertIrregToReg, F/src/deviceGpu.cpp:192-214)."""
    order, trace = {}, np.zeros(len(idx), np.int32)
    for i, p in enumerate(idx):
        trace[i] = order.setdefault(int(p), len(order))
    return np.array(list(order), np.int32), trace


def device_spread(idx, w, nc, sig_irreg):
    """Device traces -> regular traces (deviceGpu::adjoint, F/src/deviceGpu.cpp:232-246),
    float32 accumulation in device, corner order."""
    uniq, trace = device_unique(idx)
    sig_irreg = np.asarray(sig_irreg, np.float32)
    reg = np.zeros((len(uniq), sig_irreg.shape[1]), np.float32)
    for i1 in range(len(idx)):
        reg[trace[i1]] += w[i1] * sig_irreg[i1 // nc]
    return uniq, reg


def device_gather(idx, w, nc, sig_reg):
    """Regular traces -> device traces (deviceGpu::forward, F/src/deviceGpu.cpp:216-230)."""
    _, trace = device_unique(idx)
    sig_reg = np.asarray(sig_reg, np.float32)
    out = np.zeros((len(idx) // nc, sig_reg.shape[1]), np.float32)
    for i1 in range(len(idx)):
        out[i1 // nc] += w[i1] * sig_reg[trace[i1]]
    return out


def device_sinc(zc, xc, nz, nx, oz, dz, ox, dx, r=4, beta=4.14, dipole=0, zshift=0.0, xshift=0.0):
    """Kaiser-windowed sinc device weights (Hicks 2002, Geophysics 67(1)): (2r)^2 grid points per
    point, w = wz(iz) * wx(ix), w(i) = sinc(i - p) I0(beta sqrt(1 - ((i - p)/r)^2)) / I0(beta) for
    |i - p| <= r, p the coordinate in grid units; a dipole adds the shifted point with negated
    weights. Returns (idx int32, w float32), device-major, x-major inside a point."""
    from numpy import i0
    w1 = 2 * r
    npt = w1 * w1
    nc = npt * (2 if dipole == 1 else 1)
    idx = np.zeros(nc * len(zc), np.int32)
    w = np.zeros(nc * len(zc), np.float32)

    def one(p, n):
        f = int(np.floor(p))
        first = f - r + 1
        assert first >= 0 and first + w1 <= n, "stencil off the grid"
        x = first + np.arange(w1) - p
        u = x / r
        k = np.where(np.abs(u) <= 1, i0(beta * np.sqrt(np.clip(1 - u * u, 0, None))) / i0(beta), 0.0)
        return first, np.sinc(x) * k

    def point(i1, z, x, sign):
        z0, wz = one((float(np.float32(z)) - float(np.float32(oz))) / float(np.float32(dz)), nz)
        x0, wx = one((float(np.float32(x)) - float(np.float32(ox))) / float(np.float32(dx)), nx)
        for jx in range(w1):
            for jz in range(w1):
                idx[i1 + jx * w1 + jz] = (x0 + jx) * nz + z0 + jz
                w[i1 + jx * w1 + jz] = np.float32(sign * wz[jz] * wx[jx])

    for i in range(len(zc)):
        point(i * nc, zc[i], xc[i], 1.0)
        if dipole == 1:
            point(i * nc + npt, np.float32(np.float32(zc[i]) + np.float32(zshift)),
                  np.float32(np.float32(xc[i]) + np.float32(xshift)), -1.0)
    return idx, w


def prepare_source(wavelets, cidx, weights, n_reg, pos, nts, dts, sub, vel, second_derivative=True):
    """The reference's source chain of the Born-family operators (seismicOperator2D::setSources,
    F/include/seismicOperator2D.cpp:10-39) in FP32: device traces spread to their unique grid
    points (deviceGpu::adjoint, F/src/deviceGpu.cpp:232-246), second time derivative
    (F/src/secondTimeDerivative.cpp:14-39, skipped for the nonlinear operator), scaled by
    dtw^2 v^2 at each point (scaleSeismicSource, F/include/seismicOperator2D.cpp:72-86), then
    linearly interpolated to the fine time axis (F/src/interpTimeLinTbb.cpp:26-61).
    wavelets: (nDevice, nts); cidx / weights: (nDevice, nCorner) unique-point index and weight of
    every corner; pos: the n_reg unique grid indices. Returns (n_reg, ntw) float32."""
    wavelets = np.asarray(wavelets, np.float32)
    reg = np.zeros((n_reg, nts), np.float32)
    for d in range(cidx.shape[0]):
        for c in range(cidx.shape[1]):
            reg[cidx[d, c]] += np.float32(weights[d, c]) * wavelets[d]
    if second_derivative:
        reg = second_deriv(nts, dts, reg, dtype=np.float32)
    dtw = np.float32(np.float32(dts) / np.float32(sub))
    v = np.asarray(vel, np.float32).reshape(-1)[np.asarray(pos)]
    reg = reg * ((dtw * dtw) * v * v)[:, None].astype(np.float32)
    return time_interp_fwd(nts, dts, sub, reg, dtype=np.float32)
