"""Seeded synthetic workloads with the shapes of the published configurations.

The reference's examples read SEP files (Marmousi, wavelets, parfiles); there
is no dataset here, so every model, wavelet and acquisition is generated from a
seed with the documented shapes, sizes and value ranges:

* grids: physical nz x nx at 10 m, a 50-point sponge on every side, the plus
  sides rounded up so the padded interior is a multiple of 16, plus FAT=5 —
  the reference's padding rule (F/src/padFileGpuMain.cpp:37-66), with edge
  replication into the sponge (same file, :85-115) and a zero FAT ring;
* velocity: 1500 -> 3500 m/s linear in depth, optionally smoothed
  (sigma = 100 m) or with +-200 m/s Gaussian blobs (sigma = 100 m);
* reflectivity: 10 horizontal + 10 dipping (|dip| <= 15 deg) one-cell
  interfaces with amplitudes U(-0.1, 0.1);
* wavelet: Ricker (1 - 2a t^2) exp(-a t^2), a = (pi f)^2, delayed by t0
  (seis_utils/seis_utils_float/python/waveletFloatMain.py:79-98);
* sub: smallest integer with Courant vmax*dtw/min(dz,dx) <= 0.45
  (F/src/fdParam.cpp:228-240).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

FAT = 5


@dataclass
class Padding:
    nz_phys: int
    nx_phys: int
    zPadMinus: int
    zPadPlus: int
    xPadMinus: int
    xPadPlus: int

    @property
    def nz(self) -> int:
        return self.nz_phys + self.zPadMinus + self.zPadPlus + 2 * FAT

    @property
    def nx(self) -> int:
        return self.nx_phys + self.xPadMinus + self.xPadPlus + 2 * FAT

    @property
    def minPad(self) -> int:
        return min(self.zPadMinus, self.zPadPlus, self.xPadMinus, self.xPadPlus)


def padding(nz_phys: int, nx_phys: int, pad: int = 50, block: int = 16) -> Padding:
    """Reference padding rule, F/src/padFileGpuMain.cpp:37-66 (no free surface)."""
    zplus = int(math.ceil((2 * pad + nz_phys) / block)) * block - nz_phys - pad
    xplus = int(math.ceil((2 * pad + nx_phys) / block)) * block - nx_phys - pad
    return Padding(nz_phys, nx_phys, pad, zplus, pad, xplus)


def pad_model(v: np.ndarray, p: Padding) -> np.ndarray:
    """(nx_phys, nz_phys) -> (nx, nz) with edge replication and a zero FAT ring."""
    out = np.zeros((p.nx, p.nz), np.float32)
    z0, x0 = FAT + p.zPadMinus, FAT + p.xPadMinus
    core = np.pad(v, ((p.xPadMinus, p.xPadPlus), (p.zPadMinus, p.zPadPlus)), mode="edge")
    out[FAT:FAT + core.shape[0], FAT:FAT + core.shape[1]] = core
    assert z0 == FAT + p.zPadMinus and x0 == FAT + p.xPadMinus
    return out


def gradient(nz_phys, nx_phys, vtop=1500.0, vbot=3500.0) -> np.ndarray:
    z = np.linspace(vtop, vbot, nz_phys, dtype=np.float64)
    return np.repeat(z[None, :], nx_phys, axis=0)


def gaussian_smooth(v: np.ndarray, sigma_pts: float) -> np.ndarray:
    from scipy.ndimage import gaussian_filter
    return gaussian_filter(v, sigma_pts, mode="nearest")


def with_blobs(v, rng, d=10.0, n=8, sigma_m=100.0, amp=200.0):
    nx, nz = v.shape
    X, Z = np.meshgrid(np.arange(nx) * d, np.arange(nz) * d, indexing="ij")
    out = v.copy()
    for _ in range(n):
        cx, cz = rng.uniform(0, nx * d), rng.uniform(0, nz * d)
        sgn = 1.0 if rng.random() < 0.5 else -1.0
        out += sgn * amp * np.exp(-((X - cx) ** 2 + (Z - cz) ** 2) / (2 * sigma_m ** 2))
    return out


def interfaces(nz_phys, nx_phys, rng, n_flat=10, n_dip=10, max_dip_deg=15.0, amp=0.1) -> np.ndarray:
    m = np.zeros((nx_phys, nz_phys), np.float64)
    xs = np.arange(nx_phys)
    for k in range(n_flat + n_dip):
        a = rng.uniform(-amp, amp)
        z0 = rng.uniform(0.1, 0.9) * nz_phys
        dip = 0.0 if k < n_flat else math.tan(math.radians(rng.uniform(-max_dip_deg, max_dip_deg)))
        zc = np.round(z0 + dip * (xs - nx_phys / 2)).astype(int)
        ok = (zc >= 0) & (zc < nz_phys)
        m[xs[ok], zc[ok]] += a
    return m


def ricker(nts, dts, f=15.0, t0=0.1) -> np.ndarray:
    a = (math.pi * f) ** 2
    t = np.arange(nts) * dts - t0
    return ((1 - 2.0 * a * t * t) * np.exp(-a * t * t)).astype(np.float32)


def sub_for(vmax, dts, dx, courant=0.45) -> int:
    return max(1, int(math.ceil(vmax * dts / (courant * dx) - 1e-9)))


# --------------------------------------------------------------------- devices
def grid_device_positions(iz: List[int], ix: List[int], nz: int):
    """deviceGpu constructor #2 (F/src/deviceGpu.cpp:86-137): integer grid points,
    4 corners per device with weights (1, 0, 0, 0), made unique in first-seen
    order (convertIrregToReg, :201-223). Returns (unique positions, corner
    indices [nDev,4], weights [nDev,4])."""
    corners, weights = [], []
    for z, x in zip(iz, ix):
        base = x * nz + z
        corners.append([base, base + 1, base + nz, base + nz + 1])
        weights.append([1.0, 0.0, 0.0, 0.0])
    uniq, index = [], {}
    for c in corners:
        for p in c:
            if p not in index:
                index[p] = len(uniq)
                uniq.append(p)
    cidx = np.array([[index[p] for p in c] for c in corners], np.int32)
    return np.array(uniq, np.int32), cidx, np.array(weights, np.float32)


@dataclass
class Acquisition:
    src_pos: np.ndarray   # unique regular positions
    src_cidx: np.ndarray
    src_w: np.ndarray
    rec_pos: np.ndarray
    rec_cidx: np.ndarray
    rec_w: np.ndarray


def spread(signal_irreg: np.ndarray, cidx, w, n_reg) -> np.ndarray:
    """deviceGpu::adjoint (F/src/deviceGpu.cpp:245-261): irregular -> regular traces."""
    out = np.zeros((n_reg, signal_irreg.shape[1]), np.float32)
    for d in range(cidx.shape[0]):
        for c in range(cidx.shape[1]):
            out[cidx[d, c]] += w[d, c] * signal_irreg[d]
    return out


def gather(signal_reg: np.ndarray, cidx, w) -> np.ndarray:
    """deviceGpu::forward (F/src/deviceGpu.cpp:227-243): regular -> irregular traces."""
    out = np.zeros((cidx.shape[0], signal_reg.shape[1]), np.float32)
    for d in range(cidx.shape[0]):
        for c in range(cidx.shape[1]):
            out[d] += w[d, c] * signal_reg[cidx[d, c]]
    return out


@dataclass
class Workload:
    """One configuration: padded grid, fields, and per-shot acquisitions."""
    name: str
    pad: Padding
    nts: int
    dts: float
    sub: int
    dz: float
    dx: float
    vel: np.ndarray           # (nx, nz) float32 including sponge and FAT
    wavelet: np.ndarray       # (nts,) float32
    shots: List[Acquisition]
    model: Optional[np.ndarray] = None      # (nx, nz) reflectivity (Born)
    nExt: int = 1
    extra: dict = field(default_factory=dict)

    @property
    def nz(self):
        return self.pad.nz

    @property
    def nx(self):
        return self.pad.nx

    @property
    def minPad(self):
        return self.pad.minPad

    @property
    def ntw(self):
        return (self.nts - 1) * self.sub + 1

    @property
    def n_interior(self):
        return (self.nz - 2 * FAT) * (self.nx - 2 * FAT)

    @property
    def fine_steps(self):
        return (self.nts - 1) * self.sub


def surface_acquisition(p: Padding, nz, src_x_phys: int, z_phys=2) -> Acquisition:
    iz = FAT + p.zPadMinus + z_phys
    sp, sc, sw = grid_device_positions([iz], [FAT + p.xPadMinus + src_x_phys], nz)
    rx = [FAT + p.xPadMinus + x for x in range(p.nx_phys)]
    rp, rc, rw = grid_device_positions([iz] * len(rx), rx, nz)
    return Acquisition(sp, sc, sw, rp, rc, rw)


def born_workload(nz_phys=400, nx_phys=1200, nshots=32, nts=2000, dts=0.004, seed=2, d=10.0,
                  smooth=True, blobs=False) -> Workload:
    """Batched Born forward+adjoint configuration (400x1200, 32 shots, nts=2000)."""
    rng = np.random.default_rng(seed)
    p = padding(nz_phys, nx_phys)
    v = gradient(nz_phys, nx_phys)
    if blobs:
        v = with_blobs(v, rng, d)
    if smooth:
        v = gaussian_smooth(v, 100.0 / d)
    vel = pad_model(v.astype(np.float32), p)
    sub = sub_for(float(v.max()), dts, d)
    refl = pad_model(interfaces(nz_phys, nx_phys, rng).astype(np.float32), p)
    refl[:FAT + p.xPadMinus] = 0; refl[FAT + p.xPadMinus + nx_phys:] = 0
    refl[:, :FAT + p.zPadMinus] = 0; refl[:, FAT + p.zPadMinus + nz_phys:] = 0
    xs = np.linspace(0, nx_phys - 1, nshots).round().astype(int) if nshots > 1 else [nx_phys // 2]
    shots = [surface_acquisition(p, p.nz, int(x)) for x in xs]
    return Workload("born", p, nts, dts, sub, d, d, vel, ricker(nts, dts), shots, model=refl)


def tomo_workload(nz_phys=800, nx_phys=3000, nshots=96, nts=3000, n_ext=41, dts=0.004, seed=5, d=10.0) -> Workload:
    """Extended tomo / WEMVA configuration (800x3000, nExt = 41, 96 shots, nts = 3000): smoothed
    gradient background; model = Gaussian velocity anomalies (sigma 300 m, +-5 %); extended image
    (extra["ext"], (nExt, nx, nz)) = 20 interfaces times a Gaussian lag profile (sigma 3 lags)."""
    w = born_workload(nz_phys, nx_phys, nshots, nts, dts, seed, d)
    rng = np.random.default_rng(seed + 100)
    v0 = gaussian_smooth(gradient(nz_phys, nx_phys), 100.0 / d)
    z = np.arange(nz_phys)[None, :] * d
    x = np.arange(nx_phys)[:, None] * d
    dv = np.zeros((nx_phys, nz_phys))
    for _ in range(8):
        cz, cx = rng.uniform(0, nz_phys * d), rng.uniform(0, nx_phys * d)
        dv += rng.choice([-1.0, 1.0]) * np.exp(-((z - cz) ** 2 + (x - cx) ** 2) / (2 * 300.0 ** 2))
    dv = 0.05 * v0 * dv / max(1.0, float(np.abs(dv).max()))
    model = pad_model(dv.astype(np.float32), w.pad)
    model[:FAT + w.pad.xPadMinus] = 0; model[FAT + w.pad.xPadMinus + nx_phys:] = 0
    model[:, :FAT + w.pad.zPadMinus] = 0; model[:, FAT + w.pad.zPadMinus + nz_phys:] = 0
    h = (n_ext - 1) // 2
    prof = np.exp(-(np.arange(n_ext) - h) ** 2 / (2 * 3.0 ** 2)).astype(np.float32)
    w.extra["ext"] = prof[:, None, None] * w.model[None]
    w.model = model
    w.nExt = n_ext
    w.name = "tomo"
    return w


def nonlinear_workload(nz_phys=200, nx_phys=400, nts=1000, dts=0.004, seed=1, d=10.0) -> Workload:
    """Plain nonlinear forward configuration (200x400 + blobs, one shot at x=2000 m)."""
    rng = np.random.default_rng(seed)
    p = padding(nz_phys, nx_phys)
    v = with_blobs(gradient(nz_phys, nx_phys), rng, d)
    vel = pad_model(v.astype(np.float32), p)
    sub = sub_for(float(v.max()), dts, d)
    shots = [surface_acquisition(p, p.nz, int(2000.0 / d))]
    return Workload("nonlinear", p, nts, dts, sub, d, d, vel, ricker(nts, dts), shots)
