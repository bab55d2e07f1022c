"""Small seeded cases for parity tests (sizes the CPU oracle finishes in seconds)."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

import orc


@dataclass
class Case:
    scheme: orc.Scheme
    vel: np.ndarray          # (nx, nz) float32, m/s
    src_pos: list            # per shot int32 arrays (regular positions)
    rec_pos: list
    sig: list                # per shot (nSrc, ntw) float32 fine traces
    rng: np.random.Generator

    @property
    def nz(self):
        return self.scheme.nz

    @property
    def nx(self):
        return self.scheme.nx


def interior_mask(nx, nz):
    m = np.zeros((nx, nz), bool)
    m[5:nx - 5, 5:nz - 5] = True
    return m


def make_case(seed=0, nzi=48, nxi=64, nts=50, sub=3, nExt=5, minPad=8, nshots=2, dz=10.0, dx=10.0,
              dts=0.004, vmin=2000.0, vmax=2500.0) -> Case:
    rng = np.random.default_rng(seed)
    nz, nx = nzi + 10, nxi + 10
    s = orc.Scheme(nz=nz, nx=nx, nts=nts, dts=dts, sub=sub, dz=dz, dx=dx, minPad=minPad, nExt=nExt)
    # smooth random velocity
    z = np.linspace(0, 1, nz)[None, :]
    vel = vmin + (vmax - vmin) * (0.5 * z + 0.5 * rng.random((nx, nz)) * 0.3)
    vel = vel.astype(np.float32)
    src_pos, rec_pos, sig = [], [], []
    for k in range(nshots):
        ixs = 5 + int(rng.integers(3, nxi - 3))
        izs = 5 + int(rng.integers(2, 10))
        sp = np.array([ixs * nz + izs, ixs * nz + izs + 1, (ixs + 1) * nz + izs], np.int32)
        rec_iz = 5 + 4
        rp = np.array([ix * nz + rec_iz for ix in range(5, nx - 5, 2)] +
                      [ix * nz + rec_iz + 1 for ix in range(6, nx - 5, 3)], np.int32)
        src_pos.append(sp)
        rec_pos.append(rp)
        sig.append((rng.standard_normal((len(sp), s.ntw)) * 1e-2).astype(np.float32))
    return Case(s, vel, src_pos, rec_pos, sig, rng)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
