"""Generates tests/golden/reference_small.npz: outputs of the REFERENCE's own
GPU drivers (oracle/_ref — the reference's *ShotsGpuFunctions.cu compiled
unmodified for sm_100a by `make -C oracle ref`) on one small seeded case, in
FP32 (acoustic_iso_float) and FP64 (acoustic_iso_double), for every operator
family on the hot path.

The reference has no golden vectors of its own; these fixtures let the CPU
test suite pin the CPU oracle against the reference without a GPU
(tests/test_golden.py).

Run on a machine with a B200 and the oracle/_ref libraries built:

    python tests/golden/make_golden.py OUT.npz
    python tests/golden/make_golden.py --fs OUT_FS.npz   # free-surface drivers (*FsGpu) ->
                                                          # tests/golden/reference_small_fs.npz
    python tests/golden/make_golden.py --offset OUT.npz  # subsurface-offset drivers ->
                                                          # tests/golden/reference_small_offset.npz

Every input is generated here from fixed seeds and stored in the file too, so
the test does not depend on this script's random streams.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
sys.path.insert(0, os.path.join(HERE, ".."))

import refgpu  # noqa: E402
from cases import interior_mask, make_case  # noqa: E402

# The reference covers the interior with 16x16 thread blocks and requires both
# interior extents to be multiples of 16 (F/src/fdParam.cpp:259-266).
CASE = dict(seed=11, nzi=32, nxi=48, nts=30, sub=3, nExt=5, minPad=8, nshots=1)


def main(out, fs=False, offset=False):
    assert CASE["nzi"] % 16 == 0 and CASE["nxi"] % 16 == 0
    c = make_case(**CASE)
    s = c.scheme
    if fs or offset:
        import dataclasses
        s = dataclasses.replace(s, freeSurface=int(fs), extension=int(offset))
    rng = np.random.default_rng(1234)
    mask = interior_mask(c.nx, c.nz)
    sp, rp, sig = c.src_pos[0], c.rec_pos[0], c.sig[0]
    f = dict(vel=c.vel, src_pos=sp, rec_pos=rp, sig=sig,
             scheme=np.array([s.nz, s.nx, s.nts, s.sub, s.minPad, s.nExt, s.freeSurface, s.extension], np.int64),
             scheme_f=np.array([s.dz, s.dx, s.dts, s.alphaCos], np.float64))
    f["data_in"] = (rng.standard_normal((len(rp), s.nts)) * 1e-3).astype(np.float32)
    f["dm"] = (rng.standard_normal((c.nx, c.nz)) * mask).astype(np.float32)
    f["ext"] = (rng.standard_normal((s.nExt, c.nx, c.nz)) * mask).astype(np.float32)
    f["image_in"] = (rng.standard_normal((s.nExt, c.nx, c.nz)) * mask).astype(np.float32)
    f["rdata"] = (rng.standard_normal((len(rp), s.nts)) * 1e-3).astype(np.float32)
    for dt, tag in ((np.float32, "f32"), (np.float64, "f64")):
        v = c.vel.astype(dt)
        if fs:  # the reference has free-surface drivers for these families (no sloth flag, no WEMVA)
            f[f"nl_fwd_{tag}"] = refgpu.nl_fwd(s, v, sig, sp, rp, dtype=dt)
            f[f"nl_adj_{tag}"] = refgpu.nl_adj(s, v, f["data_in"], sp, rp, dtype=dt)
            f[f"born_fwd_{tag}"] = refgpu.born_fwd(s, v, f["dm"], sig, sp, rp, dtype=dt)
            f[f"born_adj_{tag}"] = refgpu.born_adj(s, v, f["data_in"], sig, sp, rp, dtype=dt)
            f[f"bornext_fwd_{tag}"] = refgpu.bornext_fwd(s, v, f["ext"], sig, sp, rp, dtype=dt)
            f[f"bornext_adj_{tag}"] = refgpu.bornext_adj(s, v, f["data_in"], sig, sp, rp, dtype=dt)
            for l1, l2 in ((1, 1), (1, 0), (0, 1)):
                k = f"l{l1}{l2}_{tag}"
                f["tomo_fwd_" + k] = refgpu.tomo_fwd(s, v, f["dm"], f["ext"], sig, sp, rp, leg1=l1, leg2=l2, dtype=dt)
                f["tomo_adj_" + k] = refgpu.tomo_adj(s, v, f["data_in"], f["ext"], sig, sp, rp, leg1=l1, leg2=l2,
                                                     dtype=dt)
            continue
        if offset:  # the offset drivers of the extended families (no sloth flag)
            f[f"bornext_fwd_{tag}"] = refgpu.bornext_fwd(s, v, f["ext"], sig, sp, rp, dtype=dt)
            f[f"bornext_adj_{tag}"] = refgpu.bornext_adj(s, v, f["data_in"], sig, sp, rp, dtype=dt)
            for l1, l2 in ((1, 1), (1, 0), (0, 1)):
                k = f"l{l1}{l2}_{tag}"
                f["tomo_fwd_" + k] = refgpu.tomo_fwd(s, v, f["dm"], f["ext"], sig, sp, rp, leg1=l1, leg2=l2, dtype=dt)
                f["tomo_adj_" + k] = refgpu.tomo_adj(s, v, f["data_in"], f["ext"], sig, sp, rp, leg1=l1, leg2=l2,
                                                     dtype=dt)
                f["wemva_fwd_" + k] = refgpu.wemva_fwd(s, v, f["dm"], sig, sp, rp, f["rdata"], leg1=l1, leg2=l2,
                                                       dtype=dt)
                f["wemva_adj_" + k] = refgpu.wemva_adj(s, v, f["image_in"], sig, sp, rp, f["rdata"], leg1=l1,
                                                       leg2=l2, dtype=dt)
            continue
        f[f"nl_fwd_{tag}"] = refgpu.nl_fwd(s, v, sig, sp, rp, dtype=dt)
        f[f"nl_adj_{tag}"] = refgpu.nl_adj(s, v, f["data_in"], sp, rp, dtype=dt)
        f[f"born_fwd_{tag}"] = refgpu.born_fwd(s, v, f["dm"], sig, sp, rp, dtype=dt)
        f[f"born_adj_{tag}"] = refgpu.born_adj(s, v, f["data_in"], sig, sp, rp, dtype=dt)
        for sl in (0, 1):
            f[f"bornext_fwd_s{sl}_{tag}"] = refgpu.bornext_fwd(s, v, f["ext"], sig, sp, rp, sloth=sl, dtype=dt)
            f[f"bornext_adj_s{sl}_{tag}"] = refgpu.bornext_adj(s, v, f["data_in"], sig, sp, rp, sloth=sl, dtype=dt)
            for l1, l2 in ((1, 1), (1, 0), (0, 1)):
                k = f"s{sl}_l{l1}{l2}_{tag}"
                f["tomo_fwd_" + k] = refgpu.tomo_fwd(s, v, f["dm"], f["ext"], sig, sp, rp, sloth=sl, leg1=l1,
                                                     leg2=l2, dtype=dt)
                f["tomo_adj_" + k] = refgpu.tomo_adj(s, v, f["data_in"], f["ext"], sig, sp, rp, sloth=sl, leg1=l1,
                                                     leg2=l2, dtype=dt)
        for l1, l2 in ((1, 1), (1, 0), (0, 1)):
            k = f"l{l1}{l2}_{tag}"
            f["wemva_fwd_" + k] = refgpu.wemva_fwd(s, v, f["dm"], sig, sp, rp, f["rdata"], leg1=l1, leg2=l2, dtype=dt)
            f["wemva_adj_" + k] = refgpu.wemva_adj(s, v, f["image_in"], sig, sp, rp, f["rdata"], leg1=l1, leg2=l2,
                                                   dtype=dt)
    np.savez_compressed(out, **f)
    print("wrote", out, len(f), "arrays")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if a not in ("--fs", "--offset")]
    fs, offset = "--fs" in sys.argv[1:], "--offset" in sys.argv[1:]
    name = "reference_small_fs.npz" if fs else ("reference_small_offset.npz" if offset else "reference_small.npz")
    main(args[0] if args else os.path.join(HERE, name), fs, offset)
