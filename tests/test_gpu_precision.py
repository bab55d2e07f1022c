"""Relative error of each stored-wavefield precision against the FP64 oracle of
the same scheme, on a medium Born case (realistic source wavelet and
reflectivity, 400 coarse samples): FP32 and FP16 with a per-slice scale must
stay within 1e-4 relative L2; BF16 is reported and bounded by 1e-2. The measured
values are printed for the record (pytest -s)."""
import numpy as np
import pytest

import orc
from cases import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def medium():
    from acoustic_isotropic_operators_b200 import synthetic as S, _capi
    import bench
    w = S.born_workload(nz_phys=96, nx_phys=160, nshots=2, nts=400)
    lib = _capi.lib()
    sigs = bench.prepare_signals(w, lib)
    s = orc.Scheme(nz=w.nz, nx=w.nx, nts=w.nts, dts=w.dts, sub=w.sub, dz=w.dz, dx=w.dx, minPad=w.minPad)
    k = orc.constants(s, w.vel, dtype=np.float32)
    return w, sigs, s, k


@pytest.mark.parametrize("wavefield,tol", [("fp32", 1e-4), ("fp16", 1e-4), ("bf16", 1e-2)])
def test_born_error_vs_fp64(medium, wavefield, tol):
    from acoustic_isotropic_operators_b200.batch import Context, Shot
    w, sigs, s, k = medium
    assert w.sub == 4
    ctx = Context(w.nz, w.nx, w.nts, w.dts, w.sub, w.dz, w.dx, w.minPad, k["v2"], k["rs"], image_fp64=True,
                  wavefield=wavefield)
    shots = [Shot(a.src_pos, a.rec_pos, sg) for a, sg in zip(w.shots, sigs)]
    d = ctx.born_forward(w.model, shots)
    d = [x.copy() for x in d]
    img = ctx.born_adjoint([Shot(a.src_pos, a.rec_pos, sg, dd) for a, sg, dd in zip(w.shots, sigs, d)])
    v64 = w.vel.astype(np.float64)
    ef = max(rel_l2(d[i], orc.born_fwd(s, v64, w.model, sigs[i], a.src_pos, a.rec_pos))
             for i, a in enumerate(w.shots))
    ref_img = sum(orc.born_adj(s, v64, d[i], sigs[i], a.src_pos, a.rec_pos) for i, a in enumerate(w.shots))
    ea = rel_l2(img, ref_img)
    print(f"\n[{wavefield}] Born forward rel err vs FP64 {ef:.2e}, adjoint {ea:.2e}")
    assert ef < tol and ea < tol
