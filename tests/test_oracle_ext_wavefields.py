"""The oracle's extended-Born wavefield outputs (restating the reference's *Wavefield drivers of
F/src/BornExtShotsGpuFunctions.cu): the data and image are those of the plain operator (non-sloth
scaling), the source wavefield is the one the Born oracle stores, and the time-lag receiver
wavefield differs from the offset one by the 2/v^3 factor only. CPU only."""
import dataclasses

import numpy as np

import orc
from cases import interior_mask, make_case, rel_l2


def test_ext_wavefield_outputs_consistent():
    c = make_case(seed=4, nts=30, nExt=5, nshots=1)
    s = c.scheme
    rng = np.random.default_rng(5)
    m = (rng.standard_normal((5, c.nx, c.nz)) * interior_mask(c.nx, c.nz)).astype(np.float32)
    args = (c.sig[0], c.src_pos[0], c.rec_pos[0])
    d0 = orc.bornext_fwd(s, c.vel, m, *args, dtype=np.float32)
    d, W, S = orc.bornext_fwd(s, c.vel, m, *args, dtype=np.float32, secondary=True)
    assert np.array_equal(d, d0) and np.abs(S).max() > 0
    _, Wb = orc.born_fwd(s, c.vel, m[2], *args, dtype=np.float32, wavefield=True)
    assert np.array_equal(W, Wb)
    dd = rng.standard_normal((len(c.rec_pos[0]), s.nts)).astype(np.float32)
    img0 = orc.bornext_adj(s, c.vel, dd, *args, dtype=np.float32)
    img, W2, R = orc.bornext_adj(s, c.vel, dd, *args, dtype=np.float32, secondary=True)
    assert np.array_equal(img, img0) and np.array_equal(W2, W)
    so = dataclasses.replace(s, extension=1)
    imgo0 = orc.bornext_adj(so, c.vel, dd, *args, dtype=np.float32)
    imgo, _, Ro = orc.bornext_adj(so, c.vel, dd, *args, dtype=np.float32, secondary=True)
    assert np.array_equal(imgo, imgo0)
    rs = orc.constants(s, c.vel, dtype=np.float32)["rs"].reshape(c.nx, c.nz)
    assert rel_l2(R, Ro * rs[None]) < 1e-6      # time lags: v^2 dtw^2 * 2/v^3; offsets: v^2 dtw^2
