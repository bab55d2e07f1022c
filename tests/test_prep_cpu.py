"""CPU: the oracle's restatement of the source chain (orc.prepare_source) against the product's
host code (aio_prepare_source, C ABI), bitwise, for the Born-family chain (with the second time
derivative) and the nonlinear one (without)."""
import ctypes as C

import numpy as np
import pytest

import orc


@pytest.mark.parametrize("second", [0, 1])
def test_prepare_source_matches_product(second):
    from acoustic_isotropic_operators_b200 import _capi as A, synthetic as S
    w = S.born_workload(nz_phys=60, nx_phys=90, nshots=3, nts=120)
    velf = np.ascontiguousarray(w.vel.reshape(-1), np.float32)
    for a in w.shots:
        wav = np.ascontiguousarray(np.repeat(w.wavelet[None, :], a.src_cidx.shape[0], axis=0), np.float32)
        out = np.zeros((len(a.src_pos), w.ntw), np.float32)
        A.check(A.lib().aio_prepare_source(second, a.src_cidx.shape[0], a.src_cidx.shape[1], A.iptr(a.src_cidx),
                                           A.fptr(a.src_w), len(a.src_pos), A.iptr(a.src_pos), w.nts,
                                           C.c_float(w.dts), w.sub, A.fptr(velf), A.fptr(wav), A.fptr(out)))
        ref = orc.prepare_source(wav, a.src_cidx, a.src_w, len(a.src_pos), a.src_pos, w.nts, w.dts, w.sub, w.vel,
                                 second_derivative=bool(second))
        assert np.array_equal(out, ref)
