"""Allocation-free nonlinear forward (aio_propShotsFwdGpu_noalloc).

This entry point is for callers that cannot let a library allocate device
memory — services that plan all device memory ahead, hosts whose allocator
owns the device heap. It keeps every temporary in
one fixed file-scope device array, so this test checks it against the regular
engine entry point on two calls in a row with different shots: anything left
over in the shared scratch from the first call would corrupt the second.
Tolerance: relative L2 1e-5, the FP32 parity bar of the other GPU tests.

Named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import orc
from cases import make_case, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-5


def test_noalloc_matches_engine_on_two_calls():
    import torch
    from acoustic_isotropic_operators_b200 import _capi
    from acoustic_isotropic_operators_b200.batch import Context, Shot

    case = make_case(seed=21, nshots=2)
    s = case.scheme
    k = orc.constants(s, case.vel, dtype=np.float32)
    ctx = Context(s.nz, s.nx, s.nts, s.dts, s.sub, s.dz, s.dx, s.minPad, k["v2"], k["rs"])
    expected = ctx.nonlinear_forward([Shot(case.src_pos[i], case.rec_pos[i], case.sig[i]) for i in range(2)])
    ctx.close()

    lib = _capi.lib()
    fn = lib.aio_propShotsFwdGpu_noalloc
    fn.argtypes = [C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_float,
                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    dev = torch.device("cuda", 0)
    v2_d = torch.from_numpy(np.ascontiguousarray(k["v2"], np.float32)).to(dev)
    stream = torch.cuda.current_stream(dev)
    for i in range(2):
        sp = np.ascontiguousarray(case.src_pos[i], np.int32)
        rp = np.ascontiguousarray(case.rec_pos[i], np.int32)
        sig_d = torch.from_numpy(case.sig[i]).to(dev)
        out_d = torch.full((len(rp), s.nts), 7.0, dtype=torch.float32, device=dev)  # must be overwritten
        torch.cuda.synchronize()
        rc = fn(s.dz, s.dx, s.nz, s.nx, s.nts, s.dts, s.sub, s.minPad, s.alphaCos, v2_d.data_ptr(),
                sig_d.data_ptr(), sp.ctypes.data, len(sp), rp.ctypes.data, len(rp), out_d.data_ptr(),
                stream.cuda_stream)
        assert rc == _capi.AIO_OK
        torch.cuda.synchronize()
        got = out_d.cpu().numpy()
        assert rel_l2(got, expected[i]) < TOL, (i, rel_l2(got, expected[i]))


def test_noalloc_rejects_oversized_grid():
    """A grid beyond the fixed scratch is refused before any device work."""
    import torch
    from acoustic_isotropic_operators_b200 import _capi
    fn = _capi.lib().aio_propShotsFwdGpu_noalloc
    fn.argtypes = [C.c_float, C.c_float, C.c_int, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_float,
                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    small = torch.zeros(16, dtype=torch.float32, device="cuda")  # valid address; the size check rejects first
    rc = fn(10.0, 10.0, 4010, 4010, 100, 0.004, 4, 50, 0.99, small.data_ptr(), None, None, 0, None, 0,
            small.data_ptr(), None)
    assert rc == _capi.AIO_ERR_ARGUMENT
