"""CPU checks of the C ABI library: it loads and exports every declared symbol."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "aio_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(aio_[A-Za-z0-9_]+)\s*\(", src)))


def test_library_exports_header():
    from acoustic_isotropic_operators_b200 import _capi
    lib = _capi.lib()
    names = declared_symbols()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_capi.EXPORTED) <= set(names)


def test_error_without_gpu_is_reported():
    """Creating a context on a machine without a usable device returns a CUDA/argument error, not a crash."""
    import torch
    if torch.cuda.is_available():
        return
    from acoustic_isotropic_operators_b200 import _capi as A
    p = A.AioParams(30, 30, 10, 2, 5, 1, 10.0, 10.0, 0.004, 0.99, 1, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0)
    h = ctypes.c_void_p()
    import numpy as np
    v2 = np.ones(900, np.float32)
    rc = A.lib().aio_context_create(ctypes.byref(p), A.fptr(v2), None, ctypes.byref(h))
    assert rc != A.AIO_OK
    assert A.lib().aio_last_error()
