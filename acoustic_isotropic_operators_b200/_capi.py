"""ctypes binding of libaio_b200.so (the C ABI declared in include/aio_b200.h).

The shared library is built in-tree (``make -C acoustic_isotropic_operators_b200/csrc``
or ``__graft_entry__.build()``). Loading fails loudly when it is missing: there
is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# AIO_B200_LIB selects another build of the same library (e.g. an experimental one).
LIB_PATH = os.environ.get("AIO_B200_LIB") or os.path.join(_HERE, "libaio_b200.so")

AIO_OK = 0
AIO_ERR_ARGUMENT = 1
AIO_ERR_CUDA = 2
AIO_ERR_MEMORY = 3
AIO_ERR_STATE = 4
AIO_MEM_HOST = 0
AIO_MEM_DEVICE = 1
AIO_NONLINEAR, AIO_BORN, AIO_BORN_EXT, AIO_TOMO_EXT, AIO_WEMVA_EXT = range(5)
AIO_WFLD_FP32, AIO_WFLD_BF16, AIO_WFLD_FP16 = range(3)
AIO_STEPPER_AUTO, AIO_STEPPER_FINE, AIO_STEPPER_BLOCKED = range(3)

EXPORTED = [
    "aio_last_error", "aio_context_create", "aio_context_destroy", "aio_context_set_velocity",
    "aio_context_wave_capacity", "aio_context_last_launches", "aio_context_stream", "aio_context_profile",
    "aio_context_stats", "aio_context_reset_stats", "aio_context_blocked_plan",
    "aio_nonlinear_forward", "aio_nonlinear_adjoint", "aio_nonlinear_forward_wavefield",
    "aio_nonlinear_adjoint_wavefield", "aio_born_forward", "aio_born_adjoint", "aio_born_adjoint_shots",
    "aio_born_ext_forward", "aio_born_ext_adjoint", "aio_tomo_ext_forward", "aio_tomo_ext_adjoint",
    "aio_wemva_ext_forward", "aio_wemva_ext_adjoint",
    "aio_getGpuInfo",
    "aio_fd_precompute", "aio_time_interp_forward", "aio_time_interp_adjoint", "aio_second_time_derivative",
    "aio_scale_seismic_source", "aio_device_spread", "aio_device_gather", "aio_prepare_source",
    "aio_initNonlinearGpu", "aio_allocateNonlinearGpu", "aio_deallocateNonlinearGpu", "aio_propShotsFwdGpu",
    "aio_propShotsFwdGpuWavefield", "aio_propShotsAdjGpu", "aio_propShotsAdjGpuWavefield",
    "aio_initBornGpu", "aio_allocateBornShotsGpu", "aio_deallocateBornShotsGpu", "aio_BornShotsFwdGpu",
    "aio_BornShotsAdjGpu",
    "aio_initBornExtGpu", "aio_allocateBornExtShotsGpu", "aio_deallocateBornExtShotsGpu",
    "aio_BornTimeShotsFwdGpu", "aio_BornTimeShotsAdjGpu",
    "aio_initTomoExtGpu", "aio_allocateTomoExtShotsGpu", "aio_deallocateTomoExtShotsGpu",
    "aio_tomoTimeShotsFwdGpu", "aio_tomoTimeShotsAdjGpu",
    "aio_initWemvaExtGpu", "aio_allocateWemvaExtShotsGpu", "aio_deallocateWemvaExtShotsGpu",
    "aio_wemvaTimeShotsFwdGpu", "aio_wemvaTimeShotsAdjGpu",
    "aio_propShotsFwdFsGpu", "aio_propShotsFwdFsGpuWavefield", "aio_propShotsAdjFsGpu",
    "aio_propShotsAdjFsGpuWavefield", "aio_BornShotsFwdFsGpu", "aio_BornShotsAdjFsGpu",
    "aio_BornTimeShotsFwdFsGpu", "aio_BornTimeShotsAdjFsGpu", "aio_tomoTimeShotsFwdFsGpu",
    "aio_tomoTimeShotsAdjFsGpu",
    "aio_BornOffsetShotsFwdGpu", "aio_BornOffsetShotsAdjGpu", "aio_BornOffsetShotsFwdFsGpu",
    "aio_BornOffsetShotsAdjFsGpu", "aio_tomoOffsetShotsFwdGpu", "aio_tomoOffsetShotsAdjGpu",
    "aio_tomoOffsetShotsFwdFsGpu", "aio_tomoOffsetShotsAdjFsGpu", "aio_wemvaOffsetShotsFwdGpu",
    "aio_wemvaOffsetShotsAdjGpu", "aio_born_forward_wavefield", "aio_born_adjoint_wavefield",
    "aio_BornShotsFwdGpuWavefield", "aio_BornShotsAdjGpuWavefield",
    "aio_born_ext_forward_wavefield", "aio_born_ext_adjoint_wavefield",
    "aio_BornTimeShotsFwdGpuWavefield", "aio_BornOffsetShotsFwdGpuWavefield", "aio_BornTimeShotsFwdFsGpuWavefield",
    "aio_BornOffsetShotsFwdFsGpuWavefield", "aio_BornTimeShotsAdjGpuWavefield", "aio_BornOffsetShotsAdjGpuWavefield",
    "aio_BornTimeShotsAdjFsGpuWavefield", "aio_BornOffsetShotsAdjFsGpuWavefield",
    "aio_dot_f64", "aio_context_graph_replays", "aio_context_set_budget",
    "aio_tomo_ext_forward_wavefield", "aio_tomo_ext_adjoint_wavefield", "aio_wemva_ext_forward_wavefield",
    "aio_wemva_ext_adjoint_wavefield", "aio_context_device_bytes", "aio_context_release_buffers",
]


class AioParams(C.Structure):
    _fields_ = [("nz", C.c_int), ("nx", C.c_int), ("nts", C.c_int), ("sub", C.c_int), ("minPad", C.c_int),
                ("nExt", C.c_int), ("dz", C.c_float), ("dx", C.c_float), ("dts", C.c_float),
                ("alphaCos", C.c_float), ("leg1", C.c_int), ("leg2", C.c_int), ("sloth", C.c_int),
                ("wavefieldPrecision", C.c_int), ("imageFp64", C.c_int), ("device", C.c_int),
                ("memBudgetBytes", C.c_longlong), ("stepper", C.c_int), ("chunkColumns", C.c_int),
                ("freeSurface", C.c_int), ("extension", C.c_int)]


class AioShot(C.Structure):
    _fields_ = [("sourcesPositionReg", C.c_void_p), ("nSourcesReg", C.c_int),
                ("receiversPositionReg", C.c_void_p), ("nReceiversReg", C.c_int),
                ("sourcesSignals", C.c_void_p), ("data", C.c_void_p), ("wemvaData", C.c_void_p),
                ("sourcesOut", C.c_void_p)]


class AioError(RuntimeError):
    """Raised when a C ABI call returns a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"aio error {code}: {msg}")
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with __graft_entry__.build() "
                              "or make -C acoustic_isotropic_operators_b200/csrc")
        L = C.CDLL(LIB_PATH)
        L.aio_last_error.restype = C.c_char_p
        L.aio_context_last_launches.restype = C.c_longlong
        L.aio_context_last_launches.argtypes = [C.c_void_p]
        L.aio_context_wave_capacity.argtypes = [C.c_void_p, C.c_int]
        L.aio_context_stream.restype = C.c_void_p
        L.aio_context_stream.argtypes = [C.c_void_p]
        L.aio_context_set_budget.argtypes = [C.c_void_p, C.c_longlong]
        L.aio_context_graph_replays.restype = C.c_longlong
        L.aio_context_graph_replays.argtypes = [C.c_void_p]
        L.aio_context_device_bytes.restype = C.c_longlong
        L.aio_context_device_bytes.argtypes = [C.c_void_p]
        L.aio_context_release_buffers.argtypes = [C.c_void_p]
        L.aio_dot_f64.argtypes = [C.c_int, C.c_int, C.c_longlong, C.c_void_p, C.c_void_p,
                                  C.POINTER(C.c_double)]
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != AIO_OK:
        raise AioError(code, lib().aio_last_error().decode())


def fptr(a):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous, "float32 C-contiguous array required"
    return a.ctypes.data_as(C.c_void_p)


def iptr(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


def dot_f64(a, b, device: int = 0) -> float:
    """sum(a * b) of two float32 host arrays of the same size, reduced in FP64 on the GPU
    (aio_dot_f64): the inner product of the dot-product tests."""
    a = np.ascontiguousarray(a, dtype=np.float32).reshape(-1)
    b = np.ascontiguousarray(b, dtype=np.float32).reshape(-1)
    assert a.size == b.size
    out = C.c_double()
    code = lib().aio_dot_f64(device, AIO_MEM_HOST, a.size, a.ctypes.data_as(C.c_void_p),
                             b.ctypes.data_as(C.c_void_p), C.byref(out))
    if code != AIO_OK:
        raise AioError(code, "aio_dot_f64 failed (see stderr)")
    return float(out.value)
