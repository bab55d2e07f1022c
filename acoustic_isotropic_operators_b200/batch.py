"""Batched operator context over the C ABI (numpy in, numpy out).

``Context`` wraps one ``aio_context``: one grid / velocity / device. Each call
runs a whole list of shots; the engine groups them into waves that fit the
device-memory budget and advances every shot of a wave with one fused stepper
launch per fine time step.

Shots are ``Shot`` objects holding regular-grid device positions (linear
indices ``ix*nz+iz``), fine-time source traces and coarse-time data, exactly
the arrays the reference's per-shot operators hand to their GPU functions.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _capi as A


@dataclass
class Shot:
    src_pos: np.ndarray                 # int32 [nSrcReg]
    rec_pos: np.ndarray                 # int32 [nRecReg]
    src_sig: Optional[np.ndarray] = None  # float32 [nSrcReg, ntw]
    data: Optional[np.ndarray] = None     # float32 [nRecReg, nts]
    wemva_data: Optional[np.ndarray] = None  # float32 [nRecReg, nts]
    src_out: Optional[np.ndarray] = None  # float32 [nSrcReg, ntw] (nonlinear adjoint output)
    _keep: list = field(default_factory=list, repr=False)

    def __post_init__(self):
        self.src_pos = np.ascontiguousarray(self.src_pos, dtype=np.int32)
        self.rec_pos = np.ascontiguousarray(self.rec_pos, dtype=np.int32)
        for name in ("src_sig", "data", "wemva_data", "src_out"):
            v = getattr(self, name)
            if v is not None:
                setattr(self, name, np.ascontiguousarray(v, dtype=np.float32))


_WFLD = {"fp32": A.AIO_WFLD_FP32, "bf16": A.AIO_WFLD_BF16, "fp16": A.AIO_WFLD_FP16}


class Context:
    """One operator instance on one GPU (grid, time axis, velocity fields)."""

    def __init__(self, nz, nx, nts, dts, sub, dz, dx, minPad, vel2Dtw2, reflectivity_scale=None, *, nExt=1,
                 alphaCos=0.99, leg1=1, leg2=1, sloth=0, wavefield="fp32", image_fp64=False, device=0,
                 mem_budget_bytes=0, stepper="auto", chunk_columns=0, free_surface=0, extension="time"):
        self.nz, self.nx, self.nts, self.sub, self.nExt = nz, nx, nts, sub, nExt
        self.ntw = (nts - 1) * sub + 1
        p = A.AioParams(nz, nx, nts, sub, minPad, nExt, dz, dx, dts, alphaCos, leg1, leg2, sloth,
                        _WFLD[wavefield], int(bool(image_fp64)), device, int(mem_budget_bytes),
                        {"auto": A.AIO_STEPPER_AUTO, "fine": A.AIO_STEPPER_FINE,
                         "blocked": A.AIO_STEPPER_BLOCKED}[stepper], int(chunk_columns), int(free_surface),
                        {"time": 0, "offset": 1}[extension])
        v2 = np.ascontiguousarray(vel2Dtw2, dtype=np.float32).reshape(-1)
        rs = None if reflectivity_scale is None else np.ascontiguousarray(reflectivity_scale,
                                                                          dtype=np.float32).reshape(-1)
        assert v2.size == nz * nx
        h = C.c_void_p()
        A.check(A.lib().aio_context_create(C.byref(p), A.fptr(v2), A.fptr(rs), C.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            A.lib().aio_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def last_launches(self) -> int:
        return int(A.lib().aio_context_last_launches(self._h))

    def set_budget(self, nbytes: int) -> None:
        """Device-memory budget for shot buffers from now on (<= 0: 93 % of free memory)."""
        A.check(A.lib().aio_context_set_budget(self._h, int(nbytes)))

    @property
    def device_bytes(self) -> int:
        """Device bytes the context holds (velocity constants and its per-call buffers)."""
        return int(A.lib().aio_context_device_bytes(self._h))

    def release_buffers(self) -> None:
        """Free the per-call buffers (and captured graphs); the next call allocates them again."""
        A.check(A.lib().aio_context_release_buffers(self._h))

    def capacity(self, family: int) -> int:
        return int(A.lib().aio_context_wave_capacity(self._h, family))

    @property
    def graph_replays(self) -> int:
        """Interval loops replayed from CUDA graphs since the context was created."""
        return int(A.lib().aio_context_graph_replays(self._h))

    @property
    def stream_ptr(self) -> int:
        return int(A.lib().aio_context_stream(self._h) or 0)

    def profile(self, sample_every: int) -> None:
        A.check(A.lib().aio_context_profile(self._h, int(sample_every)))

    def stats(self):
        """(kernels launched, timed stepper ms, timed stepper launches, their point-updates) since reset."""
        k, n = C.c_longlong(), C.c_longlong()
        ms, pts = C.c_double(), C.c_double()
        A.check(A.lib().aio_context_stats(self._h, C.byref(k), C.byref(ms), C.byref(n), C.byref(pts)))
        return int(k.value), float(ms.value), int(n.value), float(pts.value)

    def blocked_plan(self, n_shots: int) -> dict:
        """Strip rows, strips, chunk columns and chunks the blocked stepper uses for n_shots."""
        out = (C.c_int * 4)()
        A.check(A.lib().aio_context_blocked_plan(self._h, int(n_shots), out))
        return {"strip_rows": out[0], "strips": out[1], "chunk_columns": out[2], "chunks": out[3]}

    def reset_stats(self) -> None:
        A.check(A.lib().aio_context_reset_stats(self._h))

    # ------------------------------------------------------ device-resident calls
    def device_call(self, name: str, *args, shots=None):
        """Call aio_<name>(ctx, *args, nShots, shots, AIO_MEM_DEVICE) with raw device pointers.

        ``args`` are ctypes values (``ctypes.c_void_p(device_address)``, ``ctypes.c_int``...).
        ``shots`` is a list of (src_pos, rec_pos, sig_ptr, data_ptr, wemva_ptr, src_out_ptr) with
        host int32 position arrays and device addresses (ints, 0 for none).
        """
        arr = (A.AioShot * len(shots))()
        keep = []
        for i, (sp, rp, sig, dat, wd, so) in enumerate(shots):
            sp = np.ascontiguousarray(sp, np.int32)
            rp = np.ascontiguousarray(rp, np.int32)
            keep += [sp, rp]
            arr[i] = A.AioShot(A.iptr(sp), len(sp), A.iptr(rp), len(rp), sig or None, dat or None, wd or None,
                               so or None)
        fn = getattr(A.lib(), "aio_" + name)
        A.check(fn(self._h, *args, len(shots), arr, A.AIO_MEM_DEVICE))

    # ------------------------------------------------------------------ helpers
    def _shots(self, shots: Sequence[Shot], *, data_out: bool, need_sig=True, src_out=False):
        arr = (A.AioShot * len(shots))()
        for i, s in enumerate(shots):
            if data_out and (s.data is None or s.data.shape != (len(s.rec_pos), self.nts)):
                s.data = np.zeros((len(s.rec_pos), self.nts), np.float32)
            if src_out and (s.src_out is None or s.src_out.shape != (len(s.src_pos), self.ntw)):
                s.src_out = np.zeros((len(s.src_pos), self.ntw), np.float32)
            if need_sig:
                assert s.src_sig is not None and s.src_sig.shape == (len(s.src_pos), self.ntw)
            arr[i] = A.AioShot(A.iptr(s.src_pos), len(s.src_pos), A.iptr(s.rec_pos), len(s.rec_pos),
                               A.fptr(s.src_sig), A.fptr(s.data), A.fptr(s.wemva_data), A.fptr(s.src_out))
        return arr

    def _model(self, m, slices):
        m = np.ascontiguousarray(m, dtype=np.float32)
        assert m.size == slices * self.nz * self.nx
        return m

    # ---------------------------------------------------------------- operators
    def nonlinear_forward(self, shots: List[Shot]) -> List[np.ndarray]:
        arr = self._shots(shots, data_out=True)
        A.check(A.lib().aio_nonlinear_forward(self._h, len(shots), arr, A.AIO_MEM_HOST))
        return [s.data for s in shots]

    def nonlinear_adjoint(self, shots: List[Shot]) -> List[np.ndarray]:
        arr = self._shots(shots, data_out=False, need_sig=False, src_out=True)
        A.check(A.lib().aio_nonlinear_adjoint(self._h, len(shots), arr, A.AIO_MEM_HOST))
        return [s.src_out for s in shots]

    def born_forward(self, model, shots: List[Shot]) -> List[np.ndarray]:
        m = self._model(model, 1)
        arr = self._shots(shots, data_out=True)
        A.check(A.lib().aio_born_forward(self._h, A.fptr(m), len(shots), arr, A.AIO_MEM_HOST))
        return [s.data for s in shots]

    def born_adjoint(self, shots: List[Shot], model=None, add=False) -> np.ndarray:
        out = np.zeros((self.nx, self.nz), np.float32) if model is None else model
        arr = self._shots(shots, data_out=False)
        A.check(A.lib().aio_born_adjoint(self._h, A.fptr(out), int(add), len(shots), arr, A.AIO_MEM_HOST))
        return out

    def born_adjoint_shots(self, shots: List[Shot]) -> List[np.ndarray]:
        """Born adjoint with one image per shot (the shots still run in the same launches)."""
        outs = [np.zeros((self.nx, self.nz), np.float32) for _ in shots]
        ptrs = (C.c_void_p * len(shots))(*[o.ctypes.data for o in outs])
        arr = self._shots(shots, data_out=False)
        A.check(A.lib().aio_born_adjoint_shots(self._h, ptrs, len(shots), arr, A.AIO_MEM_HOST))
        return outs

    def born_forward_wavefield(self, model, shot: Shot):
        """Born forward of one shot: (data, source wavefield, scattered wavefield); the wavefields
        are (nts, nx, nz) with a zero FAT ring."""
        m = self._model(model, 1)
        arr = self._shots([shot], data_out=True)
        src = np.zeros((self.nts, self.nx, self.nz), np.float32)
        sec = np.zeros_like(src)
        A.check(A.lib().aio_born_forward_wavefield(self._h, A.fptr(m), arr, A.AIO_MEM_HOST, A.fptr(src), A.fptr(sec)))
        return shot.data, src, sec

    def born_adjoint_wavefield(self, shot: Shot):
        """Born adjoint of one shot: (image, source wavefield, receiver wavefield scaled by
        2/v^3 v^2 dtw^2), wavefields (nts, nx, nz) (the reference's adjoint wavefield driver
        returns the receiver wavefield only)."""
        out = np.zeros((self.nx, self.nz), np.float32)
        arr = self._shots([shot], data_out=False)
        src = np.zeros((self.nts, self.nx, self.nz), np.float32)
        rec = np.zeros_like(src)
        A.check(A.lib().aio_born_adjoint_wavefield(self._h, A.fptr(out), 0, arr, A.AIO_MEM_HOST, A.fptr(src),
                                                   A.fptr(rec)))
        return out, src, rec

    def born_ext_forward_wavefield(self, model, shot: Shot):
        """Extended Born forward of one shot: (data, source wavefield, scattered wavefield), the
        wavefields (nts, nx, nz) with a zero FAT ring (non-sloth time-lag scaling)."""
        m = self._model(model, self.nExt)
        arr = self._shots([shot], data_out=True)
        src = np.zeros((self.nts, self.nx, self.nz), np.float32)
        sec = np.zeros_like(src)
        A.check(A.lib().aio_born_ext_forward_wavefield(self._h, A.fptr(m), arr, A.AIO_MEM_HOST, A.fptr(src),
                                                       A.fptr(sec)))
        return shot.data, src, sec

    def born_ext_adjoint_wavefield(self, shot: Shot):
        """Extended Born adjoint of one shot: (image (nExt, nx, nz), source wavefield, receiver
        wavefield scaled by 2/v^3 v^2 dtw^2 for time lags, by v^2 dtw^2 for offsets)."""
        out = np.zeros((self.nExt, self.nx, self.nz), np.float32)
        arr = self._shots([shot], data_out=False)
        src = np.zeros((self.nts, self.nx, self.nz), np.float32)
        rec = np.zeros_like(src)
        A.check(A.lib().aio_born_ext_adjoint_wavefield(self._h, A.fptr(out), 0, arr, A.AIO_MEM_HOST, A.fptr(src),
                                                       A.fptr(rec)))
        return out, src, rec

    def _w3(self):
        return [np.zeros((self.nts, self.nx, self.nz), np.float32) for _ in range(3)]

    def tomo_forward_wavefield(self, model, ext_reflectivity, shot: Shot):
        """Tomo forward of one shot: (data, d2/dt2 of the source wavefield, the last leg's first
        and second scattered wavefields), the wavefields (nts, nx, nz) with a zero FAT ring."""
        m = self._model(model, 1)
        e = self._model(ext_reflectivity, self.nExt)
        arr = self._shots([shot], data_out=True)
        W = self._w3()
        A.check(A.lib().aio_tomo_ext_forward_wavefield(self._h, A.fptr(m), A.fptr(e), arr, A.AIO_MEM_HOST,
                                                       *[A.fptr(x) for x in W]))
        return (shot.data, *W)

    def tomo_adjoint_wavefield(self, ext_reflectivity, shot: Shot):
        """Tomo adjoint of one shot: (model, d2/dt2 of the source wavefield, receiver wavefield, the
        last leg's scattered coarse samples)."""
        out = np.zeros((self.nx, self.nz), np.float32)
        e = self._model(ext_reflectivity, self.nExt)
        arr = self._shots([shot], data_out=False)
        W = self._w3()
        A.check(A.lib().aio_tomo_ext_adjoint_wavefield(self._h, A.fptr(out), 0, A.fptr(e), arr, A.AIO_MEM_HOST,
                                                       *[A.fptr(x) for x in W]))
        return (out, *W)

    def wemva_forward_wavefield(self, model, shot: Shot):
        """WEMVA forward of one shot: (extended image, d2/dt2 of the source wavefield, receiver
        wavefield, the last leg's scattered coarse samples)."""
        m = self._model(model, 1)
        out = np.zeros((self.nExt, self.nx, self.nz), np.float32)
        arr = self._shots([shot], data_out=False)
        W = self._w3()
        A.check(A.lib().aio_wemva_ext_forward_wavefield(self._h, A.fptr(m), A.fptr(out), 0, arr, A.AIO_MEM_HOST,
                                                        *[A.fptr(x) for x in W]))
        return (out, *W)

    def wemva_adjoint_wavefield(self, image, shot: Shot):
        """WEMVA adjoint of one shot: (model, d2/dt2 of the source wavefield, receiver wavefield,
        the last leg's scattered coarse samples)."""
        im = self._model(image, self.nExt)
        out = np.zeros((self.nx, self.nz), np.float32)
        arr = self._shots([shot], data_out=False)
        W = self._w3()
        A.check(A.lib().aio_wemva_ext_adjoint_wavefield(self._h, A.fptr(out), 0, A.fptr(im), arr, A.AIO_MEM_HOST,
                                                        *[A.fptr(x) for x in W]))
        return (out, *W)

    def born_ext_forward(self, model, shots: List[Shot]) -> List[np.ndarray]:
        m = self._model(model, self.nExt)
        arr = self._shots(shots, data_out=True)
        A.check(A.lib().aio_born_ext_forward(self._h, A.fptr(m), len(shots), arr, A.AIO_MEM_HOST))
        return [s.data for s in shots]

    def born_ext_adjoint(self, shots: List[Shot], model=None, add=False) -> np.ndarray:
        out = np.zeros((self.nExt, self.nx, self.nz), np.float32) if model is None else model
        arr = self._shots(shots, data_out=False)
        A.check(A.lib().aio_born_ext_adjoint(self._h, A.fptr(out), int(add), len(shots), arr, A.AIO_MEM_HOST))
        return out

    def tomo_forward(self, model, ext_reflectivity, shots: List[Shot]) -> List[np.ndarray]:
        m = self._model(model, 1)
        e = self._model(ext_reflectivity, self.nExt)
        arr = self._shots(shots, data_out=True)
        A.check(A.lib().aio_tomo_ext_forward(self._h, A.fptr(m), A.fptr(e), len(shots), arr, A.AIO_MEM_HOST))
        return [s.data for s in shots]

    def tomo_adjoint(self, ext_reflectivity, shots: List[Shot], model=None, add=False) -> np.ndarray:
        out = np.zeros((self.nx, self.nz), np.float32) if model is None else model
        e = self._model(ext_reflectivity, self.nExt)
        arr = self._shots(shots, data_out=False)
        A.check(A.lib().aio_tomo_ext_adjoint(self._h, A.fptr(out), int(add), A.fptr(e), len(shots), arr,
                                             A.AIO_MEM_HOST))
        return out

    def wemva_forward(self, model, shots: List[Shot], image=None, add=False) -> np.ndarray:
        m = self._model(model, 1)
        out = np.zeros((self.nExt, self.nx, self.nz), np.float32) if image is None else image
        arr = self._shots(shots, data_out=False)
        A.check(A.lib().aio_wemva_ext_forward(self._h, A.fptr(m), A.fptr(out), int(add), len(shots), arr,
                                              A.AIO_MEM_HOST))
        return out

    def wemva_adjoint(self, image, shots: List[Shot], model=None, add=False) -> np.ndarray:
        im = self._model(image, self.nExt)
        out = np.zeros((self.nx, self.nz), np.float32) if model is None else model
        arr = self._shots(shots, data_out=False)
        A.check(A.lib().aio_wemva_ext_adjoint(self._h, A.fptr(out), int(add), A.fptr(im), len(shots), arr,
                                              A.AIO_MEM_HOST))
        return out
