"""Reference-named Python modules of the drop-in operator layer.

Importing this module puts acoustic_isotropic_operators_b200/pymod on sys.path
and imports the six pybind11 modules built there by
``make -C acoustic_isotropic_operators_b200/cpp``:

* ``pySepLite`` — SEP-compatible axis / hypercube / float1DReg / float2DReg /
  float3DReg (``getNdArray()`` gives a writable numpy view, slowest axis first),
  ``dictParams`` (a paramObj built from a Python dict of par-file keys),
  ``argParams`` (from ``key=value`` arguments and ``par=`` files) and the SEP .H
  dataset reader / writer ``getVector`` / ``writeVector``;
* ``pyAcoustic_iso_float_nl`` (``deviceGpu``, ``nonlinearPropShotsGpu``),
  ``pyAcoustic_iso_float_born`` (``BornShotsGpu``), ``pyAcoustic_iso_float_born_ext``
  (``BornExtShotsGpu``), ``pyAcoustic_iso_float_tomo`` (``tomoExtShotsGpu``),
  ``pyAcoustic_iso_float_wemva`` (``wemvaExtShotsGpu``) — the module, class and
  method names of the reference's pybind11 layer
  (P/python_float/pyAcoustic_iso_float_*.cpp).
"""
import os
import sys

PYMOD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "pymod")
if PYMOD not in sys.path:
    sys.path.insert(0, PYMOD)

import pySepLite  # noqa: E402,F401
import pyAcoustic_iso_float_nl  # noqa: E402,F401
import pyAcoustic_iso_float_born  # noqa: E402,F401
import pyAcoustic_iso_float_born_ext  # noqa: E402,F401
import pyAcoustic_iso_float_tomo  # noqa: E402,F401
import pyAcoustic_iso_float_wemva  # noqa: E402,F401


def vector(values, axes):
    """SEP vector over `axes` ([(n, o, d), ...], fastest first) holding `values` (numpy, slowest first)."""
    import numpy as np
    ax = [pySepLite.axis(int(n), float(o), float(d)) for n, o, d in axes]
    cls = {1: pySepLite.float1DReg, 2: pySepLite.float2DReg, 3: pySepLite.float3DReg}[len(ax)]
    v = cls(pySepLite.hypercube(ax))
    if values is not None:
        v.getNdArray()[...] = np.asarray(values, np.float32).reshape(v.getNdArray().shape)
    return v


def params(**kw):
    """paramObj from keyword arguments (par-file keys, e.g. nts=1000, iGpu=[0, 1])."""
    return pySepLite.dictParams(kw)


def io(params):
    """paramObj from command-line arguments (``key=value`` and ``par=file``), as
    ``genericIO.io(params=sys.argv)`` in the reference's Python programs."""
    return pySepLite.argParams([str(a) for a in params])


def getVector(path, ndims=0):
    """SEP vector read from the .H dataset `path` (``genericIO.defaultIO.getVector``);
    `ndims` pads the file's axes with n = 1 axes up to that many."""
    return pySepLite.getVector(path, ndims)


def writeVector(path, vec, data_format="xdr_float"):
    """Writes `vec` as the .H dataset `path` with its data in `path@`
    (``genericIO.defaultIO.writeVector``)."""
    pySepLite.writeVector(path, vec, data_format)
