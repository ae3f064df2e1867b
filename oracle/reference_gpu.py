"""TEST INFRASTRUCTURE -- ctypes front end for the reference's own CUDA kernels,
compiled from the reference sources into oracle/_ref/ by `make -C oracle ref`
(oracle/ref_shim.cu wraps the C++ launchers; the PSD launchers are already
extern "C" in psd_export_kernels.cu:204-275).  Only tests use it."""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
RASTER = os.path.join(_HERE, "_ref", "libref_raster.so")
PSD = os.path.join(_HERE, "_ref", "libref_psd.so")


def available() -> bool:
    return os.path.exists(RASTER) and os.path.exists(PSD)


_raster = _psd = None


def raster():
    global _raster
    if _raster is None:
        _raster = ctypes.CDLL(RASTER)
        _raster.ref_forward.restype = ctypes.c_int
        _raster.ref_backward.restype = ctypes.c_int
    return _raster


def psd():
    global _psd
    if _psd is None:
        _psd = ctypes.CDLL(PSD)
    return _psd
