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
RASTER16 = os.path.join(_HERE, "_ref", "libref_raster_fp16.so")


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


_raster16 = None


def raster_fp16():
    """The reference's all-half kernels, or None when they are not built."""
    global _raster16
    if _raster16 is None and os.path.exists(RASTER16):
        _raster16 = ctypes.CDLL(RASTER16)
        _raster16.ref_forward_fp16.restype = ctypes.c_int
        _raster16.ref_backward_fp16.restype = ctypes.c_int
    return _raster16
