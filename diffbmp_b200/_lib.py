"""ctypes binding of libdbmp.so (the C ABI declared in include/dbmp.h).

The library is built in-tree by ``python -m diffbmp_b200.build``.  There is
no fallback: importing this module raises if the library cannot be loaded,
and every wrapper raises ``DbmpError`` with the library's message when a call
returns a non-zero status.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# DBMP_LIBRARY selects another build of the same ABI (e.g. a tuning variant).
LIB_PATH = os.environ.get("DBMP_LIBRARY") or os.path.join(HERE, "libdbmp.so")

DBMP_OK, DBMP_ERR_INVALID, DBMP_ERR_CUDA, DBMP_ERR_CAPACITY, DBMP_ERR_UNSUPPORTED = range(5)
ATLAS_F32, ATLAS_F32_QUAD, ATLAS_F16_QUAD, ATLAS_BF16_QUAD, ATLAS_F16_PAIR, ATLAS_BF16_PAIR = range(6)
BIN_CONTENT, BIN_CULL, BIN_CONTENT_REF = 0, 1, 2

# Every symbol include/dbmp.h declares, with (restype, argtypes).
_vp, _i, _ll, _sz, _f = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_size_t, ctypes.c_float


class AdamCfg(ctypes.Structure):
    """Mirror of dbmp_adam_cfg."""
    _fields_ = [("lr", ctypes.c_float * 8), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float),
                ("eps", ctypes.c_float), ("x_max", ctypes.c_float), ("y_max", ctypes.c_float),
                ("r_min", ctypes.c_float), ("r_max", ctypes.c_float), ("clamp", ctypes.c_int32),
                ("lr_gamma", ctypes.c_float)]


class PruneCfg(ctypes.Structure):
    """Mirror of dbmp_prune_cfg."""
    _fields_ = [("every", ctypes.c_int32), ("num_iterations", ctypes.c_int32), ("no_prune_last", ctypes.c_int32),
                ("warmup", ctypes.c_int32), ("threshold", ctypes.c_float), ("pool_rows", ctypes.c_int32)]


class BlurSchedule(ctypes.Structure):
    """Mirror of dbmp_blur_schedule."""
    _fields_ = [("mode", ctypes.c_int32), ("sigma", ctypes.c_float), ("sigma_start", ctypes.c_float),
                ("sigma_end", ctypes.c_float), ("num_iterations", ctypes.c_int32)]


class Canvas(ctypes.Structure):
    """Mirror of dbmp_canvas."""
    _fields_ = [("height", ctypes.c_int32), ("width", ctypes.c_int32), ("tile_size", ctypes.c_int32),
                ("num_prims", ctypes.c_int32), ("num_templates", ctypes.c_int32),
                ("tmpl_h", ctypes.c_int32), ("tmpl_w", ctypes.c_int32), ("atlas_kind", ctypes.c_int32),
                ("bin_mode", ctypes.c_int32), ("alpha_max", ctypes.c_float), ("t_stop", ctypes.c_float),
                ("reserved", ctypes.c_int32)]


_CP = ctypes.POINTER(Canvas)
SIGNATURES = {
    "dbmp_last_error": (ctypes.c_char_p, []),
    "dbmp_version": (_i, []),
    "dbmp_num_tiles": (_i, [_CP]),
    "dbmp_template_bboxes": (_i, [_vp, _i, _i, _i, _vp, _vp]),
    "dbmp_atlas_pack": (_i, [_vp, _i, _i, _i, _i, _vp, _vp]),
    "dbmp_template_blur": (_i, [_vp, _i, _i, _i, _f, _vp, _vp]),
    "dbmp_atlas_bytes": (_sz, [_i, _i, _i, _i]),
    "dbmp_bin_workspace_bytes": (_sz, [_CP, _ll]),
    "dbmp_prim_info_bytes": (_sz, [_i]),
    "dbmp_prepare": (_i, [_CP, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dbmp_bin": (_i, [_CP, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _ll, _vp, _vp, _vp, _sz, _vp]),
    "dbmp_forward": (_i, [_CP, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dbmp_backward": (_i, [_CP, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                           _vp, _vp, _vp, _vp, _vp, _vp]),
    "dbmp_backward_noalloc": (_i, [_CP] + [_vp] * 18),
    "dbmp_forward_blend": (_i, [_CP] + [_vp] * 5 + [_f] + [_vp] * 5),
    "dbmp_backward_blend": (_i, [_CP] + [_vp] * 5 + [_f] + [_vp] * 15),
    "dbmp_backward_noalloc_max_prims": (_i, []),
    "dbmp_psd_bboxes": (_i, [_vp, _vp, _i, _i, _i, _f, _vp, _vp, _vp]),
    "dbmp_psd_layout": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "dbmp_psd_layers": (_i, [_vp] * 6 + [_i, _i, _i] + [_vp] * 4 + [_i, _f, _f, _f, _vp, _vp, _vp]),
    "dbmp_psd_rle_count": (_i, [_vp] * 4 + [_i, _ll, _i, _i] + [_vp] * 4),
    "dbmp_psd_rle_write": (_i, [_vp] * 4 + [_i, _ll, _i, _i] + [_vp] * 4 + [_ll, _vp]),
    "dbmp_count": (_i, [_CP, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dbmp_fused_fwd_bwd": (_i, [_CP, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dbmp_forward_batch": (_i, [_CP, _i, _vp, _vp, _vp, _vp, _ll, _vp, _ll, _f, _vp, _vp, _vp, _vp, _vp]),
    "dbmp_backward_batch": (_i, [_CP, _i, _vp, _vp, _vp, _vp, _ll, _vp, _ll, _f] + [_vp] * 15),
    "dbmp_grads_from_accum": (_i, [_CP] + [_vp] * 11),
    "dbmp_prune": (_i, [_CP, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dbmp_template_blur_scheduled": (_i, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp]),
    "dbmp_adam_step": (_i, [_CP, ctypes.c_void_p, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
}


class DbmpError(RuntimeError):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m diffbmp_b200.build`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


def check(rc: int, what: str = "") -> None:
    if rc != DBMP_OK:
        msg = lib.dbmp_last_error().decode(errors="replace")
        raise DbmpError(f"{what or 'dbmp'} failed (status {rc}): {msg}")


def call(name: str, *args) -> None:
    check(getattr(lib, name)(*args), name)
