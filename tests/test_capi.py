"""CPU tests of the C ABI: the library loads without a GPU, exports every
symbol include/dbmp.h declares, and rejects bad arguments before launching."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    syms = set()
    for name in os.listdir(os.path.join(ROOT, "include")):
        if name.endswith(".h"):
            text = open(os.path.join(ROOT, "include", name)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            syms |= set(re.findall(r"\b(dbmp_[a-z0-9_]+)\s*\(", text))
    return syms


def test_library_exports_header_symbols():
    from diffbmp_b200 import _lib
    syms = header_symbols()
    assert len(syms) >= 10
    missing = [s for s in sorted(syms) if not hasattr(_lib.lib, s)]
    assert not missing, missing
    # the Python binding declares a signature for every exported entry point
    assert syms <= set(_lib.SIGNATURES), sorted(syms - set(_lib.SIGNATURES))


def canvas(**kw):
    from diffbmp_b200._lib import Canvas
    d = dict(height=256, width=256, tile_size=32, num_prims=512, num_templates=1, tmpl_h=64, tmpl_w=64,
             atlas_kind=0, bin_mode=0, alpha_max=1.0, t_stop=1e-7, reserved=0)
    d.update(kw)
    return Canvas(*d.values())


def test_num_tiles_and_workspace_query():
    from diffbmp_b200._lib import lib
    assert lib.dbmp_num_tiles(ctypes.byref(canvas())) == 64
    assert lib.dbmp_num_tiles(ctypes.byref(canvas(height=200, width=136, tile_size=16))) == 13 * 9
    # per-primitive rectangles + per-tile counts and offsets; independent of the list capacity
    ws = lib.dbmp_bin_workspace_bytes(ctypes.byref(canvas()), 1 << 20)
    c = canvas()
    assert ws >= 16 * c.num_prims + 2 * 8 * (64 + 1)
    assert ws == lib.dbmp_bin_workspace_bytes(ctypes.byref(canvas()), 0)
    assert lib.dbmp_prim_info_bytes(10) == 640


@pytest.mark.parametrize("bad,msg", [
    (dict(tile_size=8), "tile_size"),
    (dict(height=0), "empty"),
    (dict(num_templates=0), "atlas"),
    (dict(t_stop=0.0), "t_stop"),
    (dict(atlas_kind=9), "atlas_kind"),
    (dict(alpha_max=-0.5), "alpha_max"),
    (dict(alpha_max=float("nan")), "alpha_max"),
])
def test_invalid_canvas_is_rejected(bad, msg):
    from diffbmp_b200._lib import lib
    assert lib.dbmp_num_tiles(ctypes.byref(canvas(**bad))) == -1
    assert msg in lib.dbmp_last_error().decode()


def test_null_pointers_are_rejected_without_launch():
    from diffbmp_b200._lib import DBMP_ERR_INVALID, lib
    cv = canvas()
    rc = lib.dbmp_forward(ctypes.byref(cv), None, None, None, None, None, None, None, None, None)
    assert rc == DBMP_ERR_INVALID and "null" in lib.dbmp_last_error().decode()
    rc = lib.dbmp_bin(ctypes.byref(cv), *([None] * 10), ctypes.c_longlong(0), None, None, None,
                      ctypes.c_size_t(0), None)
    assert rc == DBMP_ERR_INVALID
