"""GPU test of dbmp_backward_noalloc, the backward entry point for callers
that cannot allocate device memory (its gradient-sum scratch is a fixed array
inside the library).  It must give the same gradients as dbmp_backward, call
after call, since every call reuses the array.  Kept in its own file so that
it is collected last."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _scene():
    from diffbmp_b200 import workloads as wl
    return wl.make_scene("c1", seed=5, H=192, W=224, N=500)


def test_noalloc_backward_matches_backward_twice():
    from diffbmp_b200._lib import DBMP_ERR_CAPACITY, call, lib
    from diffbmp_b200.rasterizer import Atlas, Rasterizer, _ptr, _stream

    spec = _scene()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    means, radii, rot, opac, col = t(spec.means2D), t(spec.radii), t(spec.rotations), t(spec.opacities), t(spec.colors)
    sel = torch.from_numpy(spec.sel).cuda()
    atlas = Atlas(t(spec.templates))
    rz = Rasterizer(spec.H, spec.W, 32)
    _, _, state = rz.forward(means, radii, rot, opac, col, sel, atlas)
    rng = np.random.default_rng(11)
    gc = t(rng.normal(0, 1, (spec.H, spec.W, 3)))
    ga = t(rng.normal(0, 1, (spec.H, spec.W)))
    ref = rz.backward(state, gc, ga, radii, rot, opac, col, atlas)   # the allocating entry point
    cv = rz.canvas(spec.N, atlas)
    N = spec.N
    for _ in range(2):                                                 # the array is reused
        outs = [torch.full(s, float("nan"), device="cuda") for s in ((N, 2), (N,), (N,), (N,), (N, 3))]
        call("dbmp_backward_noalloc", ctypes.byref(cv), _ptr(state.prim_info), _ptr(atlas.data),
             _ptr(state.lists.offsets), _ptr(state.lists.indices), _ptr(state.T_last), _ptr(state.last_pos),
             _ptr(gc), _ptr(ga), _ptr(radii), _ptr(rot), _ptr(opac), _ptr(col), *[_ptr(o) for o in outs], _stream())
        torch.cuda.synchronize()
        for a, b in zip(outs, ref):
            torch.testing.assert_close(a, b, rtol=1e-5, atol=1e-9)

    # sizes beyond the fixed scratch are refused before any launch
    big = rz.canvas(lib.dbmp_backward_noalloc_max_prims() + 1, atlas)
    rc = lib.dbmp_backward_noalloc(ctypes.byref(big), *([None] * 17), _stream())
    assert rc == DBMP_ERR_CAPACITY
    assert b"exceed" in lib.dbmp_last_error()
