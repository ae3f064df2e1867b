"""GPU test of dbmp_backward_noalloc, the backward entry point for callers
that cannot allocate device memory (a plug-in whose host owns the device
allocator, or a frame loop that must not allocate once running).  Its
gradient-sum scratch is a fixed array inside the library, so it must give the
same gradients as dbmp_backward call after call (every call reuses the
array), allocate nothing on the device, accept N up to its stated maximum and
refuse larger N.

The test depends on no other test and passes alone in a fresh process.  Its
file name makes pytest collect it last only so that a run stopping at the
first failure has already run every other test if this one fails."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _inputs(spec):
    from diffbmp_b200.rasterizer import Atlas, Rasterizer
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    p = dict(means=t(spec.means2D), radii=t(spec.radii), rot=t(spec.rotations), opac=t(spec.opacities),
             col=t(spec.colors), sel=torch.from_numpy(spec.sel).cuda())
    atlas = Atlas(t(spec.templates))
    rz = Rasterizer(spec.H, spec.W, 32)
    _, _, state = rz.forward(p["means"], p["radii"], p["rot"], p["opac"], p["col"], p["sel"], atlas)
    rng = np.random.default_rng(11)
    p["gc"] = t(rng.normal(0, 1, (spec.H, spec.W, 3)))
    p["ga"] = t(rng.normal(0, 1, (spec.H, spec.W)))
    return p, atlas, rz, state


def _noalloc(p, atlas, rz, state, outs):
    from diffbmp_b200._lib import call
    from diffbmp_b200.rasterizer import _ptr, _stream
    cv = rz.canvas(int(p["radii"].numel()), atlas)
    call("dbmp_backward_noalloc", ctypes.byref(cv), _ptr(state.prim_info), _ptr(atlas.data),
         _ptr(state.lists.offsets), _ptr(state.lists.indices), _ptr(state.T_last), _ptr(state.last_pos),
         _ptr(p["gc"]), _ptr(p["ga"]), _ptr(p["radii"]), _ptr(p["rot"]), _ptr(p["opac"]), _ptr(p["col"]),
         *[_ptr(o) for o in outs], _stream())


def _outputs(N):
    return [torch.full(s, float("nan"), device="cuda") for s in ((N, 2), (N,), (N,), (N,), (N, 3))]


def test_noalloc_backward_matches_backward_twice():
    from diffbmp_b200 import workloads as wl
    from diffbmp_b200._lib import DBMP_ERR_CAPACITY, lib
    from diffbmp_b200.rasterizer import _stream

    spec = wl.make_scene("c1", seed=5, H=192, W=224, N=500)
    p, atlas, rz, state = _inputs(spec)
    ref = rz.backward(state, p["gc"], p["ga"], p["radii"], p["rot"], p["opac"], p["col"], atlas)  # allocating form
    outs = [_outputs(spec.N) for _ in range(3)]
    # the first call loads the library's device module (lazily, under CUDA's
    # default lazy loading), which commits the fixed array's 4 MiB; the calls
    # after it take no device memory (any allocation is at least 2 MiB)
    _noalloc(p, atlas, rz, state, outs[0])
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for o in outs[1:]:                                          # two more calls in a row share the array
        _noalloc(p, atlas, rz, state, o)
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free0 - free1 < (1 << 20), (free0, free1)
    for o in outs:
        for a, b in zip(o, ref):
            torch.testing.assert_close(a, b, rtol=1e-5, atol=1e-9)

    # sizes beyond the fixed scratch are refused before any launch
    big = rz.canvas(lib.dbmp_backward_noalloc_max_prims() + 1, atlas)
    rc = lib.dbmp_backward_noalloc(ctypes.byref(big), *([None] * 17), _stream())
    assert rc == DBMP_ERR_CAPACITY
    assert b"exceed" in lib.dbmp_last_error()


def test_noalloc_backward_at_the_limit():
    """N equal to dbmp_backward_noalloc_max_prims() uses the whole array."""
    from diffbmp_b200 import workloads as wl
    from diffbmp_b200._lib import lib
    N = int(lib.dbmp_backward_noalloc_max_prims())
    spec = wl.make_scene("c0", seed=9, H=320, W=288, N=N)
    spec.radii[:] = np.minimum(spec.radii, 6.0)               # keep the lists short
    p, atlas, rz, state = _inputs(spec)
    ref = rz.backward(state, p["gc"], p["ga"], p["radii"], p["rot"], p["opac"], p["col"], atlas)
    out = _outputs(N)
    _noalloc(p, atlas, rz, state, out)
    torch.cuda.synchronize()
    for a, b in zip(out, ref):
        torch.testing.assert_close(a, b, rtol=1e-5, atol=1e-9)
    # the last primitive's gradients are produced (its sums sit at the array's end)
    assert torch.isfinite(out[0][-1]).all()
