"""Memory test at 4096x4096 with N=100000 primitives (FP32): the backward
recomputes transmittance from the stored T entering the last contributor and
its list position, so per-pixel state is 8 bytes whatever the depth.  The
peak device memory of one forward + backward is compared with what the
reference's store-all-layers caches need (5 floats per pixel per layer at the
deepest pixel, cuda_tile_rasterizer/tile_rasterize.cu:50-82)."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_memory_4096_n100k():
    from diffbmp_b200 import workloads as wl
    from diffbmp_b200._lib import call
    from diffbmp_b200.rasterizer import Atlas, Rasterizer, _ptr, _stream
    rng = np.random.default_rng(0)
    H = W = 4096
    N = 100000
    tm = wl.soft_disk(64, 24.0)[None]
    m, r, th, v, c, sel = wl.sample_params(rng, H, W, N, 1)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    means, radii, rot, opac, col = t(m), t(r), t(th), t(v), t(c)
    s = torch.from_numpy(sel).cuda()
    atlas = Atlas(t(tm))
    rz = Rasterizer(H, W, 32)
    torch.cuda.synchronize()
    torch.cuda.reset_peak_memory_stats()
    base = torch.cuda.memory_allocated()
    color, alpha, state = rz.forward(means, radii, rot, opac, col, s, atlas)
    gc = torch.full((H, W, 3), 1e-3, device="cuda")
    grads = rz.backward(state, gc, None, radii, rot, opac, col, atlas)
    torch.cuda.synchronize()
    peak = torch.cuda.max_memory_allocated() - base
    assert all(torch.isfinite(g).all() for g in grads)
    # deepest pixel without termination, i.e. the cache depth the reference would need
    cv = rz.canvas(N, atlas)
    cv.t_stop = 0.0
    cnt = torch.zeros(10, dtype=torch.int64, device="cuda")
    call("dbmp_count", ctypes.byref(cv), _ptr(state.prim_info), _ptr(atlas.data), _ptr(state.lists.offsets),
         _ptr(state.lists.indices), _ptr(cnt), _stream())
    K = int(cnt[6].item())
    store_all = 5 * H * W * K * 4 + H * W * 4
    print(f"4096^2, N=1e5: L={state.lists.length}, peak {peak / 2**30:.2f} GiB; per-pixel state 8 B; "
          f"deepest pixel {K} layers -> store-all-layers caches {store_all / 2**30:.1f} GiB")
    assert K > 400                         # beyond the reference's default cache depth
    assert peak < store_all / 20
    assert peak < 40 * 2**30
