"""Shared implementation of the drop-in extension modules `_C` and `_C_fp16`.

The reference's extensions (cuda_tile_rasterizer/ext.cpp:5-121 and
ext_fp16.cpp:5-83) keep one process-global TileRasterizer that owns the
per-pixel caches between a forward and the following backward.  This module
keeps the same global-by-design contract (init_* replaces it) on top of
libdbmp.so: the forward keeps its ForwardState, the backward consumes it.
Every computation runs in the library's CUDA kernels; there is no fallback.
"""
from __future__ import annotations

import time

import torch

from diffbmp_b200 import rasterizer as R


class _Global:
    def __init__(self, H, W, ts, alpha_ub, fp16):
        self.H, self.W, self.ts = int(H), int(W), int(ts)
        self.alpha_ub = float(alpha_ub)
        self.fp16 = fp16
        self.kind = "f16" if fp16 else "f32"
        # an empty mapping means "every primitive in every tile" in the reference
        # (tile_rasterize.cu:171-194); the cull-square binning is its tight form
        self.rz_cull = R.Rasterizer(H, W, ts, alpha_ub, bin_mode=R.BIN_CULL)
        self.rz_map = R.Rasterizer(H, W, ts, alpha_ub, bin_mode=R.BIN_CONTENT)
        self.atlas_key = None
        self.atlas = None
        self.states = []
        self.batch_state = None     # (BatchState, rasterizer, atlas) of the last forward_batch
        self.t_fwd = self.t_bwd = 0.0
        self.n_fwd = self.n_bwd = 0

    def get_atlas(self, templates: torch.Tensor) -> R.Atlas:
        t = templates if templates.dim() == 3 else templates.unsqueeze(0)
        key = (t.data_ptr(), tuple(t.shape), t._version, t.dtype)
        if key != self.atlas_key:
            self.atlas = R.Atlas(t.float(), self.kind)
            self.atlas_key = key
        return self.atlas


_G: dict = {}


def init(H, W, ts, sigma, alpha_ub, max_prims_per_pixel, num_primitives, fp16=False):
    """init_tile_rasterizer(H, W, tile_size, sigma, alpha_upper_bound,
    max_prims_per_pixel, num_primitives): max_prims_per_pixel is accepted and
    unused (no per-layer caches exist here, depth is unbounded)."""
    _G[fp16] = _Global(H, W, ts, alpha_ub, fp16)


def _get(fp16):
    g = _G.get(fp16)
    if g is None:
        raise RuntimeError("TileRasterizer not initialized. Call init_tile_rasterizer first.")
    return g


def _f(t):
    return t.detach().to(torch.float32).contiguous()


def forward(fp16, means2D, radii, rotations, opacities, colors, colors_orig, templates, sel, c_blend, mapping,
            keep=True):
    g = _get(fp16)
    t0 = time.perf_counter()
    atlas = g.get_atlas(templates)
    m, r, th, v, c = _f(means2D).view(-1, 2), _f(radii).view(-1), _f(rotations).view(-1), _f(opacities).view(-1), \
        _f(colors).view(-1, 3)
    s = sel.to(torch.int32).contiguous().view(-1)
    has_map = mapping is not None and isinstance(mapping, torch.Tensor) and mapping.numel() > 0
    rz = g.rz_map if has_map else g.rz_cull
    # colour-map blending (tile_forward.cu:316-330) when colors_orig is given and c_blend > 0
    blend = colors_orig is not None and isinstance(colors_orig, torch.Tensor) and colors_orig.numel() > 0 \
        and float(c_blend) > 0.0
    color, alpha, state = rz.forward(m, r, th, v, c, s, atlas, mapping if has_map else None, None,
                                     _f(colors_orig) if blend else None, float(c_blend) if blend else 0.0)
    if keep:
        g.states = [(state, rz, atlas)]
    g.t_fwd += (time.perf_counter() - t0) * 1e3
    g.n_fwd += 1
    if fp16:
        return color.half(), alpha.half()
    return color, alpha, (state, rz, atlas)


def backward(fp16, grad_color, grad_alpha, radii, rotations, opacities, colors, saved=None):
    g = _get(fp16)
    if saved is None:
        if not g.states:
            raise RuntimeError("TileRasterizer not initialized or forward pass not called.")
        saved = g.states[-1]
    state, rz, atlas = saved
    t0 = time.perf_counter()
    gm, gr, gth, gv, gc = rz.backward(state, _f(grad_color), None if grad_alpha is None else _f(grad_alpha),
                                      _f(radii).view(-1), _f(rotations).view(-1), _f(opacities).view(-1),
                                      _f(colors).view(-1, 3), atlas)
    g.t_bwd += (time.perf_counter() - t0) * 1e3
    g.n_bwd += 1
    out = (gm, gr, gth, gv, gc)
    if fp16:
        out = tuple(x.half() for x in out)
    return out


def forward_batch(fp16, means2D, radii, rotations, opacities, colors, colors_orig, templates, sel, c_blend,
                  mappings):
    """B candidates (leading dimension) in one forward launch.  mappings: a
    list of B reference mapping tensors, one tensor shared by every candidate
    (the FP16 extension's form, tile_rasterize_fp16.cpp:501-560), or None
    (device binning per candidate).  Keeps the batch state for backward_batch
    and returns (color (B,H,W,3), alpha (B,H,W))."""
    g = _get(fp16)
    t0 = time.perf_counter()
    atlas = g.get_atlas(templates)
    B = int(radii.shape[0])
    m = _f(means2D).view(B, -1, 2)
    r, th, v = _f(radii).view(B, -1), _f(rotations).view(B, -1), _f(opacities).view(B, -1)
    c = _f(colors).view(B, -1, 3)
    s = sel.to(torch.int32).contiguous()
    if isinstance(mappings, torch.Tensor):
        mappings = [mappings] * B if mappings.numel() > 0 else None
    elif mappings is not None:
        mappings = [mp for mp in mappings if mp is not None and mp.numel() > 0] or None
    rz = g.rz_map if mappings is not None else g.rz_cull
    blend = colors_orig is not None and isinstance(colors_orig, torch.Tensor) and colors_orig.numel() > 0 \
        and float(c_blend) > 0.0
    color, alpha, state = rz.forward_batch(m, r, th, v, c, s, atlas, mappings, None,
                                           _f(colors_orig) if blend else None, float(c_blend) if blend else 0.0)
    g.batch_state = (state, rz, atlas)
    g.t_fwd += (time.perf_counter() - t0) * 1e3
    g.n_fwd += 1
    if fp16:
        return color.half(), alpha.half()
    return color, alpha


def backward_batch(fp16, grad_color, grad_alpha, radii, rotations, opacities, colors):
    """The five gradients of every candidate of the last forward_batch, one
    backward launch: (B,N,2), (B,N), (B,N), (B,N), (B,N,3)."""
    g = _get(fp16)
    if getattr(g, "batch_state", None) is None:
        raise RuntimeError("backward_batch must follow a forward_batch")
    state, rz, atlas = g.batch_state
    B = int(radii.shape[0])
    if state.batch != B:
        raise RuntimeError(f"backward_batch of {B} candidates after a forward_batch of {state.batch}")
    t0 = time.perf_counter()
    out = rz.backward_batch(state, _f(grad_color), None if grad_alpha is None else _f(grad_alpha),
                            _f(radii).view(B, -1), _f(rotations).view(B, -1), _f(opacities).view(B, -1),
                            _f(colors).view(B, -1, 3), atlas)
    g.t_bwd += (time.perf_counter() - t0) * 1e3
    g.n_bwd += 1
    if fp16:
        out = tuple(x.half() for x in out)
    return out


def timing_stats(fp16):
    g = _G.get(fp16)
    if g is None:
        print("No TileRasterizer instance available for timing stats.")
        return
    print("=== CUDA Tile Rasterizer Timing Statistics ===")
    print(f"Forward Pass: total {g.t_fwd:.3f} ms over {g.n_fwd} iterations (host wall time, asynchronous launches)")
    print(f"Backward Pass: total {g.t_bwd:.3f} ms over {g.n_bwd} iterations")


def reset_timing(fp16):
    g = _G.get(fp16)
    if g is not None:
        g.t_fwd = g.t_bwd = 0.0
        g.n_fwd = g.n_bwd = 0
    print("Timing statistics reset.")
