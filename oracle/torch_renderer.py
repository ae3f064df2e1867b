"""TEST AND MEASUREMENT INFRASTRUCTURE -- a torch restatement of the
reference's PyTorch per-tile renderer, the CPU path of its rasterizer.

The reference renders on the host with SimpleTileRenderer._render_tile
(pydiffbmp/core/renderer/simple_tile_renderer.py:1304-1456) over the tile
lists of _process_tiles_parallel (:479-569): per tile, the primitives of its
list are mapped into template space (_generate_tile_masks, :1459-1548:
pos = (pixel - centre) / r, rotated by the inverse rotation), the templates
(template (N-1-i) % p per primitive) are sampled with F.grid_sample
(bilinear, zeros padding, align_corners=True), alpha = sigmoid(v) alpha_max,
colour = sigmoid(c) (with c_blend = -40 the colour-map term vanishes), and
the tile is composited with VectorRenderer._transmit_over
(vector_renderer.py:706-736: cumprod transmittance, weighted sum).  Gradients
come from torch autograd through those ops.

The reference's Python cannot run where the benchmarks run, so this
restatement stands in for it as the timed CPU baseline ("port"): the same
library, the same per-tile tensor shapes and ops.  tests/test_torch_port.py
pins it to images and gradients that the reference's own renderer produced
(tests/golden/torch_*.npz).  Only tests/ and bench.py's reference arm use it.
"""
from __future__ import annotations

import torch
import torch.nn.functional as F


def render_tile(t: int, H: int, W: int, ts: int, x, y, r, theta, v, c, templates, sel, alpha_max: float,
                offsets, indices):
    """One tile of the reference's CPU path: (comp_m (h,w,3), comp_a (h,w)),
    or None for an empty tile."""
    tiles_x = (W + ts - 1) // ts
    y0, x0 = (t // tiles_x) * ts, (t % tiles_x) * ts
    y1, x1 = min(y0 + ts, H), min(x0 + ts, W)
    lo, hi = int(offsets[t]), int(offsets[t + 1])
    if hi == lo:
        return None
    idx = indices[lo:hi].long()
    tx, ty, tr, tth = x[idx], y[idx], r[idx], theta[idx]
    n = idx.numel()
    X, Y = torch.meshgrid(torch.arange(x0, x1, dtype=torch.float32), torch.arange(y0, y1, dtype=torch.float32),
                          indexing="xy")
    h, w = X.shape
    pos = torch.stack([X.expand(n, h, w) - tx.view(n, 1, 1), Y.expand(n, h, w) - ty.view(n, 1, 1)], dim=1) \
        / tr.view(n, 1, 1, 1)
    cos_t, sin_t = torch.cos(tth), torch.sin(tth)
    R_inv = torch.stack([torch.stack([cos_t, sin_t], -1), torch.stack([-sin_t, cos_t], -1)], -2)   # (n,2,2)
    uv = torch.einsum("bij,bjhw->bihw", R_inv, pos)
    grid = uv.permute(0, 2, 3, 1)
    bmp = templates[sel[idx].long()].unsqueeze(1)                          # (n,1,Ht,Wt)
    masks = F.grid_sample(bmp, grid, mode="bilinear", padding_mode="zeros", align_corners=True).squeeze(1)
    alpha = torch.sigmoid(v[idx]) * alpha_max
    rgb = torch.sigmoid(c[idx])
    a = masks * alpha.view(-1, 1, 1)
    m = a.unsqueeze(-1) * rgb.view(-1, 1, 1, 3)
    T = torch.cat([torch.ones_like(a[:1]), torch.cumprod(1.0 - a, dim=0)], dim=0)
    comp_a = 1.0 - T[-1]
    comp_m = (m * T[:-1].unsqueeze(-1)).sum(dim=0)
    return comp_m, comp_a


def render(H: int, W: int, ts: int, x, y, r, theta, v, c, templates, sel, alpha_max: float, offsets, indices,
           tiles=None):
    """The image (H,W,3) and alpha (H,W) on a black background, tile by tile
    (all tiles, or those listed in `tiles`); differentiable."""
    color = torch.zeros((H, W, 3), dtype=torch.float32)
    alpha = torch.zeros((H, W), dtype=torch.float32)
    tiles_x = (W + ts - 1) // ts
    T = tiles_x * ((H + ts - 1) // ts)
    for t in (range(T) if tiles is None else tiles):
        out = render_tile(t, H, W, ts, x, y, r, theta, v, c, templates, sel, alpha_max, offsets, indices)
        if out is None:
            continue
        y0, x0 = (t // tiles_x) * ts, (t % tiles_x) * ts
        m, a = out
        color[y0:y0 + m.shape[0], x0:x0 + m.shape[1]] = m
        alpha[y0:y0 + a.shape[0], x0:x0 + a.shape[1]] = a
    return color, alpha
