"""TEST INFRASTRUCTURE -- torch restatement of the reference's tile binning.

The reference bins primitives with float32 torch element-wise ops on the
rendering device (pydiffbmp/core/renderer/vector_renderer.py:194-252
_compute_primitive_world_bboxes and :401-444 _unified_primitive_assignment,
then simple_tile_renderer.py:721-766 _convert_masks_to_mapping).  Running this
restatement on a CUDA tensor reproduces the reference's GPU arithmetic
(torch.cos / torch.sin kernels, one rounding per op), which is the target the
device binning must match bit for bit.  Only tests/ use this module.
"""
from __future__ import annotations

import torch


def world_bboxes(x, y, r, theta, tbbox, bbox_sel):
    """vector_renderer.py:214-250 (template bbox chosen by bbox_sel)."""
    cos_t = torch.cos(theta)
    sin_t = torch.sin(theta)
    sel = tbbox[bbox_sel.long()]
    min_u, max_u, min_v, max_v = sel[:, 0], sel[:, 1], sel[:, 2], sel[:, 3]
    cu = torch.stack([min_u, max_u, min_u, max_u], dim=1)
    cv = torch.stack([min_v, min_v, max_v, max_v], dim=1)
    wx = x.unsqueeze(1) + r.unsqueeze(1) * (cu * cos_t.unsqueeze(1) - cv * sin_t.unsqueeze(1))
    wy = y.unsqueeze(1) + r.unsqueeze(1) * (cu * sin_t.unsqueeze(1) + cv * cos_t.unsqueeze(1))
    return wx.min(dim=1)[0], wx.max(dim=1)[0], wy.min(dim=1)[0], wy.max(dim=1)[0]


def tile_bounds(H, W, ts, device):
    th, tw = (H + ts - 1) // ts, (W + ts - 1) // ts
    ty = torch.arange(th, device=device).repeat_interleave(tw)
    tx = torch.arange(tw, device=device).repeat(th)
    ys = ty * ts
    ye = torch.clamp(ys + ts, max=H)
    xs = tx * ts
    xe = torch.clamp(xs + ts, max=W)
    return xs, xe, ys, ye


def mapping(H, W, ts, means2D, radii, rotations, tbbox, bbox_sel):
    """Reference mapping tensor int32 [T+1, L, offsets..., indices...]."""
    x, y = means2D[:, 0].contiguous(), means2D[:, 1].contiguous()
    bxmin, bxmax, bymin, bymax = world_bboxes(x, y, radii, rotations, tbbox, bbox_sel)
    xs, xe, ys, ye = tile_bounds(H, W, ts, means2D.device)
    xi = ~((bxmax.unsqueeze(1) < xs.unsqueeze(0)) | (bxmin.unsqueeze(1) > xe.unsqueeze(0)))
    yi = ~((bymax.unsqueeze(1) < ys.unsqueeze(0)) | (bymin.unsqueeze(1) > ye.unsqueeze(0)))
    masks = (xi & yi).t()                      # (T, N)
    counts = masks.sum(dim=1).to(torch.int32)
    offsets = torch.zeros(masks.shape[0] + 1, dtype=torch.int32, device=means2D.device)
    offsets[1:] = torch.cumsum(counts, 0).to(torch.int32)
    indices = torch.nonzero(masks, as_tuple=True)[1].to(torch.int32)   # row-major: tile, then prim
    head = torch.tensor([offsets.numel(), indices.numel()], dtype=torch.int32, device=means2D.device)
    return torch.cat([head, offsets, indices])
