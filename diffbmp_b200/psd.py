"""PSD layer export on the device (cuda_tile_rasterizer/psd_export_uint8.py:22-150
and psd_export_kernels.cu rebuilt over libdbmp.so).

``export_layers`` returns the packed uint8 RGBA crops on the device plus their
boxes; ``export_psd_layers_uint8`` mirrors the reference's
``export_psd_layers_cuda_uint8`` return value (list of (h,w,4) uint8 arrays,
their (left, top, right, bottom) boxes and original indices, skipping layers
of width or height <= 1 and fully transparent ones).  Writing the PSD file
itself (psd-tools) is left to the caller.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import call
from .rasterizer import _ptr, _stream


def _f32(t):
    return t.detach().to(torch.float32).contiguous()


def export_layers(templates, means2D, radii, rotations, vis_sig, colors_sig, sel, H, W, scale=1.0,
                  alpha_max=1.0, c_blend=0.0, colors_orig=None):
    """Returns (buffer uint8 (total,), bboxes (N,4) i32, sizes (N,2) i32,
    layer_offsets (N,) i64), all on the device.  colors_sig / vis_sig are the
    sigmoid-ed colours / opacities (psd_exporter.py:80-81)."""
    dev = means2D.device
    t = _f32(templates)
    t = t.unsqueeze(0) if t.dim() == 2 else t
    P, Ht, Wt = (int(v) for v in t.shape)
    m, r, th, v, c = (_f32(x) for x in (means2D, radii, rotations, vis_sig, colors_sig))
    m = m.view(-1, 2)
    N = int(r.numel())
    s = sel.to(device=dev, dtype=torch.int32).contiguous()
    st = _stream()
    bbox = torch.empty((N, 4), dtype=torch.int32, device=dev)
    sizes = torch.empty((N, 2), dtype=torch.int32, device=dev)
    call("dbmp_psd_bboxes", _ptr(m), _ptr(r), N, int(H), int(W), ctypes.c_float(scale), _ptr(bbox), _ptr(sizes), st)
    offs = torch.empty(max(N, 1), dtype=torch.int64, device=dev)
    blk = torch.empty(N + 1, dtype=torch.int64, device=dev)
    total = torch.empty(1, dtype=torch.int64, device=dev)
    call("dbmp_psd_layout", _ptr(sizes), N, _ptr(offs), _ptr(blk), _ptr(total), st)
    nbytes = int(total.item())            # the reference sizes its buffer on the host as well
    out = torch.empty(max(nbytes, 4), dtype=torch.uint8, device=dev)
    co = None
    if colors_orig is not None and c_blend > 0.0:
        co = _f32(colors_orig).view(-1)
    call("dbmp_psd_layers", _ptr(m), _ptr(r), _ptr(th), _ptr(c), _ptr(v), _ptr(t), P, Ht, Wt, _ptr(s), _ptr(bbox),
         _ptr(offs), _ptr(blk), N, ctypes.c_float(scale), ctypes.c_float(alpha_max), ctypes.c_float(c_blend),
         _ptr(co), _ptr(out), st)
    return out[:nbytes], bbox, sizes, offs[:N]


def export_psd_layers_uint8(templates, x, y, r, theta, v_sig, c_sig, sel, H, W, scale=1.0, alpha_max=1.0,
                            c_blend=0.0, primitive_colors=None):
    """Host-side result in the reference's format
    (cuda_tile_rasterizer/psd_export_uint8.py:125-150)."""
    means2D = torch.stack([x.float(), y.float()], 1)
    co = None
    if primitive_colors is not None and c_blend > 0.0:
        pc = primitive_colors.to(means2D.device).float()
        if pc.dim() == 4:
            co = pc[sel.long()]
        else:
            co = pc[sel.long()][:, None, None, :].expand(len(x), templates.shape[-2], templates.shape[-1], 3)
    buf, bbox, sizes, offs = export_layers(templates, means2D, r, theta, v_sig, c_sig, sel, H, W, scale, alpha_max,
                                           c_blend, co)
    hb, hs, ho, hbuf = bbox.cpu().numpy(), sizes.cpu().numpy(), offs.cpu().numpy(), buf.cpu().numpy()
    arrays, bounds, idx = [], [], []
    for i in range(len(hb)):
        w, h = hs[i]
        if w <= 1 or h <= 1:
            continue
        a = hbuf[ho[i]: ho[i] + w * h * 4].reshape(h, w, 4)
        if a[:, :, 3].max() > 0:
            arrays.append(a)
            bounds.append(tuple(int(v) for v in hb[i]))
            idx.append(i)
    return arrays, bounds, idx
