"""Drop-in for the reference extension `psd_export_cuda`
(cuda_tile_rasterizer/psd_export_bindings.cpp:38-129): outputs written in
place, bytes identical to the reference's kernels."""
import ctypes

import torch

from diffbmp_b200._lib import call
from diffbmp_b200.rasterizer import _ptr, _stream


def _check(t, dtype, name):
    if not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor")
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}")


def compute_bounding_boxes(means2D, radii, rotations, primitive_templates, global_bmp_sel, output_bounding_boxes,
                           cropped_sizes, H, W, scale_factor, alpha_upper_bound):
    _check(means2D, torch.float32, "means2D")
    _check(output_bounding_boxes, torch.int32, "output_bounding_boxes")
    N = means2D.shape[0]
    call("dbmp_psd_bboxes", _ptr(means2D.contiguous()), _ptr(radii.contiguous()), N, int(H), int(W),
         ctypes.c_float(scale_factor), _ptr(output_bounding_boxes), _ptr(cropped_sizes), _stream())


def generate_cropped_layers(means2D, radii, rotations, colors, visibility, primitive_templates, global_bmp_sel,
                            bounding_boxes, layer_offsets, cropped_output_buffer, H, W, scale_factor,
                            alpha_upper_bound, c_blend, colors_orig):
    _check(means2D, torch.float32, "means2D")
    _check(cropped_output_buffer, torch.uint8, "cropped_output_buffer")
    N = means2D.shape[0]
    t = primitive_templates.float().contiguous()
    t = t.unsqueeze(0) if t.dim() == 2 else t
    P, Ht, Wt = (int(v) for v in t.shape)
    bb = bounding_boxes.contiguous()
    sizes = torch.stack([bb[:, 2] - bb[:, 0], bb[:, 3] - bb[:, 1]], 1).to(torch.int32).contiguous()
    offs = torch.empty(max(N, 1), dtype=torch.int64, device=means2D.device)
    blk = torch.empty(N + 1, dtype=torch.int64, device=means2D.device)
    total = torch.empty(1, dtype=torch.int64, device=means2D.device)
    st = _stream()
    call("dbmp_psd_layout", _ptr(sizes), N, _ptr(offs), _ptr(blk), _ptr(total), st)
    lo = layer_offsets.to(torch.int64).contiguous()    # the caller's offsets (reference: host prefix sum)
    co = colors_orig if (colors_orig is not None and colors_orig.numel() > 0 and c_blend > 0.0) else None
    call("dbmp_psd_layers", _ptr(means2D.contiguous()), _ptr(radii.contiguous()), _ptr(rotations.contiguous()),
         _ptr(colors.contiguous()), _ptr(visibility.contiguous()), _ptr(t), P, Ht, Wt,
         _ptr(global_bmp_sel.to(torch.int32).contiguous()), _ptr(bb), _ptr(lo), _ptr(blk), N,
         ctypes.c_float(scale_factor), ctypes.c_float(alpha_upper_bound), ctypes.c_float(c_blend),
         _ptr(co.float().contiguous() if co is not None else None), _ptr(cropped_output_buffer), st)
