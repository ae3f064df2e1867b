"""Drop-in replacement for the reference package `cuda_tile_rasterizer`
(smhongok/diffbmp cuda_tile_rasterizer/__init__.py): the same public names,
signatures and autograd behaviour, over libdbmp.so's sm_100a kernels.

    TileRasterizer(image_height, image_width, tile_size=16, sigma=0.0,
                   alpha_upper_bound=1.0, max_prims_per_pixel=151,
                   num_primitives=None, use_fp16=False)
        __call__(means2D, radii, rotations, opacities, colors, colors_orig,
                 primitive_templates, global_bmp_sel, c_blend, lr_conf,
                 tile_primitive_mapping=None) -> (color (H,W,3), alpha (H,W))
        forward_batch(...) -> (B,H,W,3), (B,H,W)
    TileRasterizerFunction / TileRasterizerFunctionFP16 /
    TileRasterizerBatchFunction: torch.autograd.Function, 16 inputs, gradients
    for the first five.
    CUDA_AVAILABLE, CUDA_FP16_AVAILABLE, print/reset_cuda_timing_stats[_fp16].

Unlike the reference, a failing call raises (no silent fallback), per-pixel
depth is unbounded (max_prims_per_pixel is accepted and ignored) and an empty
mapping is binned on the device instead of listing every primitive in every
tile (same image).
"""
import torch
from torch.autograd import Function

from .cuda_tile_rasterizer import _C
from .cuda_tile_rasterizer_fp16 import _C_fp16

CUDA_AVAILABLE = True
CUDA_FP16_AVAILABLE = True


class TileRasterizer:
    """Class-based tile rasterizer (reference __init__.py:60-121)."""

    def __init__(self, image_height, image_width, tile_size=16, sigma=0.0, alpha_upper_bound=1.0,
                 max_prims_per_pixel=151, num_primitives=None, use_fp16=False):
        self.image_height = image_height
        self.image_width = image_width
        self.tile_size = tile_size
        self.sigma = sigma
        self.alpha_upper_bound = alpha_upper_bound
        self.max_prims_per_pixel = max_prims_per_pixel
        self.num_primitives = num_primitives
        self.use_fp16 = use_fp16
        if use_fp16:
            self.apply_fn = TileRasterizerFunctionFP16.apply
            _C_fp16.init_tile_rasterizer_fp16(image_height, image_width, tile_size, sigma, alpha_upper_bound,
                                              max_prims_per_pixel, num_primitives)
        else:
            self.apply_fn = TileRasterizerFunction.apply
            _C.init_tile_rasterizer(image_height, image_width, tile_size, sigma, alpha_upper_bound,
                                    max_prims_per_pixel, num_primitives)

    def __call__(self, means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates, global_bmp_sel,
                 c_blend, lr_conf, tile_primitive_mapping=None):
        return self.apply_fn(means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates,
                             global_bmp_sel, c_blend, lr_conf, tile_primitive_mapping, self.image_height,
                             self.image_width, self.tile_size, self.sigma, True)

    def forward_batch(self, means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates,
                      global_bmp_sel, c_blend, lr_conf, tile_primitive_mappings=None):
        return TileRasterizerBatchFunction.apply(means2D, radii, rotations, opacities, colors, colors_orig,
                                                 primitive_templates, global_bmp_sel, c_blend, lr_conf,
                                                 tile_primitive_mappings, self.image_height, self.image_width,
                                                 self.tile_size, self.sigma, self.use_fp16)


def _scalar(c_blend):
    return float(c_blend.item()) if isinstance(c_blend, torch.Tensor) else float(c_blend)


class TileRasterizerFunction(Function):
    """Reference __init__.py:254-340 (FP32 extension)."""

    @staticmethod
    def forward(ctx, means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates, global_bmp_sel,
                c_blend, lr_conf, tile_primitive_mapping, image_height, image_width, tile_size, sigma,
                use_class=False):
        args = [t.float() for t in (means2D, radii, rotations, opacities, colors)]
        sel = global_bmp_sel.to(torch.int32)
        ctx.save_for_backward(*args, colors_orig, primitive_templates, sel)
        ctx.c_blend = _scalar(c_blend)
        ctx.hw = (int(image_height), int(image_width))
        return _C.rasterize_tiles_class(*args, colors_orig, primitive_templates.float(), sel, ctx.c_blend,
                                        tile_primitive_mapping)

    @staticmethod
    def backward(ctx, grad_out_color, grad_out_alpha):
        means2D, radii, rotations, opacities, colors, colors_orig, templates, sel = ctx.saved_tensors
        if grad_out_color is None:
            grad_out_color = torch.zeros((*ctx.hw, 3), dtype=torch.float32, device=means2D.device)
        grads = _C.rasterize_tiles_backward_class(grad_out_color, grad_out_alpha, means2D, radii, rotations,
                                                  opacities, colors, colors_orig, templates, sel, ctx.c_blend, None)
        return (*grads, None, None, None, None, None, None, None, None, None, None, None)


class TileRasterizerFunctionFP16(Function):
    """Reference __init__.py:342-436 (FP16 extension): half tensors in and out."""

    @staticmethod
    def forward(ctx, means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates, global_bmp_sel,
                c_blend, lr_conf, tile_primitive_mapping, image_height, image_width, tile_size, sigma,
                use_class=False):
        args = [t.to(torch.float16) for t in (means2D, radii, rotations, opacities, colors)]
        sel = global_bmp_sel.to(torch.int32)
        tmpl = primitive_templates.to(torch.float16)
        ctx.save_for_backward(*args, colors_orig, tmpl, sel)
        ctx.c_blend = _scalar(c_blend)
        return _C_fp16.rasterize_tiles_class_fp16(*args, colors_orig, tmpl, sel, ctx.c_blend,
                                                  tile_primitive_mapping)

    @staticmethod
    def backward(ctx, grad_out_color, grad_out_alpha):
        means2D, radii, rotations, opacities, colors, colors_orig, templates, sel = ctx.saved_tensors
        grads = _C_fp16.rasterize_tiles_backward_class_fp16(grad_out_color, grad_out_alpha, means2D, radii,
                                                            rotations, opacities, colors, colors_orig, templates,
                                                            sel, ctx.c_blend, None)
        return (*grads, None, None, None, None, None, None, None, None, None, None, None)


class TileRasterizerBatchFunction(Function):
    """Reference __init__.py:124-252: (B,N,...) candidates, shared templates."""

    @staticmethod
    def forward(ctx, means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates, global_bmp_sel,
                c_blend, lr_conf, tile_primitive_mappings, image_height, image_width, tile_size, sigma,
                use_fp16=False):
        dt = torch.float16 if use_fp16 else torch.float32
        args = [t.to(dt).contiguous() for t in (means2D, radii, rotations, opacities, colors)]
        sel = global_bmp_sel.to(torch.int32).contiguous()
        tmpl = primitive_templates.to(dt).contiguous()
        ctx.save_for_backward(*args, tmpl, sel)
        ctx.c_blend = _scalar(c_blend)
        ctx.use_fp16 = use_fp16
        if use_fp16:
            return _C_fp16.rasterize_tiles_batch_class_fp16(*args, colors_orig, tmpl, sel, ctx.c_blend,
                                                            tile_primitive_mappings)
        return _C.rasterize_tiles_batch_class(*args, colors_orig, tmpl, sel, ctx.c_blend, tile_primitive_mappings)

    @staticmethod
    def backward(ctx, grad_out_color, grad_out_alpha):
        means2D, radii, rotations, opacities, colors, tmpl, sel = ctx.saved_tensors
        from . import _ext
        # one backward launch over every candidate (the reference loops, __init__.py:195-252)
        grads = _ext.backward_batch(ctx.use_fp16, grad_out_color, grad_out_alpha, radii, rotations, opacities, colors)
        return (*grads, None, None, None, None, None, None, None, None, None, None, None)


def print_cuda_timing_stats():
    _C.print_cuda_timing_stats()


def reset_cuda_timing_stats():
    _C.reset_cuda_timing_stats()


def print_cuda_timing_stats_fp16():
    _C_fp16.print_cuda_timing_stats_fp16()


def reset_cuda_timing_stats_fp16():
    _C_fp16.reset_cuda_timing_stats_fp16()
