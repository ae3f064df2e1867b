"""Drop-in for the reference's FP32 extension module `_C`
(cuda_tile_rasterizer/ext.cpp:110-121): same function names and argument
order, computed by libdbmp.so."""
from .. import _ext

FP16 = False


def init_tile_rasterizer(image_height, image_width, tile_size, sigma, alpha_upper_bound, max_prims_per_pixel,
                         num_primitives):
    _ext.init(image_height, image_width, tile_size, sigma, alpha_upper_bound, max_prims_per_pixel, num_primitives,
              FP16)


def rasterize_tiles_class(means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates,
                          global_bmp_sel, c_blend, tile_primitive_mapping):
    color, alpha, _ = _ext.forward(FP16, means2D, radii, rotations, opacities, colors, colors_orig,
                                   primitive_templates, global_bmp_sel, c_blend, tile_primitive_mapping)
    return color, alpha


def rasterize_tiles_backward_class(grad_out_color, grad_out_alpha, means2D, radii, rotations, opacities, colors,
                                   colors_orig, primitive_templates, global_bmp_sel, c_blend, lr_config_tensor):
    return _ext.backward(FP16, grad_out_color, grad_out_alpha, radii, rotations, opacities, colors)


def rasterize_tiles_batch_class(means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates,
                                global_bmp_sel, c_blend, tile_primitive_mappings):
    """(B,N,...) batch (tile_rasterize.cu:500-568): one forward launch over
    every candidate's tiles.  Every candidate keeps its own state, so the
    batch backward is exact for every candidate (the reference reuses the last
    candidate's caches)."""
    return _ext.forward_batch(FP16, means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates,
                              global_bmp_sel, c_blend, tile_primitive_mappings)


def rasterize_tiles_backward_batch_class(grad_out_color, grad_out_alpha, means2D, radii, rotations, opacities, colors,
                                         colors_orig, primitive_templates, global_bmp_sel, c_blend, lr_config):
    """Batch backward (tile_rasterize.cu:571-636): one launch."""
    return _ext.backward_batch(FP16, grad_out_color, grad_out_alpha, radii, rotations, opacities, colors)


def print_cuda_timing_stats():
    _ext.timing_stats(FP16)


def reset_cuda_timing_stats():
    _ext.reset_timing(FP16)
