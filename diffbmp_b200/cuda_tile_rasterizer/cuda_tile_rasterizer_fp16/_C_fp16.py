"""Drop-in for the reference's FP16 extension module `_C_fp16`
(cuda_tile_rasterizer/ext_fp16.cpp:72-83).  The reference computes everything
in half, transmittance included; here the atlas is stored in half and the
arithmetic, transmittance and gradient sums stay in FP32 (an improved-accuracy
superset).  Inputs and outputs are float16 tensors as in the reference."""
from .. import _ext

FP16 = True


def init_tile_rasterizer_fp16(image_height, image_width, tile_size, sigma, alpha_upper_bound, max_prims_per_pixel,
                              num_primitives):
    _ext.init(image_height, image_width, tile_size, sigma, alpha_upper_bound, max_prims_per_pixel, num_primitives,
              FP16)


def rasterize_tiles_class_fp16(means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates,
                               global_bmp_sel, c_blend, tile_primitive_mapping):
    return _ext.forward(FP16, means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates,
                        global_bmp_sel, c_blend, tile_primitive_mapping)


def rasterize_tiles_backward_class_fp16(grad_out_color, grad_out_alpha, means2D, radii, rotations, opacities, colors,
                                        colors_orig, primitive_templates, global_bmp_sel, c_blend, lr_config_tensor):
    return _ext.backward(FP16, grad_out_color, grad_out_alpha, radii, rotations, opacities, colors)


def rasterize_tiles_batch_class_fp16(means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates,
                                     global_bmp_sel, c_blend, tile_primitive_mapping):
    """One mapping shared by the whole batch (ext_fp16.cpp:53-70); one
    forward launch over every candidate's tiles."""
    return _ext.forward_batch(FP16, means2D, radii, rotations, opacities, colors, colors_orig, primitive_templates,
                              global_bmp_sel, c_blend, tile_primitive_mapping)


def print_cuda_timing_stats_fp16():
    _ext.timing_stats(FP16)


def reset_cuda_timing_stats_fp16():
    _ext.reset_timing(FP16)
