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
    """(B,N,...) batch; one forward per candidate like tile_rasterize.cu:500-568,
    but every candidate keeps its own state, so the batch backward is exact
    for every candidate (the reference reuses the last candidate's caches)."""
    import torch
    B = means2D.shape[0]
    maps = tile_primitive_mappings if tile_primitive_mappings is not None else []
    cols, alps, states = [], [], []
    for b in range(B):
        mp = maps[b] if b < len(maps) else None
        co = colors_orig[b] if colors_orig is not None and colors_orig.dim() == 5 else colors_orig
        c, a, st = _ext.forward(FP16, means2D[b], radii[b], rotations[b], opacities[b], colors[b], co,
                                primitive_templates, global_bmp_sel, c_blend, mp, keep=False)
        cols.append(c); alps.append(a); states.append(st)
    _ext._get(FP16).states = states
    return torch.stack(cols), torch.stack(alps)


def rasterize_tiles_backward_batch_class(grad_out_color, grad_out_alpha, means2D, radii, rotations, opacities, colors,
                                         colors_orig, primitive_templates, global_bmp_sel, c_blend, lr_config):
    import torch
    g = _ext._get(FP16)
    B = means2D.shape[0]
    if len(g.states) != B:
        raise RuntimeError("backward_batch must follow a forward_batch of the same size")
    outs = [_ext.backward(FP16, grad_out_color[b], None if grad_out_alpha is None else grad_out_alpha[b], radii[b],
                          rotations[b], opacities[b], colors[b], saved=g.states[b]) for b in range(B)]
    return tuple(torch.stack([o[k] for o in outs]) for k in range(5))


def print_cuda_timing_stats():
    _ext.timing_stats(FP16)


def reset_cuda_timing_stats():
    _ext.reset_timing(FP16)
