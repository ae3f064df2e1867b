"""Drop-in for cuda_tile_rasterizer/psd_export_uint8.py: export_psd_layers_cuda_uint8
with the reference's signature and return value (the PixelLayer helper
needs psd-tools and is imported lazily)."""
from diffbmp_b200.psd import export_psd_layers_uint8

CUDA_AVAILABLE = True


def export_psd_layers_cuda_uint8(renderer_S, x, y, r, theta, v, c, global_bmp_sel, H, W, scale_factor=1.0,
                                 alpha_upper_bound=1.0, c_blend=0.0, primitive_colors=None):
    return export_psd_layers_uint8(renderer_S, x, y, r, theta, v, c, global_bmp_sel, H, W, scale_factor,
                                   alpha_upper_bound, c_blend, primitive_colors)


def create_pixel_layers_from_numpy(numpy_arrays, bounds_list, valid_indices, names, psd_file):
    from PIL import Image
    from psd_tools.api.layers import PixelLayer   # optional dependency of PSD file writing
    layers = []
    for arr, (left, top, _, _), idx in zip(numpy_arrays, bounds_list, valid_indices):
        layer = PixelLayer.frompil(Image.fromarray(arr, "RGBA"), psd_file, names[idx], top, left)
        layers.append(layer)
    return layers
