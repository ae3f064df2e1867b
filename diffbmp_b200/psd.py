"""PSD layer export on the device (cuda_tile_rasterizer/psd_export_uint8.py:22-150
and psd_export_kernels.cu rebuilt over libdbmp.so).

``export_layers`` returns the packed uint8 RGBA crops on the device plus their
boxes; ``export_psd_layers_uint8`` mirrors the reference's
``export_psd_layers_cuda_uint8`` return value (list of (h,w,4) uint8 arrays,
their (left, top, right, bottom) boxes and original indices, skipping layers
of width or height <= 1 and fully transparent ones).

``PSDExporter`` (pydiffbmp/util/psd_exporter.py:11-501) writes the layered
PSD file itself, which the reference does with psd-tools: the channels of
every layer are PackBits-encoded on the device (dbmp_psd_rle_count /
dbmp_psd_rle_write) and the host only assembles the header, the layer records
and one blob of channel data (``encode_channel_blocks``, ``write_psd``).
"""
from __future__ import annotations

import ctypes
import struct

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


def _colors_orig(primitive_colors, sel, n, templates, device, c_blend):
    """Per-primitive colour maps (N,Ht,Wt,3) gathered by template id, or None
    (psd_export_uint8.py:89-113): (P,Ht,Wt,3) maps are gathered, (P,3)
    colours are broadcast over the template."""
    if primitive_colors is None or not c_blend > 0.0:
        return None
    pc = primitive_colors.to(device).float()
    if pc.dim() == 4:
        return pc[sel.long()]
    if pc.dim() == 2:
        return pc[sel.long()][:, None, None, :].expand(n, templates.shape[-2], templates.shape[-1], 3)
    raise ValueError(f"Unexpected primitive_colors shape: {tuple(pc.shape)}")


def export_psd_layers_uint8(templates, x, y, r, theta, v_sig, c_sig, sel, H, W, scale=1.0, alpha_max=1.0,
                            c_blend=0.0, primitive_colors=None):
    """Host-side result in the reference's format
    (cuda_tile_rasterizer/psd_export_uint8.py:125-150)."""
    means2D = torch.stack([x.float(), y.float()], 1)
    co = _colors_orig(primitive_colors, sel, len(x), templates, means2D.device, c_blend)
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


# ---------------------------------------------------------------------------
# PSD file assembly (the part the reference delegates to psd-tools).
# ---------------------------------------------------------------------------

PSD_MAX_SIDE = 30000          # width / height limit of a PSD (version 1) file
ORDER_LAYER = 0x02010003      # channel slots of a layer record: A, R, G, B
ORDER_MERGED = 0x03020100     # channels of the merged image: R, G, B, A
LAYER_CHANNEL_IDS = (-1, 0, 1, 2)


def encode_channel_blocks(buf, sizes, offsets, host_sizes, order, select, width_limit=PSD_MAX_SIDE, stream=None):
    """PackBits-encode every channel of N packed uint8 RGBA images on the device.

    ``buf`` (uint8), ``sizes`` ((N,2) i32 w,h) and ``offsets`` ((N,) i64 byte
    offset of each image) are device tensors, as ``export_layers`` returns
    them; ``host_sizes`` is the same (N,2) array on the host.  ``select`` maps
    the per-image "has a nonzero alpha byte" flags (numpy (N,) i32) to the
    images to encode, in the order their blocks go into the blob.

    Returns (blob, block_bytes, chosen): the device uint8 blob of PSD channel
    blocks (4 per chosen image, slots in ``order``, each = compression word,
    big-endian row sizes, PackBits rows), the (len(chosen), 4) block sizes and
    the chosen indices.  The host reads back only per-group sizes and flags.
    """
    dev = buf.device
    hs = np.asarray(host_sizes, dtype=np.int64).reshape(-1, 2)
    n = hs.shape[0]
    h = np.maximum(hs[:, 1], 0)
    ngroups = (h + 31) // 32
    group_base = np.zeros(n + 1, np.int64)
    group_base[1:] = np.cumsum(ngroups)
    G = int(group_base[-1])
    st = _stream(stream)
    gb = torch.from_numpy(group_base).to(dev)
    row_bytes = torch.empty(max(G, 1) * 32 * 4, dtype=torch.int16, device=dev)
    group_tot = torch.empty((max(G, 1), 4), dtype=torch.int32, device=dev)
    alpha_any = torch.zeros(max(n, 1), dtype=torch.int32, device=dev)
    call("dbmp_psd_rle_count", _ptr(buf), _ptr(sizes), _ptr(offsets), _ptr(gb), n, G, _check_order(order),
         int(width_limit), _ptr(row_bytes), _ptr(group_tot), _ptr(alpha_any), st)
    gt = group_tot[:G].cpu().numpy().astype(np.int64)
    chosen = np.asarray(select(alpha_any[:n].cpu().numpy()), dtype=np.int64).reshape(-1)
    if len(np.unique(chosen)) != len(chosen) or (len(chosen) and (chosen.min() < 0 or chosen.max() >= n)):
        raise ValueError("select must return distinct image indices")
    cs = np.zeros((G + 1, 4), np.int64)
    cs[1:] = np.cumsum(gt, axis=0)
    block = 2 + 2 * h[:, None] + (cs[group_base[1:]] - cs[group_base[:-1]])      # (n,4) bytes per block
    chan_off = np.full((n, 4), -1, np.int64)
    flat = block[chosen].reshape(-1)
    starts = np.concatenate([[0], np.cumsum(flat)[:-1]]) if len(flat) else flat
    chan_off[chosen] = starts.reshape(-1, 4)
    total = int(flat.sum())
    layer_of = np.repeat(np.arange(n), ngroups)
    gdst = chan_off[layer_of] + 2 + 2 * h[layer_of, None] + (cs[:-1] - cs[group_base[layer_of]])
    gdst[chan_off[layer_of] < 0] = -1
    out = torch.empty(max(total, 16), dtype=torch.uint8, device=dev)
    co = torch.from_numpy(chan_off).to(dev)
    gd = torch.from_numpy(np.ascontiguousarray(gdst)).to(dev)
    call("dbmp_psd_rle_write", _ptr(buf), _ptr(sizes), _ptr(offsets), _ptr(gb), n, G, _check_order(order),
         int(width_limit), _ptr(row_bytes), _ptr(co), _ptr(gd), _ptr(out), total, st)
    return out[:total], block[chosen], chosen


def _check_order(order):
    order = int(order)
    if order & ~0x03030303:
        raise ValueError(f"channel order 0x{order:08x}: each byte must be 0..3")
    return order


def _pascal4(name: str) -> bytes:
    """Pascal string padded to a multiple of 4 bytes (layer record name)."""
    raw = name.encode("mac_roman", errors="replace")[:255]
    s = bytes([len(raw)]) + raw
    return s + b"\0" * (-len(s) % 4)


def layer_record(top, left, bottom, right, channel_bytes, name, opacity=255):
    """One layer record: bounds, the four channels (ids -1, 0, 1, 2) with their
    block sizes, blend mode normal, no mask, default blending ranges, the
    name as a Pascal string and as a 'luni' (UTF-16) block."""
    rec = struct.pack(">4iH", int(top), int(left), int(bottom), int(right), 4)
    for cid, nbytes in zip(LAYER_CHANNEL_IDS, channel_bytes):
        rec += struct.pack(">hI", cid, int(nbytes))
    rec += b"8BIMnorm" + struct.pack(">4B", int(opacity), 0, 0x08, 0)
    u = name.encode("utf-16-be")
    luni = b"8BIMluni" + struct.pack(">II", 4 + len(u), len(u) // 2) + u
    ranges = struct.pack(">I", 40) + struct.pack(">I", 0x0000FFFF) * 10
    extra = struct.pack(">I", 0) + ranges + _pascal4(name) + luni
    return rec + struct.pack(">I", len(extra)) + extra


def write_psd(f, width, height, records, layer_blob, merged_blocks):
    """Writes an 8-bit RGB PSD with transparency to the binary file ``f``.

    ``records``: layer records (``layer_record``) bottom to top; ``layer_blob``:
    their channel blocks in the same order (a bytes-like object or a list of
    them); ``merged_blocks``: the merged image's four channel blocks (R, G, B,
    A), each as ``encode_channel_blocks`` writes it.  The merged image data
    takes one compression word, then every channel's row sizes, then every
    channel's rows."""
    if not (1 <= width <= PSD_MAX_SIDE and 1 <= height <= PSD_MAX_SIDE):
        raise ValueError(f"PSD canvas {width}x{height} outside 1..{PSD_MAX_SIDE}")
    blobs = layer_blob if isinstance(layer_blob, (list, tuple)) else [layer_blob]
    f.write(b"8BPS" + struct.pack(">H6xHIIHH", 1, 4, height, width, 8, 3))
    f.write(struct.pack(">II", 0, 0))            # colour mode data, image resources
    if records:
        head = struct.pack(">h", -len(records)) + b"".join(records)
        size = len(head) + sum(len(memoryview(b)) for b in blobs)
        pad = size & 1
        if 4 + size + pad + 4 > 0xFFFFFFFF:
            raise ValueError(f"layer data of {size} bytes exceeds the 4 GiB a PSD (version 1) section can hold")
        f.write(struct.pack(">II", 4 + size + pad + 4, size + pad))
        f.write(head)
        for b in blobs:
            f.write(memoryview(b))
        f.write(b"\0" * pad + struct.pack(">I", 0))  # global layer mask info
    else:
        f.write(struct.pack(">II", 8, 0) + struct.pack(">I", 0))
    rows = 2 * height
    f.write(struct.pack(">H", 1))
    for blk in merged_blocks:
        f.write(memoryview(blk)[2:2 + rows])
    for blk in merged_blocks:
        f.write(memoryview(blk)[2 + rows:])


def _solid(width, height, rgba, device):
    return torch.tensor(rgba, dtype=torch.uint8, device=device).repeat(height * width)


def _encode_image(img, device, order):
    """Channel blocks of one full-canvas (H,W,4) uint8 device image."""
    H, W = int(img.shape[0]), int(img.shape[1])
    sizes = torch.tensor([[W, H]], dtype=torch.int32, device=device)
    offs = torch.zeros(1, dtype=torch.int64, device=device)
    blob, block, _ = encode_channel_blocks(img.reshape(-1), sizes, offs, np.array([[W, H]]), order,
                                           lambda a: np.array([0]))
    return blob, block[0]


class PSDExporter:
    """Layered PSD export on the device (pydiffbmp/util/psd_exporter.py:11-501).

    Same constructor and methods as the reference: layers are added bottom to
    top, ``add_layers_batch_optimized`` puts primitive 0 on top (its layers are
    reversed, psd_exporter.py:90-99) and ``add_background_layer`` inserts a
    solid layer at the bottom.  Layer pixels come from ``export_layers`` and
    their channels are PackBits-encoded on the device; layers of width or
    height <= 1 or without a nonzero alpha are dropped, as the reference's
    export_psd_layers_cuda_uint8 does.  ``use_cuda`` is accepted and ignored:
    there is no host path.  The merged image is transparent black, like the
    reference's ``PSDImage.new(..., color=(0, 0, 0, 0))``, unless
    ``export_psd`` is given one."""

    def __init__(self, canvas_width, canvas_height, alpha_upper_bound=1.0, scale_factor=1.0, use_cuda=True,
                 c_blend=0.0, primitive_colors=None, device=None):
        self.canvas_width, self.canvas_height = int(canvas_width), int(canvas_height)
        self.alpha_upper_bound = float(alpha_upper_bound)
        self.scale_factor = float(scale_factor)
        self.use_cuda = use_cuda
        self.c_blend = float(c_blend)
        self.primitive_colors = primitive_colors
        self.export_width = int(canvas_width * scale_factor)
        self.export_height = int(canvas_height * scale_factor)
        if not (1 <= self.export_width <= PSD_MAX_SIDE and 1 <= self.export_height <= PSD_MAX_SIDE):
            raise ValueError(f"export canvas {self.export_width}x{self.export_height} outside 1..{PSD_MAX_SIDE}")
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        self._stack = []   # bottom to top: ("prims", dict) or ("solid", name, rgba)

    def add_layers_batch_optimized(self, primitive_templates, x_tensor, y_tensor, r_tensor, theta_tensor, v_tensor,
                                   c_tensor, names=None, reverse_order=True):
        """Crops every primitive into a layer (psd_exporter.py:37-107).  The
        reference looks names up as ``names[::-1][i]`` for primitive i
        (psd_export_uint8.py:180 with psd_exporter.py:95), so the default
        names run backwards: primitive i is "primitive_{N-1-i}"; kept as is."""
        N = len(x_tensor)
        if names is None:
            names = [f"primitive_{i}" for i in range(N)]
        dev = self.device
        t = primitive_templates.to(dev)
        if t.dim() == 2:
            sel = torch.zeros(N, dtype=torch.int32, device=dev)
            t = t.unsqueeze(0)
        else:
            sel = ((N - 1 - torch.arange(N, device=dev)) % t.shape[0]).int()
        means2D = torch.stack([x_tensor.to(dev).float(), y_tensor.to(dev).float()], 1)
        v = torch.sigmoid(v_tensor.to(dev).float())
        c = torch.sigmoid(c_tensor.to(dev).float())
        co = _colors_orig(self.primitive_colors, sel, N, t, dev, self.c_blend)
        buf, bbox, sizes, offs = export_layers(t, means2D, r_tensor.to(dev), theta_tensor.to(dev), v, c, sel,
                                               self.export_height, self.export_width, self.scale_factor,
                                               self.alpha_upper_bound, self.c_blend, co)
        rev = list(names)[::-1]
        self._stack.append(("prims", dict(buf=buf, bbox=bbox.cpu().numpy(), sizes=sizes, offs=offs,
                                          host_sizes=sizes.cpu().numpy(),
                                          names=[rev[i] if i < len(rev) else f"Layer_{i}" for i in range(N)])))

    def add_background_layer(self, bg_color):
        """Solid full-canvas layer named "Background" at the bottom, colour
        int(255 * c) per channel, alpha 255 (psd_exporter.py:468-492)."""
        rgb = tuple(int(bg_color[k] * 255) for k in range(3))
        self._stack.insert(0, ("solid", "Background", rgb + (255,)))

    def _encoded_layers(self):
        """(records, blobs) bottom to top."""
        W, H, dev = self.export_width, self.export_height, self.device
        records, blobs = [], []
        for kind, *rest in self._stack:
            if kind == "solid":
                name, rgba = rest
                blob, block = _encode_image(_solid(W, H, rgba, dev).view(H, W, 4), dev, ORDER_LAYER)
                records.append(layer_record(0, 0, H, W, block, name))
                blobs.append(blob)
                continue
            d = rest[0]
            hs = d["host_sizes"]
            static_ok = (hs[:, 0] > 1) & (hs[:, 1] > 1)
            # the reference keeps layers in index order, then reverses them: the
            # highest kept index is the lowest layer
            blob, blocks, chosen = encode_channel_blocks(
                d["buf"], d["sizes"], d["offs"], hs, ORDER_LAYER,
                lambda alpha_any: np.nonzero(static_ok & (alpha_any > 0))[0][::-1])
            for k, i in enumerate(chosen):
                x0, y0, x1, y1 = (int(v) for v in d["bbox"][i])
                records.append(layer_record(y0, x0, y1, x1, blocks[k], d["names"][i]))
            blobs.append(blob)
        return records, blobs

    def export_psd(self, filepath, composite=None):
        """Writes the PSD (psd_exporter.py:494-501; a .png / .tiff name gets
        the .psd extension) and returns its path.  ``composite`` (H,W,3|4)
        uint8 optionally replaces the transparent merged image."""
        if not filepath.endswith(".psd"):
            filepath = filepath.replace(".tiff", ".psd").replace(".png", ".psd")
        W, H, dev = self.export_width, self.export_height, self.device
        records, blobs = self._encoded_layers()
        if composite is None:
            merged = torch.zeros((H, W, 4), dtype=torch.uint8, device=dev)
        else:
            cimg = torch.as_tensor(composite).to(dev)
            if cimg.dtype != torch.uint8 or cimg.shape[:2] != (H, W) or cimg.shape[2] not in (3, 4):
                raise ValueError(f"composite must be uint8 ({H},{W},3|4), got {tuple(cimg.shape)} {cimg.dtype}")
            if cimg.shape[2] == 3:
                cimg = torch.cat([cimg, torch.full((H, W, 1), 255, dtype=torch.uint8, device=dev)], 2)
            merged = cimg.contiguous()
        mblob, mblock = _encode_image(merged, dev, ORDER_MERGED)
        host = [b.cpu().numpy() for b in blobs]
        m = mblob.cpu().numpy()
        cuts = np.concatenate([[0], np.cumsum(mblock)])
        with open(filepath, "wb") as f:
            write_psd(f, W, H, records, host, [m[cuts[k]:cuts[k + 1]] for k in range(4)])
        return filepath
