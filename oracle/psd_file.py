"""Oracle for PSD file assembly -- TEST INFRASTRUCTURE ONLY.

The reference writes its layered PSD with psd-tools (unpinned in
requirements.txt:25 / pyproject.toml:37, and not installed here):
``PixelLayer.frompil`` per cropped layer (cuda_tile_rasterizer/
psd_export_uint8.py:153-186), ``PSDImage.insert`` for the background
(pydiffbmp/util/psd_exporter.py:468-492) and ``PSDImage.save``
(psd_exporter.py:494-501), which RLE-compresses every channel row.  Without
psd-tools its exact bytes cannot be reproduced, so parity for the file is
defined on what a reader gets back: this module restates, from the published
Adobe Photoshop File Formats specification and the PackBits scheme it uses
(Apple Technical Note TN1023), a reader of the sections the writer emits and
a PackBits decoder.  The tests decode the device-written file with it and
compare every layer plane, bound and name with the layer pixels, which are
themselves bit-exact with the reference's CUDA kernel.

``packbits_encode`` (and ``packbits_rows_c``, the same rule compiled in
dbmp_oracle.cpp, used as the timed CPU encoder) restates the library's own
encoding rule so that the device's channel blocks can also be compared byte
for byte:
  - a maximal run of L >= 3 equal bytes becomes replicate packets of
    min(remaining, 128) bytes ([1-k, v]); a one-byte remainder becomes the
    literal packet [0, v];
  - maximal runs of one or two bytes form literal segments, written as
    128-byte literal packets and a last shorter one ([k-1, k bytes]).
Only tests import this module.
"""
from __future__ import annotations

import struct

import numpy as np


def packbits_encode(row) -> bytes:
    """PackBits encoding of one row under the rule above."""
    row = bytes(row)
    out = bytearray()
    lit = bytearray()
    i, n = 0, len(row)

    def flush():
        for k in range(0, len(lit), 128):
            chunk = lit[k:k + 128]
            out.append(len(chunk) - 1)
            out.extend(chunk)
        lit.clear()

    while i < n:
        j = i
        while j < n and row[j] == row[i]:
            j += 1
        L = j - i
        if L >= 3:
            flush()
            rem = L
            while rem > 0:
                k = min(rem, 128)
                out.append((1 - k) & 0xFF if k >= 2 else 0)
                out.append(row[i])
                rem -= k
        else:
            lit.extend(row[i:j])
        i = j
    flush()
    return bytes(out)


def packbits_decode(data, size: int) -> bytes:
    """TN1023 PackBits: header n in 0..127 copies n+1 bytes, -127..-1 repeats
    the next byte 1-n times, -128 is skipped.  Raises on malformed input or a
    length other than ``size``."""
    data = bytes(data)
    out = bytearray()
    i = 0
    while i < len(data):
        n = data[i]
        i += 1
        if n < 128:
            if i + n + 1 > len(data):
                raise ValueError("literal packet runs past the row")
            out.extend(data[i:i + n + 1])
            i += n + 1
        elif n > 128:
            if i >= len(data):
                raise ValueError("replicate packet without its byte")
            out.extend(data[i:i + 1] * (257 - n))
            i += 1
    if len(out) != size:
        raise ValueError(f"row decodes to {len(out)} bytes, expected {size}")
    return bytes(out)


def packbits_rows_c(plane: np.ndarray):
    """The same encoding of every row of a (h, w) uint8 view (any strides) by
    the compiled restatement in dbmp_oracle.cpp; returns (data, row sizes)."""
    import ctypes
    from oracle.oracle import lib
    plane = np.asarray(plane)
    h, w = plane.shape
    if plane.dtype != np.uint8 or plane.strides[0] < 0 or plane.strides[1] < 1:
        raise ValueError("a uint8 plane with positive strides is required")
    out = np.empty(h * (w + (w + 127) // 128) + 1, np.uint8)
    sizes = np.empty(max(h, 1), np.int32)
    fn = lib().orc_packbits_rows
    fn.restype = ctypes.c_longlong
    n = fn(ctypes.c_void_p(plane.ctypes.data), h, w, ctypes.c_longlong(plane.strides[0]), plane.strides[1],
           ctypes.c_void_p(out.ctypes.data), ctypes.c_longlong(out.size), ctypes.c_void_p(sizes.ctypes.data))
    if n < 0:
        raise RuntimeError("packbits output buffer too small")
    return out[:n].tobytes(), sizes[:h]


def channel_block(plane: np.ndarray) -> bytes:
    """One channel's data in a layer: compression 1, big-endian u16 row sizes,
    the rows."""
    rows = [packbits_encode(r.tobytes()) for r in np.asarray(plane, dtype=np.uint8)]
    return struct.pack(">H", 1) + b"".join(struct.pack(">H", len(r)) for r in rows) + b"".join(rows)


def _planes(buf, pos, compression, h, w, channels):
    """Decodes `channels` planes of h x w stored one after another."""
    planes = []
    if compression == 0:
        for _ in range(channels):
            planes.append(np.frombuffer(buf[pos:pos + h * w], np.uint8).reshape(h, w))
            pos += h * w
        return planes, pos
    if compression != 1:
        raise ValueError(f"compression {compression} not handled")
    counts = struct.unpack_from(f">{channels * h}H", buf, pos)
    pos += 2 * channels * h
    for c in range(channels):
        rows = []
        for y in range(h):
            k = counts[c * h + y]
            rows.append(np.frombuffer(packbits_decode(buf[pos:pos + k], w), np.uint8))
            pos += k
        planes.append(np.stack(rows) if rows else np.zeros((0, w), np.uint8))
    return planes, pos


def read_psd(data: bytes) -> dict:
    """Parses an 8-bit PSD (version 1): header, layer records (bottom to top)
    with their decoded channels, and the merged image."""
    sig, version, channels, H, W, depth, mode = struct.unpack_from(">4sH6xHIIHH", data, 0)
    if sig != b"8BPS" or version != 1:
        raise ValueError("not a version-1 PSD")
    pos = 26
    (n,) = struct.unpack_from(">I", data, pos)
    pos += 4 + n                                    # colour mode data
    (n,) = struct.unpack_from(">I", data, pos)
    pos += 4 + n                                    # image resources
    (lmi_len,) = struct.unpack_from(">I", data, pos)
    pos += 4
    lmi_end = pos + lmi_len
    layers = []
    merged_alpha_first = False
    if lmi_len:
        (li_len,) = struct.unpack_from(">I", data, pos)
        pos += 4
        li_end = pos + li_len
        if li_len:
            (count,) = struct.unpack_from(">h", data, pos)
            pos += 2
            merged_alpha_first = count < 0
            recs = []
            for _ in range(abs(count)):
                top, left, bottom, right, nch = struct.unpack_from(">4iH", data, pos)
                pos += 18
                chans = [struct.unpack_from(">hI", data, pos + 6 * k) for k in range(nch)]
                pos += 6 * nch
                bsig, blend, opacity, clipping, flags, _ = struct.unpack_from(">4s4s4B", data, pos)
                if bsig != b"8BIM":
                    raise ValueError("bad blend signature")
                pos += 12
                (extra_len,) = struct.unpack_from(">I", data, pos)
                pos += 4
                extra_end = pos + extra_len
                (mask_len,) = struct.unpack_from(">I", data, pos)
                pos += 4 + mask_len
                (ranges_len,) = struct.unpack_from(">I", data, pos)
                pos += 4 + ranges_len
                nlen = data[pos]
                name = data[pos + 1:pos + 1 + nlen].decode("mac_roman")
                pos += (1 + nlen + 3) // 4 * 4
                uname = None
                while pos + 12 <= extra_end:
                    asig, key, alen = struct.unpack_from(">4s4sI", data, pos)
                    if asig not in (b"8BIM", b"8B64"):
                        raise ValueError("bad additional-info signature")
                    body = data[pos + 12:pos + 12 + alen]
                    if key == b"luni":
                        (cnt,) = struct.unpack_from(">I", body, 0)
                        uname = body[4:4 + 2 * cnt].decode("utf-16-be")
                    pos += 12 + alen + (alen & 1)
                if pos != extra_end:
                    raise ValueError("layer extra data does not add up")
                recs.append(dict(top=top, left=left, bottom=bottom, right=right, channels=chans,
                                 blend=blend.decode(), opacity=opacity, clipping=clipping, flags=flags,
                                 name=name, unicode_name=uname))
            for rec in recs:
                h, w = rec["bottom"] - rec["top"], rec["right"] - rec["left"]
                planes = {}
                for cid, length in rec["channels"]:
                    end = pos + length
                    (comp,) = struct.unpack_from(">H", data, pos)
                    got, p2 = _planes(data, pos + 2, comp, h, w, 1)
                    if p2 != end:
                        raise ValueError(f"channel {cid} of {rec['name']!r}: length field {length}, "
                                         f"data {p2 - pos}")
                    planes[cid] = got[0]
                    pos = end
                rec["planes"] = planes
                layers.append(rec)
            if pos > li_end or li_end - pos > 1:
                raise ValueError("layer info length does not add up")
        pos = li_end
        (gm_len,) = struct.unpack_from(">I", data, pos)
        pos += 4 + gm_len
        if pos > lmi_end:
            raise ValueError("layer and mask section length does not add up")
    pos = lmi_end
    (comp,) = struct.unpack_from(">H", data, pos)
    merged, pos = _planes(data, pos + 2, comp, H, W, channels)
    if pos != len(data):
        raise ValueError(f"{len(data) - pos} trailing bytes")
    return dict(channels=channels, height=H, width=W, depth=depth, mode=mode, layers=layers,
                merged=np.stack(merged, 2), merged_alpha_first=merged_alpha_first)


def layer_rgba(layer: dict) -> np.ndarray:
    """(h, w, 4) uint8 of a decoded layer (channel ids 0, 1, 2 and -1)."""
    p = layer["planes"]
    return np.stack([p[0], p[1], p[2], p[-1]], 2)
