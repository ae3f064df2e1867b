"""CPU tests of PSD file assembly: the PackBits oracle against the TN1023
known answer and round trips over edge-case rows, the host-side document
writer read back by the oracle reader, and argument checks of the two
device entry points (rejected before any launch)."""
import ctypes
import io

import numpy as np
import pytest

from oracle import psd_file as O


def test_packbits_tn1023_known_answer():
    # the worked example of Apple Technical Note TN1023 (PackBits)
    raw = bytes.fromhex("AAAAAA80002AAAAAAAAA80002A22AAAAAAAAAAAAAAAAAAAA")
    packed = bytes.fromhex("FEAA0280002AFDAA0380002A22F7AA")
    assert O.packbits_encode(raw) == packed
    assert O.packbits_decode(packed, len(raw)) == raw


@pytest.mark.parametrize("row, packed", [
    (b"\x05", b"\x00\x05"),
    (b"\x05\x05", b"\x01\x05\x05"),                 # a pair stays literal
    (b"\x05\x05\x05", b"\xfe\x05"),
    (b"\x07" * 128, b"\x81\x07"),
    (b"\x07" * 129, b"\x81\x07\x00\x07"),           # one-byte remainder: literal packet
    (b"\x07" * 130, b"\x81\x07\xff\x07"),
    (b"\x01\x02" + b"\x09" * 3 + b"\x03", b"\x01\x01\x02\xfe\x09\x00\x03"),
])
def test_packbits_rule(row, packed):
    assert O.packbits_encode(row) == packed
    assert O.packbits_decode(packed, len(row)) == row


def _rows():
    rng = np.random.default_rng(5)
    rows = [bytes(range(256)) * 2, bytes(range(128)), bytes(range(129)), bytes(range(130)),
            b"\x00\x00\x01" * 100, b"\x01\x01\x02\x02" * 70]
    for L in (3, 127, 128, 129, 130, 131, 255, 256, 257, 384, 385):
        rows.append(b"\x11" * L)
        rows.append(bytes(range(1, 60)) + b"\x22" * L + b"\x33\x34")
    for n in (1, 2, 31, 32, 33, 300, 1000):
        rows.append(rng.integers(0, 256, n, dtype=np.uint8).tobytes())
        rows.append(rng.integers(0, 3, n, dtype=np.uint8).tobytes())      # many short runs
        rows.append(np.repeat(rng.integers(0, 256, n, dtype=np.uint8), rng.integers(1, 6, n)).tobytes())
    return rows


@pytest.mark.parametrize("i", range(len(_rows())))
def test_packbits_round_trip_and_bound(i):
    row = _rows()[i]
    enc = O.packbits_encode(row)
    assert O.packbits_decode(enc, len(row)) == row
    assert len(enc) <= len(row) + (len(row) + 127) // 128
    # no packet crosses 128 bytes, no -128 no-op is written
    pos = 0
    while pos < len(enc):
        n = enc[pos]
        assert n != 128
        pos += 2 + n if n < 128 else 2


def test_compiled_packbits_matches_restatement():
    rows = _rows()
    rng = np.random.default_rng(9)
    for row in rows[::3]:
        a = np.frombuffer(row, np.uint8).reshape(1, -1)
        data, sizes = O.packbits_rows_c(a)
        assert data == O.packbits_encode(row) and sizes.tolist() == [len(data)]
    img = (rng.integers(0, 3, (37, 301, 4)) * 70).astype(np.uint8)
    for ch in range(4):                              # a strided channel of an interleaved image
        data, sizes = O.packbits_rows_c(img[:, :, ch])
        exp = [O.packbits_encode(img[y, :, ch].tobytes()) for y in range(37)]
        assert data == b"".join(exp) and sizes.tolist() == [len(e) for e in exp]


def test_packbits_decode_rejects_malformed():
    with pytest.raises(ValueError):
        O.packbits_decode(b"\x05\x01\x02", 6)       # literal runs past the data
    with pytest.raises(ValueError):
        O.packbits_decode(b"\xfe\x01", 4)           # wrong decoded length


def _doc(layers, W, H, merged):
    """Builds a PSD with the product's writer from oracle-encoded blocks."""
    from diffbmp_b200.psd import layer_record, write_psd
    records, blobs = [], []
    for (top, left, rgba, name) in layers:
        blocks = [O.channel_block(rgba[:, :, b]) for b in (3, 0, 1, 2)]
        h, w = rgba.shape[:2]
        records.append(layer_record(top, left, top + h, left + w, [len(b) for b in blocks], name))
        blobs.extend(blocks)
    mblocks = [O.channel_block(merged[:, :, c]) for c in range(4)]
    f = io.BytesIO()
    write_psd(f, W, H, records, blobs, mblocks)
    return f.getvalue()


def test_document_writer_reads_back():
    rng = np.random.default_rng(1)
    W, H = 70, 45
    layers = []
    for k, (h, w) in enumerate([(45, 70), (1, 9), (9, 1), (33, 40), (2, 2)]):
        a = rng.integers(0, 4, (h, w, 4), dtype=np.uint8) * 60
        layers.append((int(rng.integers(0, H - h + 1)), int(rng.integers(0, W - w + 1)), a,
                       ["Background", "primitive_3", "primitive_2", "名前 ünïcode", "x" * 40][k]))
    merged = rng.integers(0, 256, (H, W, 4), dtype=np.uint8)
    doc = O.read_psd(_doc(layers, W, H, merged))
    assert (doc["width"], doc["height"], doc["channels"], doc["depth"], doc["mode"]) == (W, H, 4, 8, 3)
    assert doc["merged_alpha_first"]
    np.testing.assert_array_equal(doc["merged"], merged)
    assert len(doc["layers"]) == len(layers)
    for got, (top, left, rgba, name) in zip(doc["layers"], layers):
        h, w = rgba.shape[:2]
        assert (got["top"], got["left"], got["bottom"], got["right"]) == (top, left, top + h, left + w)
        assert [c for c, _ in got["channels"]] == [-1, 0, 1, 2]
        assert got["blend"] == "norm" and got["opacity"] == 255 and not (got["flags"] & 2)
        assert got["unicode_name"] == name
        assert got["name"] == name.encode("mac_roman", errors="replace").decode("mac_roman")
        np.testing.assert_array_equal(O.layer_rgba(got), rgba)


def test_document_without_layers():
    merged = np.zeros((3, 5, 4), np.uint8)
    doc = O.read_psd(_doc([], 5, 3, merged))
    assert doc["layers"] == [] and doc["merged"].shape == (3, 5, 4)


def test_document_rejects_oversize_canvas():
    from diffbmp_b200.psd import write_psd
    with pytest.raises(ValueError):
        write_psd(io.BytesIO(), 30001, 10, [], [], [b"\0\1"] * 4)


def test_document_rejects_layer_data_beyond_4gib():
    from diffbmp_b200.psd import layer_record, write_psd
    rec = layer_record(0, 0, 1, 1, [2, 2, 2, 2], "x")
    huge = np.lib.stride_tricks.as_strided(np.zeros(1, np.uint8), (1 << 32,), (0,))   # 4 GiB, no memory
    with pytest.raises(ValueError, match="4 GiB"):
        write_psd(io.BytesIO(), 1, 1, [rec], [huge], [b"\0\1\0\2"] * 4)


def test_layer_record_name_padding():
    from diffbmp_b200.psd import _pascal4
    for name in ("", "a", "abc", "abcd", "x" * 300):
        p = _pascal4(name)
        assert len(p) % 4 == 0 and p[0] == min(len(name), 255)


def test_rle_entry_points_reject_bad_arguments_without_launch():
    from diffbmp_b200._lib import DBMP_ERR_INVALID, lib
    ll = ctypes.c_longlong
    rc = lib.dbmp_psd_rle_count(None, None, None, None, 3, ll(2), 0x02010003, 0, None, None, None, None)
    assert rc == DBMP_ERR_INVALID and "width_limit" in lib.dbmp_last_error().decode()
    rc = lib.dbmp_psd_rle_count(None, None, None, None, 3, ll(2), 0x04010003, 100, None, None, None, None)
    assert rc == DBMP_ERR_INVALID and "channel_order" in lib.dbmp_last_error().decode()
    rc = lib.dbmp_psd_rle_count(None, None, None, None, 3, ll(2), 0x02010003, 100, None, None, None, None)
    assert rc == DBMP_ERR_INVALID and "null" in lib.dbmp_last_error().decode()
    rc = lib.dbmp_psd_rle_write(None, None, None, None, 0, ll(0), 0x02010003, 100, None, None, None, None,
                                ll(-1), None)
    assert rc == DBMP_ERR_INVALID and "out_bytes" in lib.dbmp_last_error().decode()
    # nothing to encode: accepted without touching any pointer
    assert lib.dbmp_psd_rle_count(None, None, None, None, 0, ll(0), 0x02010003, 100, None, None, None, None) == 0
