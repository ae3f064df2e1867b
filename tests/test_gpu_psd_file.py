"""GPU tests of PSD file assembly.

* The device PackBits channel blocks (dbmp_psd_rle_count / _write through
  ``encode_channel_blocks``) are byte-identical to the oracle's encoder on
  ragged images, both channel orders and partial selections, and to its
  compiled restatement on the 1024x1024 / N=5000 export case.
* ``PSDExporter`` writes a file that the oracle reader decodes to exactly the
  layers ``export_psd_layers_uint8`` returns (whose bytes the reference-kernel
  tests pin), with the reference's order (background at the bottom, primitive
  0 on top), bounds, names and filtering.
"""
import numpy as np
import pytest
import torch

from oracle import psd_file as O

pytestmark = pytest.mark.gpu


def _pack(imgs):
    sizes = np.array([[im.shape[1], im.shape[0]] for im in imgs], np.int32).reshape(-1, 2)
    offs = np.zeros(len(imgs), np.int64)
    tot = 0
    for k, im in enumerate(imgs):
        offs[k] = tot
        tot += im.size
    buf = np.zeros(max(tot, 4), np.uint8)
    for k, im in enumerate(imgs):
        buf[offs[k]:offs[k] + im.size] = im.reshape(-1)
    return buf, sizes, offs


def _images(seed):
    rng = np.random.default_rng(seed)
    shapes = [(1, 1), (1, 2), (2, 1), (3, 3), (31, 5), (32, 7), (33, 2), (64, 129), (65, 130), (5, 300),
              (40, 1), (1, 257), (97, 33), (2, 2), (300, 1000), (7, 2049)]
    imgs = []
    for h, w in shapes:
        kind = rng.integers(0, 3)
        if kind == 0:
            im = rng.integers(0, 256, (h, w, 4), dtype=np.uint8)
        elif kind == 1:
            im = (rng.integers(0, 3, (h, w, 4)) * 40).astype(np.uint8)
        else:
            im = np.zeros((h, w, 4), np.uint8)
            im[h // 4:3 * h // 4 + 1, w // 3:2 * w // 3 + 1] = [10, 20, 30, 200]
        imgs.append(im)
    imgs.append(np.zeros((20, 20, 4), np.uint8))     # fully transparent
    long = np.zeros((3, 700, 4), np.uint8)           # runs and literals across staging chunks
    long[:, 100:400] = 7
    long[1, ::2] = 9
    long[2] = rng.integers(0, 256, (700, 4))
    imgs.append(long)
    return imgs


def _expected(imgs, chosen, order):
    out = b""
    for i in chosen:
        for s in range(4):
            out += O.channel_block(imgs[i][:, :, (order >> (8 * s)) & 3])
    return out


@pytest.mark.parametrize("order", [0x02010003, 0x03020100])
@pytest.mark.parametrize("pick", ["alpha_reversed", "all", "none", "odd"])
def test_rle_blocks_match_oracle(order, pick):
    from diffbmp_b200.psd import encode_channel_blocks
    imgs = _images(11)
    buf, sizes, offs = _pack(imgs)
    sel = {"alpha_reversed": lambda a: np.nonzero(a > 0)[0][::-1], "all": lambda a: np.arange(len(a)),
           "none": lambda a: np.zeros(0, np.int64), "odd": lambda a: np.arange(1, len(a), 2)}[pick]
    blob, blocks, chosen = encode_channel_blocks(torch.from_numpy(buf).cuda(), torch.from_numpy(sizes).cuda(),
                                                 torch.from_numpy(offs).cuda(), sizes, order, sel)
    if pick == "alpha_reversed":
        assert 16 not in chosen                       # the transparent image is flagged as such
        assert list(chosen) == [i for i in range(len(imgs) - 1, -1, -1) if imgs[i][:, :, 3].any()]
    exp = _expected(imgs, chosen, order)
    got = blob.cpu().numpy().tobytes()
    assert got == exp
    assert int(blocks.sum()) == len(exp)


def test_rle_blocks_full_size_match_compiled_encoder():
    """The 1024x1024 / N=5000 export case (8 templates of 128^2, radii s W / 2
    with s log-uniform in [0.05, 0.3]; 1.0 GB of crops): every kept layer's
    four channel blocks, as the device's count and write passes produce them,
    are byte-identical to the compiled restatement of the encoder run on the
    same crops."""
    import diffbmp_b200.psd as P
    from diffbmp_b200 import workloads as wl
    W, N, n_tmpl, S = 1024, 5000, 8, 128
    rng = np.random.default_rng(0)
    tm = torch.from_numpy(np.stack([wl.random_shape(rng, S) for _ in range(n_tmpl)])).cuda()
    t = lambda a: torch.from_numpy(np.asarray(a, np.float32)).cuda()
    m = t(np.stack([rng.uniform(0, W, N), rng.uniform(0, W, N)], 1))
    r = t(np.exp(rng.uniform(np.log(0.05), np.log(0.3), N)) * W / 2)
    th = t(rng.uniform(0, 2 * np.pi, N))
    vs = torch.sigmoid(t(rng.normal(0, 1, N)))
    cs = torch.sigmoid(t(rng.normal(0, 2, (N, 3))))
    sel = torch.from_numpy(((N - 1 - np.arange(N)) % n_tmpl).astype(np.int32)).cuda()
    buf, bbox, sizes, offs = P.export_layers(tm, m, r, th, vs, cs, sel, W, W)
    hs = sizes.cpu().numpy()
    blob, blocks, chosen = P.encode_channel_blocks(buf, sizes, offs, hs, P.ORDER_LAYER,
                                                   lambda flags: np.nonzero(flags)[0])
    crops, o, got = buf.cpu().numpy(), offs.cpu().numpy(), blob.cpu().numpy()
    assert len(chosen) > 0.9 * N
    pos = 0
    for i in chosen:
        w, h = int(hs[i][0]), int(hs[i][1])
        im = crops[o[i]:o[i] + w * h * 4].reshape(h, w, 4)
        for slot in range(4):
            data, rows = O.packbits_rows_c(im[:, :, (P.ORDER_LAYER >> (8 * slot)) & 3])
            exp = b"\x00\x01" + rows.astype(">u2").tobytes() + data
            assert got[pos:pos + len(exp)].tobytes() == exp, (int(i), slot)
            pos += len(exp)
    assert pos == got.size


def test_rle_repeated_calls_identical():
    from diffbmp_b200.psd import encode_channel_blocks
    imgs = _images(12)
    buf, sizes, offs = _pack(imgs)
    args = (torch.from_numpy(buf).cuda(), torch.from_numpy(sizes).cuda(), torch.from_numpy(offs).cuda(), sizes,
            0x02010003, lambda a: np.arange(len(a)))
    a = encode_channel_blocks(*args)[0].cpu().numpy()
    b = encode_channel_blocks(*args)[0].cpu().numpy()
    assert np.array_equal(a, b)


def _scene(seed, N, H, W, scale):
    rng = np.random.default_rng(seed)
    from diffbmp_b200 import workloads as wl
    P, S = 3, 40
    tm = np.stack([wl.random_shape(rng, S) for _ in range(P)]).astype(np.float32)
    x = rng.uniform(-10, W / scale + 10, N)
    y = rng.uniform(-10, H / scale + 10, N)
    r = np.exp(rng.uniform(np.log(1.5), np.log(0.3 * min(H, W) / scale), N))
    r[:3] = [1e-3, 0.4, 2.0]
    th = rng.uniform(-7, 7, N)
    v = rng.normal(0, 2, N)
    v[5] = -60.0                                     # opacity 0: dropped as fully transparent
    c = rng.normal(0, 2, (N, 3))
    f = lambda a: torch.from_numpy(np.asarray(a, np.float32)).cuda()
    return f(tm), f(x), f(y), f(r), f(th), f(v), f(c)


@pytest.mark.parametrize("seed,N,W,H,scale,c_blend", [(0, 300, 256, 256, 1.0, 0.0), (1, 120, 136, 200, 2.0, 0.0),
                                                      (2, 90, 192, 160, 1.0, 0.4)])
def test_exporter_file_decodes_to_layers(tmp_path, seed, N, W, H, scale, c_blend):
    from diffbmp_b200.psd import PSDExporter, export_psd_layers_uint8
    tm, x, y, r, th, v, c = _scene(seed, N, H, W, scale)
    pcol = torch.rand((3, 3), generator=torch.Generator().manual_seed(seed)).cuda() if c_blend > 0 else None
    ex = PSDExporter(W, H, alpha_upper_bound=0.9, scale_factor=scale, c_blend=c_blend, primitive_colors=pcol)
    ex.add_layers_batch_optimized(tm, x, y, r, th, v, c)
    ex.add_background_layer((0.25, 0.5, 1.0))
    path = ex.export_psd(str(tmp_path / "out.png"))
    assert path.endswith("out.psd")
    doc = O.read_psd(open(path, "rb").read())
    EW, EH = int(W * scale), int(H * scale)
    assert (doc["width"], doc["height"], doc["channels"]) == (EW, EH, 4)
    assert not doc["merged"].any()

    sel = ((N - 1 - torch.arange(N, device="cuda")) % 3).int()
    arrays, bounds, idx = export_psd_layers_uint8(tm, x, y, r, th, torch.sigmoid(v), torch.sigmoid(c), sel, EH, EW,
                                                  scale, 0.9, c_blend, pcol)
    assert 5 not in idx
    layers = doc["layers"]
    assert len(layers) == 1 + len(idx)
    bg = layers[0]
    assert bg["name"] == "Background" and (bg["top"], bg["left"], bg["bottom"], bg["right"]) == (0, 0, EH, EW)
    assert np.array_equal(O.layer_rgba(bg), np.broadcast_to(np.array([63, 127, 255, 255], np.uint8), (EH, EW, 4)))
    # bottom to top: highest primitive index first
    for got, arr, (l, t, rr, b), i in zip(layers[1:], arrays[::-1], bounds[::-1], idx[::-1]):
        assert (got["left"], got["top"], got["right"], got["bottom"]) == (l, t, rr, b)
        assert got["unicode_name"] == f"primitive_{N - 1 - i}"     # the reference's name lookup
        np.testing.assert_array_equal(O.layer_rgba(got), arr)


def test_exporter_composite_and_batches(tmp_path):
    from diffbmp_b200.psd import PSDExporter
    W, H = 96, 64
    tm, x, y, r, th, v, c = _scene(4, 40, H, W, 1.0)
    ex = PSDExporter(W, H)
    ex.add_layers_batch_optimized(tm[0], x[:20], y[:20], r[:20], th[:20], v[:20], c[:20],
                                  names=[f"a{i}" for i in range(20)])
    ex.add_layers_batch_optimized(tm, x[20:], y[20:], r[20:], th[20:], v[20:], c[20:])
    comp = torch.randint(0, 256, (H, W, 3), dtype=torch.uint8, generator=torch.Generator().manual_seed(1))
    doc = O.read_psd(open(ex.export_psd(str(tmp_path / "c.psd"), composite=comp), "rb").read())
    np.testing.assert_array_equal(doc["merged"][:, :, :3], comp.numpy())
    assert (doc["merged"][:, :, 3] == 255).all()
    names = [l["unicode_name"] for l in doc["layers"]]
    first = [n for n in names if n.startswith("a")]
    assert names[:len(first)] == first             # the first batch lies below the second
    assert all(n.startswith("primitive_") for n in names[len(first):])


def test_exporter_rejects_oversize_canvas():
    from diffbmp_b200.psd import PSDExporter
    with pytest.raises(ValueError):
        PSDExporter(20000, 100, scale_factor=2.0)
