"""CPU test of the host-side planning in ``encode_channel_blocks``: group
prefix sums, channel-block offsets in file order and per-group destinations.

The two device passes are replaced by stand-ins built on the oracle's
PackBits encoder, which fill the same outputs the kernels fill (row sizes,
group totals, alpha flags; then the blocks at the planned places).  The blob
the planner lays out must equal the oracle's channel blocks of the chosen
images, in the chosen order."""
import numpy as np
import pytest
import torch

from oracle import psd_file as O


def _fake_call(name, *a):
    if name == "dbmp_psd_rle_count":
        layers, sizes, offs, gb, N, G, order, wl, row_bytes, group_tot, alpha_any, _ = a
        if N == 0 or G == 0:
            return
        L, S, LO, GB = layers.numpy(), sizes.numpy().reshape(-1, 2), offs.numpy(), gb.numpy()
        rb = row_bytes.numpy().view(np.uint16).reshape(-1, 4)
        rb[:G * 32] = 0                              # rows past a layer's end count 0, as in the kernel
        gt = group_tot.numpy().reshape(-1, 4)
        for i in range(N):
            w, h = (int(v) for v in S[i])
            img = L[LO[i]:LO[i] + w * h * 4].reshape(h, w, 4)
            if img[:, :, 3].any():
                alpha_any.numpy()[i] = 1
            for y in range(h):
                g, lane = GB[i] + y // 32, y % 32
                for s in range(4):
                    rb[g * 32 + lane, s] = len(O.packbits_encode(img[y, :, (order >> (8 * s)) & 3].tobytes()))
            for g in range(GB[i], GB[i + 1]):
                gt[g] = rb[g * 32:(g + 1) * 32].astype(np.int64).sum(0)
    elif name == "dbmp_psd_rle_write":
        layers, sizes, offs, gb, N, G, order, wl, row_bytes, chan_off, group_dst, out, out_bytes, _ = a
        if N == 0 or G == 0:
            return
        L, S, LO, GB = layers.numpy(), sizes.numpy().reshape(-1, 2), offs.numpy(), gb.numpy()
        CO, GD, OUT = chan_off.numpy().reshape(-1, 4), group_dst.numpy().reshape(-1, 4), out.numpy()
        for i in range(N):
            if (CO[i] < 0).all():
                continue
            w, h = (int(v) for v in S[i])
            img = L[LO[i]:LO[i] + w * h * 4].reshape(h, w, 4)
            for s in range(4):
                co = int(CO[i, s])
                OUT[co:co + 2] = [0, 1]
                for g in range(GB[i], GB[i + 1]):
                    pos = int(GD[g, s])
                    for y in range((g - GB[i]) * 32, min(h, (g - GB[i] + 1) * 32)):
                        enc = O.packbits_encode(img[y, :, (order >> (8 * s)) & 3].tobytes())
                        OUT[co + 2 + 2 * y:co + 4 + 2 * y] = [len(enc) >> 8, len(enc) & 255]
                        assert pos + len(enc) <= out_bytes
                        OUT[pos:pos + len(enc)] = np.frombuffer(enc, np.uint8)
                        pos += len(enc)
    else:
        raise KeyError(name)


@pytest.fixture
def planner(monkeypatch):
    import diffbmp_b200.psd as P
    monkeypatch.setattr(P, "call", _fake_call)
    monkeypatch.setattr(P, "_ptr", lambda t: t)
    monkeypatch.setattr(P, "_stream", lambda s=None: None)
    return P.encode_channel_blocks


def _case(seed):
    rng = np.random.default_rng(seed)
    imgs = []
    for h, w in [(1, 1), (2, 3), (31, 4), (32, 5), (33, 6), (70, 9), (5, 140), (20, 20), (65, 2)]:
        im = (rng.integers(0, 3, (h, w, 4)) * 50).astype(np.uint8)
        imgs.append(im)
    imgs[7][:] = 0                                   # no alpha
    return imgs


@pytest.mark.parametrize("order", [0x02010003, 0x03020100])
@pytest.mark.parametrize("pick", ["alpha_reversed", "all", "none", "every_third"])
def test_planner_lays_out_chosen_blocks(planner, order, pick):
    imgs = _case(3)
    sizes = np.array([[im.shape[1], im.shape[0]] for im in imgs], np.int32)
    offs = np.concatenate([[0], np.cumsum([im.size for im in imgs])[:-1]]).astype(np.int64)
    buf = np.concatenate([im.reshape(-1) for im in imgs])
    sel = {"alpha_reversed": lambda a: np.nonzero(a > 0)[0][::-1], "all": lambda a: np.arange(len(a)),
           "none": lambda a: np.zeros(0, np.int64), "every_third": lambda a: np.arange(len(a))[::3][::-1]}[pick]
    blob, blocks, chosen = planner(torch.from_numpy(buf), torch.from_numpy(sizes), torch.from_numpy(offs), sizes,
                                   order, sel)
    if pick == "alpha_reversed":
        assert list(chosen) == [i for i in range(len(imgs) - 1, -1, -1) if imgs[i][:, :, 3].any()]
    exp = [O.channel_block(imgs[i][:, :, (order >> (8 * s)) & 3]) for i in chosen for s in range(4)]
    assert blob.numpy().tobytes() == b"".join(exp)
    assert blocks.reshape(-1).tolist() == [len(b) for b in exp]


def test_planner_without_images(planner):
    z = np.zeros((0, 2), np.int32)
    blob, blocks, chosen = planner(torch.zeros(4, dtype=torch.uint8), torch.from_numpy(z),
                                   torch.zeros(0, dtype=torch.int64), z, 0x02010003, lambda a: np.arange(len(a)))
    assert blob.numel() == 0 and blocks.shape == (0, 4) and len(chosen) == 0


def test_planner_rejects_repeated_or_foreign_indices(planner):
    imgs = _case(4)[:3]
    sizes = np.array([[im.shape[1], im.shape[0]] for im in imgs], np.int32)
    offs = np.concatenate([[0], np.cumsum([im.size for im in imgs])[:-1]]).astype(np.int64)
    buf = np.concatenate([im.reshape(-1) for im in imgs])
    args = (torch.from_numpy(buf), torch.from_numpy(sizes), torch.from_numpy(offs), sizes, 0x02010003)
    for bad in (lambda a: np.array([0, 0]), lambda a: np.array([3]), lambda a: np.array([-1])):
        with pytest.raises(ValueError):
            planner(*args, bad)
    with pytest.raises(ValueError):
        planner(*args[:4], 0x04000000, lambda a: np.arange(3))


def test_exporter_order_names_and_filtering_on_cpu(monkeypatch, tmp_path):
    """PSDExporter's host logic with the crops from the oracle's layer
    restatement and the encoder stand-ins: background at the bottom, then the
    kept primitives from the highest index up, named through the reference's
    names[::-1][i] lookup; empty and transparent crops dropped."""
    import diffbmp_b200.psd as P
    from oracle import oracle as OO

    def crops(templates, means2D, radii, rotations, vis_sig, colors_sig, sel, H, W, scale=1.0, alpha_max=1.0,
              c_blend=0.0, colors_orig=None):
        t = templates if templates.dim() == 3 else templates.unsqueeze(0)
        m, r = means2D.numpy().astype(np.float32), radii.numpy().astype(np.float32)
        bb, sz = OO.psd_bboxes(m, r, H, W, scale)
        offs = np.concatenate([[0], np.cumsum(sz[:, 0].astype(np.int64) * sz[:, 1] * 4)[:-1]]).astype(np.int64)
        buf, _ = OO.psd_layers(m, r, rotations.numpy().astype(np.float32), colors_sig.numpy().astype(np.float32),
                               vis_sig.numpy().astype(np.float32), t.numpy().astype(np.float32),
                               sel.numpy().astype(np.int32), bb, offs, scale, alpha_max)
        return (torch.from_numpy(np.ascontiguousarray(buf, np.uint8)), torch.from_numpy(bb.astype(np.int32)),
                torch.from_numpy(sz.astype(np.int32)), torch.from_numpy(offs))

    for name, fn in (("call", _fake_call), ("_ptr", lambda t: t), ("_stream", lambda s=None: None),
                     ("export_layers", crops)):
        monkeypatch.setattr(P, name, fn)
    rng = np.random.default_rng(0)
    N, W, H = 25, 48, 40
    f = lambda a: torch.from_numpy(np.asarray(a, np.float32))
    tm = f(rng.uniform(0, 1, (3, 16, 16)))
    x, y = f(rng.uniform(0, W, N)), f(rng.uniform(0, H, N))
    r, th = f(rng.uniform(1, 8, N)), f(rng.uniform(-3, 3, N))
    r[2], x[2], y[2] = 0.2, 10.5, 10.5                # a 1x1 crop: dropped
    v, c = f(rng.normal(0, 2, N)), f(rng.normal(0, 2, (N, 3)))
    v[5] = -60.0                                      # transparent
    ex = P.PSDExporter(W, H, alpha_upper_bound=0.9, device="cpu")
    ex.add_layers_batch_optimized(tm, x, y, r, th, v, c)
    ex.add_background_layer((0.25, 0.5, 1.0))
    doc = O.read_psd(open(ex.export_psd(str(tmp_path / "t.png")), "rb").read())

    buf, bb, sz, offs = crops(tm, torch.stack([x, y], 1), r, th, torch.sigmoid(v), torch.sigmoid(c),
                              ((N - 1 - torch.arange(N)) % 3).int(), H, W, 1.0, 0.9)
    hb = buf.numpy()
    kept = []
    for i in range(N - 1, -1, -1):
        w, h = (int(t) for t in sz[i])
        a = hb[offs[i]:offs[i] + w * h * 4].reshape(h, w, 4)
        if w > 1 and h > 1 and a[:, :, 3].max() > 0:
            kept.append((i, a))
    assert 5 not in [i for i, _ in kept] and 2 not in [i for i, _ in kept]
    layers = doc["layers"]
    assert layers[0]["name"] == "Background" and len(layers) == 1 + len(kept)
    assert (O.layer_rgba(layers[0]) == np.array([63, 127, 255, 255], np.uint8)).all()
    for got, (i, a) in zip(layers[1:], kept):
        assert got["unicode_name"] == f"primitive_{N - 1 - i}"
        assert (got["left"], got["top"], got["right"], got["bottom"]) == tuple(int(t) for t in bb[i])
        np.testing.assert_array_equal(O.layer_rgba(got), a)
    assert not doc["merged"].any()
