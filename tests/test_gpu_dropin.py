"""GPU tests of the drop-in package diffbmp_b200.cuda_tile_rasterizer: the
reference's call sequences (TileRasterizer.__call__ with the renderer's
mapping, empty mapping, FP16 extension, batch API, PSD extension) give the
oracle's results."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from helpers import bin_scene, golden, split_mapping

pytestmark = pytest.mark.gpu


def scene(seed=0, H=160, W=192, N=300, P=3):
    from diffbmp_b200 import workloads as wl
    s = wl.make_scene("c1", seed, H=H, W=W, N=N)
    sel = ((N - 1 - np.arange(N)) % s.templates.shape[0]).astype(np.int32)   # the renderer API's choice
    return s, sel


def cuda(a, dt=torch.float32):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt)


@pytest.mark.parametrize("with_mapping,c_blend", [(True, 0.0), (False, 0.0), (True, 0.3)])
def test_tile_rasterizer_call_matches_oracle(with_mapping, c_blend):
    """c_blend > 0 blends the colour maps colors_orig (tile_forward.cu:316-330)."""
    import diffbmp_b200.cuda_tile_rasterizer as ctr
    s, sel = scene(1)
    ts = 32
    sc = O.Scene(s.H, s.W, ts, s.means2D, s.radii, s.rotations, s.opacities, s.colors, s.templates, sel)
    co_np = np.random.default_rng(5).uniform(0, 1, (s.N, s.templates.shape[1], s.templates.shape[2], 3))
    if c_blend > 0:
        sc.colors_orig, sc.c_blend = co_np, c_blend
    offs, idx = bin_scene(sc, O.BIN_CONTENT if with_mapping else O.BIN_CULL)
    tr = ctr.TileRasterizer(s.H, s.W, ts, 0.0, 1.0, 400, s.N)
    x, y = cuda(s.means2D[:, 0]).requires_grad_(), cuda(s.means2D[:, 1]).requires_grad_()
    r, th = cuda(s.radii).requires_grad_(), cuda(s.rotations).requires_grad_()
    v, c = cuda(s.opacities).requires_grad_(), cuda(s.colors).requires_grad_()
    co = cuda(co_np)
    lr = torch.tensor([0.1, 1, 1, 1, 1, 1, 1.0], device="cuda")
    mapping = cuda(O.mapping_tensor(offs, idx), torch.int32) if with_mapping else None
    color, alpha = tr(torch.stack([x, y], 1), r, th, v, c, co, cuda(s.templates), cuda(sel, torch.int64), c_blend,
                      lr, mapping)
    ref = O.forward(sc, offs, idx)
    band, _ = O.boundary_band(sc, offs, idx)
    err = np.abs(color.detach().cpu().numpy() - ref["color"]).max(-1)
    assert err[band == 0].max() <= 1e-5
    rng = np.random.default_rng(0)
    wc = rng.normal(0, 1, (s.H, s.W, 3)).astype(np.float32)
    ((color * cuda(wc)).sum() + alpha.sum()).backward()
    g = O.backward(sc, offs, idx, wc, np.ones((s.H, s.W), np.float32))
    ours = np.stack([x.grad.cpu().numpy(), y.grad.cpu().numpy(), r.grad.cpu().numpy(), th.grad.cpu().numpy(),
                     v.grad.cpu().numpy()] + [c.grad.cpu().numpy()[:, k] for k in range(3)], 1)
    hi = O.backward(sc, offs, idx, wc, np.ones((s.H, s.W), np.float32), edge=1e-3)
    lo = O.backward(sc, offs, idx, wc, np.ones((s.H, s.W), np.float32), edge=-1e-3)
    for k in range(8):
        assert np.linalg.norm(ours[:, k] - g[:, k]) <= 1e-4 * np.linalg.norm(g[:, k]) + \
            np.linalg.norm(hi[:, k] - lo[:, k]) + 1e-9


def test_renderer_mapping_fixture_is_accepted():
    """The reference renderer's own mapping (golden fixture) drives the
    extension directly and equals device binning."""
    import diffbmp_b200.cuda_tile_rasterizer as ctr
    d = golden("bin_c0")
    N = d["radii"].shape[0]
    rng = np.random.default_rng(2)
    v, c = rng.normal(0, 1, N).astype(np.float32), rng.normal(0, 1, (N, 3)).astype(np.float32)
    sel = np.zeros(N, np.int32)
    args = [cuda(d["means2D"]), cuda(d["radii"]), cuda(d["rotations"]), cuda(v), cuda(c), None, cuda(d["S"]),
            cuda(sel, torch.int32), 0.0]
    ctr._C.init_tile_rasterizer(256, 256, 32, 0.0, 1.0, 400, N)
    c1, a1 = ctr._C.rasterize_tiles_class(*args, cuda(d["mapping"], torch.int32))
    from diffbmp_b200.rasterizer import Atlas, Rasterizer
    rz = Rasterizer(256, 256, 32)
    c2, a2, _ = rz.forward(args[0], args[1], args[2], args[3], args[4], args[7], Atlas(args[6]))
    assert torch.equal(c1, c2) and torch.equal(a1, a2)


def test_bad_mapping_is_rejected():
    import diffbmp_b200.cuda_tile_rasterizer as ctr
    s, sel = scene(2, H=64, W=64, N=20)
    ctr._C.init_tile_rasterizer(64, 64, 32, 0.0, 1.0, 400, s.N)
    bad = torch.tensor([5, 3, 0, 1, 2, 9, 0, 1, 2], dtype=torch.int32, device="cuda")   # offsets past L
    with pytest.raises(ValueError):
        ctr._C.rasterize_tiles_class(cuda(s.means2D), cuda(s.radii), cuda(s.rotations), cuda(s.opacities),
                                     cuda(s.colors), None, cuda(s.templates), cuda(sel, torch.int32), 0.0, bad)


def test_fp16_extension_vs_oracle():
    """The FP16 extension (_C_fp16) quantises its inputs to half, as the
    reference's does; on those half-rounded inputs its image is within half
    storage and output rounding of the FP64 oracle (PSNR >= 60 dB), and its
    gradients within 1e-2 per block."""
    import diffbmp_b200.cuda_tile_rasterizer as ctr
    s, sel = scene(3)
    h = lambda a: np.asarray(a, np.float32).astype(np.float16).astype(np.float64)
    sc = O.Scene(s.H, s.W, 16, h(s.means2D), h(s.radii), h(s.rotations), h(s.opacities), h(s.colors), h(s.templates),
                 sel)
    offs, idx = bin_scene(sc, O.BIN_CULL)
    t16 = ctr.TileRasterizer(s.H, s.W, 16, 0.0, 1.0, 400, s.N, use_fp16=True)
    ps = [cuda(a).half().requires_grad_() for a in (s.means2D, s.radii, s.rotations, s.opacities, s.colors)]
    c16, a16 = t16(*ps, None, cuda(s.templates), cuda(sel, torch.int32), 0.0, None, None)
    assert c16.dtype == torch.float16
    ref = O.forward(sc, offs, idx)
    err = c16.float().detach().cpu().numpy() - ref["color"]
    psnr = 10 * np.log10(1.0 / float(np.mean(err ** 2)))
    print("fp16 extension PSNR", psnr, "max", np.abs(err).max())
    assert psnr >= 60.0
    rng = np.random.default_rng(1)
    wc = rng.normal(0, 1, (s.H, s.W, 3)).astype(np.float32)
    (c16.float() * cuda(wc)).sum().backward()
    g = O.backward(sc, offs, idx, wc, None)
    ours = np.concatenate([p.grad.float().cpu().numpy().reshape(s.N, -1) for p in ps], 1)
    for k in range(8):
        assert np.linalg.norm(ours[:, k] - g[:, k]) <= 1e-2 * np.linalg.norm(g[:, k]), k


def test_batch_api_gradients_are_per_candidate():
    """forward_batch / its backward (one launch each over every candidate's
    tiles): each candidate's image and all eight gradient blocks against the
    FP64 oracle at the single-render bars (1e-5 image, 1e-4 gradients per
    block, boundary band held to its spread)."""
    import diffbmp_b200.cuda_tile_rasterizer as ctr
    s, sel = scene(4, H=96, W=128, N=120)
    B = 3
    rng = np.random.default_rng(5)
    m = np.stack([s.means2D + rng.normal(0, 3, s.means2D.shape).astype(np.float32) for _ in range(B)])
    op = np.stack([s.opacities + rng.normal(0, 0.5, s.N).astype(np.float32) for _ in range(B)])
    tr = ctr.TileRasterizer(s.H, s.W, 32, 0.0, 1.0, 400, s.N)
    params = [cuda(m).requires_grad_(), cuda(np.stack([s.radii] * B)).requires_grad_(),
              cuda(np.stack([s.rotations] * B)).requires_grad_(), cuda(op).requires_grad_(),
              cuda(np.stack([s.colors] * B)).requires_grad_()]
    color, alpha = tr.forward_batch(*params, None, cuda(s.templates), cuda(sel, torch.int32), 0.0, None, None)
    wc = rng.normal(0, 1, (B, s.H, s.W, 3)).astype(np.float32)
    wa = rng.normal(0, 1, (B, s.H, s.W)).astype(np.float32)
    ((color * cuda(wc)).sum() + (alpha * cuda(wa)).sum()).backward()
    for b in range(B):
        sc = O.Scene(s.H, s.W, 32, m[b], s.radii, s.rotations, op[b], s.colors, s.templates, sel)
        offs, idx = bin_scene(sc, O.BIN_CULL)
        O.check_image(sc, offs, idx, color[b].detach().cpu().numpy(), alpha[b].detach().cpu().numpy(), tol=1e-5)
        ours = np.concatenate([p.grad[b].cpu().numpy().reshape(s.N, -1) for p in params], 1)
        O.check_grads(sc, offs, idx, wc[b], wa[b], ours, rel=1e-4)
