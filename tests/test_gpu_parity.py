"""GPU parity tests of the sm_100a kernels (called through libdbmp.so).

Bars (stated per test):
* tile lists and their order: bit-exact;
* FP32 image / alpha: max-abs <= 1e-5 against the FP64 oracle, except on
  pixels inside the oracle's boundary band (a fragment within 1e-3 px/texel
  of the square cull or the texel cut, where float rounding legitimately
  flips it), which must stay within the band's own spread + 1e-5;
* gradients: per parameter block ||ours - oracle|| <= 1e-4 ||oracle|| plus
  the band spread of the gradient.
"""
import numpy as np
import pytest
import torch

from oracle import binning_torch as BT
from oracle import oracle as O
from helpers import bin_scene, golden, rel_err, small_scene, split_mapping

pytestmark = pytest.mark.gpu

R = pytest.importorskip("diffbmp_b200.rasterizer")


def dev(sc: O.Scene):
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()
    return dict(means2D=t(sc.means2D), radii=t(sc.radii), rotations=t(sc.rot), opacities=t(sc.opac),
                colors=t(sc.colors), sel=torch.from_numpy(sc.sel.astype(np.int32)).cuda(),
                templates=t(sc.templates))


def ours_forward(sc, kind="f32", mapping=None, t_stop=1e-7, bin_mode=R.BIN_CONTENT):
    d = dev(sc)
    rz = R.Rasterizer(sc.H, sc.W, sc.ts, sc.alpha_max, t_stop, bin_mode)
    atlas = R.Atlas(d["templates"], kind)
    mp = None if mapping is None else torch.from_numpy(mapping).cuda()
    color, alpha, state = rz.forward(d["means2D"], d["radii"], d["rotations"], d["opacities"], d["colors"],
                                     d["sel"], atlas, mp)
    torch.cuda.synchronize()
    return color.cpu().numpy(), alpha.cpu().numpy(), state, rz, atlas, d


def check_image(sc, offs, idx, color, alpha, tol=1e-5):
    return O.check_image(sc, offs, idx, color, alpha, tol)


def check_grads(sc, offs, idx, gc, ga, ours, rel=1e-4):
    O.check_grads(sc, offs, idx, gc, ga, ours, rel)


# ---------------------------------------------------------------------------
# binning
def test_template_bboxes_gpu():
    d = golden("tmpl_bbox")
    atlas = R.Atlas(torch.from_numpy(d["S"]).cuda())
    assert np.array_equal(atlas.bbox.cpu().numpy(), d["bboxes"])


@pytest.mark.parametrize("case", ["c0", "ragged", "edges"])
def test_binning_matches_reference_gpu(case):
    d = golden(f"bin_{case}")
    S = d["S"]
    N, P = d["radii"].shape[0], S.shape[0]
    sel = ((N - 1 - np.arange(N)) % P).astype(np.int32)
    H, W, ts = int(d["H"]), int(d["W"]), int(d["ts"])
    sc = O.Scene(H, W, ts, d["means2D"], d["radii"], d["rotations"], np.zeros(N), np.zeros((N, 3)), S, sel)
    dv = dev(sc)
    rz = R.Rasterizer(H, W, ts)
    atlas = R.Atlas(dv["templates"])
    _, lists = rz.bin(dv["means2D"], dv["radii"], dv["rotations"], dv["opacities"], dv["colors"], dv["sel"], atlas)
    ours = lists.mapping_tensor().cpu().numpy()
    # the reference binning re-run with torch on this GPU
    ref_gpu = BT.mapping(H, W, ts, dv["means2D"], dv["radii"], dv["rotations"], atlas.bbox, dv["sel"]).cpu().numpy()
    assert np.array_equal(ours, ref_gpu)
    # and the reference's own output (torch on CPU) stored in the fixture
    assert np.array_equal(ours, d["mapping"])


# (2000, 2000, 16): the per-slice count arrays exceed the shared-memory staging
# limit, so the in-place scan path of the counts kernel runs
@pytest.mark.parametrize("H,W,ts,N,seed", [(256, 256, 32, 512, 0), (200, 136, 16, 300, 1), (1024, 768, 32, 3000, 2),
                                           (64, 64, 16, 1, 3), (100, 300, 32, 0, 4), (2000, 2000, 16, 1500, 5)])
def test_binning_random_gpu(H, W, ts, N, seed):
    sc = small_scene(seed, H=H, W=W, N=N, P=3, size=48, ts=ts, rmin=1.0, rmax=0.3 * min(H, W))
    dv = dev(sc)
    rz = R.Rasterizer(H, W, ts)
    atlas = R.Atlas(dv["templates"])
    _, lists = rz.bin(dv["means2D"], dv["radii"], dv["rotations"], dv["opacities"], dv["colors"], dv["sel"], atlas)
    ref = BT.mapping(H, W, ts, dv["means2D"], dv["radii"], dv["rotations"], atlas.bbox, dv["sel"])
    assert torch.equal(lists.mapping_tensor(), ref)
    # cull-square mode against the oracle's exact float predicate
    rzc = R.Rasterizer(H, W, ts, bin_mode=R.BIN_CULL)
    _, lc = rzc.bin(dv["means2D"], dv["radii"], dv["rotations"], dv["opacities"], dv["colors"], dv["sel"], atlas)
    offs, idx = bin_scene(sc, O.BIN_CULL)
    assert np.array_equal(lc.mapping_tensor().cpu().numpy(), O.mapping_tensor(offs, idx))


# ---------------------------------------------------------------------------
# forward / backward
SCENES = {
    "c0": lambda: _spec_scene("c0", 0),
    "atlas128": lambda: _spec_scene("c1", 1, H=256, W=256, N=800),
    "ragged16": lambda: small_scene(5, H=200, W=136, N=150, P=3, size=48, ts=16, rmin=3, rmax=50),
    "nonsquare": lambda: small_scene(6, H=120, W=90, N=60, P=2, size=40, ts=32, nonsquare=True, amax=0.8),
}


def _spec_scene(cfg, seed, **over):
    from diffbmp_b200 import workloads as wl
    s = wl.make_scene(cfg, seed, **over)
    return O.Scene(s.H, s.W, 32, s.means2D, s.radii, s.rotations, s.opacities, s.colors, s.templates, s.sel,
                   s.alpha_max)


@pytest.mark.parametrize("kind", ["f32", "f32q"])
@pytest.mark.parametrize("name", list(SCENES))
def test_forward_parity_gpu(name, kind):
    """f32: reference atlas layout; f32q: packed quads with the clearance-grid skip."""
    sc = SCENES[name]()
    offs, idx = bin_scene(sc)
    color, alpha, state, *_ = ours_forward(sc, kind=kind)
    r = check_image(sc, offs, idx, color, alpha)
    # per-pixel last contributor never exceeds the oracle's fragment list
    assert state.last_pos.max().item() < max(len(idx), 1)
    print(name, r["max_err"], r["sensitive"])


@pytest.mark.parametrize("kind", ["f32", "f32q"])
@pytest.mark.parametrize("name", list(SCENES))
def test_backward_parity_gpu(name, kind):
    sc = SCENES[name]()
    offs, idx = bin_scene(sc)
    color, alpha, state, rz, atlas, d = ours_forward(sc, kind=kind)
    rng = np.random.default_rng(7)
    gc = rng.normal(0, 1, (sc.H, sc.W, 3)).astype(np.float32)
    ga = rng.normal(0, 1, (sc.H, sc.W)).astype(np.float32)
    grads = rz.backward(state, torch.from_numpy(gc).cuda(), torch.from_numpy(ga).cuda(), d["radii"],
                        d["rotations"], d["opacities"], d["colors"], atlas)
    ours = np.concatenate([g.cpu().numpy().reshape(sc.N, -1) for g in grads], 1)
    check_grads(sc, offs, idx, gc, ga, ours)


@pytest.mark.parametrize("kind", ["f32q", "f16", "f16q", "bf16", "bf16q"])
def test_storage_kinds_track_fp32_gpu(kind):
    """Every storage kind renders within its quantisation error of the FP32
    kernels and yields gradients within 1e-2 (half) / 5e-2 (bfloat16) relative."""
    sc = SCENES["atlas128"]()
    c32, a32, st32, rz, atlas32, d = ours_forward(sc)
    ck, ak, stk, rzk, atlask, _ = ours_forward(sc, kind=kind)
    tol = {"f32q": 1e-5, "f16": 2e-3, "f16q": 2e-3, "bf16": 2e-2, "bf16q": 2e-2}[kind]
    assert np.abs(ck - c32).max() <= tol
    rng = np.random.default_rng(2)
    gc = torch.from_numpy(rng.normal(0, 1, (sc.H, sc.W, 3)).astype(np.float32)).cuda()
    g32 = rz.backward(st32, gc, None, d["radii"], d["rotations"], d["opacities"], d["colors"], atlas32)
    gk = rzk.backward(stk, gc, None, d["radii"], d["rotations"], d["opacities"], d["colors"], atlask)
    gtol = {"f32q": 1e-4, "f16": 1e-2, "f16q": 1e-2, "bf16": 5e-2, "bf16q": 5e-2}[kind]
    for a, b in zip(gk, g32):
        assert rel_err(a.cpu().numpy(), b.cpu().numpy()) < gtol


def test_caller_mapping_equals_device_binning_gpu():
    """A caller-supplied reference mapping and the device binning render the same image."""
    sc = SCENES["atlas128"]()
    offs, idx = bin_scene(sc)
    c1, a1, *_ = ours_forward(sc)
    c2, a2, *_ = ours_forward(sc, mapping=O.mapping_tensor(offs, idx))
    assert np.array_equal(c1, c2) and np.array_equal(a1, a2)


def test_autograd_function_gpu():
    sc = SCENES["c0"]()
    d = dev(sc)
    rz = R.Rasterizer(sc.H, sc.W, sc.ts)
    atlas = R.Atlas(d["templates"])
    params = [d[k].clone().requires_grad_(True) for k in ("means2D", "radii", "rotations", "opacities", "colors")]
    color, alpha = R.rasterize(*params, d["sel"], atlas, rz)
    rng = np.random.default_rng(3)
    wc = torch.from_numpy(rng.normal(0, 1, (sc.H, sc.W, 3)).astype(np.float32)).cuda()
    wa = torch.from_numpy(rng.normal(0, 1, (sc.H, sc.W)).astype(np.float32)).cuda()
    ((color * wc).sum() + (alpha * wa).sum()).backward()
    offs, idx = bin_scene(sc)
    ours = np.concatenate([p.grad.cpu().numpy().reshape(sc.N, -1) for p in params], 1)
    check_grads(sc, offs, idx, wc.cpu().numpy(), wa.cpu().numpy(), ours)


@pytest.mark.parametrize("kind,min_psnr", [("f32q", 90.0), ("f16", 60.0), ("f16q", 60.0), ("bf16", 45.0),
                                           ("bf16q", 45.0)])
def test_precision_forms_gpu(kind, min_psnr):
    sc = SCENES["atlas128"]()
    offs, idx = bin_scene(sc)
    color, alpha, *_ = ours_forward(sc, kind=kind)
    ref = O.forward(sc, offs, idx)
    mse = float(np.mean((color - ref["color"]) ** 2))
    psnr = 10 * np.log10(1.0 / max(mse, 1e-30))
    print(kind, "PSNR", psnr, "max", np.abs(color - ref["color"]).max())
    assert psnr >= min_psnr


# ---------------------------------------------------------------------------
# clearance grid of the packed atlases
def _grid_bruteforce(t, cap=64, max_cells=128):
    """Per cell: min over support texels (> 5e-7 or NaN) of the L-infinity
    distance from the cell's coordinate range to the texel, capped (the
    definition, evaluated directly)."""
    Ht, Wt = t.shape

    def shape(n):
        s = 0
        while -(-n // (1 << s)) > max_cells:
            s += 1
        return s, -(-n // (1 << s))
    sx, gx = shape(Wt)
    sy, gy = shape(Ht)
    ys, xs = np.nonzero(~(t <= 5e-7))
    out = np.full((gy, gx), cap, np.int64)
    for iy in range(gy):
        ylo, yhi = iy << sy, min((iy + 1) << sy, Ht - 1)
        dy = np.maximum(0, np.maximum(ylo - ys, ys - yhi))
        for ix in range(gx):
            xlo, xhi = ix << sx, min((ix + 1) << sx, Wt - 1)
            dx = np.maximum(0, np.maximum(xlo - xs, xs - xhi))
            if len(xs):
                out[iy, ix] = min(cap, int(np.maximum(dx, dy).min()))
    return out


@pytest.mark.parametrize("kind,rec_bytes,extra_row", [("f32q", 16, 0), ("f16", 4, 1), ("bf16q", 8, 0)])
@pytest.mark.parametrize("Ht,Wt", [(40, 72), (130, 130), (300, 20)])
def test_clearance_grid_matches_definition_gpu(kind, rec_bytes, extra_row, Ht, Wt):
    from diffbmp_b200 import workloads as wl
    rng = np.random.default_rng(Ht * 7 + Wt)
    P = 3
    T = np.zeros((P, Ht, Wt), np.float32)
    for p in range(P):
        sh = wl.random_shape(rng, max(Ht, Wt))[:Ht, :Wt]
        T[p] = np.where(sh > 0.5, sh, 0.0)          # hard zero outside the shape
    T[2, Ht // 3, Wt // 2] = np.nan                   # NaN texels count as support
    T[2, 1, 1] = -0.5                                 # negative texels do not
    T[1, 2, Wt - 3] = 4e-7                            # nor texels at or below 5e-7
    T[0, Ht - 2, 3] = 6e-7                            # above it they do
    atlas = R.Atlas(torch.from_numpy(T).cuda(), kind)
    raw = atlas.data.cpu().numpy()
    off = (P * (Ht + extra_row) * Wt * rec_bytes + 255) // 256 * 256
    for p in range(P):
        want = _grid_bruteforce(T[p])
        n = want.size
        got = raw[off + p * n: off + (p + 1) * n].reshape(want.shape).astype(np.int64)
        assert np.array_equal(got, want), (p, np.argwhere(got != want)[:5])
    assert raw.size == off + P * want.size


@pytest.mark.parametrize("kind", ["f32q", "f16", "bf16"])
@pytest.mark.parametrize("name", list(SCENES))
@pytest.mark.parametrize("t_stop", [1e-6, 0.0])
def test_clearance_grid_never_skips_a_fragment_gpu(name, kind, t_stop):
    """The counting walk evaluates the grid test on every walked warp entry:
    none that the grid skips may hold a fragment."""
    import ctypes
    from diffbmp_b200._lib import call
    sc = SCENES[name]()
    color, alpha, state, rz, atlas, d = ours_forward(sc, kind=kind)
    cv = rz.canvas(sc.N, atlas)
    cv.t_stop = t_stop
    cnt = torch.zeros(10, dtype=torch.int64, device="cuda")
    call("dbmp_count", ctypes.byref(cv), R._ptr(state.prim_info), R._ptr(atlas.data), R._ptr(state.lists.offsets),
         R._ptr(state.lists.indices), R._ptr(cnt), R._stream())
    c = cnt.tolist()
    print(name, kind, t_stop, "walked", c[3], "empty", c[7], "grid skips", c[8], "bad", c[9])
    assert c[9] == 0
    assert c[8] <= c[7]
    if name == "atlas128":        # random shapes leave empty cells (the c0 soft disk has none)
        assert c[8] > 0


# ---------------------------------------------------------------------------
# colour-map blending (c_blend > 0)
@pytest.mark.parametrize("name", ["c0", "atlas128", "ragged16", "nonsquare"])
def test_colour_map_blend_parity_gpu(name):
    """dbmp_forward_blend / dbmp_backward_blend against the FP64 oracle with
    the reference's blend semantics, at the FP32 bars."""
    sc = SCENES[name]()
    rng = np.random.default_rng(11)
    P, Ht, Wt = sc.templates.shape
    cm = rng.uniform(0, 1, (sc.N, Ht, Wt, 3)).astype(np.float32)
    sc.colors_orig, sc.c_blend = cm.astype(np.float64), 0.35
    offs, idx = bin_scene(sc)
    d = dev(sc)
    rz = R.Rasterizer(sc.H, sc.W, sc.ts, sc.alpha_max, 1e-7)
    atlas = R.Atlas(d["templates"])
    tcm = torch.from_numpy(cm).cuda()
    color, alpha, state = rz.forward(d["means2D"], d["radii"], d["rotations"], d["opacities"], d["colors"],
                                     d["sel"], atlas, None, None, tcm, 0.35)
    torch.cuda.synchronize()
    r = check_image(sc, offs, idx, color.cpu().numpy(), alpha.cpu().numpy())
    print(name, "image", r["max_err"])
    gc = rng.normal(0, 1, (sc.H, sc.W, 3)).astype(np.float32)
    ga = rng.normal(0, 1, (sc.H, sc.W)).astype(np.float32)
    grads = rz.backward(state, torch.from_numpy(gc).cuda(), torch.from_numpy(ga).cuda(), d["radii"],
                        d["rotations"], d["opacities"], d["colors"], atlas)
    ours = np.concatenate([g.cpu().numpy().reshape(sc.N, -1) for g in grads], 1)
    check_grads(sc, offs, idx, gc, ga, ours)
    # the blend changes the image: c_blend = 0 renders something else
    c0, *_ = rz.forward(d["means2D"], d["radii"], d["rotations"], d["opacities"], d["colors"], d["sel"], atlas)
    assert (c0 - color).abs().max().item() > 1e-3


def test_colour_map_blend_rejects_bad_input_gpu():
    sc = SCENES["c0"]()
    d = dev(sc)
    rz = R.Rasterizer(sc.H, sc.W, sc.ts)
    atlas = R.Atlas(d["templates"])
    with pytest.raises(ValueError):
        rz.forward(d["means2D"], d["radii"], d["rotations"], d["opacities"], d["colors"], d["sel"], atlas,
                   None, None, torch.zeros(3, device="cuda"), 0.5)


# ---------------------------------------------------------------------------
# template blur (the reference's gaussian_blur of the atlas)
def test_template_blur_matches_reference_gpu():
    """dbmp_template_blur against the reference's gaussian_blur run on the
    fixture atlas (tests/golden/blur.npz), within float32 summation-order
    rounding; Atlas(sigma=) renders with the blurred texels but bins with the
    unblurred content bboxes, as VectorRenderer does."""
    import ctypes
    from diffbmp_b200._lib import call
    gd = golden("blur")
    S = torch.from_numpy(gd["S"]).cuda()
    P, Ht, Wt = S.shape
    for sg, want in zip(gd["sigmas"], gd["blurred"]):
        out = torch.empty_like(S)
        call("dbmp_template_blur", R._ptr(S), P, Ht, Wt, ctypes.c_float(float(sg)), R._ptr(out), R._stream())
        err = (out.cpu() - torch.from_numpy(want)).abs().max().item()
        print("sigma", float(sg), "max err", err)
        assert err <= 2e-6
    a = R.Atlas(S, "f32", sigma=1.5)
    a0 = R.Atlas(S, "f32")
    assert torch.equal(a.bbox, a0.bbox)
    assert (a.data.cpu() - torch.from_numpy(gd["blurred"][1])).abs().max().item() <= 2e-6
    aq = a.with_kind("f16q")
    assert torch.equal(aq.bbox, a0.bbox)
