"""CPU tests of the oracle: pinned against golden vectors produced by the
reference's own Python code (tests/golden/make_golden.py), closed-form
known answers for the kernel semantics, and an FP64 finite-difference check
of its backward."""
import numpy as np
import pytest

from oracle import oracle as O
from helpers import bin_scene, golden, rel_err, small_scene, split_mapping


def test_template_bboxes_match_reference():
    d = golden("tmpl_bbox")
    assert np.array_equal(O.template_bboxes(d["S"]), d["bboxes"])


@pytest.mark.parametrize("case", ["c0", "ragged", "edges"])
def test_binning_matches_reference(case):
    d = golden(f"bin_{case}")
    S = d["S"]
    N = d["radii"].shape[0]
    P, Ht, Wt = S.shape
    tb = O.template_bboxes(S)
    assert np.array_equal(tb, d["tbbox"])
    sel = (N - 1 - np.arange(N)) % P          # the renderer API's template choice
    offs, idx = O.bin_tiles(int(d["H"]), int(d["W"]), int(d["ts"]), d["means2D"], d["radii"],
                            d["rotations"], sel, tb, Ht, Wt)
    assert np.array_equal(O.mapping_tensor(offs, idx), d["mapping"])


@pytest.mark.parametrize("case", ["disk64", "ragged"])
def test_torch_path_matches_reference(case):
    """Forward image/alpha and all six gradient blocks of the reference's
    PyTorch renderer, reproduced by the oracle's SEM_TORCH mode."""
    d = golden(f"torch_{case}")
    sc = O.Scene(d["H"], d["W"], d["ts"], d["means2D"], d["radii"], d["rotations"], d["opacities"],
                 d["colors"], d["S"], d["sel"], float(d["amax"]))
    offs, idx = split_mapping(d["mapping"])
    f = O.forward(sc, offs, idx, sem=O.SEM_TORCH)
    assert np.abs(f["color"] - d["image"]).max() < 5e-6
    assert np.abs(f["alpha"] - d["alpha"]).max() < 5e-6
    g = O.backward(sc, offs, idx, d["wc"], d["wa"], sem=O.SEM_TORCH)
    refs = [d["g_x"], d["g_y"], d["g_r"], d["g_theta"], d["g_v"], d["g_c"][:, 0], d["g_c"][:, 1], d["g_c"][:, 2]]
    for k, ref in enumerate(refs):
        assert rel_err(g[:, k], ref) < 2e-5, f"gradient block {k}"


def _one_prim_scene(tmpl, mx, my, r, th=0.0, v=0.3, c=(0.2, -0.4, 1.1), H=40, W=48, amax=1.0, extra=None):
    prims = [(mx, my, r, th, v, c)] + (extra or [])
    m = np.array([[p[0], p[1]] for p in prims])
    return O.Scene(H, W, 16, m, [p[2] for p in prims], [p[3] for p in prims], [p[4] for p in prims],
                   [p[5] for p in prims], tmpl, [0] * len(prims), amax)


def _render(sc):
    offs, idx = bin_scene(sc, O.BIN_CULL)
    return O.forward(sc, offs, idx)


def sig(x):
    return 1.0 / (1.0 + np.exp(-np.asarray(x, np.float64)))


def test_kat_constant_template_square():
    """A constant-1 template gives alpha = sigmoid(v) exactly on the cull square."""
    sc = _one_prim_scene(np.ones((8, 8), np.float32), 20.25, 17.5, 5.0, v=0.3)
    f = _render(sc)
    yy, xx = np.mgrid[0:40, 0:48]
    inside = (np.abs(xx - 20.25) <= 5.0) & (np.abs(yy - 17.5) <= 5.0)
    a = sig(0.3)
    assert np.allclose(f["alpha"][inside], a, atol=1e-15) and np.all(f["alpha"][~inside] == 0)
    assert np.allclose(f["color"][inside], a * sig([0.2, -0.4, 1.1]), atol=1e-15)


def test_kat_two_layer_composite():
    c1, c2 = (0.5, -1.0, 2.0), (-0.3, 0.8, 0.1)
    sc = _one_prim_scene(np.ones((8, 8), np.float32), 20.0, 20.0, 6.0, v=0.7, c=c1,
                         extra=[(24.0, 22.0, 6.0, 0.0, -0.2, c2)])
    f = _render(sc)
    a1, a2 = sig(0.7), sig(-0.2)
    both = f["color"][20, 24]
    assert np.allclose(both, a1 * sig(c1) + (1 - a1) * a2 * sig(c2), atol=1e-14)
    assert abs(f["alpha"][20, 24] - (1 - (1 - a1) * (1 - a2))) < 1e-14


def test_kat_full_occlusion():
    c1 = (0.5, -1.0, 2.0)
    sc = _one_prim_scene(np.ones((8, 8), np.float32), 20.0, 20.0, 6.0, v=60.0, c=c1,
                         extra=[(22.0, 20.0, 6.0, 0.0, 0.0, (3.0, 3.0, 3.0))])
    f = _render(sc)
    assert np.allclose(f["color"][20, 22], sig(c1), atol=1e-15)
    assert f["alpha"][20, 22] == 1.0


def test_kat_colour_map_blend():
    """c_blend > 0 (tile_forward.cu:316-330): colour = (1-cb) sigmoid(c) + cb c_o, with
    c_o the colour map sampled at the texel coordinate (clamped, edge-repeating);
    the colour-logit gradient is gC a T sigma'(c) without (1-cb), as the
    reference computes it (tile_backward.cu:254-262)."""
    Ht = Wt = 9
    cm = np.zeros((1, Ht, Wt, 3))
    cm[..., 0] = np.linspace(0, 1, Wt)[None, :]           # red ramps with the texel column
    cm[..., 1] = 0.25
    cm[..., 2] = np.linspace(1, 0, Ht)[:, None]           # blue ramps down the rows
    sc = _one_prim_scene(np.ones((Ht, Wt), np.float32), 20.0, 20.0, 4.0, v=0.3)
    sc.colors_orig, sc.c_blend = cm, 0.4
    f = _render(sc)
    a, cb, sc_ = sig(0.3), 0.4, sig([0.2, -0.4, 1.1])
    # pixel (x=22, y=19): texel (x, y) = ((2/4)+1)*4, ((-1/4)+1)*4 = (6, 3)
    co = np.array([6 / 8, 0.25, 1 - 3 / 8])
    assert np.allclose(f["color"][19, 22], a * ((1 - cb) * sc_ + cb * co), atol=1e-14)
    offs, idx = bin_scene(sc, O.BIN_CULL)
    gc = np.zeros((40, 48, 3), np.float32)
    gc[19, 22] = (1.0, 2.0, -1.0)
    g = O.backward(sc, offs, idx, gc, None)
    assert np.allclose(g[0, 5:8], np.array([1.0, 2.0, -1.0]) * a * sc_ * (1 - sc_), atol=1e-14)
    # the opacity gradient sees the blended colour
    assert g[0, 4] == pytest.approx(np.dot([1.0, 2.0, -1.0], (1 - cb) * sc_ + cb * co) * a * (1 - sig(0.3)),
                                    abs=1e-13)


def test_kat_texel_edge_is_inclusive():
    """tex_x == Wt-1 is sampled (hard cut is `x > W-1`, tile_common.h:177)."""
    t = np.zeros((8, 8), np.float32)
    t[:, 7] = 1.0
    sc = _one_prim_scene(t, 20.0, 20.0, 4.0, v=5.0)    # hx = 3.5 -> dx = 4 maps to tex 7
    f = _render(sc)
    assert f["alpha"][20, 24] == pytest.approx(sig(5.0), abs=1e-15)
    # dx = 3 -> tex 6.125: bilinear weight 0.125 on the hot column
    assert f["alpha"][20, 23] == pytest.approx(0.125 * sig(5.0), abs=1e-15)
    assert f["alpha"][20, 25] == 0.0                    # culled (|dx| > hw = 4)


def test_kat_quarter_turn():
    """phi = pi/2 maps template column x to image row: u = dy/r, v = -dx/r."""
    t = np.zeros((9, 9), np.float32)
    t[:, 6] = 1.0                                        # u = (6/4)-1 = +0.5
    sc = _one_prim_scene(t, 20.0, 20.0, 4.0, th=np.pi / 2, v=4.0)
    f = _render(sc)
    row = f["alpha"][22, 16:25]                           # dy = +2 -> u = +0.5
    assert np.allclose(row[1:8], sig(4.0), atol=1e-12)
    assert f["alpha"][21, 20] < 1e-12 and f["alpha"][23, 20] < 1e-12


def test_termination_bounds_image_error():
    sc = small_scene(3, N=60)
    offs, idx = bin_scene(sc)
    full = O.forward(sc, offs, idx)
    cut = O.forward(sc, offs, idx, t_stop=1e-4)
    assert np.abs(full["color"] - cut["color"]).max() <= 1e-4
    assert cut["stats"]["live"] <= full["stats"]["live"]


def test_finite_difference_gradcheck_fp64():
    """Central differences (h = 1e-6) of the FP64 forward against the
    backward, on every centre / radius / rotation / opacity / colour
    parameter of a 64x64, N=32 scene with one 32x32 soft disk."""
    from diffbmp_b200 import workloads as wl
    spec = wl.make_scene("c3", seed=4)
    sc = O.Scene(spec.H, spec.W, 32, spec.means2D, spec.radii, spec.rotations, spec.opacities, spec.colors,
                 spec.templates, spec.sel)
    offs, idx = bin_scene(sc, O.BIN_CULL)
    rng = np.random.default_rng(1)
    wc = rng.normal(0, 1, (sc.H, sc.W, 3)).astype(np.float32)
    wa = rng.normal(0, 1, (sc.H, sc.W)).astype(np.float32)

    def loss(s):
        f = O.forward(s, offs, idx)
        return float((f["color"] * wc).sum() + (f["alpha"] * wa).sum())

    g = O.backward(sc, offs, idx, wc, wa)
    h = 1e-6
    fields = [("means2D", 0), ("means2D", 1), ("radii", None), ("rot", None), ("opac", None),
              ("colors", 0), ("colors", 1), ("colors", 2)]
    checked = skipped = 0
    for k, (name, col) in enumerate(fields):
        fd = np.zeros(sc.N)
        for n in range(sc.N):
            arr = getattr(sc, name)
            sl = (n, col) if col is not None else (n,)
            x0 = arr[sl]
            arr[sl] = x0 + h; lp = loss(sc)
            arr[sl] = x0 - h; lm = loss(sc)
            arr[sl] = x0; l0 = loss(sc)
            # a one-sided slope pair that disagrees marks a crossed cull / cut edge
            if abs((lp - l0) - (l0 - lm)) > 1e-3 * max(abs(lp - l0), 1e-9) + 1e-9:
                fd[n] = np.nan; skipped += 1
            else:
                fd[n] = (lp - lm) / (2 * h); checked += 1
        ok = ~np.isnan(fd)
        assert rel_err(g[ok, k], fd[ok], floor=1e-9) < 1e-5, f"block {k} ({name})"
    assert checked >= 8 * sc.N - 8, (checked, skipped)


def test_band_covers_texel_grid_lines():
    """A point 1e-7 texel below a texel grid line: float32 can round its
    coordinate onto the line, where the bilinear gradient jumps (the value
    does not).  The +-edge band runs give its two one-sided gradients, the
    plain run one of them, and the image does not move."""
    from diffbmp_b200 import workloads as wl
    T = wl.random_shape(np.random.default_rng(4), 32)[None]
    hy, r, py = 15.5, 10.0, 20
    my = py - r * ((10.0 - 1e-7) / hy - 1.0)          # texel row of pixel row py: 10 - 1e-7
    # centre x 17.3: no pixel of row py lies on the cull square or the texel cut
    sc = O.Scene(40, 40, 32, np.array([[17.3, my]]), np.array([r]), np.array([0.0]), np.array([2.0]),
                 np.zeros((1, 3)), T, np.zeros(1, np.int32))
    offs, idx = bin_scene(sc, O.BIN_CULL)
    gc = np.zeros((40, 40, 3), np.float32)
    gc[py, :, :] = 1.0                                  # only row py carries gradient
    g0 = O.backward(sc, offs, idx, gc, None)
    hi = O.backward(sc, offs, idx, gc, None, edge=1e-3)
    lo = O.backward(sc, offs, idx, gc, None, edge=-1e-3)
    assert np.abs(hi - lo)[0, 1] > 1e-3 * np.abs(g0[0, 1])        # the y-gradient jumps across the line
    assert np.allclose(g0, lo) or np.allclose(g0, hi)
    f0, fh, fl = (O.forward(sc, offs, idx, edge=e)["color"][py] for e in (0.0, 1e-3, -1e-3))
    inner = slice(10, 25)                               # pixels away from the cull / cut edges
    assert np.allclose(f0[inner], fh[inner], atol=1e-9) and np.allclose(f0[inner], fl[inner], atol=1e-9)
