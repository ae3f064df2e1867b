"""Generates the golden fixtures in tests/golden/ by running the reference's own
Python code (smhongok/diffbmp, pydiffbmp package) on the CPU.

Run by hand in a checkout that has the reference next to it:

    python tests/golden/make_golden.py --reference /path/to/diffbmp

The reference's optional dependencies that are absent here (cairosvg,
psd_tools, piq, ...) are replaced by empty stub modules; none of them is on
the code paths exercised below.  Fixtures produced:

* tmpl_bbox.npz   -- SimpleTileRenderer._compute_primitive_bboxes
                     (pydiffbmp/core/renderer/simple_tile_renderer.py:130-171)
* bin_<case>.npz  -- _unified_primitive_assignment + _convert_masks_to_mapping
                     (vector_renderer.py:401-444, simple_tile_renderer.py:721-766)
* blur.npz         -- gaussian_blur (pydiffbmp/util/utils.py:22-67) of a small
                     atlas at several sigmas, as VectorRenderer applies it
                     (vector_renderer.py:80-96)
* torch_<case>.npz -- the PyTorch per-tile renderer (_process_tiles_parallel with
                     CUDA off, simple_tile_renderer.py:479-569, 1304-1550):
                     image, alpha and autograd gradients of
                     sum(image*wc) + sum(alpha*wa) for seeded weights wc, wa.
"""
from __future__ import annotations

import argparse
import json
import importlib.abc
import importlib.machinery
import os
import sys
from unittest import mock

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

_STUBS = {"cairosvg", "psd_tools", "piq", "matplotlib", "svgpathtools", "svgwrite", "scour",
          "fontTools", "pyvista", "moviepy", "pylrc", "wandb", "clip", "lpips"}


class _StubFinder(importlib.abc.MetaPathFinder, importlib.abc.Loader):
    def find_spec(self, name, path, target=None):
        if name.split(".")[0] in _STUBS:
            return importlib.machinery.ModuleSpec(name, self, is_package=True)
        return None

    def create_module(self, spec):
        m = mock.MagicMock()
        m.__path__ = []
        m.__spec__ = spec
        m.__name__ = spec.name
        return m

    def exec_module(self, module):
        pass


def load_reference(ref_root: str):
    if not ref_root or not os.path.isdir(os.path.join(ref_root, "pydiffbmp")):
        raise SystemExit(f"reference checkout not found at {ref_root!r}: pass --reference or set DIFFBMP_REFERENCE")
    os.environ["WANDB_MODE"] = "disabled"
    sys.meta_path.insert(0, _StubFinder())
    sys.path.insert(0, ref_root)
    import torch  # noqa: F401
    from pydiffbmp.core.renderer import simple_tile_renderer as str_
    str_.CUDA_AVAILABLE = False      # take the PyTorch per-tile path
    return str_


def make_renderer(str_, H, W, S, ts, amax):
    import torch
    P, Ht, Wt = S.shape
    co = torch.zeros(P, Ht, Wt, 3)
    R = str_.SimpleTileRenderer((H, W), torch.from_numpy(S), tile_size=ts, alpha_upper_bound=amax,
                                device="cpu", c_blend=-40.0, primitive_colors=co)
    R._forward_compute_time_accum = 0.0
    return R


def tile_bounds(H, W, ts):
    import torch
    th, tw = (H + ts - 1) // ts, (W + ts - 1) // ts
    ty = torch.arange(th).repeat_interleave(tw)
    tx = torch.arange(tw).repeat(th)
    ys = ty * ts
    ye = torch.clamp(ys + ts, max=H)
    xs = tx * ts
    xe = torch.clamp(xs + ts, max=W)
    return xs, xe, ys, ye


def scene_params(rng, H, W, N, rmin, rmax, off_canvas=0.0):
    cx = rng.uniform(-off_canvas * W, (1 + off_canvas) * W, N)
    cy = rng.uniform(-off_canvas * H, (1 + off_canvas) * H, N)
    r = np.exp(rng.uniform(np.log(rmin), np.log(rmax), N))
    th = rng.uniform(0, 2 * np.pi, N)
    v = rng.normal(0, 1.2, N)
    c = rng.normal(0, 1.5, (N, 3))
    return (np.stack([cx, cy], 1).astype(np.float32), r.astype(np.float32), th.astype(np.float32),
            v.astype(np.float32), c.astype(np.float32))


def gen_bin_case(str_, name, H, W, ts, S, N, seed, rmin, rmax, off_canvas=0.0, special=None):
    import torch
    rng = np.random.default_rng(seed)
    means2D, r, th, v, c = scene_params(rng, H, W, N, rmin, rmax, off_canvas)
    if special is not None:
        special(means2D, r, th)
    R = make_renderer(str_, H, W, S, ts, 1.0)
    xs, xe, ys, ye = tile_bounds(H, W, ts)
    x = torch.from_numpy(means2D[:, 0].copy()); y = torch.from_numpy(means2D[:, 1].copy())
    masks = R._unified_primitive_assignment(x, y, torch.from_numpy(r), torch.from_numpy(th),
                                            xs, xe, ys, ye)
    mapping = R._convert_masks_to_mapping(masks, xs, xe, ys, ye).numpy().astype(np.int32)
    np.savez_compressed(os.path.join(HERE, f"bin_{name}.npz"), H=H, W=W, ts=ts, S=S,
                        means2D=means2D, radii=r, rotations=th, mapping=mapping,
                        tbbox=np.array(R.primitive_bboxes, np.float32))
    print(f"bin_{name}: N={N} L={mapping[1]}")


def gen_torch_case(str_, name, H, W, ts, S, N, seed, rmin, rmax, amax):
    import torch
    rng = np.random.default_rng(seed)
    means2D, r, th, v, c = scene_params(rng, H, W, N, rmin, rmax)
    P = S.shape[0]
    R = make_renderer(str_, H, W, S, ts, amax)
    x = torch.tensor(means2D[:, 0], requires_grad=True)
    y = torch.tensor(means2D[:, 1], requires_grad=True)
    rr = torch.tensor(r, requires_grad=True)
    tt = torch.tensor(th, requires_grad=True)
    vv = torch.tensor(v, requires_grad=True)
    cc = torch.tensor(c, requires_grad=True)
    gsel = (torch.arange(N) % P).flip(0)
    out = torch.zeros(H, W, 3)
    img, alpha = R._process_tiles_parallel(x, y, rr, tt, vv, cc, 0.0, None, gsel, out, None,
                                           return_alpha=True)
    wc = torch.from_numpy(rng.normal(0, 1, (H, W, 3)).astype(np.float32))
    wa = torch.from_numpy(rng.normal(0, 1, (H, W)).astype(np.float32))
    ((img * wc).sum() + (alpha * wa).sum()).backward()
    xs, xe, ys, ye = tile_bounds(H, W, ts)
    masks = R._unified_primitive_assignment(x.detach(), y.detach(), rr.detach(), tt.detach(),
                                            xs, xe, ys, ye)
    mapping = R._convert_masks_to_mapping(masks, xs, xe, ys, ye).numpy().astype(np.int32)
    np.savez_compressed(
        os.path.join(HERE, f"torch_{name}.npz"), H=H, W=W, ts=ts, S=S, amax=amax,
        means2D=means2D, radii=r, rotations=th, opacities=v, colors=c, sel=gsel.numpy().astype(np.int32),
        mapping=mapping, image=img.detach().numpy(), alpha=alpha.detach().numpy(),
        wc=wc.numpy(), wa=wa.numpy(),
        g_x=x.grad.numpy(), g_y=y.grad.numpy(), g_r=rr.grad.numpy(), g_theta=tt.grad.numpy(),
        g_v=vv.grad.numpy(), g_c=cc.grad.numpy())
    print(f"torch_{name}: N={N} image sum={float(img.sum()):.4f}")


# Options of the recorded fit loop: ExponentialLR decay, the adaptive blur
# schedule and pruning, as the reference's opt_conf names them.
FIT_LOOP_CONF = {
    "num_iterations": 50,
    "learning_rate": {"default": 0.01, "gain_x": 10.0, "gain_y": 10.0, "gain_r": 10.0, "gain_v": 1.5,
                      "gain_theta": 1.0, "gain_c": 1.0},
    "loss_config": {"type": "mse"},
    "do_decay": True, "decay_rate": 0.95,
    "do_adapt_gaussian_blur": True, "blur_sigma_start": 2.0, "blur_sigma_end": 0.0,
    "pruning": {"do_pruning": True, "prune_iterations": 5, "no_prune_last_iterations": 10,
                "no_prune_warmup_iterations": 20, "prune_threshold": 0.3},
    "bg_color": "white",
}


def gen_fit_loop(str_):
    """Runs the reference's optimisation loop (SimpleTileRenderer.
    _optimize_parameters_whole, simple_tile_renderer.py:913-1228) on its CPU
    path for the 256x256 / N=512 soft-disk scene with FIT_LOOP_CONF, and
    records per iteration the learning rate of each Adam parameter group at
    its step, the blur sigma handed to the renderer, and each prune: its
    iteration, the opacity logits it saw and the primitives it replaced.  The
    initializer is a stand-in whose reinitialize_subset hands out consecutive
    rows of a seeded pool (the reference's own initializers are outside this
    path)."""
    import tempfile
    import torch
    from diffbmp_b200 import workloads as wl
    from diffbmp_b200.fitting import fallback_pool
    s = wl.make_scene("c0", 0)
    N = s.N
    pool = fallback_pool(np.random.default_rng(17), s.H, s.W, 4 * N)
    R = make_renderer(str_, s.H, s.W, s.templates, 32, 1.0)
    R.output_path = tempfile.mkdtemp()
    str_.vram_used_by_pid = lambda pid=None: 0          # NVML is absent on this host
    rec = dict(lrs=[], sigmas=[], prune_its=[], prune_v=[], prune_idx=[])
    orig_step = torch.optim.Adam.step

    def step(self, *a, **k):
        rec["lrs"].append([g["lr"] for g in self.param_groups])
        return orig_step(self, *a, **k)
    orig_render = R.render_from_params

    def render(*a, **k):
        rec["sigmas"].append(float(k.get("sigma", 0.0)))
        # render_from_params picks the per-tile path only when torch sees a GPU
        # (simple_tile_renderer.py:249); its sequential CPU path does not run as
        # written, so the per-tile path (CPU fallback inside) is forced here
        real = torch.cuda.is_available
        torch.cuda.is_available = lambda: True
        try:
            return orig_render(*a, **k)
        finally:
            torch.cuda.is_available = real
    orig_prune = R.do_prune

    def do_prune(x, y, r, v, theta, c, prune_conf, initializer, target_image):
        v0 = v.detach().clone()
        x0 = x.detach().clone()
        orig_prune(x, y, r, v, theta, c, prune_conf, initializer, target_image)
        rec["prune_its"].append(len(rec["sigmas"]))
        rec["prune_v"].append(v0.numpy())
        rec["prune_idx"].append(np.nonzero((x.detach() != x0).numpy() | (v.detach() != v0).numpy())[0])

    class Initializer:
        decrease_max_radius = 0

        def __init__(self):
            self.cursor = 0

        def reinitialize_subset(self, n, target, device):
            rows = torch.from_numpy(pool[[(self.cursor + i) % len(pool) for i in range(n)]])
            self.cursor += n
            return (rows[:, 0], rows[:, 1], rows[:, 2], rows[:, 4], rows[:, 3], rows[:, 5:8])

    R.render_from_params = render
    R.do_prune = do_prune
    torch.optim.Adam.step = step
    try:
        leaf = lambda a: torch.tensor(np.ascontiguousarray(a), requires_grad=True)
        x, y = leaf(s.means2D[:, 0]), leaf(s.means2D[:, 1])
        r, th, v, c = leaf(s.radii), leaf(s.rotations), leaf(s.opacities), leaf(s.colors)
        import copy
        R._optimize_parameters_whole(x, y, r, v, th, c, torch.from_numpy(s.target), copy.deepcopy(FIT_LOOP_CONF),
                                     initializer=Initializer())
    finally:
        torch.optim.Adam.step = orig_step
    idx = np.concatenate(rec["prune_idx"]) if rec["prune_idx"] else np.zeros(0, np.int64)
    np.savez_compressed(
        os.path.join(HERE, "fit_loop.npz"), N=N, lrs=np.array(rec["lrs"], np.float64),
        sigmas=np.array(rec["sigmas"], np.float64), prune_its=np.array(rec["prune_its"], np.int64),
        prune_v=np.stack(rec["prune_v"]) if rec["prune_v"] else np.zeros((0, N), np.float32),
        prune_counts=np.array([len(i) for i in rec["prune_idx"]], np.int64), prune_idx=idx.astype(np.int64),
        pool=pool, conf=json.dumps(FIT_LOOP_CONF), decay_rate=FIT_LOOP_CONF["decay_rate"], sigma_start=FIT_LOOP_CONF["blur_sigma_start"],
        sigma_end=FIT_LOOP_CONF["blur_sigma_end"], iterations=FIT_LOOP_CONF["num_iterations"],
        final=np.concatenate([t.detach().numpy().reshape(N, -1) for t in (x, y, r, th, v, c)], 1))
    print(f"fit_loop: {len(rec['lrs'])} steps, prunes at {rec['prune_its']} replacing "
          f"{[len(i) for i in rec['prune_idx']]}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("DIFFBMP_REFERENCE"),
                    help="root of the reference checkout (or set DIFFBMP_REFERENCE)")
    ap.add_argument("--only", default=None, help="regenerate one fixture group only (e.g. fit_loop)")
    args = ap.parse_args()
    str_ = load_reference(args.reference)
    if args.only == "fit_loop":
        gen_fit_loop(str_)
        return
    from diffbmp_b200 import workloads as wl
    import torch

    # template bboxes: soft disk, random shapes, an empty and a one-texel template
    rng = np.random.default_rng(11)
    shapes = [wl.soft_disk(64, 24.0), wl.random_shape(rng, 64), wl.random_shape(rng, 64),
              np.zeros((64, 64), np.float32)]
    one = np.zeros((64, 64), np.float32); one[7, 50] = 0.5
    shapes.append(one)
    edge = np.zeros((64, 64), np.float32); edge[:, 0] = 1e-6; edge[0, :] = 2e-6
    shapes.append(edge)
    S = np.stack(shapes)
    R = make_renderer(str_, 64, 64, S, 32, 1.0)
    np.savez_compressed(os.path.join(HERE, "tmpl_bbox.npz"), S=S,
                        bboxes=np.array(R.primitive_bboxes, np.float32))
    print("tmpl_bbox:", R.primitive_bboxes)

    disk64 = wl.soft_disk(64, 24.0)[None]
    rng = np.random.default_rng(5)
    atlas3 = np.stack([wl.random_shape(rng, 48) for _ in range(3)])
    gen_bin_case(str_, "c0", 256, 256, 32, disk64, 512, 1, 0.05 * 256, 0.3 * 256)
    gen_bin_case(str_, "ragged", 200, 136, 16, atlas3, 300, 2, 3.0, 60.0, off_canvas=0.2)

    def special(m, r, th):
        m[0] = (-500.0, -500.0); r[0] = 3.0             # far off canvas
        m[1] = (64.0, 32.0); r[1] = 1e-7                 # degenerate radius
        m[2] = (100.0, 100.0); r[2] = 5000.0             # covers everything
        m[3] = (32.0, 32.0); th[3] = np.float32(np.pi / 2)
        m[4] = (31.999998, 95.5); r[4] = 0.5; th[4] = 0.0
    gen_bin_case(str_, "edges", 128, 160, 32, disk64, 64, 3, 2.0, 40.0, special=special)

    rng = np.random.default_rng(9)
    gen_torch_case(str_, "disk64", 64, 64, 32, wl.soft_disk(32, 12.0)[None], 32, 21, 4.0, 20.0, 1.0)
    atlas_ns = np.stack([wl.random_shape(rng, 40)[:24, :] for _ in range(3)])  # 24x40, non-square
    gen_torch_case(str_, "ragged", 80, 96, 16, atlas_ns, 48, 22, 3.0, 25.0, 0.8)
    torch.set_num_threads(1)
    gen_blur(args.reference)
    torch.set_num_threads(os.cpu_count() or 1)
    gen_fit_loop(str_)


def gen_blur(ref_root):
    import torch
    from pydiffbmp.util.utils import gaussian_blur
    from diffbmp_b200 import workloads as wl
    rng = np.random.default_rng(13)
    S = np.stack([wl.random_shape(rng, 40) for _ in range(3)]).astype(np.float32)
    S[1, 3:9, 30:36] = 1.0                      # a hard-edged block
    sigmas = np.array([0.5, 1.5, 2.0, 0.0], np.float32)
    out = []
    for sg in sigmas:
        b = gaussian_blur(torch.from_numpy(S).unsqueeze(0), float(sg)).squeeze(0)
        out.append(b.numpy().astype(np.float32))
    np.savez_compressed(os.path.join(HERE, "blur.npz"), S=S, sigmas=sigmas, blurred=np.stack(out))
    print("blur:", [float(np.abs(o - S).max()) for o in out])


if __name__ == "__main__":
    main()
