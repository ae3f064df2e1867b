"""GPU tests of the fitting step: the fused fwd+L2+bwd kernel against the
plain kernels + torch loss gradient, CUDA-graph replay against eager
execution, list-overflow recovery, and the Adam step against torch.optim.Adam."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

from diffbmp_b200 import workloads as wl  # noqa: E402


def make(spec, kind="f32", fused=True, **cfg):
    from diffbmp_b200.fitting import FitConfig, ImageFitter
    from diffbmp_b200.rasterizer import Atlas
    atlas = Atlas(torch.from_numpy(spec.templates).cuda(), kind)
    return ImageFitter(spec.means2D, spec.radii, spec.rotations, spec.opacities, spec.colors, spec.sel, atlas,
                       spec.target, spec.background, FitConfig(fused=fused, **cfg))


@pytest.fixture(scope="module")
def spec():
    return wl.make_scene("c1", seed=3, H=256, W=320, N=600)


def test_fused_gradient_equals_plain(spec):
    a, b = make(spec, fused=True), make(spec, fused=False)
    for j in (a, b):
        j.adam_cfg.lr[:] = [0.0] * 8          # keep parameters fixed: compare gradients only
        j.step()
        j.sync()
    ga, gb = a.gacc.cpu().numpy(), b.gacc.cpu().numpy()
    for k in range(8):
        rel = np.linalg.norm(ga[:, k] - gb[:, k]) / max(np.linalg.norm(gb[:, k]), 1e-30)
        assert rel < 1e-5, (k, rel)
    assert abs(a.loss() - b.loss()) <= 1e-6 * b.loss()


def test_graph_replay_equals_eager(spec):
    a, b = make(spec), make(spec)
    for _ in range(3):
        a.step()
    a.sync()
    b.step(); b.sync()
    b.capture()
    b.step(); b.step()
    b.sync()
    for k, v in a.params().items():
        assert torch.equal(v, b.params()[k]), k


def test_overflow_steps_are_replayed_exactly(spec):
    a, b = make(spec), make(spec)
    for _ in range(4):
        a.step()
    a.sync()
    # shrink b's capacity below the list length: every step overflows, is
    # skipped on the device, and sync() replays it after regrowing
    b.rz.capacity = 16
    b.rz._ws = None
    b.rz._ensure(b.cv, 16)
    for _ in range(4):
        b.step()
    assert b.sync() >= 4
    for k, v in a.params().items():
        assert torch.equal(v, b.params()[k]), k


def test_adam_matches_torch_optimizer(spec):
    """dbmp_adam_step == torch.optim.Adam (per-group lr) + the reference clamp,
    given the same gradients."""
    j = make(spec, fused=False)
    p0 = {k: v.clone() for k, v in j.params().items()}
    j.step(); j.sync()
    g = [t.clone() for t in j.grads]                      # finalized FP32 gradients of step 1
    ref = {k: v.clone().requires_grad_(True) for k, v in p0.items()}
    lr = [float(x) for x in j.adam_cfg.lr]
    opt = torch.optim.Adam([
        {"params": [ref["means2D"]], "lr": lr[0]},          # x and y share gain 10 here
        {"params": [ref["radii"]], "lr": lr[2]},
        {"params": [ref["rotations"]], "lr": lr[3]},
        {"params": [ref["opacities"]], "lr": lr[4]},
        {"params": [ref["colors"]], "lr": lr[5]}])
    for t, gg in zip([ref["means2D"], ref["radii"], ref["rotations"], ref["opacities"], ref["colors"]], g):
        t.grad = gg
    opt.step()
    with torch.no_grad():
        ref["means2D"][:, 0].clamp_(0, spec.W - 1); ref["means2D"][:, 1].clamp_(0, spec.H - 1)
        ref["radii"].clamp_(2.0, float(min(spec.H, spec.W) // 4))
    for k, v in j.params().items():
        torch.testing.assert_close(v, ref[k].detach(), rtol=2e-5, atol=2e-5)


def test_params_flat_layout_and_shape_check():
    """The five parameter tensors are views of params_flat, in the order
    centres, radii, rotations, opacity logits, colour logits; parameters that
    disagree on N are rejected."""
    import numpy as np
    import pytest
    import torch
    from diffbmp_b200 import workloads as wl
    from diffbmp_b200.fitting import FitConfig, ImageFitter
    from diffbmp_b200.rasterizer import Atlas
    s = wl.make_scene("c0", 1)
    atlas = Atlas(torch.from_numpy(s.templates).cuda(), "f16q")
    f = ImageFitter(s.means2D, s.radii, s.rotations, s.opacities, s.colors, s.sel, atlas, s.target, s.background,
                    FitConfig())
    N = s.N
    flat = f.params_flat.cpu().numpy()
    want = np.concatenate([np.asarray(a, np.float32).reshape(-1)
                           for a in (s.means2D, s.radii, s.rotations, s.opacities, s.colors)])
    assert flat.shape == (8 * N,) and np.array_equal(flat, want)
    for k, v in f.params().items():
        assert v.untyped_storage().data_ptr() == f.params_flat.untyped_storage().data_ptr(), k
    with pytest.raises(ValueError):
        ImageFitter(s.means2D[:-1], s.radii, s.rotations, s.opacities, s.colors, s.sel, atlas, s.target,
                    s.background, FitConfig())


def test_loop_decay_blur_prune_step_by_step():
    """The device loop with ExponentialLR decay, the adaptive blur schedule and
    pruning (the options recorded in tests/golden/fit_loop.npz from the
    reference's loop), checked at every one of its 50 steps against a replica
    of that one step started from the device's state: the reference's prune
    rule with the same replacement rows, the templates blurred with this
    step's sigma (dbmp_template_blur), the render's L2 gradients through the
    autograd path (plain kernels), and torch.optim.Adam with the learning rates
    the reference's own scheduler produced at that step, then the clamp.  The
    first 10 steps run eagerly, the rest replay one captured CUDA graph."""
    import ctypes
    import json
    from diffbmp_b200 import fitting as F
    from diffbmp_b200._lib import call
    from diffbmp_b200.rasterizer import Atlas, Rasterizer, _ptr, _stream, rasterize
    from helpers import golden
    fx = golden("fit_loop")
    s = wl.make_scene("c0", 0)                   # the scene and N the reference loop ran with
    N = s.N
    assert N == int(fx["N"])
    cfg = F.FitConfig.from_opt_conf(json.loads(str(fx["conf"])), pool=fx["pool"], fused=True)
    tmpl = torch.from_numpy(s.templates).cuda()
    job = F.ImageFitter(s.means2D, s.radii, s.rotations, s.opacities, s.colors, s.sel, Atlas(tmpl, "f32"),
                        s.target, s.background, cfg)
    target = torch.from_numpy(s.target).cuda()
    bg = torch.from_numpy(s.background).cuda()
    sel = torch.from_numpy(s.sel).cuda()
    pool = torch.from_numpy(fx["pool"]).cuda()
    cursor = replaced = 0
    keys = ("means2D", "radii", "rotations", "opacities", "colors")
    for k in range(cfg.num_iterations):
        p0 = {key: v.detach().clone() for key, v in job.params().items()}
        m0, v0 = job.adam_m.clone(), job.adam_v.clone()
        if k == 10:
            job.capture()
        job.step()
        assert job.sync() == 0
        # -- replica of iteration k ------------------------------------------
        q = p0
        if F.prune_due(cfg, k):
            low = torch.nonzero(torch.sigmoid(q["opacities"]) < cfg.prune.threshold).flatten()
            rows = pool[(cursor + torch.arange(low.numel(), device="cuda")) % pool.shape[0]]
            cursor += low.numel()
            replaced += low.numel()
            q["means2D"][low] = rows[:, 0:2]
            q["radii"][low], q["rotations"][low], q["opacities"][low] = rows[:, 2], rows[:, 3], rows[:, 4]
            q["colors"][low] = rows[:, 5:8]
        # the gradients the device used, from its raw sums and the pruned parameters
        g_dev = [torch.empty_like(q[key]) for key in keys]
        call("dbmp_grads_from_accum", ctypes.byref(job.cv), _ptr(job.gacc), _ptr(q["radii"]), _ptr(q["rotations"]),
             _ptr(q["opacities"]), _ptr(q["colors"]), *[_ptr(g) for g in g_dev], _stream())
        # the same gradients through the autograd render with this step's blurred templates
        sig = F.blur_sigma_at(cfg, k)
        atlas_k = Atlas(tmpl, "f32", sigma=sig)
        leaves = [q[key].clone().requires_grad_(True) for key in keys]
        rz = Rasterizer(s.H, s.W, 32)
        color, alpha = rasterize(*leaves, sel, atlas_k, rz)
        img = color + (1 - alpha).unsqueeze(-1) * bg
        torch.nn.functional.mse_loss(img, target).backward()
        for key, a, b in zip(keys, g_dev, leaves):
            rel = (a - b.grad).norm() / b.grad.norm().clamp_min(1e-30)
            assert rel < 1e-4, (k, key, float(rel), sig)
        # torch.optim.Adam from the device's moments with the reference's learning rates at step k
        lr = [float(x) for x in fx["lrs"][k]]                    # x, y, r, v, theta, c
        ref = {key: q[key].clone().requires_grad_(True) for key in keys}
        opt = torch.optim.Adam([{"params": [ref["means2D"]], "lr": lr[0]}, {"params": [ref["radii"]], "lr": lr[2]},
                                {"params": [ref["rotations"]], "lr": lr[4]}, {"params": [ref["opacities"]], "lr": lr[3]},
                                {"params": [ref["colors"]], "lr": lr[5]}])
        cols = {"means2D": slice(0, 2), "radii": 2, "rotations": 3, "opacities": 4, "colors": slice(5, 8)}
        for key, g in zip(keys, g_dev):
            t = ref[key]
            t.grad = g
            opt.state[t] = {"step": torch.tensor(float(k)), "exp_avg": m0[:N, cols[key]].clone().view_as(t),
                            "exp_avg_sq": v0[:N, cols[key]].clone().view_as(t)}
        opt.step()
        with torch.no_grad():
            ref["means2D"][:, 0].clamp_(0, s.W - 1)
            ref["means2D"][:, 1].clamp_(0, s.H - 1)
            ref["radii"].clamp_(2.0, float(min(s.H, s.W) // 4))
        for key in keys:
            torch.testing.assert_close(job.params()[key], ref[key].detach(), rtol=2e-5, atol=2e-5,
                                       msg=lambda m, key=key: f"iteration {k}, {key}: {m}")
    assert replaced > 0 and int(job.prune_state[3].item()) == replaced


def test_upload_params_double_buffered(spec):
    """ImageFitter.upload_params (copy stream, two staging buffers) gives
    each step the parameters uploaded for it, like a plain copy before the step."""
    a, b = make(spec), make(spec)
    rng = np.random.default_rng(8)
    base = a.params_flat.cpu()
    hosts = [(base + torch.from_numpy(rng.normal(0, 0.5, base.shape).astype(np.float32))).pin_memory()
             for _ in range(3)]
    a.capture()
    for h in hosts:
        a.upload_params(h)
        a.step()
        b.params_flat.copy_(h.cuda())
        b.step()
    a.sync(); b.sync()
    assert torch.equal(a.params_flat, b.params_flat)
    assert abs(a.loss() - b.loss()) <= 1e-12 * max(1.0, abs(b.loss()))
