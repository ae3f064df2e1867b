"""GPU tests of the pydiffbmp renderer API drop-in (diffbmp_b200/pydiffbmp):
SimpleTileRenderer.render_from_params / render_from_params_batch and
DiffBMPWrapper.render / render_batch against the FP64 oracle at the parity
bars (image <= 1e-5 max-abs, gradients <= 1e-4 relative per parameter block,
boundary band held to its spread), with the renderer's template assignment
(N-1-i) % p, a background image, blurred templates and return_alpha."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from helpers import bin_scene

pytestmark = pytest.mark.gpu


def _cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def _setup(seed=0, H=160, W=192, N=300, P=3, amax=0.8):
    from diffbmp_b200 import workloads as wl
    rng = np.random.default_rng(seed)
    S = np.stack([wl.random_shape(rng, 48) for _ in range(P)]).astype(np.float32)
    s = wl.make_scene("c1", seed, H=H, W=W, N=N, templates=S)
    bg = rng.uniform(0, 1, (H, W, 3)).astype(np.float32)
    sel = ((N - 1 - np.arange(N)) % P).astype(np.int32)
    return s, S, bg, sel, amax


def _leaves(s, shift=None):
    m = s.means2D if shift is None else s.means2D + shift
    return [_cuda(m[:, 0]).requires_grad_(), _cuda(m[:, 1]).requires_grad_(), _cuda(s.radii).requires_grad_(),
            _cuda(s.rotations).requires_grad_(), _cuda(s.opacities).requires_grad_(), _cuda(s.colors).requires_grad_()]


def _grads(leaves):
    x, y, r, th, v, c = leaves
    return np.stack([x.grad.cpu().numpy(), y.grad.cpu().numpy(), r.grad.cpu().numpy(), th.grad.cpu().numpy(),
                     v.grad.cpu().numpy()] + [c.grad.cpu().numpy()[:, k] for k in range(3)], 1)


def _check(s, templates, sel, amax, means2D, img, alpha, bg, wc, wa, ours):
    """Composite over bg against the oracle; gradients through the composite:
    dL/dC = wc, dL/dA = wa - sum_c wc * bg."""
    sc = O.Scene(s.H, s.W, 32, means2D, s.radii, s.rotations, s.opacities, s.colors, templates, sel, amax)
    offs, idx = bin_scene(sc)
    # the composite C + (1 - A) bg is within tol when C and A are within tol / 2 each (bg in [0, 1])
    color = img - (1.0 - alpha)[..., None] * bg
    O.check_image(sc, offs, idx, color, alpha, tol=5e-6)
    ga = (wa - (wc * bg).sum(-1)).astype(np.float32)
    O.check_grads(sc, offs, idx, wc, ga, ours, rel=1e-4)


@pytest.mark.parametrize("is_final", [False, True])
def test_render_from_params_vs_oracle(is_final):
    """With sigma > 0 the renderer holds blurred templates; is_final renders
    the unblurred ones; binning uses the unblurred content bboxes either way."""
    from diffbmp_b200.pydiffbmp.core.renderer.simple_tile_renderer import SimpleTileRenderer
    s, S, bg, sel, amax = _setup(0)
    R = SimpleTileRenderer((s.H, s.W), _cuda(S), tile_size=32, alpha_upper_bound=amax, sigma=1.5)
    leaves = _leaves(s)
    img, alpha = R.render_from_params(*leaves, return_alpha=True, I_bg=_cuda(bg), is_final=is_final)
    rng = np.random.default_rng(1)
    wc = rng.normal(0, 1, (s.H, s.W, 3)).astype(np.float32)
    wa = rng.normal(0, 1, (s.H, s.W)).astype(np.float32)
    ((img * _cuda(wc)).sum() + (alpha * _cuda(wa)).sum()).backward()
    templates = S if is_final else R.S_blurred.float().cpu().numpy()
    if not is_final:    # the blurred templates are the pinned template blur's (dbmp_template_blur)
        assert np.abs(templates - S).max() > 1e-3
    _check(s, templates, sel, amax, s.means2D, img.detach().cpu().numpy(), alpha.detach().cpu().numpy(), bg, wc, wa,
           _grads(leaves))


def test_render_from_params_colour_maps_vs_oracle():
    """c_blend > 0: the primitive colour maps c_o[(N-1-i) % p] blend in."""
    from diffbmp_b200.pydiffbmp.core.renderer.simple_tile_renderer import SimpleTileRenderer
    s, S, bg, sel, amax = _setup(2)
    co = np.random.default_rng(3).uniform(0, 1, (S.shape[0], S.shape[1], S.shape[2], 3)).astype(np.float32)
    R = SimpleTileRenderer((s.H, s.W), _cuda(S), alpha_upper_bound=amax, c_blend=0.4, primitive_colors=_cuda(co))
    leaves = _leaves(s)
    img = R.render_from_params(*leaves, I_bg=_cuda(bg))
    wc = np.random.default_rng(4).normal(0, 1, (s.H, s.W, 3)).astype(np.float32)
    (img * _cuda(wc)).sum().backward()
    sc = O.Scene(s.H, s.W, 32, s.means2D, s.radii, s.rotations, s.opacities, s.colors, S, sel, amax,
                 colors_orig=co[sel], c_blend=0.4)
    offs, idx = bin_scene(sc)
    ref = O.forward(sc, offs, idx)
    ref_img = ref["color"] + (1 - ref["alpha"])[..., None] * bg
    band, band_a = O.boundary_band(sc, offs, idx)
    err = np.abs(img.detach().cpu().numpy() - ref_img).max(-1)
    assert err[(band == 0) & (band_a == 0)].max() <= 1e-5
    ga = -(wc * bg).sum(-1).astype(np.float32)
    O.check_grads(sc, offs, idx, wc, ga, _grads(leaves), rel=1e-4)


def test_render_from_params_batch_vs_oracle_and_single():
    """A batch of candidates (some outside the clamp range: the batch clamps
    their values, gradients pass through) in one launch per direction; each
    candidate against the oracle, and equal to rendering it alone."""
    from diffbmp_b200.pydiffbmp.core.renderer.simple_tile_renderer import SimpleTileRenderer
    s, S, bg, sel, amax = _setup(5, N=200)
    R = SimpleTileRenderer((s.H, s.W), _cuda(S), alpha_upper_bound=amax)
    rng = np.random.default_rng(6)
    B = 4
    shifts = [rng.normal(0, 4, s.means2D.shape).astype(np.float32) for _ in range(B)]
    shifts[1][:5] = -50.0                                  # off canvas: clamped to x, y = 0
    cands = [_leaves(s, sh) for sh in shifts]
    outs = R.render_from_params_batch([tuple(c) for c in cands], return_alpha=True, I_bg=_cuda(bg))
    wcs = [rng.normal(0, 1, (s.H, s.W, 3)).astype(np.float32) for _ in range(B)]
    loss = sum((img * _cuda(wc)).sum() for (img, _), wc in zip(outs, wcs))
    loss.backward()
    for b in range(B):
        m = s.means2D + shifts[b]
        mc = np.stack([np.clip(m[:, 0], 0, s.W - 1), np.clip(m[:, 1], 0, s.H - 1)], 1).astype(np.float32)
        s_b = type(s)(**{**s.__dict__, "radii": np.clip(s.radii, 2.0, min(s.H, s.W) // 4).astype(np.float32)})
        img, alpha = outs[b]
        _check(s_b, S, sel, amax, mc, img.detach().cpu().numpy(), alpha.detach().cpu().numpy(), bg, wcs[b],
               np.zeros((s.H, s.W), np.float32), _grads(cands[b]))
    # the batch launch renders each candidate exactly as a single render of its clamped values
    m = s.means2D + shifts[2]
    x2, y2 = _cuda(np.clip(m[:, 0], 0, s.W - 1)), _cuda(np.clip(m[:, 1], 0, s.H - 1))
    r2 = _cuda(np.clip(s.radii, 2.0, min(s.H, s.W) // 4))
    img2 = R.render_from_params(x2, y2, r2, _cuda(s.rotations), _cuda(s.opacities), _cuda(s.colors), I_bg=_cuda(bg))
    assert torch.equal(img2, outs[2][0])


def test_diffbmp_wrapper_render_and_batch():
    from diffbmp_b200.pydiffbmp.core.renderer.simple_tile_renderer import SimpleTileRenderer
    from diffbmp_b200.pydiffbmp.diffbmp_wrapper import DiffBMPWrapper
    s, S, bg, sel, amax = _setup(7, N=150)
    # values the batch path's clamp leaves unchanged (x in [0, W-1], y in [0, H-1], r in [2, min(H,W)//4])
    s.radii[:] = np.clip(s.radii, 2.0, min(s.H, s.W) // 4)
    s.means2D[:] = np.clip(s.means2D - 3.0, 0.0, [s.W - 4.0, s.H - 4.0])
    w = DiffBMPWrapper("cuda").set_primitive(_cuda(S))
    w.canvas_size = (s.H, s.W)
    leaves = _leaves(s)
    rgba = w.render(*leaves, background=_cuda(bg), blur_sigma=0.0, return_alpha=True, alpha_upper_bound=amax)
    assert rgba.shape == (s.H, s.W, 4)
    R = SimpleTileRenderer((s.H, s.W), _cuda(S), alpha_upper_bound=amax)
    img, alpha = R.render_from_params(*[t.detach() for t in leaves], return_alpha=True, I_bg=_cuda(bg))
    assert torch.equal(rgba[..., :3], img) and torch.equal(rgba[..., 3], alpha)
    batch = w.render_batch([tuple(leaves), tuple(_leaves(s, np.float32(3.0)))], background=_cuda(bg),
                           blur_sigma=0.0, alpha_upper_bound=amax)
    assert len(batch) == 2 and torch.equal(batch[0], img)


def test_optimize_parameters_runs_the_device_loop():
    """The reference's fit-loop entry point: parameters are fitted in place on
    the device, with the decay, blur schedule and pruning options of its
    opt_conf, and the L2 loss falls."""
    from diffbmp_b200 import workloads as wl
    from diffbmp_b200.pydiffbmp.core.renderer.simple_tile_renderer import SimpleTileRenderer
    s = wl.make_scene("c0", 3)
    R = SimpleTileRenderer((s.H, s.W), _cuda(s.templates), alpha_upper_bound=1.0)
    x, y, r, th, v, c = [t.detach() for t in _leaves(s)]
    x0 = x.clone()
    bg = torch.ones((s.H, s.W, 3), device="cuda")
    target = _cuda(s.target)
    before = torch.mean((R.render_from_params(x, y, r, th, v, c, I_bg=bg) - target) ** 2).item()
    conf = {"num_iterations": 40, "learning_rate": {"default": 0.01}, "do_decay": True, "decay_rate": 0.99,
            "do_adapt_gaussian_blur": True, "blur_sigma_start": 1.0, "blur_sigma_end": 0.0,
            "pruning": {"do_pruning": True, "prune_iterations": 10, "no_prune_last_iterations": 5,
                        "no_prune_warmup_iterations": 15, "prune_threshold": 0.2}}
    out = R.optimize_parameters(x, y, r, v, th, c, target, conf)
    assert out[0] is x and not torch.equal(x, x0)
    after = torch.mean((R.render_from_params(x, y, r, th, v, c, I_bg=bg) - target) ** 2).item()
    print("loss", before, "->", after)
    assert after < 0.8 * before
    with pytest.raises(ValueError):
        R.optimize_parameters(x, y, r, v, th, c, target, {**conf, "loss_config": {"type": "perceptual"}})
