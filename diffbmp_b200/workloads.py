"""Seeded synthetic scenes for the rasterizer's reference workloads.

The reference evaluates on image-fitting jobs (a target image, an atlas of
alpha bitmaps and N bitmap primitives).  No dataset ships with this package;
these generators produce inputs with the same shapes and value distributions:

* ``c0`` -- 256x256, N=512, one 64x64 soft disk  alpha = sigmoid((24 - rho)/2)
* ``c1`` -- 1024x1024, N=5000, 8 random 128x128 star / ring / blob bitmaps
* ``c2`` -- 2048x2048, N=20000, 16 random 256x256 bitmaps
* ``c3`` -- 64x64, N=32, one 32x32 soft disk (gradient check); 4096x4096, N=1e5
* ``c4`` -- serving jobs with canvases in {256,512,1024,2048}^2 and log-uniform N

Primitive parameters follow the reference's parameterisation
(pydiffbmp/core/renderer/simple_tile_renderer.py:173-266): centres in pixels,
``radii`` the half extent of the template square (tile_forward.cu:200-205),
rotations in radians, opacity and colour given as logits (the kernels apply
the sigmoid, tile_forward.cu:226-284).  "Depth uniform in [0,1]" is realised by
stable-sorting primitives by depth, because the reference composites in
ascending primitive index within each tile (index 0 frontmost).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def soft_disk(size: int, radius: float, softness: float = 2.0) -> np.ndarray:
    """alpha = sigmoid((radius - rho)/softness), rho = distance from the centre."""
    c = (size - 1) / 2.0
    yy, xx = np.mgrid[0:size, 0:size].astype(np.float64)
    rho = np.sqrt((xx - c) ** 2 + (yy - c) ** 2)
    return (1.0 / (1.0 + np.exp(-(radius - rho) / softness))).astype(np.float32)


def _soft(d: np.ndarray) -> np.ndarray:
    # signed distance (positive outside) -> alpha with a ~2 px 10-90% edge
    return (1.0 / (1.0 + np.exp(d / 0.5))).astype(np.float32)


def random_shape(rng: np.random.Generator, size: int) -> np.ndarray:
    """One random star, ring or blob bitmap with soft 2-px edges."""
    c = (size - 1) / 2.0
    yy, xx = np.mgrid[0:size, 0:size].astype(np.float64)
    dx, dy = xx - c, yy - c
    rho = np.sqrt(dx * dx + dy * dy)
    ang = np.arctan2(dy, dx)
    kind = rng.integers(0, 3)
    R = size * rng.uniform(0.28, 0.45)
    if kind == 0:  # star
        k = int(rng.integers(4, 9))
        depth = rng.uniform(0.25, 0.5)
        rad = R * (1.0 - depth * 0.5 * (1.0 + np.cos(k * ang + rng.uniform(0, 2 * np.pi))))
        d = rho - rad
    elif kind == 1:  # ring
        w = R * rng.uniform(0.15, 0.35)
        d = np.abs(rho - (R - w)) - w
    else:  # blob: union of soft circles
        d = np.full_like(rho, 1e9)
        for _ in range(int(rng.integers(3, 7))):
            cx, cy = rng.uniform(-0.3, 0.3, 2) * size
            rr = size * rng.uniform(0.12, 0.25)
            d = np.minimum(d, np.sqrt((dx - cx) ** 2 + (dy - cy) ** 2) - rr)
    return _soft(d)


def smooth_field(rng: np.random.Generator, H: int, W: int, n: int = 8,
                 noise: float = 0.0) -> np.ndarray:
    """(H,W,3) sum of n random 2-D sinusoids per channel, rescaled to [0,1]."""
    xs = np.arange(W, dtype=np.float64)
    ys = np.arange(H, dtype=np.float64)
    out = np.zeros((H, W, 3), np.float32)
    for ch in range(3):
        # sum_k a_k sin(u_k + v_k) = sum_k a_k (cos v_k sin u_k + sin v_k cos u_k), one (H,2n)@(2n,W) product
        A = np.zeros((H, 2 * n)); B = np.zeros((2 * n, W))
        for k in range(n):
            fx, fy = rng.uniform(-4, 4, 2)
            ph = rng.uniform(0, 2 * np.pi)
            a = rng.uniform(0.5, 1.0)
            u = 2 * np.pi * fx * xs / W + ph
            v = 2 * np.pi * fy * ys / H
            A[:, 2 * k], A[:, 2 * k + 1] = a * np.cos(v), a * np.sin(v)
            B[2 * k], B[2 * k + 1] = np.sin(u), np.cos(u)
        f = (A @ B).astype(np.float32)
        f -= f.min()
        f /= max(float(f.max()), 1e-12)
        out[..., ch] = f
    if noise > 0:
        out += noise * rng.standard_normal(out.shape, dtype=np.float32)
    return out.astype(np.float32)


@dataclass
class SceneSpec:
    H: int
    W: int
    N: int
    means2D: np.ndarray          # (N,2) f32 pixels
    radii: np.ndarray            # (N,) f32 pixels (half extent)
    rotations: np.ndarray        # (N,) f32 radians
    opacities: np.ndarray        # (N,) f32 logits
    colors: np.ndarray           # (N,3) f32 logits
    templates: np.ndarray        # (P,Ht,Wt) f32 in [0,1]
    sel: np.ndarray              # (N,) int32 template id per primitive
    target: np.ndarray           # (H,W,3) f32
    background: np.ndarray       # (H,W,3) f32 (white)
    alpha_max: float = 1.0
    meta: dict = field(default_factory=dict)


def sample_params(rng: np.random.Generator, H: int, W: int, N: int, P: int,
                  sel_mode: str = "uniform"):
    """Config parameter distributions: centre U(canvas), radius log-U[0.05,0.3]
    x canvas, rotation U[0,2pi), RGB U[0,1] (as clipped logits), opacity
    sigmoid(N(0,1)) (as logits), depth U[0,1] realised by index order."""
    canvas = float(min(H, W))
    cx = rng.uniform(0, W, N)
    cy = rng.uniform(0, H, N)
    s = np.exp(rng.uniform(np.log(0.05), np.log(0.3), N))
    r = s * canvas
    th = rng.uniform(0, 2 * np.pi, N)
    rgb = rng.uniform(0, 1, (N, 3))
    logits_c = np.clip(np.log(np.maximum(rgb, 1e-9)) - np.log(np.maximum(1 - rgb, 1e-9)), -20, 20)
    v = rng.normal(0.0, 1.0, N)
    depth = rng.uniform(0, 1, N)
    if sel_mode == "uniform":
        sel = rng.integers(0, P, N)
    else:  # the renderer API's (N-1-i) % P
        sel = (N - 1 - np.arange(N)) % P
    order = np.argsort(depth, kind="stable")
    means2D = np.stack([cx, cy], 1)[order]
    return (means2D.astype(np.float32), r[order].astype(np.float32), th[order].astype(np.float32),
            v[order].astype(np.float32), logits_c[order].astype(np.float32),
            sel[order].astype(np.int32) if sel_mode == "uniform" else sel.astype(np.int32))


def make_scene(config: str, seed: int = 0, **over) -> SceneSpec:
    """Builds the seeded scene of one reference workload ("c0".."c3mem")."""
    rng = np.random.default_rng(seed)
    if config == "c0":
        H = W = 256; N = 512; templates = soft_disk(64, 24.0)[None]; noise = 0.0
    elif config == "c1":
        H = W = 1024; N = 5000; templates = np.stack([random_shape(rng, 128) for _ in range(8)]); noise = 0.02
    elif config == "c2":
        H = W = 2048; N = 20000; templates = np.stack([random_shape(rng, 256) for _ in range(16)]); noise = 0.02
    elif config == "c3":
        H = W = 64; N = 32; templates = soft_disk(32, 12.0)[None]; noise = 0.0
    elif config == "c3mem":
        H = W = 4096; N = 100000; templates = soft_disk(64, 24.0)[None]; noise = 0.0
    else:
        raise ValueError(f"unknown config {config!r}")
    H = over.get("H", H); W = over.get("W", W); N = over.get("N", N)
    if "templates" in over:
        templates = over["templates"]
    P = templates.shape[0]
    means2D, r, th, v, c, sel = sample_params(rng, H, W, N, P, over.get("sel_mode", "uniform"))
    target = smooth_field(rng, H, W, noise=noise)
    bg = np.ones((H, W, 3), np.float32)
    return SceneSpec(H, W, N, means2D, r, th, v, c, templates.astype(np.float32), sel, target, bg,
                     alpha_max=over.get("alpha_max", 1.0), meta=dict(config=config, seed=seed))


def smooth_field_device(rng: np.random.Generator, H: int, W: int, device, n: int = 8, noise: float = 0.0):
    """smooth_field built on a torch device (same construction, float32)."""
    import torch
    xs = torch.arange(W, dtype=torch.float32, device=device)
    ys = torch.arange(H, dtype=torch.float32, device=device)
    chans = []
    for _ in range(3):
        p = rng.uniform(size=(n, 4))
        fx, fy = -4 + 8 * p[:, 0], -4 + 8 * p[:, 1]
        ph, a = 2 * np.pi * p[:, 2], 0.5 + 0.5 * p[:, 3]
        t = lambda z: torch.tensor(z, dtype=torch.float32, device=device)
        u = 2 * np.pi * t(fx)[:, None] * xs[None] / W + t(ph)[:, None]          # (n, W)
        v = 2 * np.pi * t(fy)[:, None] * ys[None] / H                           # (n, H)
        A = torch.cat([t(a)[:, None] * torch.cos(v), t(a)[:, None] * torch.sin(v)], 0).T   # (H, 2n)
        B = torch.cat([torch.sin(u), torch.cos(u)], 0)                          # (2n, W)
        f = A @ B
        f = f - f.min()
        chans.append(f / f.max().clamp_min(1e-12))
    out = torch.stack(chans, -1)
    if noise > 0:
        g = torch.Generator(device=device).manual_seed(int(rng.integers(0, 2**62)))
        out += noise * torch.randn(out.shape, generator=g, device=device)
    return out.contiguous()


_WHITE = {}


def white_background(H: int, W: int, device):
    """A white (H,W,3) background on `device`, one read-only tensor per size
    shared by every job of that size."""
    import torch
    key = (H, W, str(device))
    if key not in _WHITE:
        _WHITE[key] = torch.ones((H, W, 3), dtype=torch.float32, device=device)
    return _WHITE[key]


def make_job(rng: np.random.Generator, atlas: np.ndarray, sizes=(256, 512, 1024, 2048),
             n_range=(256, 20000), device=None) -> SceneSpec:
    """One serving job: W and H drawn independently from `sizes`, N log-uniform
    in n_range, primitives drawn from the shared atlas.  With `device` the
    target and background are built there as torch tensors."""
    H = int(rng.choice(sizes)); W = int(rng.choice(sizes))
    N = int(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]))))
    P = atlas.shape[0]
    means2D, r, th, v, c, sel = sample_params(rng, H, W, N, P, "uniform")
    if device is not None:
        target = smooth_field_device(rng, H, W, device, noise=0.02)
        bg = white_background(H, W, device)
    else:
        target = smooth_field(rng, H, W, noise=0.02)
        bg = np.ones((H, W, 3), np.float32)
    return SceneSpec(H, W, N, means2D, r, th, v, c, atlas, sel, target, bg,
                     meta=dict(config="c4"))
