"""Shared test helpers: seeded scenes and oracle comparisons."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O
from diffbmp_b200 import workloads as wl

GOLDEN = __import__("os").path.join(__import__("os").path.dirname(__file__), "golden")


def golden(name):
    return np.load(f"{GOLDEN}/{name}.npz")


def split_mapping(mp):
    T1 = int(mp[0])
    return mp[2:2 + T1], mp[2 + T1:]


def small_scene(seed=0, H=96, W=80, N=40, P=2, size=32, ts=32, rmin=4.0, rmax=30.0, amax=1.0,
                nonsquare=False):
    rng = np.random.default_rng(seed)
    if nonsquare:
        S = np.stack([wl.random_shape(rng, size)[: size * 3 // 4] for _ in range(P)])
    else:
        S = np.stack([wl.random_shape(rng, size) for _ in range(P)])
    cx = rng.uniform(0, W, N); cy = rng.uniform(0, H, N)
    r = np.exp(rng.uniform(np.log(rmin), np.log(rmax), N))
    th = rng.uniform(0, 2 * np.pi, N)
    v = rng.normal(0, 1, N); c = rng.normal(0, 1.5, (N, 3))
    sel = rng.integers(0, P, N)
    f = lambda a: np.asarray(a, np.float32)   # the kernels take float32 inputs
    return O.Scene(H, W, ts, f(np.stack([cx, cy], 1)), f(r), f(th), f(v), f(c), f(S), sel, amax)


def bin_scene(sc: O.Scene, mode=O.BIN_CONTENT):
    tb = O.template_bboxes(sc.templates)
    P, Ht, Wt = sc.templates.shape
    return O.bin_tiles(sc.H, sc.W, sc.ts, sc.means2D, sc.radii, sc.rot, sc.sel, tb, Ht, Wt, mode)


def rel_err(a, b, floor=1e-12):
    return float(np.linalg.norm(np.asarray(a, np.float64) - np.asarray(b, np.float64)) /
                 max(np.linalg.norm(np.asarray(b, np.float64)), floor))
