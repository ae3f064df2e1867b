"""MEASUREMENT INFRASTRUCTURE -- times the reference's own PyTorch renderer on
the host CPU (SimpleTileRenderer._process_tiles_parallel with CUDA off,
pydiffbmp/core/renderer/simple_tile_renderer.py:479-569, c_blend = -40 so the
colour is the pure sigmoid as in the CUDA kernels), forward + backward of
sum(image * wc) + sum(alpha * wa), on a seeded scene of the given workload.
It needs the reference checkout (its Python imports), so it runs where that
checkout is, not on a GPU box:

    python oracle/time_reference_cpu.py --reference /path/to/diffbmp --configs c0 --reps 3

Prints one JSON line per config: median seconds per forward + backward, the
thread count used, and the tile-mapping time (the reference's Python binning)
separately.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("DIFFBMP_REFERENCE"),
                    help="root of the reference checkout (or set DIFFBMP_REFERENCE)")
    ap.add_argument("--configs", default="c0")
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    import make_golden as MG
    str_ = MG.load_reference(a.reference)
    import torch
    from diffbmp_b200 import workloads as wl
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    for cfg in a.configs.split(","):
        s = wl.make_scene(cfg, seed=0)
        R = MG.make_renderer(str_, s.H, s.W, s.templates, 32, 1.0)
        P = s.templates.shape[0]
        rng = np.random.default_rng(1)
        wc = torch.from_numpy(rng.normal(0, 1, (s.H, s.W, 3)).astype(np.float32))
        wa = torch.from_numpy(rng.normal(0, 1, (s.H, s.W)).astype(np.float32))
        times, bin_times = [], []
        for _ in range(a.reps):
            x = torch.tensor(s.means2D[:, 0], requires_grad=True)
            y = torch.tensor(s.means2D[:, 1], requires_grad=True)
            rr = torch.tensor(s.radii, requires_grad=True)
            tt = torch.tensor(s.rotations, requires_grad=True)
            vv = torch.tensor(s.opacities, requires_grad=True)
            cc = torch.tensor(s.colors, requires_grad=True)
            gsel = torch.from_numpy(s.sel.astype(np.int64))
            out = torch.zeros(s.H, s.W, 3)
            t0 = time.perf_counter()
            img, alpha = R._process_tiles_parallel(x, y, rr, tt, vv, cc, 0.0, None, gsel, out, None,
                                                   return_alpha=True)
            ((img * wc).sum() + (alpha * wa).sum()).backward()
            times.append(time.perf_counter() - t0)
            xs, xe, ys, ye = MG.tile_bounds(s.H, s.W, 32)
            t0 = time.perf_counter()
            masks = R._unified_primitive_assignment(x.detach(), y.detach(), rr.detach(), tt.detach(),
                                                    xs, xe, ys, ye)
            R._convert_masks_to_mapping(masks, xs, xe, ys, ye)
            bin_times.append(time.perf_counter() - t0)
        print(json.dumps({"config": cfg, "canvas": [s.H, s.W], "N": s.N, "threads": threads,
                          "fwd_bwd_s_median": float(np.median(times)), "fwd_bwd_s_all": times,
                          "binning_s_median": float(np.median(bin_times)), "P": P}), flush=True)


if __name__ == "__main__":
    main()
