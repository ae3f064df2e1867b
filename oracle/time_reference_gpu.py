"""MEASUREMENT INFRASTRUCTURE -- times the reference's own CUDA kernels (built
from the reference sources into oracle/_ref/ by `make -C oracle ref`) beside
this repository's kernels on the same scenes and the same GPU.

    python oracle/time_reference_gpu.py [--configs c0,c1] [--reps 20] [--psd 1024:5000]

Per config it prints one JSON line with:
* ref_fwd_bwd_ms: one reference forward + backward as the reference runs it
  (tile_rasterize.cu:297-498,638-780): cache and output memsets, the forward
  kernel, the backward kernel, a device synchronisation after each;
  K (cache slots per pixel) is set to the deepest pixel + 16 so the caches
  never overflow, and the caches are 5*H*W*K floats;
* ours_plain_fwd_bwd_ms: this repository's FP32 forward + backward on the
  same tile lists (reference-layout atlas, no early-termination change);
* ref_fp16_fwd_bwd_ms: the same for the reference's all-half extension
  (_C_fp16), with K = the longest tile list (its half-precision fragment
  test can exceed the FP32 depth; a pixel never takes more slots than its
  tile has entries);
* ours_fused_f16q_ms: one full fit iteration here (device binning, fused
  forward + L2 + backward, Adam) with the FP16 quad atlas, graph replayed.
A config whose caches would exceed 120 GB, or whose cache index H*W*K would
not fit a 32-bit int, is reported as skipped with the reason; the reference
kernel is not launched there.  The tile lists come from this repository's
binning, which is bit-identical to the reference's.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import sys
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from oracle import reference_gpu as RG  # noqa: E402

P_ = lambda t: ctypes.c_void_p(t.data_ptr()) if t is not None else None


def dev(a, dt=np.float32):
    return torch.from_numpy(np.ascontiguousarray(a, dt)).cuda()


def deepest_pixel(rz, atlas, state, N):
    from diffbmp_b200._lib import call
    from diffbmp_b200.rasterizer import _ptr, _stream
    cv = rz.canvas(N, atlas)
    cv.t_stop = 0.0
    cnt = torch.zeros(10, dtype=torch.int64, device="cuda")
    call("dbmp_count", ctypes.byref(cv), _ptr(state.prim_info), _ptr(atlas.data), _ptr(state.lists.offsets),
         _ptr(state.lists.indices), _ptr(cnt), _stream())
    return int(cnt[6].item())


def time_config(cfg, reps):
    from diffbmp_b200 import workloads as wl
    from diffbmp_b200.fitting import FitConfig, ImageFitter
    from diffbmp_b200.rasterizer import Atlas, Rasterizer
    s = wl.make_scene(cfg, seed=0)
    H, W, N = s.H, s.W, s.N
    P, Ht, Wt = s.templates.shape
    d = dict(m=dev(s.means2D), r=dev(s.radii), th=dev(s.rotations), v=dev(s.opacities), c=dev(s.colors),
             t=dev(s.templates), s=dev(s.sel, np.int32))
    atlas = Atlas(d["t"])
    rz = Rasterizer(H, W, 32)
    color, alpha, state = rz.forward(d["m"], d["r"], d["th"], d["v"], d["c"], d["s"], atlas)
    torch.cuda.synchronize()
    K = deepest_pixel(rz, atlas, state, N) + 16
    out = {"config": cfg, "canvas": [H, W], "N": N, "tile_list_entries": state.lists.length,
           "deepest_pixel": K - 16, "K": K}
    gc = torch.randn((H, W, 3), device="cuda") * 1e-3
    ga = torch.zeros((H, W), device="cuda")

    # ours: plain FP32 forward + backward on the same lists
    def ours():
        _, _, st = rz.forward(d["m"], d["r"], d["th"], d["v"], d["c"], d["s"], atlas,
                              mapping=state.lists.mapping_tensor())
        rz.backward(st, gc, ga, d["r"], d["th"], d["v"], d["c"], atlas)
    for _ in range(3):
        ours()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        ours()
    torch.cuda.synchronize()
    out["ours_plain_fwd_bwd_ms"] = (time.perf_counter() - t0) / reps * 1e3

    # ours: a fused FP16-quad fit iteration (binning included), graph replayed
    a16 = Atlas(d["t"], "f16q")
    job = ImageFitter(s.means2D, s.radii, s.rotations, s.opacities, s.colors, s.sel, a16, s.target, s.background,
                      FitConfig(fused=True))
    job.capture()
    for _ in range(5):
        job.step()
    job.sync(); torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        job.step()
    torch.cuda.synchronize()
    out["ours_fused_f16q_ms"] = (time.perf_counter() - t0) / reps * 1e3

    cache_bytes = 5 * H * W * K * 4
    if H * W * K >= 2 ** 31:
        out["ref_fwd_bwd_ms"] = None
        out["ref_skipped"] = f"cache index H*W*K = {H * W * K} does not fit a 32-bit int"
        return out
    if cache_bytes > 120e9:
        out["ref_fwd_bwd_ms"] = None
        out["ref_skipped"] = f"caches of {cache_bytes / 1e9:.0f} GB"
        return out
    del color, alpha
    caches = torch.zeros(5 * H * W * K + 8 * K, dtype=torch.float32, device="cuda")
    counts = torch.zeros(H * W, dtype=torch.int32, device="cuda")
    sig = torch.zeros(8 * N + 8, dtype=torch.float32, device="cuda")
    offs = state.lists.offsets
    idx = state.lists.indices
    L = state.lists.length
    rcol = torch.zeros((H, W, 3), device="cuda")
    ralp = torch.zeros((H, W), device="cuda")
    rg = [torch.zeros(sh, device="cuda") for sh in ((N, 2), (N,), (N,), (N,), (N, 3))]
    Lr = RG.raster()

    def ref():
        rc = Lr.ref_forward(H, W, 32, ctypes.c_float(1.0), N, P, Ht, Wt, K, P_(d["m"]), P_(d["r"]), P_(d["th"]),
                            P_(d["v"]), P_(d["c"]), P_(d["t"]), P_(d["s"]), P_(offs), offs.numel(), P_(idx), L,
                            P_(rcol), P_(ralp), P_(caches), P_(counts), P_(sig))
        assert rc == 0
        rc = Lr.ref_backward(H, W, 32, ctypes.c_float(1.0), N, P, Ht, Wt, K, P_(d["m"]), P_(d["r"]), P_(d["th"]),
                             P_(d["v"]), P_(d["c"]), P_(d["t"]), P_(d["s"]), P_(offs), offs.numel(), P_(idx), L,
                             P_(gc), P_(ga), P_(caches), P_(counts), P_(sig), *[P_(t) for t in rg])
        assert rc == 0
    for _ in range(2):
        ref()
    t0 = time.perf_counter()
    n = max(3, reps // 4)
    for _ in range(n):
        ref()
    out["ref_fwd_bwd_ms"] = (time.perf_counter() - t0) / n * 1e3
    out["ref_cache_gb"] = cache_bytes / 1e9
    out["speedup_fused_f16q_vs_ref"] = out["ref_fwd_bwd_ms"] / out["ours_fused_f16q_ms"]
    out["speedup_plain_vs_ref"] = out["ref_fwd_bwd_ms"] / out["ours_plain_fwd_bwd_ms"]
    del caches
    torch.cuda.empty_cache()

    # the reference's all-half extension (_C_fp16): its fragment test runs in
    # half precision, so its per-pixel depth can differ from the FP32 count;
    # K = the longest tile list bounds it (one slot per list entry at most)
    Lr16 = RG.raster_fp16()
    if Lr16 is None:
        out["ref_fp16_skipped"] = "reference FP16 kernels not built"
        return out
    K16 = int((offs[1:] - offs[:-1]).max().item())
    out["K_fp16"] = K16
    if H * W * K16 >= 2 ** 31 or 5 * H * W * K16 * 2 > 120e9:
        out["ref_fp16_skipped"] = f"K = longest tile list = {K16}: cache index or size out of range"
        return out
    h = lambda t: t.half().contiguous()
    d16 = {k: h(v) for k, v in d.items() if k != "s"}
    caches16 = torch.zeros(5 * H * W * K16 + 8 * K16, dtype=torch.float16, device="cuda")
    sig16 = torch.zeros(8 * N + 8, dtype=torch.float16, device="cuda")
    rcol16 = torch.zeros((H, W, 3), dtype=torch.float16, device="cuda")
    ralp16 = torch.zeros((H, W), dtype=torch.float16, device="cuda")
    gc16, ga16 = h(gc), h(ga)
    rg16 = [torch.zeros(sh, dtype=torch.float16, device="cuda") for sh in ((N, 2), (N,), (N,), (N,), (N, 3))]

    def ref16():
        rc = Lr16.ref_forward_fp16(H, W, 32, ctypes.c_float(1.0), N, P, Ht, Wt, K16, P_(d16["m"]), P_(d16["r"]),
                                   P_(d16["th"]), P_(d16["v"]), P_(d16["c"]), P_(d16["t"]), P_(d["s"]), P_(offs),
                                   offs.numel(), P_(idx), L, P_(rcol16), P_(ralp16), P_(caches16), P_(counts),
                                   P_(sig16))
        assert rc == 0
        rc = Lr16.ref_backward_fp16(H, W, 32, ctypes.c_float(1.0), N, P, Ht, Wt, K16, P_(d16["m"]), P_(d16["r"]),
                                    P_(d16["th"]), P_(d16["v"]), P_(d16["c"]), P_(d16["t"]), P_(d["s"]), P_(offs),
                                    offs.numel(), P_(idx), L, P_(gc16), P_(ga16), P_(caches16), P_(counts),
                                    P_(sig16), *[P_(t) for t in rg16])
        assert rc == 0
    for _ in range(2):
        ref16()
    t0 = time.perf_counter()
    for _ in range(n):
        ref16()
    out["ref_fp16_fwd_bwd_ms"] = (time.perf_counter() - t0) / n * 1e3
    out["speedup_fused_f16q_vs_ref_fp16"] = out["ref_fp16_fwd_bwd_ms"] / out["ours_fused_f16q_ms"]
    return out


def time_psd(W, N, reps):
    """The PSD crop kernels on the export case of a W x W canvas with N
    primitives (8 templates of 128^2, centres uniform, radii s W / 2 with s
    log-uniform in [0.05, 0.3]): the reference's generate_cropped_layers
    launch (psd_export_kernels.cu:219-270, one thread per primitive for every
    16x16 tile of the canvas) and this repository's dbmp_psd_layers on the
    same boxes and offsets, each timed with CUDA events over `reps` launches."""
    from diffbmp_b200 import workloads as wl
    from diffbmp_b200.psd import export_layers
    from diffbmp_b200._lib import call
    from diffbmp_b200.rasterizer import _ptr, _stream
    rng = np.random.default_rng(0)
    P, S = 8, 128
    tm = dev(np.stack([wl.random_shape(rng, S) for _ in range(P)]))
    m = dev(np.stack([rng.uniform(0, W, N), rng.uniform(0, W, N)], 1))
    r = dev(np.exp(rng.uniform(np.log(0.05), np.log(0.3), N)) * W / 2)
    th = dev(rng.uniform(0, 2 * np.pi, N))
    v = dev(1 / (1 + np.exp(-rng.normal(0, 1, N))))
    c = dev(1 / (1 + np.exp(-rng.normal(0, 2, (N, 3)))))
    sel = dev((N - 1 - np.arange(N)) % P, np.int32)
    buf, bbox, sizes, offs = export_layers(tm, m, r, th, v, c, sel, W, W, 1.0, 0.9, 0.0, None)
    hs = sizes.cpu().numpy()
    total = int((hs[:, 0].astype(np.int64) * hs[:, 1] * 4).sum())
    out = {"psd_case": f"{W}x{W}, N={N}", "crop_bytes": total}
    if total >= 2 ** 31:
        out["ref_skipped"] = "the reference's layer offsets are 32-bit and the crops exceed 2^31 bytes"
        return out
    ro = dev(np.concatenate([[0], np.cumsum(hs[:, 0].astype(np.int64) * hs[:, 1] * 4)[:-1]]), np.int32)
    rbuf = torch.zeros(total, dtype=torch.uint8, device="cuda")
    L = RG.psd()
    blk = torch.zeros(N + 1, dtype=torch.int64, device="cuda")
    lo = torch.zeros(N, dtype=torch.int64, device="cuda")
    tb = torch.zeros(1, dtype=torch.int64, device="cuda")
    call("dbmp_psd_layout", _ptr(sizes), N, _ptr(lo), _ptr(blk), _ptr(tb), _stream())

    def ref():
        L.launch_generate_cropped_layers(P_(m), P_(r), P_(th), P_(c), P_(v), P_(tm), P_(sel), P_(bbox), P_(ro),
                                         P_(rbuf), N, W, W, S, S, ctypes.c_float(1.0), ctypes.c_float(0.9),
                                         ctypes.c_float(0.0), None, W, W)

    def ours():
        call("dbmp_psd_layers", _ptr(m), _ptr(r), _ptr(th), _ptr(c), _ptr(v), _ptr(tm), P, S, S, _ptr(sel),
             _ptr(bbox), _ptr(lo), _ptr(blk), N, ctypes.c_float(1.0), ctypes.c_float(0.9), ctypes.c_float(0.0), None,
             _ptr(buf), _stream())

    for name, fn in (("ref_psd_layers_ms", ref), ("ours_psd_layers_ms", ours)):
        fn(); torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record(); e1.synchronize()
        out[name] = e0.elapsed_time(e1) / reps
    out["bytes_equal"] = bool(torch.equal(rbuf, buf))
    out["speedup"] = out["ref_psd_layers_ms"] / out["ours_psd_layers_ms"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--configs", default="c0,c1")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--psd", default="", help="PSD crop cases W:N,... (e.g. 1024:5000,2048:20000)")
    a = ap.parse_args()
    if not RG.available():
        print(json.dumps({"unavailable": "reference kernels not built (make -C oracle ref)"}))
        return
    for cfg in [c for c in a.configs.split(",") if c]:
        print(json.dumps(time_config(cfg, a.reps)), flush=True)
        torch.cuda.empty_cache()
    for case in [c for c in a.psd.split(",") if c]:
        W, N = (int(x) for x in case.split(":"))
        print(json.dumps(time_psd(W, N, a.reps)), flush=True)
        torch.cuda.empty_cache()


if __name__ == "__main__":
    main()
