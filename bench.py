"""Benchmark of the DiffBMP B200 tile rasterizer.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config c2|c1|c0] [--fast]

Workload (default): the precision-form configuration -- 2048x2048 canvas,
N=20000 primitives drawn from a 16-bitmap 256x256 atlas, one image-fitting
iteration per step (device binning + forward + L2 loss + backward + Adam).
``value`` is iterations/s of the FP16-storage fused step (half-precision
bilinear-quad atlas), replayed from a CUDA graph with every input resident in
HBM; the plain FP32 kernels (unfused forward / backward, FP32 atlas in the
reference layout) and the FP16 pair-layout atlas are timed beside it on the
same scene.  ``e2e`` is the same iteration through the public Python API with the
primitive parameters uploaded from pinned host memory before each step and
each step's loss read back by the host (one step in flight: the host reads
step k-1's loss while step k runs).  Multi-GPU (torchrun): every rank fits its own
independent job (replicas, no collective on the data path); value sums the
ranks' iterations over the slowest rank's time.

``--impl reference`` times the reference's CPU path -- its PyTorch per-tile
renderer, restated in oracle/torch_renderer.py and pinned to its own outputs
-- on all host cores, fwd+bwd on a bounded sample of the canvas's tiles per
step, extrapolated by tile count; the FP64 restatement of the reference's
kernel algorithm is reported beside it.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

# the serving loop runs one stream per active job group: give them hardware queues
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd iters/s at 2048^2 N=20k (FP16-storage fused vs plain FP32)"
HEADLINE_KIND = "f16q"          # FP16 bilinear-quad atlas
HEADLINE_KERNEL = "fused_kernel<32, F16_QUAD>"
# DRAM bytes of one fused_kernel launch (FP16 quad atlas) on the 2048^2 / N=20k
# scene, from one ncu capture (read 108.3 MB + write 3.8 MB); null for other configs.
FUSED_DRAM_BYTES_C2 = 112.057e6


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=["c0", "c1", "c2"])
    ap.add_argument("--fast", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--dist-backend", default="nccl", choices=["nccl", "gloo"],
                    help="process-group backend under torchrun (gloo: the CPU-only reference arm)")
    ap.add_argument("--serving-jobs", type=int, default=2000,
                    help="jobs of the serving stream measured beside the headline (0: skip)")
    ap.add_argument("--no-psd", action="store_true", help="skip the PSD export section")
    ap.add_argument("--profile", default=None,
                    choices=["f16", "f32", "bf16", "f32q", "f16q", "bf16q", "plain", "psd"],
                    help="profiling mode: one job of this form, --warmup + --steps eager steps, no timing line "
                         "(psd: one PSD export of the 1024^2 / N=5000 case: crop kernel, count and write passes)")
    return ap.parse_args()


def dist_setup(args, backend="nccl"):
    """One process per GPU (torchrun env).  backend "gloo" runs the same
    barrier / max-over-ranks plumbing without GPUs (used by the CPU tests)."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    elif backend == "nccl" and torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """SM clocks and throttle reasons of the GPU, sampled during the timed
    region by a host thread polling NVML about every millisecond (a timed
    region of 20 steps lasts ~15 ms; nvidia-smi's 100 ms period would miss it),
    with nvidia-smi as the fallback where NVML is unavailable."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0, period_s=0.001):
        self.index, self.period = index, period_s
        self.samples = []          # (sm_mhz, max_mhz, reason bitmask)
        self.source = None
        self._stop = threading.Event()
        self._thread = self._proc = None

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        try:   # the CUDA device's own UUID (CUDA_VISIBLE_DEVICES may renumber devices)
            import torch
            uuid = str(torch.cuda.get_device_properties(self.index).uuid)
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
            phys = int(vis[self.index]) if self.index < len(vis) and vis[self.index].strip().isdigit() else self.index
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(phys)

    def _poll(self, nv, h):
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self._stop.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), mx,
                                     nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
            except Exception:
                break
            time.sleep(self.period)

    def _read_smi(self):
        for line in self._proc.stdout:
            f = [x.strip() for x in line.split(",")]
            try:
                mask = sum(bit for (name, bit), v in zip(self.REASONS.items(), f[5:9]) if v.lower() == "active")
                self.samples.append((float(f[1]), float(f[2]), mask))
            except (ValueError, IndexError):
                continue

    def __enter__(self):
        try:
            nv, h = self._nvml_handle()
            self.source = "nvml, ~1 ms"
            self._thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
        except Exception:
            vis = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")
            idx = vis[self.index].strip() if self.index < len(vis) and vis[self.index].strip().isdigit() \
                else str(self.index)
            try:
                self._proc = subprocess.Popen(["nvidia-smi", f"--id={idx}", f"--query-gpu={self.QUERY}",
                                               "--format=csv,noheader,nounits", "-lms", "100"],
                                              stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self.source = "nvidia-smi, 100 ms"
                self._thread = threading.Thread(target=self._read_smi, daemon=True)
            except Exception:
                self._thread = None
        if self._thread is not None:
            self._thread.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        if self._thread is not None:
            self._thread.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        mhz = [s[0] for s in self.samples]
        mask = 0
        for s in self.samples:
            mask |= int(s[2])
        return {"sm_mhz": float(np.median(mhz)), "sm_max_mhz": float(self.samples[-1][1]),
                "reasons": sorted(n for n, bit in self.REASONS.items() if mask & bit),
                "samples": len(self.samples), "source": self.source}


def fp32_simt_peak_tflops(torch):
    """Measured FP32 (non-tensor) peak: cuBLAS SGEMM 8192^3 with TF32 disabled."""
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn(n, n, device="cuda")
        b = torch.randn(n, n, device="cuda")
        for _ in range(2):
            a @ b
        torch.cuda.synchronize()
        best = 1e9
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(); a @ b; e1.record(); e1.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        return 2.0 * n ** 3 / best / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def build_job(spec, kind, fused, torch):
    from diffbmp_b200.fitting import FitConfig, ImageFitter
    from diffbmp_b200.rasterizer import Atlas
    atlas = Atlas(torch.from_numpy(spec.templates).cuda(), kind)
    cfg = FitConfig(lr=0.01, fused=fused)
    return ImageFitter(spec.means2D, spec.radii, spec.rotations, spec.opacities, spec.colors, spec.sel, atlas,
                       spec.target, spec.background, cfg)


def time_steps(job, steps, warmup, torch, world, graph=True):
    for _ in range(warmup):
        job.step()
    job.sync()
    if graph:
        job.capture()
        job.step(); job.sync()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        job.step()
    e1.record(st)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(world)
    replayed = job.sync()
    return e0.elapsed_time(e1) / 1e3, replayed


def kernel_time(job, fn, reps, torch):
    """Average duration of one launch of `fn` on the current stream (CUDA events)."""
    st = torch.cuda.current_stream()
    fn(); torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def counts(job, torch):
    import ctypes
    from diffbmp_b200._lib import call
    from diffbmp_b200.rasterizer import _ptr, _stream
    c = torch.zeros(10, dtype=torch.int64, device="cuda")
    call("dbmp_count", ctypes.byref(job.cv), _ptr(job.prim_info), _ptr(job.atlas.data), _ptr(job.offsets),
         _ptr(job.rz._idx), _ptr(c), _stream())
    return [int(v) for v in c.tolist()]


class CpuReference:
    """The reference algorithm on the host cores through the oracle port
    (FP64, all host threads, no early termination).  Bins the scene once;
    sample(px_rows) times forward + backward over the first px_rows pixel rows
    and returns the time extrapolated to the whole canvas."""

    def __init__(self, spec, ts=32):
        from oracle import oracle as O
        self.O, self.spec, self.ts = O, spec, ts
        self.sc = O.Scene(spec.H, spec.W, ts, spec.means2D, spec.radii, spec.rotations, spec.opacities,
                          spec.colors, spec.templates, spec.sel, spec.alpha_max)
        tb = O.template_bboxes(spec.templates)
        P, Ht, Wt = spec.templates.shape
        self.offs, self.idx = O.bin_tiles(spec.H, spec.W, ts, spec.means2D, spec.radii, spec.rotations, spec.sel,
                                          tb, Ht, Wt)
        self.tiles_x = (spec.W + ts - 1) // ts

    def sample(self, px_rows, nthreads=0):
        O, sc, spec, ts = self.O, self.sc, self.spec, self.ts
        Hs = max(1, min(spec.H, int(px_rows)))
        sub = O.Scene(Hs, spec.W, ts, sc.means2D, sc.radii, sc.rot, sc.opac, sc.colors, sc.templates, sc.sel,
                      sc.alpha_max)
        so = self.offs[: ((Hs + ts - 1) // ts) * self.tiles_x + 1]
        si = self.idx[: so[-1]]
        gc = np.ones((Hs, spec.W, 3), np.float32) * 1e-3
        t0 = time.perf_counter()
        O.forward(sub, so, si, nthreads=nthreads)
        O.backward(sub, so, si, gc, None, nthreads=nthreads)
        return (time.perf_counter() - t0) * spec.H / Hs

    def rows_for_budget(self, seconds_per_sample):
        """Pixel rows per sample so that one sample takes about the given time;
        at least one row per host thread (the oracle runs rows in parallel)."""
        base = int(min(self.spec.H, max(1, os.cpu_count() or 1)))
        per_row = self.sample(base) / self.spec.H   # whole-canvas time from a `base`-row sample
        return int(min(self.spec.H, max(base, seconds_per_sample / max(per_row, 1e-9))))


PRECISION_KINDS = ("f32", "f16q", "f16", "bf16q", "bf16")


def precision_band(spec, ts=32):
    """Pixel rows [y0, y1) of the precision comparison: 8 tile rows at the
    middle of the canvas (the whole canvas when it has at most 8 tile rows)."""
    rows = 8 * ts
    if spec.H <= rows:
        return 0, spec.H
    y0 = (spec.H // 2 - rows // 2) // ts * ts
    return y0, y0 + rows


def render_band(spec, kind, band, torch):
    """Forward render of the scene (its initial parameters) with atlas storage
    `kind`; returns the band's (color, alpha) on the host."""
    from diffbmp_b200.rasterizer import Atlas, Rasterizer
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    atlas = Atlas(t(spec.templates), kind)
    rz = Rasterizer(spec.H, spec.W, 32)      # the fit step's t_stop
    color, alpha, _ = rz.forward(t(spec.means2D), t(spec.radii), t(spec.rotations), t(spec.opacities),
                                 t(spec.colors), t(spec.sel), atlas)
    y0, y1 = band
    out = color[y0:y1].cpu().numpy(), alpha[y0:y1].cpu().numpy()
    del color, alpha, atlas, rz
    return out


def precision_vs_oracle(spec, band, renders, ts=32):
    """PSNR and max-abs error of each storage kind's image (rendered over the
    scene's background) against the FP64 oracle's render of the same band of
    rows (the reference kernels' semantics, every fragment, no termination)."""
    from oracle import oracle as O
    y0, y1 = band
    tb = O.template_bboxes(spec.templates)
    P, Ht, Wt = spec.templates.shape
    offs, idx = O.bin_tiles(spec.H, spec.W, ts, spec.means2D, spec.radii, spec.rotations, spec.sel, tb, Ht, Wt)
    tx = (spec.W + ts - 1) // ts
    t0, t1 = (y0 // ts) * tx, ((y1 + ts - 1) // ts) * tx
    so = (offs[t0:t1 + 1] - offs[t0]).astype(np.int32)
    si = idx[offs[t0]:offs[t1]]
    m = spec.means2D.astype(np.float64).copy()
    m[:, 1] -= y0                  # exact in float64: the band's pixel offsets are unchanged
    sc = O.Scene(y1 - y0, spec.W, ts, m, spec.radii, spec.rotations, spec.opacities, spec.colors, spec.templates,
                 spec.sel, spec.alpha_max)
    t_start = time.perf_counter()
    ref = O.forward(sc, so, si)
    t_oracle = time.perf_counter() - t_start
    bg = spec.background[y0:y1].astype(np.float64)
    ref_img = ref["color"] + (1.0 - ref["alpha"])[..., None] * bg
    out = {"band": f"pixel rows {y0}-{y1 - 1} of {spec.H} ({(y1 - y0) // ts} tile rows), full width",
           "checker": "FP64 oracle render (reference kernel semantics, every fragment, no termination)",
           "image": "rendered = C + (1 - A) * background, PSNR with peak 1.0",
           "oracle_s": t_oracle}
    for kind, (color, alpha) in renders.items():
        img = color.astype(np.float64) + (1.0 - alpha.astype(np.float64))[..., None] * bg
        err = np.abs(img - ref_img)
        mse = float(np.mean(err ** 2))
        out[kind] = {"psnr_db": 10 * np.log10(1.0 / max(mse, 1e-30)), "max_abs": float(err.max()),
                     "alpha_max_abs": float(np.abs(alpha - ref["alpha"]).max())}
    return out


def run_serving(n_jobs, seed, torch, subsample=5, load=0.8):
    """Serving workload: a stream of fit-an-image jobs (canvas sides drawn from
    {256,512,1024,2048}, N log-uniform in [256,20000], the shared 16-bitmap
    atlas, 100 Adam iterations each) through the continuous-batching server
    with FP16 atlas storage and the fused step.

    * capacity: every job queued at the start; jobs/s is the service rate;
    * latency: Poisson arrivals at `load` x that measured rate (a stated,
      sub-saturating rate), so p50 / p99 measure service rather than backlog;
    * baselines: the same jobs (every `subsample`-th of the stream) solved one
      at a time, each set up as the server sets it up and replayed from a CUDA
      graph -- with the plain FP32 kernels (the denominator of the 3x target)
      and with the fused FP16 step (what continuous batching itself adds)."""
    from diffbmp_b200 import serving, workloads as wl
    rng = np.random.default_rng(100 + seed)
    atlas = np.stack([wl.random_shape(rng, 256) for _ in range(16)])
    reqs = serving.poisson_requests(n_jobs, 1.0, atlas, seed=seed, iterations=100, device="cuda")
    unit_arrivals = [r.arrival for r in reqs]       # a Poisson stream at rate 1, rescaled below
    torch.cuda.synchronize()
    t_atlas = torch.from_numpy(atlas).cuda()
    srv = serving.Server(t_atlas, kind=HEADLINE_KIND, fused=True, max_slots=48, hbm_budget=150e9)
    warm = serving.poisson_requests(2, 200.0, atlas, seed=seed + 999, iterations=5, sizes=(256,), device="cuda")
    srv.run(warm, realtime=False)
    cap = serving.summarize(srv.run(reqs, realtime=False))
    rate = load * cap["jobs_per_s"]
    for r, a in zip(reqs, unit_arrivals):
        r.arrival = a / rate
    res = srv.run(reqs, realtime=True)
    lat = serving.summarize(res)
    sub = reqs[::subsample]
    seq_plain, t_plain, _ = serving.run_sequential(sub, t_atlas, kind="f32", fused=False, graphs=True)
    seq_fused, t_fused, dev_fused = serving.run_sequential(sub, t_atlas, kind=HEADLINE_KIND, fused=True, graphs=True)
    device_rate = len(sub) / dev_fused          # the fused jobs' iterations alone
    plain_rate, fused_rate = len(sub) / t_plain, len(sub) / t_fused
    served = {r.job_id: r.loss for r in res}
    d_fused = max(abs(served[q.job_id] - f.loss) / max(abs(f.loss), 1e-30) for q, f in zip(sub, seq_fused))
    return {"jobs": cap["jobs"], "iterations_per_job": 100,
            "capacity_jobs_per_s": cap["jobs_per_s"],
            "arrival_rate_per_s": rate, "arrival_rate_note": f"Poisson at {load:.0%} of the measured capacity",
            "jobs_per_s": lat["jobs_per_s"], "p50_s": lat["p50_s"], "p99_s": lat["p99_s"],
            "mean_final_l2": lat["mean_loss"], "replayed_steps": cap["replayed"] + lat["replayed"],
            "sequential_plain_fp32_graphed_jobs_per_s": plain_rate,
            "sequential_fused_f16_graphed_jobs_per_s": fused_rate,
            "fused_f16_iterations_only_jobs_per_s": device_rate,
            "fused_f16_iterations_only_note": "the same jobs' 100 iterations each, one job at a time, device time "
                                              "(CUDA events) without set-up or host waits",
            "baseline_sample": f"every {subsample}th job of the stream ({len(sub)} jobs), one at a time",
            "capacity_vs_sequential_plain_fp32": cap["jobs_per_s"] / plain_rate,
            "capacity_vs_sequential_fused_f16": cap["jobs_per_s"] / fused_rate,
            "sequential_plain_mean_final_l2": float(np.mean([r.loss for r in seq_plain])),
            "served_mean_final_l2_same_jobs": float(np.mean([served[q.job_id] for q in sub])),
            "served_vs_sequential_fused_max_rel_l2_diff": d_fused,
            "what": "continuous batching: admission by slots (48) + 150 GB HBM budget, resident job state, per-job "
                    "CUDA graph (bin + fused fwd/bwd + Adam) on the least-loaded of 16 streams, up to 3 "
                    "iterations ahead of the host"}


def psd_case(torch, W, N, P_, S, seed=0):
    """Inputs of the PSD export case: W x W canvas, N primitives, P_ templates
    of S^2 texels, radii s*W/2 with s log-uniform in [0.05, 0.3]."""
    from diffbmp_b200 import workloads as wl
    rng = np.random.default_rng(seed)
    tm = torch.from_numpy(np.stack([wl.random_shape(rng, S) for _ in range(P_)])).cuda()
    t = lambda a: torch.from_numpy(np.asarray(a, np.float32)).cuda()
    m = t(np.stack([rng.uniform(0, W, N), rng.uniform(0, W, N)], 1))
    r = t(np.exp(rng.uniform(np.log(0.05), np.log(0.3), N)) * W / 2)
    th = t(rng.uniform(0, 2 * np.pi, N))
    vs = torch.sigmoid(t(rng.normal(0, 1, N)))
    cs = torch.sigmoid(t(rng.normal(0, 2, (N, 3))))
    sel = torch.from_numpy(((N - 1 - np.arange(N)) % P_).astype(np.int32)).cuda()
    return tm, m, r, th, vs, cs, sel


def psd_export_once(torch, W, N, P_, S):
    """One device export of the case: crops, then the layers' PackBits channel blocks."""
    import diffbmp_b200.psd as P
    tm, m, r, th, vs, cs, sel = psd_case(torch, W, N, P_, S)
    buf, bbox, sizes, offs = P.export_layers(tm, m, r, th, vs, cs, sel, W, W)
    blob, blocks, chosen = P.encode_channel_blocks(buf, sizes, offs, sizes.cpu().numpy(), P.ORDER_LAYER,
                                                   lambda flags: np.nonzero(flags)[0])
    torch.cuda.synchronize()
    return {"crop_bytes": int(buf.numel()), "encoded_bytes": int(blob.numel()), "layers": int(len(chosen))}


def run_psd(torch, peaks):
    """PSD layer export on the device at 1024^2 / N=5000 and 2048^2 / N=20000
    (templates of the scene configs, radii s*W/2 with s log-uniform in
    [0.05, 0.3], sigmoid-ed colours and opacities): CUDA-event time of each
    library call -- the crop kernel (dbmp_psd_layers) and the two PackBits
    passes of the file's channel data (dbmp_psd_rle_count / _write) -- with
    its algorithmic bytes and the fraction of the measured HBM copy peak."""
    import diffbmp_b200.psd as P
    hbm = peaks.get("hbm_gbs")
    times = {}
    real_call = P.call

    def timed_call(name, *a):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        real_call(name, *a)
        e1.record()
        e1.synchronize()
        times.setdefault(name, []).append(e0.elapsed_time(e1) / 1e3)

    out = {"what": "CUDA events around each library call; bytes: crop kernel = crop bytes written, count pass = "
                   "crop bytes read, write pass = crop bytes read + encoded bytes written",
           "peak_gbs": hbm}
    P.call = timed_call
    try:
        for cfg, (W, N, P_, S) in (("c1", (1024, 5000, 8, 128)), ("c2", (2048, 20000, 16, 256))):
            tm, m, r, th, vs, cs, sel = psd_case(torch, W, N, P_, S)
            best = {}
            for _ in range(3):          # the first pass warms up; the best of the other two counts
                times.clear()
                buf, bbox, sizes, offs = P.export_layers(tm, m, r, th, vs, cs, sel, W, W)
                hs = sizes.cpu().numpy()
                blob, blocks, chosen = P.encode_channel_blocks(buf, sizes, offs, hs, P.ORDER_LAYER,
                                                               lambda flags: np.nonzero(flags)[0])
                for k in ("dbmp_psd_layers", "dbmp_psd_rle_count", "dbmp_psd_rle_write"):
                    best[k] = min(best.get(k, 1e9), times[k][0])
                crop, enc = int(buf.numel()), int(blob.numel())
                del buf, blob
            moved = {"dbmp_psd_layers": crop, "dbmp_psd_rle_count": crop, "dbmp_psd_rle_write": crop + enc}
            out[cfg] = {"canvas": [W, W], "N": N, "crop_bytes": crop, "encoded_bytes": enc}
            for k, t in best.items():
                gbs = moved[k] / t / 1e9
                out[cfg][k] = {"ms": t * 1e3, "GB_per_s": gbs, "frac_of_hbm": gbs / hbm if hbm else None}
            torch.cuda.empty_cache()
    finally:
        P.call = real_call
    return out


class TorchReference:
    """The reference's PyTorch per-tile renderer on the host cores (its CPU
    path, restated in oracle/torch_renderer.py and pinned to the reference's
    own outputs): forward + backward of an evenly spaced sample of tiles,
    extrapolated to the canvas by tile count (a whole-canvas backward is out
    of reach at 2048^2: its saved per-tile tensors alone run to hundreds of GB)."""

    def __init__(self, spec, ts=32):
        import torch
        from oracle import oracle as O
        from oracle import torch_renderer as TR
        self.TR, self.spec, self.ts = TR, spec, ts
        P, Ht, Wt = spec.templates.shape
        tb = O.template_bboxes(spec.templates)
        offs, idx = O.bin_tiles(spec.H, spec.W, ts, spec.means2D, spec.radii, spec.rotations, spec.sel, tb, Ht, Wt)
        self.offs, self.idx = torch.from_numpy(offs), torch.from_numpy(idx)
        self.T = int(offs.size - 1)
        self.tmpl, self.sel = torch.from_numpy(spec.templates), torch.from_numpy(spec.sel)
        leaf = lambda a: torch.tensor(np.ascontiguousarray(a, np.float32), requires_grad=True)
        self.p = [leaf(spec.means2D[:, 0]), leaf(spec.means2D[:, 1]), leaf(spec.radii), leaf(spec.rotations),
                  leaf(spec.opacities), leaf(spec.colors)]
        torch.set_num_threads(os.cpu_count() or 1)

    def sample(self, k):
        """Seconds per fwd+bwd of the whole canvas, from k tiles spaced
        evenly over the canvas (each tile's L2-style loss backpropagated)."""
        tiles = np.unique(np.linspace(0, self.T - 1, max(1, int(k))).astype(np.int64))
        t0 = time.perf_counter()
        for t in tiles:
            out = self.TR.render_tile(int(t), self.spec.H, self.spec.W, self.ts, *self.p, self.tmpl, self.sel,
                                      self.spec.alpha_max, self.offs, self.idx)
            if out is not None:
                m, a = out
                ((m * m).sum() + a.sum()).backward()
        return (time.perf_counter() - t0) * self.T / len(tiles)

    def tiles_for_budget(self, seconds):
        per_tile = self.sample(2) / self.T
        return int(min(self.T, max(2, seconds / max(per_tile, 1e-9))))


def run_reference(args):
    """--impl reference: the reference's CPU path -- its PyTorch per-tile
    renderer (restated in oracle/torch_renderer.py, pinned to its outputs) --
    on the host cores, fwd+bwd on a bounded sample of tiles per step; the FP64
    restatement of its CUDA kernels' algorithm (oracle port) is timed once
    beside it and reported as a second figure."""
    import torch
    rank, world, _ = dist_setup(args, args.dist_backend)
    if rank != 0:
        barrier(world)
        finish(world)
        return
    from diffbmp_b200 import workloads as wl
    spec = wl.make_scene(args.config, seed=0)
    cores = os.cpu_count() or 1
    ref = TorchReference(spec)
    # each step is a bounded sample (evenly spaced tiles) so that the whole
    # run stays within about three minutes whatever --steps / --warmup are
    k = ref.tiles_for_budget(min(3.0, 150.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        ref.sample(k)
    times = [ref.sample(k) for _ in range(args.steps)]
    per_iter = float(np.median(times))
    value = 1.0 / per_iter
    port = CpuReference(spec)
    rows = port.rows_for_budget(5.0)
    t_port = port.sample(rows)
    sample = (f"fwd+bwd of the reference's PyTorch per-tile renderer on {k} of {ref.T} tiles (evenly spaced) per "
              f"step, extrapolated to the canvas by tile count")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "iters/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_iter * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{args.config}: {sample}", "canvas": [spec.H, spec.W], "N": spec.N,
                       "tile_size": 32, "threads": torch.get_num_threads()},
            "cpu_baseline": {"value": value, "unit": "iters/s", "cores": cores, "kind": "port",
                             "sample": sample,
                             "what": "torch restatement of SimpleTileRenderer._render_tile / _transmit_over "
                                     "(oracle/torch_renderer.py), pinned to the reference renderer's images "
                                     "and gradients"},
            "fp64_port": {"value": 1.0 / t_port, "unit": "iters/s", "cores": cores,
                          "sample": f"FP64 restatement of the reference CUDA kernels' algorithm (no termination), "
                                    f"fwd+bwd on {rows} of {spec.H} pixel rows, extrapolated"},
            "e2e": {"value": value, "unit": "iters/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    barrier(world)
    finish(world)


def finish(world):
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    rank, world, local = dist_setup(args)
    from diffbmp_b200 import workloads as wl
    spec = wl.make_scene(args.config, seed=rank)
    if args.profile == "psd":
        print(json.dumps({"profile": "psd", "export": psd_export_once(torch, 1024, 5000, 8, 128)}))
        return
    if args.profile:
        kind = "f32" if args.profile == "plain" else args.profile
        job = build_job(spec, kind, args.profile != "plain", torch)
        for _ in range(args.warmup + args.steps):
            job.step()
        job.sync()
        torch.cuda.synchronize()
        print(json.dumps({"profile": args.profile, "steps": args.warmup + args.steps, "loss": job.loss()}))
        return
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass

    # --- headline: FP16-storage fused step, graph replayed ----------------
    job = build_job(spec, HEADLINE_KIND, True, torch)
    for _ in range(3):   # a timed region with a skipped (overflowed) step is discarded
        with ClockSampler(local) as clk:
            t_fused, replayed = time_steps(job, args.steps, args.warmup, torch, world)
        if max_over_ranks(float(replayed), world) == 0:
            break
    clocks = clk.summary()
    t_fused = max_over_ranks(t_fused, world)
    loss_fused = job.loss()

    # --- plain FP32 kernels on the same scene -----------------------------
    plain = build_job(spec, "f32", False, torch)
    t_plain, _ = time_steps(plain, args.steps, args.warmup, torch, world)
    t_plain = max_over_ranks(t_plain, world)
    fused32 = build_job(spec, "f32", True, torch)
    t_fused32, _ = time_steps(fused32, args.steps, args.warmup, torch, world)
    t_fused32 = max_over_ranks(t_fused32, world)
    pair = build_job(spec, "f16", True, torch)
    t_pair, _ = time_steps(pair, args.steps, args.warmup, torch, world)
    t_pair = max_over_ranks(t_pair, world)
    t_bf16 = {}
    for kind in ("bf16q", "bf16"):        # BF16 storage, quad and pair layouts
        j = build_job(spec, kind, True, torch)
        t, _ = time_steps(j, args.steps, args.warmup, torch, world)
        t_bf16[kind] = max_over_ranks(t, world)
        j.graph = None
        del j
    # precision renders: each storage kind's image of the scene's initial
    # parameters, the band of rows compared with the FP64 oracle below
    band = precision_band(spec)
    renders = {kind: render_band(spec, kind, band, torch) for kind in PRECISION_KINDS}

    # --- e2e through the public API with host buffers ---------------------
    e2e_job = build_job(spec, HEADLINE_KIND, True, torch)
    # the step's inputs: the five parameter arrays, packed host-side as
    # ImageFitter.params_flat lays them out, uploaded with one copy
    host = torch.from_numpy(np.concatenate([np.asarray(getattr(spec, k), np.float32).reshape(-1) for k in
                                            ("means2D", "radii", "rotations", "opacities", "colors")])).pin_memory()
    loss_host = torch.zeros(2, dtype=torch.float64).pin_memory()   # ring of two step results
    done = [torch.cuda.Event(), torch.cuda.Event()]
    dev_params = e2e_job.params_flat
    h2d = host.numel() * 4
    losses = []

    def e2e_step(i):
        # one step in flight: step i is enqueued (inputs H2D through the
        # double-buffered upload, iteration, loss D2H), then the host waits for
        # step i - 1 and reads its loss
        e2e_job.upload_params(host)
        e2e_job.step()
        loss_host[i % 2:i % 2 + 1].copy_(e2e_job.loss_dev, non_blocking=True)
        done[i % 2].record()
        if i > 0:
            done[(i - 1) % 2].synchronize()
            losses.append(float(loss_host[(i - 1) % 2]))

    def e2e_finish(n):
        done[(n - 1) % 2].synchronize()
        losses.append(float(loss_host[(n - 1) % 2]))
    for i in range(args.warmup):
        e2e_step(i)
    e2e_finish(args.warmup)
    e2e_job.sync()
    torch.cuda.synchronize(); barrier(world)
    t0 = time.perf_counter()
    for i in range(args.steps):
        e2e_step(i)
    e2e_finish(args.steps)
    t_e2e = time.perf_counter() - t0
    assert len(losses) == args.warmup + args.steps and all(np.isfinite(losses))
    t_e2e = max_over_ranks(t_e2e, world)

    # --- roofline of the dominant kernel (fused fwd+bwd), CUDA events ------
    import ctypes
    from diffbmp_b200._lib import call
    from diffbmp_b200.rasterizer import _ptr, _stream

    def fused_launch():
        call("dbmp_fused_fwd_bwd", ctypes.byref(job.cv), _ptr(job.prim_info), _ptr(job.atlas.data),
             _ptr(job.offsets), _ptr(job.rz._idx), _ptr(job.target), _ptr(job.background), None, _ptr(job.gacc),
             _ptr(job.loss_dev), None, _stream())
    job._enqueue(); torch.cuda.synchronize()
    t_kernel = kernel_time(job, fused_launch, max(5, args.steps // 4), torch)
    cand, frag, L, went, slots, miss, _, empty, clear, bad = counts(job, torch)
    flop = 12.0 * cand + 144.0 * frag
    fp32_peak = fp32_simt_peak_tflops(torch)
    achieved = flop / t_kernel / 1e12

    FUSED_DRAM_BYTES = FUSED_DRAM_BYTES_C2 if args.config == "c2" else None
    ms_step = t_fused / args.steps * 1e3
    value = world * args.steps / t_fused
    line = {
        "metric": METRIC, "value": value, "unit": "iters/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.config}: {spec.H}x{spec.W} canvas, N={spec.N}, "
                               f"{spec.templates.shape[0]}x{spec.templates.shape[1]}x{spec.templates.shape[2]} atlas; "
                               "one fit iteration per step (device binning, fused fwd+L2+bwd, Adam) with FP16 bilinear-quad atlas "
                               "storage and FP32 arithmetic, CUDA-graph replay",
                   "canvas": [spec.H, spec.W], "N": spec.N, "tile_size": 32, "t_stop": job.cfg.t_stop,
                   "l2": "per-step working set (target 50 MB + background 50 MB + tile lists 28 MB) exceeds the 126 MB L2",
                   "parallelism": f"replicas x{world}", "tile_list_entries": L, "replayed_steps": replayed},
        "plain_fp32": {"iters_per_s": world * args.steps / t_plain, "ms_per_step": t_plain / args.steps * 1e3,
                       "what": "unfused forward + torch L2 gradient + backward, FP32 atlas, graph replay"},
        "fused_fp32": {"iters_per_s": world * args.steps / t_fused32, "ms_per_step": t_fused32 / args.steps * 1e3,
                       "what": "fused kernel, FP32 atlas in the reference layout"},
        "fused_f16_pair": {"iters_per_s": world * args.steps / t_pair, "ms_per_step": t_pair / args.steps * 1e3,
                           "what": "fused kernel, FP16 atlas as horizontal texel pairs (half the FP32 bytes)"},
        "fused_bf16_quad": {"iters_per_s": world * args.steps / t_bf16["bf16q"],
                            "ms_per_step": t_bf16["bf16q"] / args.steps * 1e3,
                            "what": "fused kernel, BF16 bilinear-quad atlas"},
        "fused_bf16_pair": {"iters_per_s": world * args.steps / t_bf16["bf16"],
                            "ms_per_step": t_bf16["bf16"] / args.steps * 1e3,
                            "what": "fused kernel, BF16 atlas as horizontal texel pairs"},
        "speedup_vs_plain_fp32": (world * args.steps / t_fused) / (world * args.steps / t_plain),
        "loss_after": loss_fused,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak, "traffic": FUSED_DRAM_BYTES,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of this "
                                       "kernel on this workload (the committed fused-kernel profile)",
                     "kernel": HEADLINE_KERNEL, "kernel_ms": t_kernel * 1e3,
                     "flop_model": "12*C + 144*F_live (C pairs passing cull, F_live fragments composited)",
                     "C": cand, "F_live": frag, "warp_entries": went, "live_pixel_slots": slots,
                     "footprint_rejects": miss, "empty_warp_entries": empty, "grid_skips": clear,
                     "grid_skips_with_fragment": bad,
                     "peak_source": "measured in-run: cuBLAS SGEMM 8192^3, TF32 off (FP32 SIMT pipe)",
                     "hbm_peak_gbs_measured": peaks.get("hbm_gbs")},
        "e2e": {"value": world * args.steps / t_e2e, "unit": "iters/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 8,
                "what": "public API: every step's parameters H2D from pinned host (ImageFitter.upload_params: copy "
                        "stream, two staging buffers), ImageFitter.step(), loss D2H read by the host every step, "
                        "one step in flight"},
        "gpu_launches": 6 * args.steps,
        "gpu_launches_note": "ours per step: prepare, counts, bin_rows, fused, adam, step_increment "
                             "(+ three memsets -- the binning difference arrays, the loss and the gradient "
                             "sums -- and the two kernels of one CUB exclusive scan over the tile counts)",
        "clocks": clocks,
    }
    if args.serving_jobs > 0 and world == 1:   # the serving stream is a single-GPU measurement
        # measured on a clean device: the jobs above and their graphs are released first
        for j in (job, plain, fused32, pair, e2e_job):
            j.graph = None
        del job, plain, fused32, pair, e2e_job, dev_params
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        line["serving"] = run_serving(args.serving_jobs, rank, torch)
    if world == 1 and not args.no_psd:
        torch.cuda.synchronize()
        torch.cuda.empty_cache()          # the serving loop's cached blocks belong to its streams
        line["psd"] = run_psd(torch, peaks)
    if rank == 0 and world == 1 and not args.fast:
        # the same leg renders the precision band with the FP64 oracle, the
        # checker of the storage kinds' images rendered above
        line["precision"] = precision_vs_oracle(spec, band, renders)
        ref = TorchReference(spec)
        k = ref.tiles_for_budget(15.0)           # about 15 s of CPU work
        t_cpu = ref.sample(k)
        port = CpuReference(spec)
        rows = port.rows_for_budget(4.0)
        t_port = port.sample(rows)
        line["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": "iters/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": f"fwd+bwd of the reference's PyTorch per-tile renderer (restated, pinned "
                                          f"to its outputs) on {k} of {ref.T} tiles, evenly spaced, extrapolated "
                                          f"to the canvas by tile count",
                                "fp64_port": {"value": 1.0 / t_port, "unit": "iters/s",
                                              "sample": f"FP64 restatement of the reference kernels' algorithm "
                                                        f"(no termination), fwd+bwd on {rows} of {spec.H} pixel "
                                                        f"rows, extrapolated"}}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        for j in (job, plain, fused32, pair, e2e_job):
            j.graph = None
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
