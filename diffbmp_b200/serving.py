"""Continuous-batching server for fit-an-image jobs.

Replaces the reference's only batching -- a host loop calling the single-image
forward/backward once per candidate (cuda_tile_rasterizer/tile_rasterize.cu:500-636,
simple_tile_renderer.py:268-429) -- with a request loop:

* jobs arrive over time (``JobRequest.arrival`` seconds after start) and are
  admitted into a slot as soon as a slot is free and their estimated device
  memory fits the HBM budget;
* an admitted job stays resident in HBM (``ImageFitter``: parameters, Adam
  moments, target, tile lists, scratch) and its fit iteration (binning, fused
  forward + L2 + backward, Adam) is captured once in a CUDA graph;
* every active job advances independently on its own stream of a pool, at
  most ``depth`` iterations ahead of the host, so iterations of small and
  large canvases overlap on the device instead of waiting for each other;
* a job retires when its device step counter reaches its iteration count;
  list-capacity overflows are detected there and the skipped iterations are
  replayed (exact results);
* latency = retirement time - arrival time; throughput = retired jobs over
  the span from the first arrival to the last retirement.
"""
from __future__ import annotations

import collections
import gc
import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import torch

from .fitting import FitConfig, ImageFitter
from .rasterizer import Atlas


@dataclass
class JobRequest:
    job_id: int
    arrival: float               # seconds after the server starts
    spec: object                 # workloads.SceneSpec
    iterations: int = 100


@dataclass
class JobResult:
    job_id: int
    arrival: float
    admitted: float
    done: float
    loss: float
    replayed: int
    params: Optional[dict] = None

    @property
    def latency(self):
        return self.done - self.arrival


def list_capacity_bound(spec, tile_size=32) -> int:
    """Upper bound of a job's tile-list length from its parameters on the
    host: the binning box of a primitive (its template's content box, rotated)
    lies within the square of half-width r*sqrt(2) about its centre, and the
    inclusive tile test adds at most one tile per side; non-finite geometry
    is binned into every tile."""
    H, W = spec.H, spec.W
    tx, ty = (W + tile_size - 1) // tile_size, (H + tile_size - 1) // tile_size
    r = np.abs(np.asarray(spec.radii, np.float64))
    finite = np.isfinite(r) & np.isfinite(np.asarray(spec.rotations, np.float64)) & \
        np.isfinite(np.asarray(spec.means2D, np.float64)).all(-1)
    side = np.ceil(2.0 * np.sqrt(2.0) * np.where(finite, r, 0.0) / tile_size) + 2.0
    per = np.minimum(side, tx) * np.minimum(side, ty)
    return int(np.where(finite, per, tx * ty).sum()) + 4096


def estimate_bytes(spec, tile_size=32) -> int:
    """Upper estimate of one job's resident device memory: target and
    background images, per-pixel state, the tile lists at list_capacity_bound,
    and the per-primitive state."""
    H, W, N = spec.H, spec.W, spec.N
    T = ((H + tile_size - 1) // tile_size) * ((W + tile_size - 1) // tile_size)
    L = list_capacity_bound(spec, tile_size)
    return int(2 * H * W * 12 + H * W * 8 + L * 4 + N * 512 + (T + 1) * 64)


@dataclass
class _Slot:
    req: JobRequest
    fitter: ImageFitter
    stream: torch.cuda.Stream
    admitted: float
    issued: int = 0
    events: collections.deque = field(default_factory=collections.deque)
    nbytes: int = 0


class Server:
    """Request loop over a shared atlas.  ``kind``: atlas storage ("f16" for
    the precision form, "f32" plain); ``fused``: fused fwd/bwd kernel."""

    def __init__(self, atlas_templates: torch.Tensor, kind="f16", fused=True, max_slots=48,
                 hbm_budget=150e9, n_streams=16, depth=3, graphs=True, lr=0.01, keep_params=False):
        self.atlas = Atlas(atlas_templates, kind)
        self.cfg = FitConfig(lr=lr, fused=fused)
        self.max_slots = max_slots
        self.budget = float(hbm_budget)
        self.streams = [torch.cuda.Stream() for _ in range(n_streams)]
        self.admit_stream = torch.cuda.Stream()
        self.depth = depth
        self.graphs = graphs
        self.keep_params = keep_params

    def _reserve(self, requests: List[JobRequest]):
        """Grows the device allocator's cache to the resident jobs' estimated
        total (within the HBM budget) before serving: job set-up then carves its
        buffers from cached memory instead of allocating device memory while
        the device is busy, which stalled the host for up to 0.2 s.  The
        allocator reuses a cached block only on the stream it was allocated
        on, so the blocks are allocated on the admission stream: one large
        block for the large pool, and 1 MB blocks for the small pool's
        segments (tensors of up to 1 MB: counters, offsets, small jobs' state)."""
        # at most max_slots jobs are resident at once: the largest max_slots estimates bound them
        est = sorted(estimate_bytes(r.spec, self.cfg.tile_size) for r in requests)[-self.max_slots:]
        want = min(self.budget, float(sum(est)))
        free, _ = torch.cuda.mem_get_info()
        want = int(min(want, 0.8 * free))
        with torch.cuda.stream(self.admit_stream):
            if want > (1 << 26):
                block = torch.empty(want, dtype=torch.uint8, device="cuda")
                del block
            # segments for the jobs that can be resident at once, not for the whole stream
            small = [torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
                     for _ in range(16 * min(len(requests), self.max_slots))]
            del small

    def _admit(self, req: JobRequest, now: float, stream) -> _Slot:
        """Sets a job up on the admission stream, which carries no iterations,
        so its uploads never wait behind other jobs' work; the lists are sized
        from list_capacity_bound (no device read-back).  The job's stream then
        waits for the set-up."""
        s = req.spec
        adm = self.admit_stream
        adm.wait_stream(torch.cuda.default_stream())   # job tensors may come from the default stream
        with torch.cuda.stream(adm):
            f = ImageFitter(s.means2D, s.radii, s.rotations, s.opacities, s.colors, s.sel, self.atlas, s.target,
                            s.background, self.cfg, list_capacity=list_capacity_bound(s, self.cfg.tile_size))
            if self.graphs:
                f.capture()
        stream.wait_stream(adm)
        return _Slot(req, f, stream, now)

    def run(self, requests: List[JobRequest], realtime=True) -> List[JobResult]:
        """Serves `requests`.  realtime: admit each at its arrival time (else
        all are queued at the start and latencies count from 0)."""
        # the loop allocates an event per iteration: a garbage-collector pass in
        # the middle of it would stall issuing, so collection pauses until the end
        gc.collect()
        gc_was_enabled = gc.isenabled()
        gc.disable()
        try:
            return self._run(requests, realtime)
        finally:
            if gc_was_enabled:
                gc.enable()

    def _run(self, requests: List[JobRequest], realtime: bool) -> List[JobResult]:
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        self._reserve(requests)
        active: List[_Slot] = []
        results: List[JobResult] = []
        used = 0
        t0 = time.perf_counter()
        clock = lambda: time.perf_counter() - t0
        load = {id(st): 0 for st in self.streams}        # active jobs per stream
        inflight = collections.deque()                   # events of issued iterations, in issue order

        def admit():
            # arrived jobs, while slots and the HBM budget allow
            nonlocal used
            now = clock()
            while pending and (pending[0].arrival <= now or not realtime) and len(active) < self.max_slots:
                est = estimate_bytes(pending[0].spec, self.cfg.tile_size)
                if used + est > self.budget and active:
                    break
                req = pending.popleft()
                # the least-loaded stream: a new job does not queue behind several others
                stream = min(self.streams, key=lambda st: load[id(st)])
                load[id(stream)] += 1
                slot = self._admit(req, max(now, req.arrival) if realtime else now, stream)
                slot.nbytes = est
                used += est
                active.append(slot)

        while pending or active:
            admit()
            progressed = False
            for slot in list(active):
                # retire finished iterations
                while slot.events and slot.events[0].query():
                    slot.events.popleft()
                    progressed = True
                f = slot.fitter
                if slot.issued >= slot.req.iterations and not slot.events:
                    # the last iteration staged the step count and loss on the host;
                    # only a skipped (overflowed) step needs the synchronising path
                    replayed = 0
                    done, loss = f.staged_result()
                    if done < f.steps_enqueued:
                        with torch.cuda.stream(slot.stream):
                            replayed = f.sync()
                            loss = f.loss()
                    params = {k: v.detach().clone() for k, v in f.params().items()} if self.keep_params else None
                    # without realtime arrivals every request is queued at the start
                    arrival = slot.req.arrival if realtime else 0.0
                    results.append(JobResult(slot.req.job_id, arrival, slot.admitted, clock(), loss,
                                             replayed, params))
                    active.remove(slot)
                    load[id(slot.stream)] -= 1
                    used -= slot.nbytes
                    progressed = True
                    admit()   # the freed slot takes the next waiting job at once
                    continue
                # issue up to `depth` iterations ahead of the host
                while slot.issued < slot.req.iterations and len(slot.events) < self.depth:
                    with torch.cuda.stream(slot.stream):
                        f.step()
                        if slot.issued + 1 == slot.req.iterations:
                            f.stage_result()
                        ev = torch.cuda.Event()
                        ev.record(slot.stream)
                    slot.events.append(ev)
                    inflight.append(ev)
                    slot.issued += 1
                    progressed = True
            if not progressed:
                if active:
                    # nothing to issue: wait for the earliest-issued iteration still
                    # running (the device retires work roughly in issue order)
                    while inflight and inflight[0].query():
                        inflight.popleft()
                    if inflight:
                        inflight.popleft().synchronize()
                    else:
                        time.sleep(0.0002)
                elif pending and realtime:
                    time.sleep(max(0.0, min(0.002, pending[0].arrival - clock())))
        torch.cuda.synchronize()
        return results


def poisson_requests(n, rate, atlas, seed=0, iterations=100, sizes=(256, 512, 1024, 2048), n_range=(256, 20000),
                     device=None):
    """n jobs of the serving workload, exponential inter-arrival times at `rate`
    jobs/s, drawn from the shared atlas (targets built on `device` if given)."""
    from . import workloads as wl
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        reqs.append(JobRequest(i, t, wl.make_job(rng, atlas, sizes, n_range, device), iterations))
    return reqs


def summarize(results: List[JobResult]):
    lat = np.array([r.latency for r in results])
    span = max(r.done for r in results) - min(r.arrival for r in results)
    return dict(jobs=len(results), jobs_per_s=len(results) / span, p50_s=float(np.percentile(lat, 50)),
                p99_s=float(np.percentile(lat, 99)), mean_loss=float(np.mean([r.loss for r in results])),
                replayed=int(sum(r.replayed for r in results)))


def run_sequential(requests: List[JobRequest], atlas_templates, kind="f32", fused=False, lr=0.01, graphs=False):
    """One job at a time, to completion: the baselines of the serving target.
    Each job is set up as the server sets one up (lists sized from
    list_capacity_bound, the iteration captured in a CUDA graph when
    `graphs`), then runs its iterations and reads its result.  Returns
    (results, wall seconds, device seconds of the iterations alone)."""
    atlas = Atlas(atlas_templates, kind)
    cfg = FitConfig(lr=lr, fused=fused)
    out = []
    device_s = 0.0
    t0 = time.perf_counter()
    for req in requests:
        s = req.spec
        f = ImageFitter(s.means2D, s.radii, s.rotations, s.opacities, s.colors, s.sel, atlas, s.target,
                        s.background, cfg, list_capacity=list_capacity_bound(s, cfg.tile_size))
        if graphs:
            f.capture()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(req.iterations):
            f.step()
        e1.record()
        rep = f.sync()
        device_s += e0.elapsed_time(e1) / 1e3
        out.append(JobResult(req.job_id, 0.0, 0.0, time.perf_counter() - t0, f.loss(), rep))
    return out, time.perf_counter() - t0, device_s
