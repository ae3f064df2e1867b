"""Image fitting on the device: the reference's optimisation loop
(pydiffbmp/core/renderer/simple_tile_renderer.py:913-1228,
_optimize_parameters_whole) rebuilt as a sync-free step of library kernels.

One ``ImageFitter`` holds one job resident in HBM: FP32 master parameters,
Adam moments, the target and background, the atlas in its storage kind, the
tile-list buffers and scratch.  ``step()`` enqueues

    dbmp_bin -> dbmp_fused_fwd_bwd -> dbmp_adam_step          (fused form)
    dbmp_bin -> dbmp_forward -> L2 gradient -> dbmp_backward -> dbmp_adam_step   (plain form)

with no host synchronisation, so it can be captured in a CUDA graph.  If the
tile lists outgrow their capacity the bin call flags it on the device and the
later kernels of that step leave every state untouched; ``sync()`` detects the
skipped steps (the device step counter lags) and replays them after growing
the capacity, so results are exactly those of an unlimited capacity.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import AdamCfg, call, lib
from .rasterizer import Atlas, Rasterizer, _ptr, _stream, DEFAULT_T_STOP

# Reference defaults (pydiffbmp/util/constants.py:24-38): base lr and gains,
# ExponentialLR factor, fixed blur sigma.
LR_GAINS = dict(x=10.0, y=10.0, r=10.0, v=1.5, theta=1.0, c=1.0)
DECAY_RATE = 0.99
BLUR_SIGMA = 1.0
BLUR_MODES = {"none": 0, "fixed": 1, "adaptive": 2}


@dataclass
class PruneConfig:
    """The reference's pruning (restart) options, opt_conf["pruning"]
    (simple_tile_renderer.py:980-981,1007-1013): every `every` iterations
    inside (warmup, num_iterations - no_prune_last), primitives with
    sigmoid(opacity) < threshold are re-initialised.  `pool` (R,8) holds the
    replacement parameters (x, y, r, theta, opacity logit, colour logits) that
    the reference draws from its initializer at each prune; rows are used in
    order, cyclically (``fallback_pool`` draws them as the reference's
    _fallback_random_init does)."""
    pool: object
    threshold: float = 0.3
    every: int = 5
    no_prune_last: int = 10
    warmup: int = 20


def fallback_pool(rng: np.random.Generator, H: int, W: int, rows: int) -> np.ndarray:
    """Replacement rows drawn as the reference's _fallback_random_init
    (simple_tile_renderer.py:1272-1282): x U[0,W), y U[0,H), r U[0,1) *
    min(H,W)/20 + 2, opacity logit -2, theta U[0,2pi), colour logits U[0,1)."""
    out = np.empty((rows, 8), np.float32)
    out[:, 0] = rng.random(rows) * W
    out[:, 1] = rng.random(rows) * H
    out[:, 2] = rng.random(rows) * (min(H, W) / 20) + 2
    out[:, 3] = rng.random(rows) * 2 * np.pi
    out[:, 4] = -2.0
    out[:, 5:8] = rng.random((rows, 3))
    return out


@dataclass
class FitConfig:
    lr: float = 0.01
    gains: dict = field(default_factory=lambda: dict(LR_GAINS))
    betas: tuple = (0.9, 0.999)
    eps: float = 1e-8
    tile_size: int = 32
    alpha_max: float = 1.0
    t_stop: float = DEFAULT_T_STOP
    fused: bool = True
    headroom: float = 1.3
    # the rest of the reference's loop (simple_tile_renderer.py:970-981):
    num_iterations: int = 0          # iterations of the whole fit (blur / prune schedules)
    decay_rate: float = 1.0          # ExponentialLR gamma (do_decay: DECAY_RATE); 1: no decay
    blur: str = "none"               # "fixed" (do_gaussian_blur) or "adaptive" (do_adapt_gaussian_blur)
    blur_sigma: float = BLUR_SIGMA
    blur_sigma_start: float = 2.0
    blur_sigma_end: float = 0.0
    prune: PruneConfig | None = None

    @classmethod
    def from_opt_conf(cls, opt_conf: dict, pool=None, **over) -> "FitConfig":
        """The settings of the reference's optimisation config (the
        "optimization" block read by _optimize_parameters_whole,
        simple_tile_renderer.py:939-981): learning_rate.default and gains,
        num_iterations, do_decay / decay_rate, do_gaussian_blur / blur_sigma,
        do_adapt_gaussian_blur / blur_sigma_start / blur_sigma_end and pruning.
        Pruning needs `pool`, the replacement rows of PruneConfig."""
        lr_conf = opt_conf.get("learning_rate", {})
        gains = dict(LR_GAINS)
        for k in ("x", "y", "r", "v", "theta", "c"):
            gains[k] = float(lr_conf.get(f"gain_{k}", gains[k]))
        blur = "adaptive" if opt_conf.get("do_adapt_gaussian_blur") else \
            "fixed" if opt_conf.get("do_gaussian_blur") else "none"
        pr = opt_conf.get("pruning", {})
        prune = None
        if pr.get("do_pruning", False):
            if pool is None:
                raise ValueError("pruning needs the replacement pool (PruneConfig.pool)")
            prune = PruneConfig(pool, float(pr.get("prune_threshold", 0.3)), int(pr.get("prune_iterations", 5)),
                                int(pr.get("no_prune_last_iterations", 10)),
                                int(pr.get("no_prune_warmup_iterations", 20)))
        kw = dict(lr=float(lr_conf.get("default", 0.1)), gains=gains,
                  num_iterations=int(opt_conf.get("num_iterations", 100)),
                  decay_rate=float(opt_conf.get("decay_rate", DECAY_RATE)) if opt_conf.get("do_decay") else 1.0,
                  blur=blur, blur_sigma=float(opt_conf.get("blur_sigma", BLUR_SIGMA)),
                  blur_sigma_start=float(opt_conf.get("blur_sigma_start", 2.0)),
                  blur_sigma_end=float(opt_conf.get("blur_sigma_end", 0.0)), prune=prune)
        kw.update(over)
        return cls(**kw)


# Host statements of the loop's schedules; the device kernels (dbmp_adam_step,
# dbmp_template_blur_scheduled, dbmp_prune) evaluate the same expressions from
# the device step count.
def lr_schedule(cfg: FitConfig, N: int, it: int) -> list:
    """Learning rates of the reference's Adam groups (x, y, r, v, theta, c) at
    iteration it: lr * gain (v: * 1000/N) * decay_rate^it
    (simple_tile_renderer.py:961-973, ExponentialLR stepped once per iteration)."""
    g, d = cfg.gains, cfg.decay_rate ** it
    return [cfg.lr * g["x"] * d, cfg.lr * g["y"] * d, cfg.lr * g["r"] * d,
            cfg.lr * g["v"] * (1000.0 / max(N, 1)) * d, cfg.lr * g["theta"] * d, cfg.lr * g["c"] * d]


def blur_sigma_at(cfg: FitConfig, it: int) -> float:
    """Template blur sigma of iteration it (simple_tile_renderer.py:1015-1022)."""
    if cfg.blur == "adaptive":
        progress = it / cfg.num_iterations
        return cfg.blur_sigma_start * (1 - progress) + cfg.blur_sigma_end * progress
    if cfg.blur == "fixed":
        return cfg.blur_sigma
    return 0.0


def prune_due(cfg: FitConfig, it: int) -> bool:
    """Whether iteration it prunes (simple_tile_renderer.py:1007-1012)."""
    p = cfg.prune
    return (p is not None and it != 0 and it % p.every == 0 and it < cfg.num_iterations - p.no_prune_last
            and it > p.warmup)


def prune_selection(cfg: FitConfig, opacity_logits) -> np.ndarray:
    """Indices the prune replaces: sigmoid(v) < threshold in float32
    (simple_tile_renderer.py:1244-1254), ascending."""
    v = np.asarray(opacity_logits, np.float32)
    with np.errstate(over="ignore"):
        sig = (np.float32(1) / (np.float32(1) + np.exp(-v))).astype(np.float32)
    return np.nonzero(sig < np.float32(cfg.prune.threshold))[0]


def _upload(a: np.ndarray, device) -> torch.Tensor:
    """Host array to the device through pinned memory, asynchronously on the
    current stream: a copy from pageable memory would first wait for every
    kernel queued on that stream, which on a busy device (a serving loop
    admitting jobs) blocks the host for the duration of other jobs' work."""
    return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().to(device, non_blocking=True)


def _dev_f32(a, device, copy=True):
    if isinstance(a, torch.Tensor):
        t = a.detach().to(device=device, dtype=torch.float32).contiguous()
        return t.clone() if copy and t.data_ptr() == a.data_ptr() else t
    return _upload(np.asarray(a, np.float32), device)


class ImageFitter:
    """One fit-an-image job resident on the device."""

    def __init__(self, means2D, radii, rotations, opacities, colors, sel, atlas: Atlas, target,
                 background=None, config: FitConfig | None = None, device=None, list_capacity: int | None = None):
        """list_capacity: tile-list entries to provision.  By default the
        current lists are counted on the device (one host synchronisation);
        a caller that knows an upper bound (list_capacity_bound) avoids it.
        A bound that turns out short is still exact: an overflowed binning
        skips its step, and sync() grows the lists and replays it."""
        self.cfg = cfg = config or FitConfig()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        dev = self.device
        # the five parameter arrays are views of one (N*8,) buffer, params_flat
        # (centres, radii, rotations, opacity logits, colour logits), so that a
        # caller can upload all of them with one copy
        parts = [_dev_f32(a, dev, copy=False).reshape(-1) for a in (means2D, radii, rotations, opacities, colors)]
        n = int(parts[1].numel())
        if [int(t.numel()) for t in parts] != [2 * n, n, n, n, 3 * n]:
            raise ValueError("means2D (N,2), radii, rotations, opacities (N) and colors (N,3) disagree on N")
        self.params_flat = torch.cat(parts) if n > 0 else torch.zeros(0, dtype=torch.float32, device=dev)
        o = [0, 2 * n, 3 * n, 4 * n, 5 * n, 8 * n]
        self.means2D = self.params_flat[o[0]:o[1]].view(-1, 2)
        self.radii = self.params_flat[o[1]:o[2]]
        self.rotations = self.params_flat[o[2]:o[3]]
        self.opacities = self.params_flat[o[3]:o[4]]
        self.colors = self.params_flat[o[4]:o[5]].view(-1, 3)
        self.sel = (sel.to(device=dev, dtype=torch.int32) if isinstance(sel, torch.Tensor)
                    else _upload(np.asarray(sel, np.int32), dev)).contiguous()
        self.N = int(self.radii.numel())
        # read-only images: no private copy is needed
        self.target = _dev_f32(target, dev, copy=False)
        self.H, self.W = int(self.target.shape[0]), int(self.target.shape[1])
        self.background = _dev_f32(background, dev, copy=False) if background is not None else None
        self.atlas = atlas
        self.rz = Rasterizer(self.H, self.W, cfg.tile_size, cfg.alpha_max, cfg.t_stop, device=dev)
        self.cv = self.rz.canvas(self.N, atlas)
        N8 = (max(self.N, 1), 8)
        self.adam_m = torch.zeros(N8, dtype=torch.float32, device=dev)
        self.adam_v = torch.zeros(N8, dtype=torch.float32, device=dev)
        self.gacc = torch.zeros(N8, dtype=torch.float64, device=dev)
        self.loss_dev = torch.zeros(1, dtype=torch.float64, device=dev)
        self.step_count = torch.zeros(1, dtype=torch.int32, device=dev)
        self.flags = torch.zeros(2, dtype=torch.int32, device=dev)    # [L, overflow]
        self.prim_info = torch.empty((max(self.N, 1), 16), dtype=torch.float32, device=dev)
        # zero lists until the first successful binning: an overflowed first bin renders nothing
        self.offsets = torch.zeros(self.rz.T + 1, dtype=torch.int32, device=dev)
        if not cfg.fused:
            self.color = torch.empty((self.H, self.W, 3), dtype=torch.float32, device=dev)
            self.alpha = torch.empty((self.H, self.W), dtype=torch.float32, device=dev)
            self.T_last = torch.empty((self.H, self.W), dtype=torch.float32, device=dev)
            self.last_pos = torch.empty((self.H, self.W), dtype=torch.int32, device=dev)
            self.grads = [torch.empty(s, dtype=torch.float32, device=dev)
                          for s in ((self.N, 2), (self.N,), (self.N,), (self.N,), (self.N, 3))]
        g = cfg.gains
        lr = cfg.lr
        lrs = [lr * g["x"], lr * g["y"], lr * g["r"], lr * g["theta"], lr * g["v"] * (1000.0 / max(self.N, 1))] + \
              [lr * g["c"]] * 3
        self.adam_cfg = AdamCfg((ctypes.c_float * 8)(*lrs), cfg.betas[0], cfg.betas[1], cfg.eps,
                                float(self.W - 1), float(self.H - 1), 2.0, float(min(self.H, self.W) // 4), 1,
                                float(cfg.decay_rate))
        # blur schedule: the job re-blurs the atlas's templates into its own
        # texel buffer every step (the content bboxes stay the unblurred ones)
        self.blur = None
        if cfg.blur != "none":
            if cfg.blur not in BLUR_MODES:
                raise ValueError(f"blur must be one of {sorted(BLUR_MODES)}, not {cfg.blur!r}")
            if cfg.blur == "adaptive" and cfg.num_iterations < 1:
                raise ValueError("the adaptive blur schedule needs FitConfig.num_iterations")
            self.atlas = atlas.private_copy()
            self.cv = self.rz.canvas(self.N, self.atlas)
            self.blur = _lib.BlurSchedule(BLUR_MODES[cfg.blur], cfg.blur_sigma, cfg.blur_sigma_start,
                                          cfg.blur_sigma_end, int(cfg.num_iterations))
            self._blurred = (self.atlas.data if self.atlas.kind == _lib.ATLAS_F32
                             else torch.empty_like(self.atlas.templates))
            self._blur_step()     # this iteration's texels before the first binning / render
        self.prune = None
        if cfg.prune is not None:
            pc = cfg.prune
            if cfg.num_iterations < 1:
                raise ValueError("pruning needs FitConfig.num_iterations")
            pool = pc.pool if isinstance(pc.pool, torch.Tensor) else torch.from_numpy(np.asarray(pc.pool, np.float32))
            self.prune_pool = pool.to(device=dev, dtype=torch.float32).contiguous().view(-1, 8)
            self.prune_state = torch.zeros(4, dtype=torch.int32, device=dev)
            self.prune = _lib.PruneCfg(int(pc.every), int(cfg.num_iterations), int(pc.no_prune_last),
                                       int(pc.warmup), float(pc.threshold), int(self.prune_pool.shape[0]))
        self.steps_enqueued = 0
        self.graph = None
        self._host_state = None   # pinned (step count, loss) staged by stage_result()
        if list_capacity is None:
            self._grow(self._count())
        else:
            self.rz._ensure(self.cv, int(list_capacity))

    # -- capacity ----------------------------------------------------------
    def _count(self) -> int:
        """Counts the current tile-list length (one host sync)."""
        cap, self.rz.capacity = self.rz.capacity, 0
        self.rz._ensure(self.cv, 0)
        ws, wsb = self.rz._ws_ptr()
        call("dbmp_bin", ctypes.byref(self.cv), *self._param_ptrs(), _ptr(self.atlas.bbox), _ptr(self.prim_info),
             _ptr(self.offsets), None, ctypes.c_longlong(0), _ptr(self.flags),
             ctypes.c_void_p(self.flags.data_ptr() + 4), ws, ctypes.c_size_t(wsb), _stream())
        self.rz.capacity = cap
        return int(self.flags[0].item())

    def _grow(self, L: int):
        want = int(L * self.cfg.headroom) + 4096
        if want > self.rz.capacity:
            self.rz._ensure(self.cv, want)
            self.graph = None

    def _param_ptrs(self):
        return [_ptr(self.means2D), _ptr(self.radii), _ptr(self.rotations), _ptr(self.opacities),
                _ptr(self.colors), _ptr(self.sel)]

    # -- one iteration -------------------------------------------------------
    def _blur_step(self, st=None):
        """This iteration's blurred texels (blur schedule on the device step count)."""
        st = st if st is not None else _stream()
        a = self.atlas
        call("dbmp_template_blur_scheduled", _ptr(a.templates), a.P, a.Ht, a.Wt, ctypes.byref(self.blur),
             _ptr(self.step_count), _ptr(self._blurred), st)
        if a.kind != _lib.ATLAS_F32:
            call("dbmp_atlas_pack", _ptr(self._blurred), a.P, a.Ht, a.Wt, a.kind, _ptr(a.data), st)

    def _enqueue(self):
        st = _stream()
        cv = self.cv
        rz = self.rz
        ws, wsb = rz._ws_ptr()
        skip = ctypes.c_void_p(self.flags.data_ptr() + 4)
        # the reference's iteration order: prune, blur, render, loss, backward,
        # Adam step, lr decay, clamp (simple_tile_renderer.py:1003-1131)
        if self.prune is not None:
            call("dbmp_prune", ctypes.byref(cv), ctypes.byref(self.prune), _ptr(self.step_count),
                 _ptr(self.prune_pool), _ptr(self.prune_state), _ptr(self.means2D), _ptr(self.radii),
                 _ptr(self.rotations), _ptr(self.opacities), _ptr(self.colors), None, st)
        if self.blur is not None:
            self._blur_step(st)
        call("dbmp_bin", ctypes.byref(cv), *self._param_ptrs(), _ptr(self.atlas.bbox), _ptr(self.prim_info),
             _ptr(self.offsets), _ptr(rz._idx), ctypes.c_longlong(rz.capacity), _ptr(self.flags), skip, ws,
             ctypes.c_size_t(wsb), st)
        if self.cfg.fused:
            call("dbmp_fused_fwd_bwd", ctypes.byref(cv), _ptr(self.prim_info), _ptr(self.atlas.data),
                 _ptr(self.offsets), _ptr(rz._idx), _ptr(self.target), _ptr(self.background), None,
                 _ptr(self.gacc), _ptr(self.loss_dev), skip, st)
        else:
            # plain form: forward kernel, the reference's torch composite + MSE
            # gradient (simple_tile_renderer.py:704-707, loss_functions.py:20-40),
            # backward kernel.  An overflowed bin leaves stale lists, but the
            # Adam step below is skipped and the step replayed, as in fused form.
            call("dbmp_forward", ctypes.byref(cv), _ptr(self.prim_info), _ptr(self.atlas.data), _ptr(self.offsets),
                 _ptr(rz._idx), _ptr(self.color), _ptr(self.alpha), _ptr(self.T_last), _ptr(self.last_pos), st)
            img = self.color if self.background is None else self.color + (1 - self.alpha).unsqueeze(-1) * self.background
            d = img - self.target
            self.loss_dev.copy_((d * d).mean().double().view(1))
            gC = d * (2.0 / d.numel())
            gA = -(gC * self.background).sum(-1) if self.background is not None else None
            call("dbmp_backward", ctypes.byref(cv), _ptr(self.prim_info), _ptr(self.atlas.data), _ptr(self.offsets),
                 _ptr(rz._idx), _ptr(self.T_last), _ptr(self.last_pos), _ptr(gC), _ptr(gA), _ptr(self.radii),
                 _ptr(self.rotations), _ptr(self.opacities), _ptr(self.colors), _ptr(self.gacc),
                 *[_ptr(g) for g in self.grads], st)
        call("dbmp_adam_step", ctypes.byref(cv), ctypes.byref(self.adam_cfg), _ptr(self.gacc), _ptr(self.means2D),
             _ptr(self.radii), _ptr(self.rotations), _ptr(self.opacities), _ptr(self.colors), _ptr(self.adam_m),
             _ptr(self.adam_v), _ptr(self.step_count), skip, st)

    def upload_params(self, host_params: torch.Tensor):
        """Sets the parameters from a pinned host tensor laid out as
        params_flat ((N*8,) f32: centres, radii, rotations, opacity and colour
        logits), without stalling the device: the host-to-device copy runs on
        a copy stream into one of two staging buffers, so it overlaps the work
        already queued, and the current stream only waits for it and copies
        device to device before the next step reads the parameters."""
        if host_params.numel() != self.params_flat.numel():
            raise ValueError(f"{host_params.numel()} values for {self.params_flat.numel()} parameters")
        if not hasattr(self, "_staging"):
            self._copy_stream = torch.cuda.Stream(self.device)
            self._staging = [torch.empty_like(self.params_flat) for _ in range(2)]
            self._staged = [torch.cuda.Event(), torch.cuda.Event()]
            self._consumed = [None, None]
            self._slot = 0
        k = self._slot
        self._slot ^= 1
        cs = self._copy_stream
        if self._consumed[k] is not None:          # the device copy that last read this buffer is done
            cs.wait_event(self._consumed[k])
        with torch.cuda.stream(cs):
            self._staging[k].copy_(host_params.view(-1), non_blocking=True)
        self._staged[k].record(cs)
        cur = torch.cuda.current_stream(self.device)
        cur.wait_event(self._staged[k])
        self.params_flat.copy_(self._staging[k], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(cur)
        self._consumed[k] = ev

    def step(self):
        """Enqueues one fit iteration (no host synchronisation)."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._enqueue()
        self.steps_enqueued += 1

    def capture(self):
        """Captures one iteration in a CUDA graph; later step() calls replay it.

        Uses capture_begin/capture_end directly: the torch.cuda.graph context
        manager also synchronises the device, runs the garbage collector and
        empties the allocator cache on every capture, which costs a serving
        loop up to hundreds of milliseconds per admitted job."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            g.capture_begin()
            try:
                self._enqueue()
            finally:
                g.capture_end()
        torch.cuda.current_stream().wait_stream(s)
        self.graph = g

    def sync(self) -> int:
        """Waits for the queued steps; replays any that a list overflow skipped.
        Returns the number of replayed steps."""
        replayed = 0
        while True:
            done = int(self.step_count.item())
            missing = self.steps_enqueued - done
            if missing <= 0:
                return replayed
            self._grow(self._count())
            self.steps_enqueued = done
            for _ in range(missing):
                self.step()
            replayed += missing

    def loss(self) -> float:
        return float(self.loss_dev.item())

    def stage_result(self):
        """Enqueues copies of the device step count and loss into pinned host
        memory on the current stream; once that stream has passed them,
        staged_result() reads them without synchronising."""
        if self._host_state is None:
            self._host_state = (torch.zeros(1, dtype=torch.int32).pin_memory(),
                                torch.zeros(1, dtype=torch.float64).pin_memory())
        self._host_state[0].copy_(self.step_count, non_blocking=True)
        self._host_state[1].copy_(self.loss_dev, non_blocking=True)

    def staged_result(self):
        """(completed steps, loss) as staged by the last stage_result()."""
        return int(self._host_state[0][0]), float(self._host_state[1][0])

    def render(self) -> torch.Tensor:
        """Current image (H,W,3) over the background (forward only)."""
        color, alpha, _ = self.rz.forward(self.means2D, self.radii, self.rotations, self.opacities, self.colors,
                                          self.sel, self.atlas)
        if self.background is None:
            return color
        return color + (1 - alpha).unsqueeze(-1) * self.background

    def params(self):
        return dict(means2D=self.means2D, radii=self.radii, rotations=self.rotations, opacities=self.opacities,
                    colors=self.colors)
