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

# Reference defaults (pydiffbmp/util/constants.py:24-31): base lr and gains.
LR_GAINS = dict(x=10.0, y=10.0, r=10.0, v=1.5, theta=1.0, c=1.0)


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
                                float(self.W - 1), float(self.H - 1), 2.0, float(min(self.H, self.W) // 4), 1)
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
    def _enqueue(self):
        st = _stream()
        cv = self.cv
        rz = self.rz
        ws, wsb = rz._ws_ptr()
        skip = ctypes.c_void_p(self.flags.data_ptr() + 4)
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
