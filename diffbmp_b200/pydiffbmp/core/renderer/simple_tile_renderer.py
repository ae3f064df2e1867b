"""Drop-in for the reference's SimpleTileRenderer
(pydiffbmp/core/renderer/simple_tile_renderer.py) on libdbmp.so.

Same constructor, attributes and methods on the rasterizer's path:

* ``render_from_params(x, y, r, theta, v, c, return_alpha, I_bg, sigma,
  lr_conf, is_final)`` (reference :173-266): template (N-1-i) % p per
  primitive, the blurred templates unless ``is_final``, background composite
  C + (1-A) I_bg, differentiable in the six parameter tensors;
* ``render_from_params_batch(params_list, return_alpha, I_bg)`` (:268-429):
  the candidates are clamped as there and rendered by ONE forward launch over
  all their tiles (and one backward launch), not a loop over candidates;
* ``optimize_parameters`` / ``_optimize_parameters_whole`` (:913-1228): the
  fit loop -- Adam with the reference's per-parameter gains, ExponentialLR
  decay, the blur schedule, pruning and the clamp -- as CUDA-graph-replayed
  device steps (diffbmp_b200.fitting.ImageFitter).

Differences from the reference, by design: no CPU or PyTorch fallback (a
failing call raises); per-pixel depth is unbounded (``max_prims_per_pixel`` is
accepted and unused); ``use_fp16`` stores the atlas in FP16 and computes in
FP32 (the reference computes everything in half); the colour maps are gathered
per primitive only when ``c_blend > 0``.  As in the reference's CUDA path, the
per-call ``sigma`` argument of render_from_params has no effect (its
TileConfig.sigma is unused by its kernels); the fit loop's blur schedule
re-blurs the templates as the reference's CPU path does.
"""
from __future__ import annotations

from typing import Any, Optional

import numpy as np
import torch

from diffbmp_b200.fitting import FitConfig, ImageFitter, fallback_pool, prune_due
from diffbmp_b200.rasterizer import Atlas, Rasterizer, rasterize, rasterize_batch

MAX_PRIMS_PER_PIXEL = 400          # pydiffbmp/util/constants.py:21 (unused: depth is unbounded here)

# Named backgrounds of _get_background_for_render (simple_tile_renderer.py:862-911),
# the standard RGB values of those colours.
BACKGROUNDS = {"white": (1.0, 1.0, 1.0), "black": (0.0, 0.0, 0.0), "red": (1.0, 0.0, 0.0),
               "orange": (1.0, 0.647, 0.0), "yellow": (1.0, 1.0, 0.0), "green": (0.0, 1.0, 0.0),
               "blue": (0.0, 0.0, 1.0), "indigo": (0.294, 0.0, 0.510), "violet": (0.580, 0.0, 0.827),
               "purple": (0.580, 0.0, 0.827), "gray": (0.5, 0.5, 0.5), "grey": (0.5, 0.5, 0.5),
               "pink": (1.0, 0.753, 0.796), "cyan": (0.0, 1.0, 1.0), "magenta": (1.0, 0.0, 1.0)}


class SimpleTileRenderer:
    """Tile renderer of bitmap primitives over a template atlas S (p,Ht,Wt)."""

    def __init__(self, canvas_size, S: torch.Tensor, tile_size: int = 32, max_prims_per_pixel: int = None,
                 alpha_upper_bound: float = 0.5, device: str = "cuda", use_fp16: bool = False, gamma: float = 1.0,
                 output_path: str = None, sigma: float = 0.0, c_blend: float = 0.0,
                 primitive_colors: Optional[torch.Tensor] = None):
        self.H, self.W = (int(v) for v in canvas_size)
        self.alpha_upper_bound = float(alpha_upper_bound)
        self.device = torch.device(device)
        self.use_fp16 = bool(use_fp16)
        self.gamma = gamma
        self.output_path = output_path
        self.c_blend = float(c_blend)
        self.c_o = primitive_colors.clone().to(self.device).float() if primitive_colors is not None else None
        self.tile_size = int(tile_size)
        self.tiles_h = (self.H + self.tile_size - 1) // self.tile_size
        self.tiles_w = (self.W + self.tile_size - 1) // self.tile_size
        self.max_prims_per_pixel = max_prims_per_pixel if max_prims_per_pixel is not None else MAX_PRIMS_PER_PIXEL
        S = S.to(self.device)
        self.S = S.half() if self.use_fp16 else S
        self.sigma = float(sigma)
        # storage of the precision form: FP16 texels with FP32 arithmetic
        kind = "f16q" if self.use_fp16 else "f32"
        self._atlas = Atlas(S.float(), kind)
        self._atlas_blurred = Atlas(S.float(), kind, sigma=self.sigma) if self.sigma > 0.0 else None
        self.S_blurred = self._atlas_blurred.templates.to(self.S.dtype) if self._atlas_blurred is not None else None
        # content bboxes of the unblurred templates (vector_renderer.py:103-104)
        self.primitive_bboxes = [tuple(b) for b in self._atlas.bbox.tolist()]
        self._rz = Rasterizer(self.H, self.W, self.tile_size, self.alpha_upper_bound, device=self.device)
        self.cuda_rasterizer = self._rz

    # -- helpers -------------------------------------------------------------
    def _num_templates(self) -> int:
        return self._atlas.P

    def _global_bmp_sel(self, N: int) -> torch.Tensor:
        """Template of primitive i: (N-1-i) % p (simple_tile_renderer.py:221-224)."""
        return (torch.arange(N, device=self.device, dtype=torch.int32) % self._num_templates()).flip(0).contiguous()

    def _atlas_for(self, is_final: bool) -> Atlas:
        return self._atlas_blurred if (self._atlas_blurred is not None and not is_final) else self._atlas

    def _colour_maps(self, sel: torch.Tensor):
        if self.c_blend > 0.0 and self.c_o is not None:
            return self.c_o[sel.long()]
        return None

    def _out(self, color, alpha, I_bg, return_alpha):
        out = color if I_bg is None else color + (1 - alpha).unsqueeze(-1) * I_bg.to(color.dtype)
        if self.use_fp16:
            out, alpha = out.half(), alpha.half()
        return (out, alpha) if return_alpha else out

    def _clamp_params_inplace(self, x, y, r):
        """x in [0, W-1], y in [0, H-1], r in [2, min(H,W)//4] (simple_tile_renderer.py:122-128)."""
        with torch.no_grad():
            x.clamp_(0.0, float(self.W - 1))
            y.clamp_(0.0, float(self.H - 1))
            r.clamp_(2.0, float(min(self.H, self.W) // 4))

    # -- rendering -------------------------------------------------------------
    def render_from_params(self, x: torch.Tensor, y: torch.Tensor, r: torch.Tensor, theta: torch.Tensor,
                           v: torch.Tensor, c: torch.Tensor, return_alpha: bool = False, I_bg: torch.Tensor = None,
                           sigma: float = 0.0, lr_conf: dict = None, is_final: bool = False):
        """(H,W,3) image, or (image, alpha (H,W)) with return_alpha."""
        N = int(x.shape[0])
        sel = self._global_bmp_sel(N)
        means2D = torch.stack([x.float(), y.float()], dim=1)
        cmap = self._colour_maps(sel)
        color, alpha = rasterize(means2D, r.float(), theta.float(), v.float(), c.float(), sel,
                                 self._atlas_for(is_final), self._rz, None, cmap, self.c_blend if cmap is not None
                                 else 0.0)
        return self._out(color, alpha, I_bg, return_alpha)

    def render_from_params_batch(self, params_list: list, return_alpha: bool = False, I_bg: torch.Tensor = None):
        """List of (x, y, r, theta, v, c) candidates with the same N -> list of
        images (or (image, alpha) pairs); one forward launch for the batch."""
        B = len(params_list)
        if B == 0:
            return []
        N = int(params_list[0][0].shape[0])
        means2D = torch.stack([torch.stack([p[0].float(), p[1].float()], dim=1) for p in params_list], dim=0)
        radii = torch.stack([p[2].float() for p in params_list], dim=0)
        rotations = torch.stack([p[3].float() for p in params_list], dim=0)
        opacities = torch.stack([p[4].float() for p in params_list], dim=0)
        colors = torch.stack([p[5].float() for p in params_list], dim=0)
        # the reference clamps the stacked candidates (values only; the
        # gradients pass through, simple_tile_renderer.py:313-320)
        with torch.no_grad():
            means2D[:, :, 0].clamp_(0.0, float(self.W - 1))
            means2D[:, :, 1].clamp_(0.0, float(self.H - 1))
            radii.clamp_(2.0, float(min(self.H, self.W) // 4))
        sel = self._global_bmp_sel(N)
        cmap = self._colour_maps(sel)
        atlas = self._atlas_blurred if self._atlas_blurred is not None else self._atlas
        color, alpha = rasterize_batch(means2D, radii, rotations, opacities, colors, sel, atlas, self._rz, None, cmap,
                                       self.c_blend if cmap is not None else 0.0)
        return [self._out(color[b], alpha[b], I_bg, return_alpha) for b in range(B)]

    # -- fitting -----------------------------------------------------------------
    def _get_background_for_render(self, bg_type: str = "white", export: bool = False) -> torch.Tensor:
        if bg_type == "random":
            if export:
                return torch.ones((self.H, self.W, 3), device=self.device)
            return torch.rand((self.H, self.W, 3), device=self.device)
        if bg_type not in BACKGROUNDS:
            raise ValueError(f"Unsupported bg_type: {bg_type}. Supported: {sorted(BACKGROUNDS) + ['random']}")
        return torch.tensor(BACKGROUNDS[bg_type], device=self.device).expand(self.H, self.W, 3).contiguous()

    def optimize_parameters(self, x, y, r, v, theta, c, target_image, opt_conf: dict, target_binary_mask=None,
                            initializer: Optional[Any] = None):
        """Fits the parameters to target_image (vector_renderer.py:1128-1148)."""
        return self._optimize_parameters_whole(x, y, r, v, theta, c, target_image, opt_conf, target_binary_mask,
                                               initializer)

    def _optimize_parameters_whole(self, x, y, r, v, theta, c, target_image, opt_conf: dict,
                                   target_binary_mask=None, initializer: Optional[Any] = None):
        """The reference's loop (simple_tile_renderer.py:913-1228) on the
        device: num_iterations graph-replayed steps of binning, fused forward +
        L2 loss + backward, Adam with the per-group gains and ExponentialLR
        decay, the blur schedule, pruning and the clamp.  Returns the fitted
        (x, y, r, v, theta, c), also written into the given tensors.

        The L2 loss (loss_config type "mse", loss_functions.py:20-40) is the
        one the device step fuses.  Pruning draws its replacement rows from
        `initializer.reinitialize_subset` up front (enough for every scheduled
        prune to replace all N primitives), or, without an initializer, as the
        reference's _fallback_random_init does."""
        loss_type = opt_conf.get("loss_config", {"type": "mse"}).get("type", "mse")
        if loss_type != "mse":
            raise ValueError(f"loss type {loss_type!r}: the device fit step computes the L2 loss (mse) only")
        if target_image.shape[-1] != 3:
            raise ValueError("the device fit step takes an RGB target (H,W,3)")
        N = int(x.shape[0])
        cfg = FitConfig.from_opt_conf(opt_conf, pool=np.zeros((1, 8), np.float32),
                                      tile_size=self.tile_size, alpha_max=self.alpha_upper_bound)
        if cfg.prune is not None:
            prunes = sum(1 for k in range(cfg.num_iterations) if prune_due(cfg, k))
            rows = max(1, prunes * N)
            if initializer is not None and hasattr(initializer, "reinitialize_subset"):
                nx, ny, nr, nv, nth, nc = initializer.reinitialize_subset(rows, target_image[:, :, :3], self.device)
                pool = torch.cat([t.reshape(rows, -1).float().to(self.device) for t in (nx, ny, nr, nth, nv, nc)], 1)
            else:
                pool = torch.from_numpy(fallback_pool(np.random.default_rng(), self.H, self.W, rows))
            cfg.prune.pool = pool
        sel = self._global_bmp_sel(N)
        atlas = self._atlas_blurred if (self._atlas_blurred is not None and cfg.blur == "none") else self._atlas
        bg = self._get_background_for_render(opt_conf.get("bg_color", "white"))
        means2D = torch.stack([x.detach().float(), y.detach().float()], dim=1)
        job = ImageFitter(means2D, r.detach().float(), theta.detach().float(), v.detach().float(),
                          c.detach().float(), sel, atlas, target_image.to(self.device).float(), bg, cfg,
                          device=self.device)
        for k in range(cfg.num_iterations):
            if k == 1:
                job.capture()           # iteration 0 ran eagerly; the rest replay one graph
            job.step()
        job.sync()
        self.last_loss = job.loss()
        with torch.no_grad():
            x.copy_(job.means2D[:, 0]); y.copy_(job.means2D[:, 1]); r.copy_(job.radii)
            theta.copy_(job.rotations); v.copy_(job.opacities); c.copy_(job.colors)
        return x, y, r, v, theta, c
