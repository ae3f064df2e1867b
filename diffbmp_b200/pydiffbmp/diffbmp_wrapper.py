"""Drop-in for the reference's DiffBMPWrapper (pydiffbmp/diffbmp_wrapper.py)
on the rasterizer's path: ``render`` (:247-343) and ``render_batch``
(:345-435) with the reference's signatures, over this package's
SimpleTileRenderer (one multi-candidate launch per batch).

The reference fills the primitive from files with its asset loaders
(``load_primitive``, :52-130) and the canvas size from its initializers
(``initialize_params``, :132-245); both lie outside the rasterizer's path.
Here the caller hands the loaded bitmaps over with ``set_primitive(S,
colors)`` and sets ``canvas_size``.
"""
from __future__ import annotations

from typing import Optional, Tuple, Union

import torch

from .core.renderer.simple_tile_renderer import SimpleTileRenderer


class DiffBMPWrapper:
    """Functional rendering of bitmap primitives with parameters passed per call."""

    def __init__(self, device: str = "cuda"):
        self.device = torch.device(device)
        self.primitive = None
        self.renderer = None
        self.canvas_size = None

    def set_primitive(self, S: torch.Tensor, colors: Optional[torch.Tensor] = None) -> "DiffBMPWrapper":
        """The primitive bitmaps S (p,Ht,Wt) or (Ht,Wt) in [0,1] and their
        colour maps (p,Ht,Wt,3) -- what the reference's load_primitive keeps
        (diffbmp_wrapper.py:122-127).  Resets the renderer."""
        S = S.to(self.device).float()
        p = S.shape[0] if S.dim() == 3 else 1
        if colors is None:
            colors = torch.zeros(p, S.shape[-2], S.shape[-1], 3, device=self.device)
        self.primitive = {"S": S, "colors": colors.to(self.device).float()}
        self.renderer = None
        return self

    def _background(self, background, H, W):
        if isinstance(background, str):
            if background == "white":
                return torch.ones((H, W, 3), device=self.device, dtype=torch.float32)
            if background == "black":
                return torch.zeros((H, W, 3), device=self.device, dtype=torch.float32)
            if background == "random":
                return torch.rand((H, W, 3), device=self.device, dtype=torch.float32)
            raise ValueError(f"Unknown background type: {background}")
        if isinstance(background, torch.Tensor):
            return background.to(self.device)
        return None

    def _ensure_renderer(self, blur_sigma, tile_size, alpha_upper_bound, c_blend, use_fp16):
        if self.primitive is None:
            raise ValueError("Primitive not set. Call set_primitive() first.")
        if self.canvas_size is None:
            raise ValueError("Canvas size not set: assign canvas_size = (H, W) first.")
        H, W = self.canvas_size
        if self.renderer is None:
            # the reference renders canvases up to 64 px with 12-px tiles so that
            # they have more than 4 tiles (diffbmp_wrapper.py:296-299); the tile
            # sizes here are 16 and 32, and 16 keeps such canvases multi-tile
            ts = 16 if min(H, W) <= 64 else tile_size
            self.renderer = SimpleTileRenderer((H, W), self.primitive["S"], tile_size=ts,
                                               alpha_upper_bound=alpha_upper_bound, device=str(self.device),
                                               use_fp16=use_fp16, sigma=blur_sigma, c_blend=c_blend,
                                               primitive_colors=self.primitive["colors"])
        return self.renderer

    def render(self, x: torch.Tensor, y: torch.Tensor, r: torch.Tensor, theta: torch.Tensor, v: torch.Tensor,
               c: torch.Tensor, background: Optional[Union[str, torch.Tensor]] = "white", blur_sigma: float = 1.0,
               return_alpha: bool = False, tile_size: int = 32, alpha_upper_bound: float = 0.5,
               c_blend: float = 0.0, use_fp16: bool = False) -> torch.Tensor:
        """(H,W,3) image, or (H,W,4) RGBA with return_alpha; differentiable."""
        R = self._ensure_renderer(blur_sigma, tile_size, alpha_upper_bound, c_blend, use_fp16)
        H, W = self.canvas_size
        out = R.render_from_params(x=x, y=y, r=r, theta=theta, v=v, c=c, return_alpha=return_alpha,
                                   I_bg=self._background(background, H, W), sigma=0.0, is_final=False)
        if return_alpha:
            rendered, alpha = out
            return torch.cat([rendered, alpha.unsqueeze(-1)], dim=-1)
        return out

    def render_batch(self, params_list: list, background: Optional[Union[str, torch.Tensor]] = "white",
                     blur_sigma: float = 1.0, return_alpha: bool = False, tile_size: int = 32,
                     alpha_upper_bound: float = 0.5, c_blend: float = 0.0, use_fp16: bool = False) -> list:
        """Renders every (x, y, r, theta, v, c) candidate with one launch.
        Returns the renderer's list for the batch: images, or (image, alpha)
        pairs with return_alpha (as the reference's batch path returns them)."""
        R = self._ensure_renderer(blur_sigma, tile_size, alpha_upper_bound, c_blend, use_fp16)
        H, W = self.canvas_size
        return R.render_from_params_batch(params_list, return_alpha=return_alpha,
                                          I_bg=self._background(background, H, W))
