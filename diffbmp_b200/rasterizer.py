"""Torch-facing host layer over libdbmp.so.

PyTorch supplies device memory and streams; every computation is one of the
library's CUDA kernels.  Tensors must be CUDA tensors; nothing here falls
back to a CPU or PyTorch implementation.

Main objects:

* ``Atlas``       -- a template atlas resident on the device in one storage
                     kind (f32 reference layout, or f32/f16/bf16 bilinear quads)
                     plus its per-template content bboxes.
* ``Rasterizer``  -- one canvas (H, W, tile size): binning, forward, backward
                     and the fused fit step; owns the scratch it reuses.
* ``rasterize``   -- autograd entry point (``RasterizeFunction``).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib
from ._lib import (ATLAS_BF16_PAIR, ATLAS_BF16_QUAD, ATLAS_F16_PAIR, ATLAS_F16_QUAD, ATLAS_F32, ATLAS_F32_QUAD,
                   BIN_CONTENT, BIN_CONTENT_REF, BIN_CULL, Canvas, DbmpError, call, lib)

# Atlas storage kinds: "f32" is the reference layout; the precision form
# stores half / bfloat16 texels as horizontal pairs ("f16", "bf16", two 4-byte
# loads per bilinear sample) or as full bilinear quads ("f16q", "bf16q", "f32q").
KIND_NAMES = {"f32": ATLAS_F32, "f32q": ATLAS_F32_QUAD, "f16q": ATLAS_F16_QUAD, "bf16q": ATLAS_BF16_QUAD,
              "f16": ATLAS_F16_PAIR, "bf16": ATLAS_BF16_PAIR}

DEFAULT_T_STOP = 1e-6   # image error <= t_stop * max colour, well inside the 1e-5 parity bar


def _ptr(t: Optional[torch.Tensor]):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _need_cuda(*ts):
    for t in ts:
        if t is not None and not t.is_cuda:
            raise ValueError("diffbmp_b200 kernels need CUDA tensors (no CPU fallback exists)")


def _f32(t: torch.Tensor) -> torch.Tensor:
    return t.detach().to(torch.float32).contiguous()


class Atlas:
    """Template atlas on the device.  ``templates``: (P,Ht,Wt) or (Ht,Wt).
    ``sigma`` > 0 renders with Gaussian-blurred templates while the content
    bboxes (binning) stay those of the unblurred ones, as the reference's
    VectorRenderer does (vector_renderer.py:80-104)."""

    def __init__(self, templates: torch.Tensor, kind: str | int = "f32", sigma: float = 0.0):
        t = templates if templates.dim() == 3 else templates.unsqueeze(0)
        _need_cuda(t)
        self.templates = _f32(t)
        self.sigma = float(sigma)
        self.P, self.Ht, self.Wt = (int(v) for v in self.templates.shape)
        self.kind = KIND_NAMES[kind] if isinstance(kind, str) else int(kind)
        st = _stream()
        self.bbox = torch.empty((self.P, 4), dtype=torch.float32, device=t.device)
        call("dbmp_template_bboxes", _ptr(self.templates), self.P, self.Ht, self.Wt, _ptr(self.bbox), st)
        if self.sigma > 0.0:
            blurred = torch.empty_like(self.templates)
            call("dbmp_template_blur", _ptr(self.templates), self.P, self.Ht, self.Wt, ctypes.c_float(self.sigma),
                 _ptr(blurred), st)
            self.templates = blurred
        if self.kind == ATLAS_F32:
            self.data = self.templates
        else:
            nbytes = int(lib.dbmp_atlas_bytes(self.P, self.Ht, self.Wt, self.kind))
            self.data = torch.empty(nbytes, dtype=torch.uint8, device=t.device)
            call("dbmp_atlas_pack", _ptr(self.templates), self.P, self.Ht, self.Wt, self.kind, _ptr(self.data), st)

    def private_copy(self) -> "Atlas":
        """An atlas of the same kind, templates and content bboxes with its own
        texel buffer (filled by the caller), for a job that re-derives its
        texels every step (the fit loop's blur schedule)."""
        a = Atlas.__new__(Atlas)
        a.templates, a.sigma, a.bbox = self.templates, self.sigma, self.bbox
        a.P, a.Ht, a.Wt, a.kind = self.P, self.Ht, self.Wt, self.kind
        a.data = torch.empty_like(self.data)
        return a

    def with_kind(self, kind) -> "Atlas":
        a = Atlas(self.templates, kind)
        a.bbox, a.sigma = self.bbox, self.sigma   # keep the unblurred content bboxes
        return a


@dataclass
class TileLists:
    """CSR tile lists of one binning: offsets (T+1) and indices (>= L entries)."""
    offsets: torch.Tensor
    indices: torch.Tensor
    length: int

    def mapping_tensor(self) -> torch.Tensor:
        """The reference's int32 wire format [T+1, L, offsets..., indices...]."""
        head = torch.tensor([self.offsets.numel(), self.length], dtype=torch.int32, device=self.offsets.device)
        return torch.cat([head, self.offsets, self.indices[: self.length]])


@dataclass
class BatchState:
    """Forward state of a batch of candidates (Rasterizer.forward_batch):
    records (B*N,16), lists offsets (B,T+1) / indices (B,stride), per-pixel
    T_last / last_pos (B,H,W), the colour maps of a blended render."""
    prim_info: torch.Tensor
    offsets: torch.Tensor
    indices: torch.Tensor
    T_last: torch.Tensor
    last_pos: torch.Tensor
    colors_orig: Optional[torch.Tensor] = None
    cmap_stride: int = 0
    c_blend: float = 0.0

    @property
    def batch(self) -> int:
        return int(self.offsets.shape[0])


@dataclass
class ForwardState:
    prim_info: torch.Tensor
    lists: TileLists
    T_last: torch.Tensor
    last_pos: torch.Tensor
    colors_orig: Optional[torch.Tensor] = None   # colour maps of a blended render
    c_blend: float = 0.0


def lists_from_mapping(mapping: torch.Tensor, num_tiles: int, num_prims: int) -> TileLists:
    """Views a reference mapping tensor (simple_tile_renderer.py:757-766) as
    TileLists after validating it, so that no kernel can read outside it."""
    _need_cuda(mapping)
    m = mapping.to(torch.int32).contiguous()
    if m.dim() != 1 or m.numel() < num_tiles + 3:
        raise ValueError(f"tile mapping has {m.numel()} entries, need at least {num_tiles + 3}")
    offs = m[2:3 + num_tiles]
    idx = m[3 + num_tiles:]
    head = torch.stack([m[0], m[1], offs.min(), offs.max(), offs[-1]]).tolist()
    T1, L, omin, omax, olast = head
    if T1 != num_tiles + 1:
        raise ValueError(f"tile mapping is for {T1 - 1} tiles, canvas has {num_tiles}")
    if L != idx.numel() or olast != L or omin < 0 or omax > L:
        raise ValueError(f"inconsistent tile mapping (L={L}, indices={idx.numel()}, offsets in [{omin},{omax}], "
                         f"last offset {olast})")
    if idx.numel() == 0:
        idx = torch.zeros(1, dtype=torch.int32, device=m.device)
    return TileLists(offs, idx, int(L))


class Rasterizer:
    """One canvas.  Holds the binning capacity and scratch between calls."""

    def __init__(self, height: int, width: int, tile_size: int = 32, alpha_max: float = 1.0,
                 t_stop: float = DEFAULT_T_STOP, bin_mode: int = BIN_CONTENT, device=None):
        self.H, self.W, self.ts = int(height), int(width), int(tile_size)
        self.alpha_max = float(alpha_max)
        self.t_stop = float(t_stop)
        self.bin_mode = int(bin_mode)
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.tiles_x = (self.W + self.ts - 1) // self.ts
        self.tiles_y = (self.H + self.ts - 1) // self.ts
        self.T = self.tiles_x * self.tiles_y
        self.capacity = 0
        self._ws = None
        self._idx = None
        self._small = torch.zeros(2, dtype=torch.int32, device=self.device)   # total L, overflow flag

    def canvas(self, N: int, atlas: Atlas) -> Canvas:
        return Canvas(self.H, self.W, self.ts, int(N), atlas.P, atlas.Ht, atlas.Wt, atlas.kind, self.bin_mode,
                      self.alpha_max, self.t_stop, 0)

    # -- binning -----------------------------------------------------------
    def _ensure(self, cv: Canvas, cap: int):
        if cap > self.capacity or self._ws is None:
            self.capacity = int(cap)
            nbytes = int(lib.dbmp_bin_workspace_bytes(ctypes.byref(cv), self.capacity))
            self._ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=self.device)
            self._idx = torch.empty(max(self.capacity, 1), dtype=torch.int32, device=self.device)
        nbytes = int(lib.dbmp_bin_workspace_bytes(ctypes.byref(cv), self.capacity))
        if self._ws.numel() < nbytes + 256:
            self._ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=self.device)

    def _ws_ptr(self):
        base = self._ws.data_ptr()
        return ctypes.c_void_p((base + 255) & ~255), self._ws.numel() - 256

    def bin(self, means2D, radii, rotations, opacities, colors, sel, atlas: Atlas, stream=None):
        """Device binning.  Returns (prim_info, TileLists).  Synchronises once
        to learn the list length (the reference reads it with .item() too)."""
        N = int(radii.shape[0])
        cv = self.canvas(N, atlas)
        st = _stream(stream)
        prim_info = torch.empty((max(N, 1), 16), dtype=torch.float32, device=self.device)
        offsets = torch.empty(self.T + 1, dtype=torch.int32, device=self.device)
        args = [_ptr(means2D), _ptr(radii), _ptr(rotations), _ptr(opacities), _ptr(colors), _ptr(sel),
                _ptr(atlas.bbox), _ptr(prim_info), _ptr(offsets)]
        for _ in range(3):
            self._ensure(cv, self.capacity)
            ws, wsb = self._ws_ptr()
            # each binning owns its index list: a ForwardState must stay valid
            # while later forwards on this canvas run (batch APIs keep several)
            indices = torch.empty(max(self.capacity, 1), dtype=torch.int32, device=self.device)
            call("dbmp_bin", ctypes.byref(cv), *args, _ptr(indices), ctypes.c_longlong(self.capacity),
                 _ptr(self._small), ctypes.c_void_p(self._small.data_ptr() + 4), ws, ctypes.c_size_t(wsb), st)
            L, overflow = self._small.tolist()
            if not overflow:
                return prim_info, TileLists(offsets, indices, int(L))
            self._ensure(cv, int(L * 1.25) + 4096)
        raise DbmpError("binning capacity did not converge")

    def prepare(self, means2D, radii, rotations, opacities, colors, sel, atlas: Atlas, stream=None):
        N = int(radii.shape[0])
        cv = self.canvas(N, atlas)
        prim_info = torch.empty((max(N, 1), 16), dtype=torch.float32, device=self.device)
        call("dbmp_prepare", ctypes.byref(cv), _ptr(means2D), _ptr(radii), _ptr(rotations), _ptr(opacities),
             _ptr(colors), _ptr(sel), _ptr(prim_info), _stream(stream))
        return prim_info

    # -- forward / backward -------------------------------------------------
    def forward(self, means2D, radii, rotations, opacities, colors, sel, atlas: Atlas,
                mapping: Optional[torch.Tensor] = None, stream=None, colors_orig: Optional[torch.Tensor] = None,
                c_blend: float = 0.0):
        """Returns (color (H,W,3), alpha (H,W), ForwardState).  With
        colors_orig (N,Ht,Wt,3) and c_blend in (0, 1], fragment colours blend
        the per-primitive colour maps (dbmp_forward_blend)."""
        _need_cuda(means2D, radii, rotations, opacities, colors, sel)
        N = int(radii.shape[0])
        cmap = self._colour_maps(colors_orig, c_blend, N, atlas)
        if mapping is not None and mapping.numel() > 0:
            lists = lists_from_mapping(mapping, self.T, N)
            prim_info = self.prepare(means2D, radii, rotations, opacities, colors, sel, atlas, stream)
        else:
            prim_info, lists = self.bin(means2D, radii, rotations, opacities, colors, sel, atlas, stream)
        cv = self.canvas(N, atlas)
        color = torch.empty((self.H, self.W, 3), dtype=torch.float32, device=self.device)
        alpha = torch.empty((self.H, self.W), dtype=torch.float32, device=self.device)
        T_last = torch.empty((self.H, self.W), dtype=torch.float32, device=self.device)
        last_pos = torch.empty((self.H, self.W), dtype=torch.int32, device=self.device)
        if cmap is None:
            call("dbmp_forward", ctypes.byref(cv), _ptr(prim_info), _ptr(atlas.data), _ptr(lists.offsets),
                 _ptr(lists.indices), _ptr(color), _ptr(alpha), _ptr(T_last), _ptr(last_pos), _stream(stream))
            return color, alpha, ForwardState(prim_info, lists, T_last, last_pos)
        call("dbmp_forward_blend", ctypes.byref(cv), _ptr(prim_info), _ptr(atlas.data), _ptr(lists.offsets),
             _ptr(lists.indices), _ptr(cmap), ctypes.c_float(c_blend), _ptr(color), _ptr(alpha), _ptr(T_last),
             _ptr(last_pos), _stream(stream))
        return color, alpha, ForwardState(prim_info, lists, T_last, last_pos, cmap, float(c_blend))

    # -- batches of candidates -------------------------------------------------
    def bin_batch(self, means2D, radii, rotations, opacities, colors, sel, atlas: Atlas, stream=None):
        """Device binning of B candidates (leading dimension of every parameter
        tensor; sel (N) shared or (B,N)) into slots of shared buffers: records
        (B*N,16), offsets (B,T+1), indices (B,capacity).  One host
        synchronisation reads the B list lengths."""
        B, N = int(radii.shape[0]), int(radii.shape[1])
        cv = self.canvas(N, atlas)
        st = _stream(stream)
        prim = torch.empty((max(B * N, 1), 16), dtype=torch.float32, device=self.device)
        offsets = torch.empty((B, self.T + 1), dtype=torch.int32, device=self.device)
        small = torch.zeros((B, 2), dtype=torch.int32, device=self.device)    # per candidate: L, overflow
        sel2 = sel if sel.dim() == 2 else sel.unsqueeze(0).expand(B, -1)
        for _ in range(3):
            self._ensure(cv, self.capacity)
            ws, wsb = self._ws_ptr()
            cap = max(self.capacity, 1)
            indices = torch.empty((B, cap), dtype=torch.int32, device=self.device)
            for b in range(B):
                call("dbmp_bin", ctypes.byref(cv), _ptr(means2D[b]), _ptr(radii[b]), _ptr(rotations[b]),
                     _ptr(opacities[b]), _ptr(colors[b]), _ptr(sel2[b]), _ptr(atlas.bbox),
                     ctypes.c_void_p(prim.data_ptr() + b * N * 64), _ptr(offsets[b]), _ptr(indices[b]),
                     ctypes.c_longlong(self.capacity), _ptr(small[b]), ctypes.c_void_p(small[b].data_ptr() + 4),
                     ws, ctypes.c_size_t(wsb), st)
            Ls = small.cpu()
            if not bool(Ls[:, 1].any()):
                return prim, offsets, indices
            self._ensure(cv, int(int(Ls[:, 0].max()) * 1.25) + 4096)
        raise DbmpError("binning capacity did not converge")

    def forward_batch(self, means2D, radii, rotations, opacities, colors, sel, atlas: Atlas, mappings=None,
                      stream=None, colors_orig: Optional[torch.Tensor] = None, c_blend: float = 0.0):
        """B candidates of this canvas in one launch.  means2D (B,N,2), radii /
        rotations / opacities (B,N), colors (B,N,3), sel (N) or (B,N);
        mappings: None (device binning) or B reference mapping tensors;
        colors_orig (N,Ht,Wt,3) shared or (B,N,Ht,Wt,3).  Returns
        (color (B,H,W,3), alpha (B,H,W), BatchState)."""
        _need_cuda(means2D, radii, rotations, opacities, colors, sel)
        B, N = int(radii.shape[0]), int(radii.shape[1])
        st = _stream(stream)
        if mappings is not None and len(mappings) > 0:
            if len(mappings) != B:
                raise ValueError(f"{len(mappings)} mappings for {B} candidates")
            lists = [lists_from_mapping(m, self.T, N) for m in mappings]
            stride = max(max(l.length for l in lists), 1)
            offsets = torch.stack([l.offsets for l in lists])
            indices = torch.zeros((B, stride), dtype=torch.int32, device=self.device)
            for b, l in enumerate(lists):
                indices[b, :l.length] = l.indices[:l.length]
            prim = torch.empty((max(B * N, 1), 16), dtype=torch.float32, device=self.device)
            cv = self.canvas(N, atlas)
            sel2 = sel if sel.dim() == 2 else sel.unsqueeze(0).expand(B, -1)
            for b in range(B):
                call("dbmp_prepare", ctypes.byref(cv), _ptr(means2D[b]), _ptr(radii[b]), _ptr(rotations[b]),
                     _ptr(opacities[b]), _ptr(colors[b]), _ptr(sel2[b]),
                     ctypes.c_void_p(prim.data_ptr() + b * N * 64), st)
        else:
            prim, offsets, indices = self.bin_batch(means2D, radii, rotations, opacities, colors, sel, atlas, stream)
        cmap, cstride = None, 0
        if colors_orig is not None and colors_orig.numel() > 0 and float(c_blend) > 0.0:
            if colors_orig.dim() == 5:
                cmap = self._colour_maps(colors_orig.reshape(B * N, *colors_orig.shape[2:]), c_blend, B * N, atlas)
                cstride = N * atlas.Ht * atlas.Wt * 3
            else:
                cmap = self._colour_maps(colors_orig, c_blend, N, atlas)
        cv = self.canvas(N, atlas)
        dev = self.device
        color = torch.empty((B, self.H, self.W, 3), dtype=torch.float32, device=dev)
        alpha = torch.empty((B, self.H, self.W), dtype=torch.float32, device=dev)
        T_last = torch.empty((B, self.H, self.W), dtype=torch.float32, device=dev)
        last_pos = torch.empty((B, self.H, self.W), dtype=torch.int32, device=dev)
        call("dbmp_forward_batch", ctypes.byref(cv), B, _ptr(prim), _ptr(atlas.data), _ptr(offsets), _ptr(indices),
             ctypes.c_longlong(indices.shape[1]), _ptr(cmap), ctypes.c_longlong(cstride),
             ctypes.c_float(c_blend if cmap is not None else 0.0), _ptr(color), _ptr(alpha), _ptr(T_last),
             _ptr(last_pos), st)
        return color, alpha, BatchState(prim, offsets, indices, T_last, last_pos, cmap, cstride,
                                        float(c_blend) if cmap is not None else 0.0)

    def backward_batch(self, state: BatchState, grad_color, grad_alpha, radii, rotations, opacities, colors,
                       atlas: Atlas, stream=None):
        """The five gradients of each candidate, in one launch: (B,N,2),
        (B,N), (B,N), (B,N), (B,N,3)."""
        B, N = int(radii.shape[0]), int(radii.shape[1])
        cv = self.canvas(N, atlas)
        dev = self.device
        gc = _f32(grad_color)
        ga = _f32(grad_alpha) if grad_alpha is not None else None
        acc = torch.empty((max(B * N, 1), 8), dtype=torch.float64, device=dev)
        outs = [torch.empty(sh, dtype=torch.float32, device=dev)
                for sh in ((B, N, 2), (B, N), (B, N), (B, N), (B, N, 3))]
        call("dbmp_backward_batch", ctypes.byref(cv), B, _ptr(state.prim_info), _ptr(atlas.data),
             _ptr(state.offsets), _ptr(state.indices), ctypes.c_longlong(state.indices.shape[1]),
             _ptr(state.colors_orig), ctypes.c_longlong(state.cmap_stride), ctypes.c_float(state.c_blend),
             _ptr(state.T_last), _ptr(state.last_pos), _ptr(gc), _ptr(ga), _ptr(radii), _ptr(rotations),
             _ptr(opacities), _ptr(colors), _ptr(acc), *[_ptr(o) for o in outs], _stream(stream))
        return tuple(outs)

    @staticmethod
    def _colour_maps(colors_orig, c_blend, N, atlas: Atlas):
        """The (N,Ht,Wt,3) f32 colour maps of a blended render, or None."""
        if colors_orig is None or colors_orig.numel() == 0 or float(c_blend) <= 0.0:
            return None
        if not 0.0 < float(c_blend) <= 1.0:
            raise ValueError(f"c_blend {c_blend} outside [0, 1]")
        _need_cuda(colors_orig)
        cm = _f32(colors_orig)
        if cm.numel() != N * atlas.Ht * atlas.Wt * 3:
            raise ValueError(f"colors_orig has {cm.numel()} values, expected N*Ht*Wt*3 = "
                             f"{N}*{atlas.Ht}*{atlas.Wt}*3")
        return cm

    def backward(self, state: ForwardState, grad_color, grad_alpha, radii, rotations, opacities, colors,
                 atlas: Atlas, stream=None):
        """Returns the reference's five gradients: (means2D (N,2), radii (N),
        rotations (N), opacities (N), colors (N,3)), float32."""
        N = int(radii.shape[0])
        cv = self.canvas(N, atlas)
        dev = self.device
        gc = _f32(grad_color)
        ga = _f32(grad_alpha) if grad_alpha is not None else None
        acc = torch.empty((max(N, 1), 8), dtype=torch.float64, device=dev)
        g_means = torch.empty((N, 2), dtype=torch.float32, device=dev)
        g_r = torch.empty(N, dtype=torch.float32, device=dev)
        g_rot = torch.empty(N, dtype=torch.float32, device=dev)
        g_op = torch.empty(N, dtype=torch.float32, device=dev)
        g_col = torch.empty((N, 3), dtype=torch.float32, device=dev)
        if state.colors_orig is None:
            call("dbmp_backward", ctypes.byref(cv), _ptr(state.prim_info), _ptr(atlas.data),
                 _ptr(state.lists.offsets), _ptr(state.lists.indices), _ptr(state.T_last), _ptr(state.last_pos),
                 _ptr(gc), _ptr(ga), _ptr(radii), _ptr(rotations), _ptr(opacities), _ptr(colors), _ptr(acc),
                 _ptr(g_means), _ptr(g_r), _ptr(g_rot), _ptr(g_op), _ptr(g_col), _stream(stream))
        else:
            call("dbmp_backward_blend", ctypes.byref(cv), _ptr(state.prim_info), _ptr(atlas.data),
                 _ptr(state.lists.offsets), _ptr(state.lists.indices), _ptr(state.colors_orig),
                 ctypes.c_float(state.c_blend), _ptr(state.T_last), _ptr(state.last_pos),
                 _ptr(gc), _ptr(ga), _ptr(radii), _ptr(rotations), _ptr(opacities), _ptr(colors), _ptr(acc),
                 _ptr(g_means), _ptr(g_r), _ptr(g_rot), _ptr(g_op), _ptr(g_col), _stream(stream))
        return g_means, g_r, g_rot, g_op, g_col


class RasterizeFunction(torch.autograd.Function):
    """Differentiable render of bitmap primitives (hand-written backward).

    forward(means2D (N,2), radii (N), rotations (N), opacities (N), colors (N,3),
            sel (N) int, atlas, rasterizer, mapping, colors_orig, c_blend)
        -> (color (H,W,3), alpha (H,W))
    Gradients flow to the five parameter tensors, as in the reference's
    TileRasterizerFunction (cuda_tile_rasterizer/__init__.py:254-340); the
    colour maps colors_orig get none, as there.
    """

    @staticmethod
    def forward(ctx, means2D, radii, rotations, opacities, colors, sel, atlas, rasterizer, mapping=None,
                colors_orig=None, c_blend=0.0):
        m, r, th, v, c = (_f32(t) for t in (means2D, radii, rotations, opacities, colors))
        s = sel.detach().to(torch.int32).contiguous()
        color, alpha, state = rasterizer.forward(m.view(-1, 2), r.view(-1), th.view(-1), v.view(-1),
                                                 c.view(-1, 3), s.view(-1), atlas, mapping, None,
                                                 None if colors_orig is None else colors_orig.detach(),
                                                 float(c_blend))
        ctx.state = state
        ctx.atlas = atlas
        ctx.rasterizer = rasterizer
        ctx.shapes = (means2D.shape, radii.shape, rotations.shape, opacities.shape, colors.shape)
        ctx.save_for_backward(r, th, v, c)
        return color, alpha

    @staticmethod
    def backward(ctx, grad_color, grad_alpha):
        r, th, v, c = ctx.saved_tensors
        rz: Rasterizer = ctx.rasterizer
        if grad_color is None:
            grad_color = torch.zeros((rz.H, rz.W, 3), dtype=torch.float32, device=r.device)
        gm, gr, gth, gv, gc = rz.backward(ctx.state, grad_color, grad_alpha, r.view(-1), th.view(-1), v.view(-1),
                                          c.view(-1, 3), ctx.atlas)
        sh = ctx.shapes
        return (gm.view(sh[0]), gr.view(sh[1]), gth.view(sh[2]), gv.view(sh[3]), gc.view(sh[4]),
                None, None, None, None, None, None)


class RasterizeBatchFunction(torch.autograd.Function):
    """Differentiable render of B candidates in one launch per direction.

    forward(means2D (B,N,2), radii (B,N), rotations (B,N), opacities (B,N),
            colors (B,N,3), sel (N) or (B,N), atlas, rasterizer, mappings,
            colors_orig, c_blend) -> (color (B,H,W,3), alpha (B,H,W))
    Gradients flow to the five parameter tensors of every candidate, as in the
    reference's TileRasterizerBatchFunction (cuda_tile_rasterizer/__init__.py:
    124-252), whose backward loops over the candidates.
    """

    @staticmethod
    def forward(ctx, means2D, radii, rotations, opacities, colors, sel, atlas, rasterizer, mappings=None,
                colors_orig=None, c_blend=0.0):
        B = int(radii.shape[0])
        m, r, th, v, c = (_f32(t) for t in (means2D, radii, rotations, opacities, colors))
        s = sel.detach().to(torch.int32).contiguous()
        color, alpha, state = rasterizer.forward_batch(m.view(B, -1, 2), r.view(B, -1), th.view(B, -1),
                                                       v.view(B, -1), c.view(B, -1, 3), s, atlas, mappings, None,
                                                       None if colors_orig is None else colors_orig.detach(),
                                                       float(c_blend))
        ctx.state, ctx.atlas, ctx.rasterizer = state, atlas, rasterizer
        ctx.shapes = (means2D.shape, radii.shape, rotations.shape, opacities.shape, colors.shape)
        ctx.save_for_backward(r, th, v, c)
        return color, alpha

    @staticmethod
    def backward(ctx, grad_color, grad_alpha):
        r, th, v, c = ctx.saved_tensors
        rz: Rasterizer = ctx.rasterizer
        B = int(ctx.state.batch)
        if grad_color is None:
            grad_color = torch.zeros((B, rz.H, rz.W, 3), dtype=torch.float32, device=r.device)
        g = rz.backward_batch(ctx.state, grad_color, grad_alpha, r.view(B, -1), th.view(B, -1), v.view(B, -1),
                              c.view(B, -1, 3), ctx.atlas)
        sh = ctx.shapes
        return (g[0].view(sh[0]), g[1].view(sh[1]), g[2].view(sh[2]), g[3].view(sh[3]), g[4].view(sh[4]),
                None, None, None, None, None, None)


def rasterize_batch(means2D, radii, rotations, opacities, colors, sel, atlas: Atlas, rasterizer: Rasterizer,
                    mappings=None, colors_orig: Optional[torch.Tensor] = None, c_blend: float = 0.0):
    return RasterizeBatchFunction.apply(means2D, radii, rotations, opacities, colors, sel, atlas, rasterizer,
                                        mappings, colors_orig, c_blend)


def rasterize(means2D, radii, rotations, opacities, colors, sel, atlas: Atlas, rasterizer: Rasterizer,
              mapping: Optional[torch.Tensor] = None, colors_orig: Optional[torch.Tensor] = None,
              c_blend: float = 0.0):
    return RasterizeFunction.apply(means2D, radii, rotations, opacities, colors, sel, atlas, rasterizer, mapping,
                                   colors_orig, c_blend)
