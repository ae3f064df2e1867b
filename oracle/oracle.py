"""TEST INFRASTRUCTURE -- the CPU oracle for DiffBMP's tile rasterizer.

ctypes front end over ``libdbmp_oracle.so`` (built from ``dbmp_oracle.cpp`` by
``make -C oracle``).  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline / reference legs of ``bench.py`` may import this module; the
product package ``diffbmp_b200`` never does.

Every function mirrors one piece of the reference (smhongok/diffbmp):

* ``template_bboxes``  -- pydiffbmp/core/renderer/vector_renderer.py:151-192
* ``world_bboxes``     -- pydiffbmp/core/renderer/vector_renderer.py:194-252
* ``bin_tiles``        -- vector_renderer.py:401-444 + simple_tile_renderer.py:721-766
* ``forward``          -- cuda_tile_rasterizer/cuda_kernels/tile_forward.cu:96-398
* ``backward``         -- cuda_tile_rasterizer/cuda_kernels/tile_backward.cu:102-452
* ``psd_bboxes``       -- cuda_tile_rasterizer/cuda_kernels/psd_export_kernels.cu:12-55
* ``psd_layers``       -- cuda_tile_rasterizer/cuda_kernels/psd_export_kernels.cu:61-198
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libdbmp_oracle.so")

SEM_KERNEL = 0   # the reference CUDA kernels' sampling/cull semantics
SEM_TORCH = 1    # the reference PyTorch per-tile path (grid_sample zeros padding)

BIN_CONTENT = 0  # world bbox of the template's nonzero texels (renderer API)
BIN_CULL = 1     # square cull box (equivalent to the all-primitives default mapping)
BIN_CONTENT_REF = 2  # as BIN_CONTENT with the bbox of template (N-1-i) % P whatever sel says

_lib = None


def build() -> str:
    """Compiles the oracle library if it is missing or stale; returns its path."""
    src = os.path.join(_HERE, "dbmp_oracle.cpp")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE, "libdbmp_oracle.so"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _lib.orc_bin.restype = ctypes.c_longlong
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def template_bboxes(S: np.ndarray) -> np.ndarray:
    S = _f32(S)
    if S.ndim == 2:
        S = S[None]
    P, Ht, Wt = S.shape
    out = np.zeros((P, 4), np.float32)
    lib().orc_template_bboxes(_p(S), P, Ht, Wt, _p(out))
    return out


def world_bboxes(means2D, radii, rot, bbox_sel, tbbox) -> np.ndarray:
    means2D, radii, rot, tbbox = _f32(means2D), _f32(radii), _f32(rot), _f32(tbbox)
    bbox_sel = _i32(bbox_sel)
    N = radii.shape[0]
    out = np.zeros((N, 4), np.float32)
    rc = lib().orc_world_bboxes(_p(means2D), _p(radii), _p(rot), _p(bbox_sel), _p(tbbox), N,
                                tbbox.shape[0], _p(out))
    if rc != 0:
        raise ValueError("template index out of range")
    return out


def bin_tiles(H, W, ts, means2D, radii, rot, sel, tbbox, Ht, Wt, mode=BIN_CONTENT):
    """Returns (offsets int32 (T+1,), indices int32 (L,)) in the reference order."""
    means2D, radii, rot, tbbox = _f32(means2D), _f32(radii), _f32(rot), _f32(tbbox)
    sel = _i32(sel)
    N = radii.shape[0]
    T = ((W + ts - 1) // ts) * ((H + ts - 1) // ts)
    offs = np.zeros(T + 1, np.int32)
    L = lib().orc_bin(H, W, ts, _p(means2D), _p(radii), _p(rot), _p(sel), _p(tbbox), N,
                      tbbox.shape[0], Ht, Wt, mode, _p(offs), None, 0)
    idx = np.zeros(max(L, 1), np.int32)
    lib().orc_bin(H, W, ts, _p(means2D), _p(radii), _p(rot), _p(sel), _p(tbbox), N,
                  tbbox.shape[0], Ht, Wt, mode, _p(offs), _p(idx), ctypes.c_longlong(L))
    return offs, idx[:L]


def mapping_tensor(offs: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """The reference wire format: int32 [T+1, L, offsets..., indices...]
    (simple_tile_renderer.py:757-766)."""
    return np.concatenate([np.array([offs.size, idx.size], np.int32), offs, idx]).astype(np.int32)


class Scene:
    """Inputs of one render, as the reference extension receives them."""

    def __init__(self, H, W, ts, means2D, radii, rot, opac, colors, templates, sel,
                 alpha_max=1.0, colors_orig=None, c_blend=0.0):
        self.H, self.W, self.ts = int(H), int(W), int(ts)
        # parameters are kept in float64: the kernels' float32 inputs convert
        # exactly, and finite-difference checks can perturb them below 1 ulp(f32)
        self.means2D = _f64(means2D).reshape(-1, 2)
        self.radii = _f64(radii).reshape(-1)
        self.rot = _f64(rot).reshape(-1)
        self.opac = _f64(opac).reshape(-1)
        self.colors = _f64(colors).reshape(-1, 3)
        t = _f64(templates)
        self.templates = t[None] if t.ndim == 2 else t
        self.sel = _i32(sel).reshape(-1)
        self.alpha_max = float(alpha_max)
        # per-primitive colour maps (N,Ht,Wt,3) in [0,1] and their blend weight
        # (tile_forward.cu:316-330); used when both are given and c_blend > 0
        self.colors_orig = None if colors_orig is None else _f64(colors_orig)
        self.c_blend = float(c_blend)

    def _cmap_args(self):
        use = self.colors_orig is not None and self.c_blend > 0
        return (_p(self.colors_orig) if use else None, ctypes.c_double(self.c_blend if use else 0.0))

    @property
    def N(self):
        return self.radii.shape[0]

    def _args(self):
        P, Ht, Wt = self.templates.shape
        return (self.H, self.W, self.ts, self.N, _p(self.means2D), _p(self.radii), _p(self.rot),
                _p(self.opac), _p(self.colors), P, Ht, Wt, _p(self.templates), _p(self.sel),
                ctypes.c_double(self.alpha_max))


def forward(scene: Scene, offs, idx, sem=SEM_KERNEL, t_stop=0.0, nthreads=0, edge=0.0):
    """Returns dict(color (H,W,3) f64, alpha (H,W) f64, T_last, last_pos, stats).
    ``edge`` shifts the cull / texel-cut boundaries (see dbmp_oracle.cpp)."""
    offs, idx = _i32(offs), _i32(idx)
    if idx.size == 0:
        idx = np.zeros(1, np.int32)
    H, W = scene.H, scene.W
    color = np.zeros((H, W, 3), np.float64)
    alpha = np.zeros((H, W), np.float64)
    tl = np.zeros((H, W), np.float64)
    lp = np.zeros((H, W), np.int32)
    stats = np.zeros(5, np.int64)
    lib().orc_forward_cmap(*scene._args(), int(sem), ctypes.c_double(t_stop), ctypes.c_double(edge),
                           _p(offs), _p(idx),
                           _p(color), _p(alpha), _p(tl), _p(lp), _p(stats), int(nthreads), *scene._cmap_args())
    return dict(color=color, alpha=alpha, T_last=tl, last_pos=lp,
                stats=dict(candidates=int(stats[0]), fragments=int(stats[1]),
                           live=int(stats[2]), max_depth=int(stats[3])))


def backward(scene: Scene, offs, idx, grad_color, grad_alpha, sem=SEM_KERNEL, t_stop=0.0,
             nthreads=0, edge=0.0):
    """Returns the (N,8) float64 gradients: means.x, means.y, radius, rotation,
    opacity logit, colour logits r,g,b."""
    offs, idx = _i32(offs), _i32(idx)
    if idx.size == 0:
        idx = np.zeros(1, np.int32)
    gc = _f32(grad_color).reshape(scene.H, scene.W, 3)
    ga = None if grad_alpha is None else _f32(grad_alpha).reshape(scene.H, scene.W)
    g = np.zeros((scene.N, 8), np.float64)
    lib().orc_backward_cmap(*scene._args(), int(sem), ctypes.c_double(t_stop), ctypes.c_double(edge),
                            _p(offs), _p(idx),
                            _p(gc), _p(ga), _p(g), int(nthreads), *scene._cmap_args())
    return g


def split_grads(g: np.ndarray):
    """(N,8) -> the reference's five gradient tensors (means2D, radii, rotations,
    opacities, colors) as returned by rasterize_tiles_backward_class."""
    return g[:, 0:2], g[:, 2], g[:, 3], g[:, 4], g[:, 5:8]


def psd_bboxes(means2D, radii, H, W, scale=1.0):
    means2D, radii = _f32(means2D), _f32(radii)
    N = radii.shape[0]
    bb = np.zeros((N, 4), np.int32)
    sz = np.zeros((N, 2), np.int32)
    lib().orc_psd_bboxes(_p(means2D), _p(radii), N, H, W, ctypes.c_float(scale), _p(bb), _p(sz))
    return bb, sz


def psd_layers(means2D, radii, rot, colors_sig, vis_sig, templates, sel, bboxes, offsets,
               scale=1.0, alpha_max=1.0):
    """Returns (buffer uint8, ambiguous uint8) for the packed cropped RGBA layers."""
    means2D, radii, rot = _f32(means2D), _f32(radii), _f32(rot)
    colors_sig, vis_sig = _f32(colors_sig), _f32(vis_sig)
    t = _f32(templates)
    t = t[None] if t.ndim == 2 else t
    sel, bboxes = _i32(sel), _i32(bboxes)
    offsets = np.ascontiguousarray(offsets, dtype=np.int64)
    N = radii.shape[0]
    sizes = (bboxes[:, 2] - bboxes[:, 0]) * (bboxes[:, 3] - bboxes[:, 1]) * 4
    total = int(offsets[-1] + sizes[-1]) if N else 0
    out = np.zeros(max(total, 1), np.uint8)
    amb = np.zeros(max(total, 1), np.uint8)
    P, Ht, Wt = t.shape
    lib().orc_psd_layers(_p(means2D), _p(radii), _p(rot), _p(colors_sig), _p(vis_sig), P, Ht, Wt,
                         _p(t), _p(sel), _p(bboxes), _p(offsets), N, ctypes.c_float(scale),
                         ctypes.c_float(alpha_max), _p(out), _p(amb))
    return out[:total], amb[:total]


def boundary_band(scene: Scene, offs, idx, edge=1e-3, t_stop=0.0, nthreads=0):
    """Per-pixel spread of the image between renders whose cull and texel-cut
    boundaries are widened and narrowed by `edge` (and whose bilinear cell
    choice moves by two float32 ulps of the texel coordinate, where the
    bilinear gradient jumps): non-zero where a float rounding difference
    at a primitive's boundary can flip a fragment.
    Returns (spread_color (H,W), spread_alpha (H,W))."""
    hi = forward(scene, offs, idx, SEM_KERNEL, t_stop, nthreads, edge=+edge)
    lo = forward(scene, offs, idx, SEM_KERNEL, t_stop, nthreads, edge=-edge)
    return np.abs(hi["color"] - lo["color"]).max(-1), np.abs(hi["alpha"] - lo["alpha"])


def check_image(scene: Scene, offs, idx, color, alpha, tol=1e-5, ref=None, nthreads=0):
    """Compares a float32 render (color (H,W,3), alpha (H,W)) with this
    oracle's FP64 render.  Pixels outside the boundary band must be within
    `tol` max-abs; pixels inside it (a fragment within 1e-3 px/texel of a
    cull or texel-cut boundary, where any float rounding can flip it) within
    the band's own spread + tol.  Raises AssertionError; returns a summary."""
    ref = forward(scene, offs, idx, nthreads=nthreads) if ref is None else ref
    band_c, band_a = boundary_band(scene, offs, idx, edge=1e-3, nthreads=nthreads)
    ec = np.abs(np.asarray(color, np.float64) - ref["color"]).max(-1)
    ea = np.abs(np.asarray(alpha, np.float64) - ref["alpha"])
    sens = (band_c > 0) | (band_a > 0)
    assert ec[~sens].max(initial=0) <= tol, ("color", ec[~sens].max(initial=0))
    assert ea[~sens].max(initial=0) <= tol, ("alpha", ea[~sens].max(initial=0))
    assert np.all(ec[sens] <= band_c[sens] + tol), ("color in band", float((ec - band_c)[sens].max()))
    assert np.all(ea[sens] <= band_a[sens] + tol), ("alpha in band", float((ea - band_a)[sens].max()))
    return dict(max_err=float(max(ec[~sens].max(initial=0), ea[~sens].max(initial=0))),
                sensitive=int(sens.sum()), ref=ref)


def check_grads(scene: Scene, offs, idx, grad_color, grad_alpha, ours, rel=1e-4, nthreads=0, verbose=True):
    """Per parameter block k of the (N,8) gradients:
    ||ours - oracle|| <= rel ||oracle|| + ||oracle(+edge) - oracle(-edge)||
    (the band spread of the gradient, edge = 1e-3: fragments within 1e-3 of
    the cull square or the texel cut, and points within two float32 ulps of
    a texel grid line, where the bilinear gradient jumps).  Returns the
    per-block relative errors."""
    ref = backward(scene, offs, idx, grad_color, grad_alpha, nthreads=nthreads)
    hi = backward(scene, offs, idx, grad_color, grad_alpha, nthreads=nthreads, edge=1e-3)
    lo = backward(scene, offs, idx, grad_color, grad_alpha, nthreads=nthreads, edge=-1e-3)
    ours = np.asarray(ours, np.float64).reshape(scene.N, 8)
    errs = []
    for k in range(8):
        spread = np.linalg.norm(hi[:, k] - lo[:, k])
        err = np.linalg.norm(ours[:, k] - ref[:, k])
        nrm = np.linalg.norm(ref[:, k])
        if verbose:
            print(f"  block {k}: err {err:.3e} |ref| {nrm:.3e} band {spread:.3e}")
        assert err <= rel * nrm + spread + 1e-9, (k, err, nrm, spread)
        errs.append(err / max(nrm, 1e-30))
    return errs
