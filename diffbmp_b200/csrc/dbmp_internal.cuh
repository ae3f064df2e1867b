// Shared device-side definitions of the DiffBMP B200 tile rasterizer.
#pragma once

#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/dbmp.h"

namespace dbmp {

// Per-primitive record derived once per iteration by the preparation kernel.
// 64 bytes, read with four 16-byte loads by the raster kernels.
//   tex_x = a00*dx + a01*dy + hx,  tex_y = a10*dx + a11*dy + hy
// with dx = px - mx, dy = py - my (integer pixel coordinates, no +0.5, as in
// cuda_tile_rasterizer/cuda_kernels/tile_forward.cu:191-192) and
// hx = (Wt-1)/2, hy = (Ht-1)/2.  The affine coefficients fold the reference's
// r_inv, rotation and texel scaling (tile_forward.cu:250-264).
struct __align__(16) PrimInfo {
  float mx, my, hw, hh;      // centre, square-cull half extents (tile_forward.cu:194-210)
  float a00, a01, a10, a11;  // inverse affine to texel coordinates
  float alpha0, cr, cg, cb;  // alpha_max*sigmoid(opacity), sigmoid(colour logits)
  int tmpl;                  // template id, -1 when the primitive yields no fragments
  float rinv, cs, sn;        // reference r_inv and rotation cos/sin (backward chain)
};
static_assert(sizeof(PrimInfo) == 64, "PrimInfo must be 64 bytes");

// Texel storage of the template atlas.
enum AtlasKind : int {
  ATLAS_F32 = DBMP_ATLAS_F32,            // (P,Ht,Wt) float32, the reference layout
  ATLAS_F32_QUAD = DBMP_ATLAS_F32_QUAD,  // (P,Ht,Wt) x 4 float32 bilinear quads
  ATLAS_F16_QUAD = DBMP_ATLAS_F16_QUAD,  // (P,Ht,Wt) x 4 half
  ATLAS_BF16_QUAD = DBMP_ATLAS_BF16_QUAD // (P,Ht,Wt) x 4 bfloat16
};

struct Geom {
  int H, W, TS, tilesX, tilesY, T;
  int N, P, Ht, Wt;
  float hx, hy;        // (Wt-1)/2, (Ht-1)/2
  float rxy, ryx;      // hx/hy, hy/hx (rotation gradient of non-square templates)
  float alpha_max;
  float t_stop;
};

// Quad of bilinear neighbours (v00, v01, v10, v11) of texel (x0, y0); entries
// outside the template read 0 (tile_common.h:188-194).
struct Quad { float v00, v01, v10, v11; };

template <int KIND> struct AtlasFetch;

template <> struct AtlasFetch<ATLAS_F32> {
  static __device__ __forceinline__ Quad get(const void* atlas, int tmpl, int Ht, int Wt, int x0, int y0) {
    const float* t = static_cast<const float*>(atlas) + (size_t)tmpl * Ht * Wt + (size_t)y0 * Wt + x0;
    const bool xr = x0 + 1 < Wt, yr = y0 + 1 < Ht;
    Quad q;
    q.v00 = __ldg(t);
    q.v01 = xr ? __ldg(t + 1) : 0.f;
    q.v10 = yr ? __ldg(t + Wt) : 0.f;
    q.v11 = (xr && yr) ? __ldg(t + Wt + 1) : 0.f;
    return q;
  }
};

template <> struct AtlasFetch<ATLAS_F32_QUAD> {
  static __device__ __forceinline__ Quad get(const void* atlas, int tmpl, int Ht, int Wt, int x0, int y0) {
    const float4 v = __ldg(static_cast<const float4*>(atlas) + (size_t)tmpl * Ht * Wt + (size_t)y0 * Wt + x0);
    return Quad{v.x, v.y, v.z, v.w};
  }
};

template <> struct AtlasFetch<ATLAS_F16_QUAD> {
  static __device__ __forceinline__ Quad get(const void* atlas, int tmpl, int Ht, int Wt, int x0, int y0) {
    const uint2 raw = __ldg(static_cast<const uint2*>(atlas) + (size_t)tmpl * Ht * Wt + (size_t)y0 * Wt + x0);
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&raw.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&raw.y));
    return Quad{a.x, a.y, b.x, b.y};
  }
};

template <> struct AtlasFetch<ATLAS_BF16_QUAD> {
  static __device__ __forceinline__ Quad get(const void* atlas, int tmpl, int Ht, int Wt, int x0, int y0) {
    const uint2 raw = __ldg(static_cast<const uint2*>(atlas) + (size_t)tmpl * Ht * Wt + (size_t)y0 * Wt + x0);
    const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.x));
    const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&raw.y));
    return Quad{a.x, a.y, b.x, b.y};
  }
};

// Template mask at texel coordinate (tx, ty): bilinear with a hard zero
// outside [0,Wt-1]x[0,Ht-1] (tile_common.h:175-198), clamped to [0,1]
// (tile_forward.cu:271, same operand order).  A NaN coordinate passes the
// reference's range test, converts to texel 0 and clamps to 1 through
// fmaxf(0, fminf(1, NaN)); the same happens here.  When GRAD is set also
// returns d(mask)/d(tex) before the clamp (tile_common.h:201-239).
template <int KIND, bool GRAD>
__device__ __forceinline__ float sample_mask(const void* atlas, int tmpl, int Ht, int Wt, float tx, float ty,
                                             float* gx, float* gy) {
  if (tx < 0.f || tx > (float)(Wt - 1) || ty < 0.f || ty > (float)(Ht - 1)) {
    if (GRAD) { *gx = 0.f; *gy = 0.f; }
    return 0.f;
  }
  // tx, ty in [0, W-1] (or NaN -> 0): truncation is floor and stays in range
  const int x0 = __float2int_rz(tx), y0 = __float2int_rz(ty);
  const float wx = tx - (float)x0, wy = ty - (float)y0;
  const Quad q = AtlasFetch<KIND>::get(atlas, tmpl, Ht, Wt, x0, y0);
  const float top = fmaf(wx, q.v01 - q.v00, q.v00);
  const float bot = fmaf(wx, q.v11 - q.v10, q.v10);
  const float m = fmaf(wy, bot - top, top);
  if (GRAD) {
    *gx = fmaf(wy, (q.v11 - q.v10) - (q.v01 - q.v00), q.v01 - q.v00);
    *gy = bot - top;
  }
  return fmaxf(0.f, fminf(1.f, m));
}

__device__ __forceinline__ float sigmoid_precise(float x) {
  // branch-stable logistic (tile_common.h:125-133) with IEEE exp/div
  if (x >= 0.f) { const float z = expf(-x); return 1.f / (1.f + z); }
  const float z = expf(x);
  return z / (1.f + z);
}

// Thread-local error string shared by every entry point.
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);

#define DBMP_CHECK_LAUNCH(what)                                  \
  do {                                                           \
    cudaError_t _e = cudaGetLastError();                         \
    if (_e != cudaSuccess) return ::dbmp::cuda_status(_e, what); \
  } while (0)

}  // namespace dbmp
