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
// With a half or bfloat16 atlas (the precision form) the opacity and colours
// are stored in FP16 as well: the third word then holds the bit patterns of
// the half pairs (alpha0, cr) and (cg, cb) in alpha0 and cr, and zeros.
struct __align__(16) PrimInfo {
  float mx, my, hw, hh;      // centre, square-cull half extents (tile_forward.cu:194-210)
  float a00, a01, a10, a11;  // inverse affine to texel coordinates
  float alpha0, cr, cg, cb;  // alpha_max*sigmoid(opacity), sigmoid(colour logits)
  int toff;                  // first element of the template in the atlas, or kNoFrag
  int goff;                  // first cell of the template's clearance grid (packed atlases)
  int gext;                  // clearance a warp footprint needs to be skipped (> kGridCap: never)
  int pad;
};
static_assert(sizeof(PrimInfo) == 64, "PrimInfo must be 64 bytes");

// toff sentinel kNoFrag: the primitive never yields a fragment.  Set for an
// invalid template id (tile_forward.cu:211-216,274) and for NaN geometry (a NaN
// centre, or a NaN in the inverse affine from a NaN or infinite rotation).  For
// NaN geometry this is what the reference kernel computes as built with its
// own flags (--use_fast_math): run side by side, no such primitive changes its
// image, although its source, read literally, would clamp a NaN mask to 1
// (tile_common.h:177-197, tile_forward.cu:271).
constexpr int kNoFrag = -1;

// Texel storage of the template atlas.
enum AtlasKind : int {
  ATLAS_F32 = DBMP_ATLAS_F32,              // (P,Ht,Wt) float32, the reference layout
  ATLAS_F32_QUAD = DBMP_ATLAS_F32_QUAD,    // (P,Ht,Wt) x 4 float32 bilinear quads
  ATLAS_F16_QUAD = DBMP_ATLAS_F16_QUAD,    // (P,Ht,Wt) x 4 half
  ATLAS_BF16_QUAD = DBMP_ATLAS_BF16_QUAD,  // (P,Ht,Wt) x 4 bfloat16
  ATLAS_F16_PAIR = DBMP_ATLAS_F16_PAIR,    // (P,Ht+1,Wt) x 2 half (x, x+1), zero last row
  ATLAS_BF16_PAIR = DBMP_ATLAS_BF16_PAIR   // (P,Ht+1,Wt) x 2 bfloat16
};

// Elements (texel records) per template for a storage kind.
__host__ __device__ inline int template_records(int kind, int Ht, int Wt) {
  return (kind == ATLAS_F16_PAIR || kind == ATLAS_BF16_PAIR) ? (Ht + 1) * Wt : Ht * Wt;
}

// Clearance grid of the packed atlas kinds.  Template texels are grouped in
// cells of 2^gsx x 2^gsy; a cell stores the L-infinity distance, in texels and
// capped at kGridCap, from its coordinate range to the nearest "support"
// texel: value > kGridSupport or NaN.  The bilinear mask is a convex
// combination of its four texels, so it can pass the fragment test
// mask > 1e-6 (tile_forward.cu:271-276) only next to a support texel
// (kGridSupport = 5e-7 leaves room for rounding and for half / bfloat16
// storage).  A point whose clamped texel coordinate falls in a cell with
// clearance D has no support texel within L-infinity distance < D, so a warp
// footprint whose texel-space box (half extent e around the footprint centre)
// satisfies e + 1 <= D yields no fragment.  The grid follows the texel
// records, 256-byte aligned.
constexpr int kGridCap = 64;
constexpr float kGridSupport = 5e-7f;
#ifndef DBMP_GRID_CELLS
#define DBMP_GRID_CELLS 128
#endif
constexpr int kGridMaxCells = DBMP_GRID_CELLS;   // cells per axis at most

__host__ __device__ inline void grid_shape(int n, int* shift, int* cells) {
  int s = 0;
  while (((n + (1 << s) - 1) >> s) > kGridMaxCells) ++s;
  *shift = s;
  *cells = (n + (1 << s) - 1) >> s;
}

__host__ __device__ inline bool atlas_has_grid(int kind) { return kind != ATLAS_F32; }

// Atlas kinds of the precision form: texels, opacity and colours in 16 bits.
__host__ __device__ constexpr bool half_record(int kind) {
  return kind == ATLAS_F16_QUAD || kind == ATLAS_BF16_QUAD || kind == ATLAS_F16_PAIR || kind == ATLAS_BF16_PAIR;
}

// Bytes of the texel records of an atlas kind (a packed atlas's grid follows them).
__host__ __device__ inline size_t atlas_record_bytes(int P, int Ht, int Wt, int kind) {
  const size_t recs = (size_t)P * template_records(kind, Ht, Wt);
  switch (kind) {
    case ATLAS_F32: return recs * 4;
    case ATLAS_F32_QUAD: return recs * 16;
    case ATLAS_F16_QUAD: case ATLAS_BF16_QUAD: return recs * 8;
    case ATLAS_F16_PAIR: case ATLAS_BF16_PAIR: return recs * 4;
    default: return 0;
  }
}
__host__ __device__ inline size_t atlas_grid_offset(int P, int Ht, int Wt, int kind) {
  return (atlas_record_bytes(P, Ht, Wt, kind) + 255) & ~(size_t)255;
}

// Thread layout of the tile walk: one CTA per TS x TS tile, NP pixels per
// thread, each warp owning an FW x FH footprint.
// DBMP_SQUARE_FOOTPRINT: with 2 pixels per thread, an 8x8 warp footprint
// (the second pixel 4 rows below the first) instead of 16x4.
#ifndef DBMP_SQUARE_FOOTPRINT
#define DBMP_SQUARE_FOOTPRINT 1
#endif
template <int TS, int NP>
struct Layout {
  static_assert(NP == 1 || NP == 2 || NP == 4, "pixels per thread");
  static constexpr bool kSq = DBMP_SQUARE_FOOTPRINT && NP == 2;
  static constexpr int FW = kSq ? 8 : (NP >= 2 ? 16 : 8);     // warp footprint
  static constexpr int FH = kSq ? 8 : (NP == 4 ? 8 : 4);
  static constexpr int WPR = TS / FW;              // warps per footprint row
  static constexpr int NW = (TS / FW) * (TS / FH);
  static constexpr int NT = NW * 32;
  static __host__ __device__ __forceinline__ int ox(int p) { return kSq ? 0 : 8 * (p & 1); }
  static __host__ __device__ __forceinline__ int oy(int p) { return kSq ? 4 * p : 4 * (p >> 1); }
};

// Pixels per thread of each tile size (tuned on B200).
template <int TS> struct DefaultNP;
#ifndef DBMP_NP32
#define DBMP_NP32 2
#endif
template <> struct DefaultNP<32> { static constexpr int v = DBMP_NP32; };
template <> struct DefaultNP<16> { static constexpr int v = 1; };

struct Geom {
  // operand pairs of the packed pixel-pair arithmetic (both halves equal)
  float2 k23;          // 2^23
  float2 m1;           // -1
  float2 nhx, nhy;     // -hx, -hy
  float2 rxy2, nryx2;  // hx/hy, -hy/hx
  unsigned kbias;      // 0x4B000000 (Wt + 1): the 2^23 bias of two floored coordinates in a record index
  int H, W, TS, tilesX, tilesY, T;
  int N, P, Ht, Wt;
  int kind;            // AtlasKind of the atlas the kernels read
  float hx, hy;        // (Wt-1)/2, (Ht-1)/2
  float rxy, ryx;      // hx/hy, hy/hx (rotation gradient of non-square templates)
  float wm1, hm1;      // Wt-1, Ht-1
  float alpha_max;
  float t_stop;
  float fhx, fhy;      // half extents (pixels) of the warp footprint of this tile size
  int gsx, gsy;        // clearance grid: log2 of the cell size in texels
  int gGx, gGy;        // clearance grid: cells per template row / column
  long long grid_off;  // byte offset of the clearance grid in a packed atlas
};

// Bilinear neighbours of texel (x0, y0) in difference form: v00, d01 =
// v01 - v00, v10, d11 = v11 - v10; neighbours outside the template read 0
// (tile_common.h:188-194).  The packed kinds store this form; the reference
// layout takes the differences after the loads.
struct Quad { float v00, d01, v10, d11; };

template <int KIND> struct AtlasFetch;

template <> struct AtlasFetch<ATLAS_F32> {
  using Raw = float4;
  // the four neighbours as loaded: (v00, v01, v10, v11)
  static __device__ __forceinline__ float4 get_raw(const void* atlas, int off, int Ht, int Wt, int x0, int y0) {
    const float* t = static_cast<const float*>(atlas) + off + y0 * Wt + x0;
    const bool xr = x0 + 1 < Wt, yr = y0 + 1 < Ht;
    return make_float4(__ldg(t), xr ? __ldg(t + 1) : 0.f, yr ? __ldg(t + Wt) : 0.f,
                       (xr && yr) ? __ldg(t + Wt + 1) : 0.f);
  }
  static __device__ __forceinline__ Quad get(const void* atlas, int off, int Ht, int Wt, int x0, int y0) {
    const float4 v = get_raw(atlas, off, Ht, Wt, x0, y0);
    return Quad{v.x, v.y - v.x, v.z, v.w - v.z};
  }
};

// Packed kinds: load() fetches record i (= off + y0 Wt + x0; int or unsigned)
// as stored, unpack() turns it into a Quad, at() does both.
template <> struct AtlasFetch<ATLAS_F32_QUAD> {
  using Raw = float4;
  template <typename I>
  static __device__ __forceinline__ Raw load(const void* atlas, I i, int Wt) {
    return __ldg(static_cast<const float4*>(atlas) + i);
  }
  static __device__ __forceinline__ Quad unpack(const Raw& v) { return Quad{v.x, v.y, v.z, v.w}; }
  template <typename I>
  static __device__ __forceinline__ Quad at(const void* atlas, I i, int Wt) { return unpack(load(atlas, i, Wt)); }
  static __device__ __forceinline__ Quad get(const void* atlas, int off, int Ht, int Wt, int x0, int y0) {
    return at(atlas, off + y0 * Wt + x0, Wt);
  }
};

__device__ __forceinline__ float2 h2f(unsigned u) { return __half22float2(*reinterpret_cast<const __half2*>(&u)); }
__device__ __forceinline__ float2 b2f(unsigned u) {
  return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u));
}

template <> struct AtlasFetch<ATLAS_F16_QUAD> {
  using Raw = uint2;
  template <typename I>
  static __device__ __forceinline__ Raw load(const void* atlas, I i, int Wt) {
    return __ldg(static_cast<const uint2*>(atlas) + i);
  }
  static __device__ __forceinline__ Quad unpack(const Raw& r) {
    const float2 a = h2f(r.x), b = h2f(r.y);
    return Quad{a.x, a.y, b.x, b.y};
  }
  template <typename I>
  static __device__ __forceinline__ Quad at(const void* atlas, I i, int Wt) { return unpack(load(atlas, i, Wt)); }
  static __device__ __forceinline__ Quad get(const void* atlas, int off, int Ht, int Wt, int x0, int y0) {
    return at(atlas, off + y0 * Wt + x0, Wt);
  }
};

template <> struct AtlasFetch<ATLAS_BF16_QUAD> {
  using Raw = uint2;
  template <typename I>
  static __device__ __forceinline__ Raw load(const void* atlas, I i, int Wt) {
    return __ldg(static_cast<const uint2*>(atlas) + i);
  }
  static __device__ __forceinline__ Quad unpack(const Raw& r) {
    const float2 a = b2f(r.x), b = b2f(r.y);
    return Quad{a.x, a.y, b.x, b.y};
  }
  template <typename I>
  static __device__ __forceinline__ Quad at(const void* atlas, I i, int Wt) { return unpack(load(atlas, i, Wt)); }
  static __device__ __forceinline__ Quad get(const void* atlas, int off, int Ht, int Wt, int x0, int y0) {
    return at(atlas, off + y0 * Wt + x0, Wt);
  }
};

template <> struct AtlasFetch<ATLAS_F16_PAIR> {
  using Raw = uint2;   // (record i, record i + Wt): rows y and y + 1; row Ht is the zero pad
  template <typename I>
  static __device__ __forceinline__ Raw load(const void* atlas, I i, int Wt) {
    const unsigned* p = static_cast<const unsigned*>(atlas) + i;
    return make_uint2(__ldg(p), __ldg(p + Wt));
  }
  static __device__ __forceinline__ Quad unpack(const Raw& r) {
    const float2 a = h2f(r.x), b = h2f(r.y);
    return Quad{a.x, a.y, b.x, b.y};
  }
  template <typename I>
  static __device__ __forceinline__ Quad at(const void* atlas, I i, int Wt) { return unpack(load(atlas, i, Wt)); }
  static __device__ __forceinline__ Quad get(const void* atlas, int off, int Ht, int Wt, int x0, int y0) {
    return at(atlas, off + y0 * Wt + x0, Wt);
  }
};

template <> struct AtlasFetch<ATLAS_BF16_PAIR> {
  using Raw = uint2;
  template <typename I>
  static __device__ __forceinline__ Raw load(const void* atlas, I i, int Wt) {
    const unsigned* p = static_cast<const unsigned*>(atlas) + i;
    return make_uint2(__ldg(p), __ldg(p + Wt));
  }
  static __device__ __forceinline__ Quad unpack(const Raw& r) {
    const float2 a = b2f(r.x), b = b2f(r.y);
    return Quad{a.x, a.y, b.x, b.y};
  }
  template <typename I>
  static __device__ __forceinline__ Quad at(const void* atlas, I i, int Wt) { return unpack(load(atlas, i, Wt)); }
  static __device__ __forceinline__ Quad get(const void* atlas, int off, int Ht, int Wt, int x0, int y0) {
    return at(atlas, off + y0 * Wt + x0, Wt);
  }
};

// floor(v) for 0 <= v < 2^23 without a float<->int conversion: adding 2^23
// with round-toward-zero leaves floor(v) in the low mantissa bits.
__device__ __forceinline__ int floor_small(float v, float* fl) {
  const float b = __fadd_rz(v, 8388608.f);
  *fl = b - 8388608.f;
  return __float_as_int(b) - 0x4B000000;
}

__device__ __forceinline__ float sigmoid_precise(float x) {
  // branch-stable logistic (tile_common.h:125-133) with IEEE exp/div
  if (x >= 0.f) { const float z = expf(-x); return 1.f / (1.f + z); }
  const float z = expf(x);
  return z / (1.f + z);
}

// Optimiser step arguments (dbmp_adam_cfg as the kernels take it).
struct AdamArgs {
  float lr[8];            // per parameter: x, y, r, theta, v, c_r, c_g, c_b
  float beta1, beta2, eps;
  float x_max, y_max, r_min, r_max;
  int clamp;
  float gamma;            // ExponentialLR factor per completed step (1: none)
};

// Pruning arguments (dbmp_prune_cfg).
struct PruneArgs {
  int every, num_iterations, no_last, warmup;
  float threshold;
  int pool_rows;
};

// Thread-local error string shared by every entry point.
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);

#define DBMP_CHECK_LAUNCH(what)                                  \
  do {                                                           \
    cudaError_t _e = cudaGetLastError();                         \
    if (_e != cudaSuccess) return ::dbmp::cuda_status(_e, what); \
  } while (0)

}  // namespace dbmp
