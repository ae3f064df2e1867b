// Forward / backward / fused tile compositing kernels.
//
// A tile of TS x TS pixels is walked by NW warps (one or more CTAs); each thread owns NP pixels
// (NP = 4, 2 or 1) of a compact warp footprint (16x8, 8x8 or 8x4 pixels) so
// that a primitive's square cull is mostly warp-uniform and the warp's texel
// fetches stay close together in the atlas.
//
// Every warp walks the tile's primitive list on its own, without CTA
// barriers: it stages 32 list entries at a time into a warp-private shared
// buffer (lane i loads entry i's 64-byte PrimInfo record and runs the
// warp-footprint cull and the clearance-grid test for it), and a ballot of
// the survivors gives the entries the warp composites, in list order in the
// forward walk and in reverse order in the backward walk.  Per entry a thread
// first computes the texel coordinates of all its pixels and issues their
// texel loads (addresses of pixels without a fragment are redirected to texel
// 0 of the template, so every load is in bounds), then composites them
// branch-free.  A warp stops when all its pixels are below t_stop; the
// backward walk of a warp starts at its own last contributor and adds its
// warp-reduced per-primitive sums straight into the FP64 accumulator.  With 2
// pixels per thread (32x32 tiles) both pixels go through the arithmetic as one
// float2 of packed FP32x2 instructions, and the forward walk issues the
// texel loads of two entries before compositing either.
#include "dbmp_internal.cuh"

namespace dbmp {

constexpr int kChunk = 32;   // list entries staged per warp at a time (one per lane)
constexpr unsigned kFull = 0xffffffffu;

// Conservative warp-uniform rejection: true when the primitive's cull square
// misses every pixel of the warp footprint (1 px margin for rounding; NaN
// never rejects, matching the reference's cull).
__device__ __forceinline__ bool footprint_miss(const float4& g0, float x0, float x1, float y0, float y1) {
  return (g0.x - g0.z > x1 + 1.f) || (g0.x + g0.z < x0 - 1.f) || (g0.y - g0.w > y1 + 1.f) ||
         (g0.y + g0.w < y0 - 1.f);
}

// Warp-uniform: true when every pixel of the warp footprint passes the
// primitive's square cull with a 1 px margin, so the per-pixel cull can be
// skipped (false for NaN geometry, which then takes the per-pixel path).
__device__ __forceinline__ bool footprint_inside(const float4& g0, float x0, float x1, float y0, float y1) {
  return (g0.x - g0.z <= x0 - 1.f) && (g0.x + g0.z >= x1 + 1.f) && (g0.y - g0.w <= y0 - 1.f) &&
         (g0.y + g0.w >= y1 + 1.f);
}

// Warp-uniform: true when the template's clearance grid shows that no pixel
// of the warp footprint (centre (cx, cy)) can get a fragment from this
// primitive.  The footprint centre's texel coordinate is clamped into the
// template (clamping only shortens distances to its texels), and its cell's
// clearance is compared with the primitive's requirement gext.
__device__ __forceinline__ bool grid_clear(const Geom& g, const unsigned char* __restrict__ grid, const float4& g0,
                                           const float4& g1, int goff, int gext, float cx, float cy) {
  const float dx = cx - g0.x, dy = cy - g0.y;
  const float tx = fminf(fmaxf(fmaf(g1.x, dx, fmaf(g1.y, dy, g.hx)), 0.f), g.wm1);
  const float ty = fminf(fmaxf(fmaf(g1.z, dx, fmaf(g1.w, dy, g.hy)), 0.f), g.hm1);
  float unused;
  const int ix = floor_small(tx, &unused) >> g.gsx;
  const int iy = floor_small(ty, &unused) >> g.gsy;
  return (int)__ldg(grid + goff + iy * g.gGx + ix) >= gext;
}

// Texel coordinates, sampling position and fetched neighbours of one pixel.
struct Sample {
  float tx, ty, wx, wy;
  bool ok;    // pixel live, inside the cull square and inside [0,W-1]x[0,H-1]
  Quad q;
};

// Phase 1 of an entry: texel coordinates of every pixel of the thread (the
// inverse affine is linear, so pixel p is pixel 0 plus a multiple of a column
// of A) and whether the pixel can yield a fragment (live, inside the cull
// square, inside [0,W-1]x[0,H-1]).
// FAST: the warp footprint lies inside the cull square and its texel-space
// box inside the template (with margin), so every pixel passes both tests.
template <int NP, class L, bool FAST>
__device__ __forceinline__ void entry_coords(const Geom& g, const float4& g0, const float4& g1, bool inside,
                                             const float (&pxf)[NP], const float (&pyf)[NP],
                                             const bool (&live)[NP], Sample (&s)[NP]) {
  const float dx0 = pxf[0] - g0.x, dy0 = pyf[0] - g0.y;
  const float tx0 = fmaf(g1.x, dx0, fmaf(g1.y, dy0, g.hx));
  const float ty0 = fmaf(g1.z, dx0, fmaf(g1.w, dy0, g.hy));
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    float tx = tx0, ty = ty0;
    if (L::ox(p)) { tx = fmaf((float)L::ox(p), g1.x, tx); ty = fmaf((float)L::ox(p), g1.z, ty); }
    if (L::oy(p)) { tx = fmaf((float)L::oy(p), g1.y, tx); ty = fmaf((float)L::oy(p), g1.w, ty); }
    if (FAST) {
      s[p].ok = live[p];
    } else {
      bool cull_ok = inside;
      if (!inside) cull_ok = !(fabsf(pxf[p] - g0.x) > g0.z || fabsf(pyf[p] - g0.y) > g0.w);
      const bool in_rng = tx >= 0.f && tx <= g.wm1 && ty >= 0.f && ty <= g.hm1;
      s[p].ok = live[p] && cull_ok && in_rng;
    }
    s[p].tx = tx;
    s[p].ty = ty;
  }
}

// Phase 2 for one pixel: sampling position and texel fetch (texel 0 of the
// template when the pixel cannot yield a fragment, so the load is in bounds).
template <int KIND, bool FAST>
__device__ __forceinline__ void entry_fetch(const Geom& g, const void* __restrict__ atlas, int toff, Sample& s) {
  // FAST: every pixel's coordinate lies inside the template, no redirection needed
  const float tx = (FAST || s.ok) ? s.tx : 0.f, ty = (FAST || s.ok) ? s.ty : 0.f;
  float fx, fy;
  const int x0 = floor_small(tx, &fx);
  const int y0 = floor_small(ty, &fy);
  s.wx = tx - fx;
  s.wy = ty - fy;
  s.q = AtlasFetch<KIND>::get(atlas, toff, g.Ht, g.Wt, x0, y0);
}

// Texel coordinates and texel fetches of all pixels of the thread for one
// entry (fast: the entry's warp-uniform interior bit).
template <int NP, class L, int KIND>
__device__ __forceinline__ void entry_sample(const Geom& g, const void* __restrict__ atlas, int toff,
                                             const float4& g0, const float4& g1, bool inside, bool fast,
                                             const float (&pxf)[NP], const float (&pyf)[NP],
                                             const bool (&live)[NP], Sample (&s)[NP]) {
  if (fast) {
    entry_coords<NP, L, true>(g, g0, g1, inside, pxf, pyf, live, s);
#pragma unroll
    for (int p = 0; p < NP; ++p) entry_fetch<KIND, true>(g, atlas, toff, s[p]);
  } else {
    entry_coords<NP, L, false>(g, g0, g1, inside, pxf, pyf, live, s);
#pragma unroll
    for (int p = 0; p < NP; ++p) entry_fetch<KIND, false>(g, atlas, toff, s[p]);
  }
}

// Bilinear mask and, with GRAD, its texel-space gradient.  The reference
// clamps the mask to [0,1] (tile_forward.cu:271, NaN -> 1); only the upper
// clamp is applied here, since every caller discards masks failing the
// fragment test mask > 1e-6, which the lower clamp cannot change.
template <bool GRAD>
__device__ __forceinline__ float blend(const Sample& s, float* gx, float* gy) {
  const float dt = s.q.d01, db = s.q.d11;
  const float top = fmaf(s.wx, dt, s.q.v00);
  const float bot = fmaf(s.wx, db, s.q.v10);
  const float m = fmaf(s.wy, bot - top, top);
  if (GRAD) {
    *gx = fmaf(s.wy, db - dt, dt);
    *gy = bot - top;
  }
  return fminf(1.f, m);
}

// ---------------------------------------------------------------------------
// Pixel pairs.  With 2 pixels per thread the per-entry arithmetic of both
// pixels runs as one float2 (x: pixel 0, y: pixel 1) through the packed FP32x2
// instructions of sm_100, one instruction for both pixels.  Each packed
// operation rounds exactly like its scalar counterpart; constant operands come
// as pairs from the kernel parameters (Geom) or the staged record.  Packed
// operations issue to the FMA-heavy pipe only, while scalar FP32 operations
// may also use the FMA-lite pipe, so some steps stay scalar to keep both pipes
// busy (measured on B200: the forward's blend and colour accumulation, the
// backward's colour and per-primitive product terms).
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
// b - a, as the exact FMA a * -1 + b
__device__ __forceinline__ float2 sub2(const Geom& g, float2 b, float2 a) { return __ffma2_rn(a, g.m1, b); }

// Texel coordinates, sampling weights and neighbours of a thread's two pixels.
struct PairSample {
  float2 tx, ty;             // texel coordinates (not redirected)
  float2 wx, wy;             // bilinear weights of the fetched texel
  float2 v00, d01, v10, d11;  // neighbours in difference form (Quad)
  bool ok0, ok1;             // pixel can yield a fragment (as Sample::ok)
};

// A pixel pair's sample with its texel loads issued but not yet consumed.
template <int KIND>
struct PairPre {
  float2 wx, wy;
  typename AtlasFetch<KIND>::Raw r0, r1;   // the two pixels' records as loaded
  bool ok0, ok1;
};

// Coordinates, weights and texel loads of both pixels for one entry; tx, ty
// (optional) receive the texel coordinates.
template <class L, int KIND, bool FAST>
__device__ __forceinline__ void pair_prep(const Geom& g, const void* __restrict__ atlas, int toff,
                                          const float4& g0, const float4& g1, bool inside, const float (&pxf)[2],
                                          const float (&pyf)[2], const bool (&live)[2], PairPre<KIND>& s,
                                          float2* ptx = nullptr, float2* pty = nullptr) {
  Sample c[2];
  entry_coords<2, L, FAST>(g, g0, g1, inside, pxf, pyf, live, c);
  s.ok0 = c[0].ok;
  s.ok1 = c[1].ok;
  if (ptx) {
    *ptx = make_float2(c[0].tx, c[1].tx);
    *pty = make_float2(c[0].ty, c[1].ty);
  }
  // pixels without a fragment sample texel 0 of the template (in bounds)
  const float2 tx = make_float2((FAST || c[0].ok) ? c[0].tx : 0.f, (FAST || c[1].ok) ? c[1].tx : 0.f);
  const float2 ty = make_float2((FAST || c[0].ok) ? c[0].ty : 0.f, (FAST || c[1].ok) ? c[1].ty : 0.f);
  // floor as in floor_small: adding 2^23 rounding toward zero
  const float2 bx = __fadd2_rz(tx, g.k23), by = __fadd2_rz(ty, g.k23);
  const float2 fx = fma2(g.m1, g.k23, bx), fy = fma2(g.m1, g.k23, by);
  s.wx = sub2(g, tx, fx);
  s.wy = sub2(g, ty, fy);
  if constexpr (KIND == ATLAS_F32) {
    const int x0 = __float_as_int(bx.x) - 0x4B000000, y0 = __float_as_int(by.x) - 0x4B000000;
    const int x1 = __float_as_int(bx.y) - 0x4B000000, y1 = __float_as_int(by.y) - 0x4B000000;
    s.r0 = AtlasFetch<KIND>::get_raw(atlas, toff, g.Ht, g.Wt, x0, y0);
    s.r1 = AtlasFetch<KIND>::get_raw(atlas, toff, g.Ht, g.Wt, x1, y1);
  } else {
    // record index toff + y0 Wt + x0 straight from the biased bit patterns
    // (2^23 + x0, 2^23 + y0): the bias is one constant per entry, and the
    // unsigned arithmetic wraps back to the in-range index
    const unsigned c = (unsigned)toff - g.kbias;
    s.r0 = AtlasFetch<KIND>::load(atlas, __float_as_uint(by.x) * (unsigned)g.Wt + __float_as_uint(bx.x) + c, g.Wt);
    s.r1 = AtlasFetch<KIND>::load(atlas, __float_as_uint(by.y) * (unsigned)g.Wt + __float_as_uint(bx.y) + c, g.Wt);
  }
}

// Consumes the loads of pair_prep: weights and neighbours as pairs (the
// neighbours in difference form); tx, ty are not set.
template <int KIND>
__device__ __forceinline__ void pair_unpack(const Geom& g, const PairPre<KIND>& p, PairSample& s) {
  s.wx = p.wx;
  s.wy = p.wy;
  s.ok0 = p.ok0;
  s.ok1 = p.ok1;
  if constexpr (KIND == ATLAS_F32) {
    // reference layout: both pixels' differences as packed subtractions
    s.v00 = make_float2(p.r0.x, p.r1.x);
    s.v10 = make_float2(p.r0.z, p.r1.z);
    s.d01 = sub2(g, make_float2(p.r0.y, p.r1.y), s.v00);
    s.d11 = sub2(g, make_float2(p.r0.w, p.r1.w), s.v10);
  } else {
    const Quad q0 = AtlasFetch<KIND>::unpack(p.r0), q1 = AtlasFetch<KIND>::unpack(p.r1);
    s.v00 = make_float2(q0.v00, q1.v00);
    s.d01 = make_float2(q0.d01, q1.d01);
    s.v10 = make_float2(q0.v10, q1.v10);
    s.d11 = make_float2(q0.d11, q1.d11);
  }
}

// Both phases for one entry, with the texel coordinates.
template <class L, int KIND, bool FAST>
__device__ __forceinline__ void pair_sample(const Geom& g, const void* __restrict__ atlas, int toff,
                                            const float4& g0, const float4& g1, bool inside, const float (&pxf)[2],
                                            const float (&pyf)[2], const bool (&live)[2], PairSample& s) {
  PairPre<KIND> p;
  pair_prep<L, KIND, FAST>(g, atlas, toff, g0, g1, inside, pxf, pyf, live, p, &s.tx, &s.ty);
  pair_unpack<KIND>(g, p, s);
}

// Bilinear mask of both pixels (upper-clamped as in blend()) and, with GRAD, its texel-space
// gradient: the operations of blend() on pairs.  PACKED: as FP32x2 instructions;
// otherwise as scalar ones (same roundings).
template <bool GRAD, bool PACKED = true>
__device__ __forceinline__ float2 pair_blend(const Geom& g, const PairSample& s, float2* gx, float2* gy) {
  if (!PACKED) {
    const float top0 = fmaf(s.wx.x, s.d01.x, s.v00.x), top1 = fmaf(s.wx.y, s.d01.y, s.v00.y);
    const float bot0 = fmaf(s.wx.x, s.d11.x, s.v10.x), bot1 = fmaf(s.wx.y, s.d11.y, s.v10.y);
    const float d0 = bot0 - top0, d1 = bot1 - top1;
    if (GRAD) {
      *gx = make_float2(fmaf(s.wy.x, s.d11.x - s.d01.x, s.d01.x), fmaf(s.wy.y, s.d11.y - s.d01.y, s.d01.y));
      *gy = make_float2(d0, d1);
    }
    return make_float2(fminf(1.f, fmaf(s.wy.x, d0, top0)), fminf(1.f, fmaf(s.wy.y, d1, top1)));
  }
  const float2 dt = s.d01, db = s.d11;
  const float2 top = fma2(s.wx, dt, s.v00);
  const float2 bot = fma2(s.wx, db, s.v10);
  const float2 d = sub2(g, bot, top);
  const float2 m = fma2(s.wy, d, top);
  if (GRAD) {
    *gx = fma2(s.wy, sub2(g, db, dt), dt);
    *gy = d;
  }
  return make_float2(fminf(1.f, m.x), fminf(1.f, m.y));
}

// Colour-map sample (tile_forward.cu:17-89): the texel coordinate is clamped
// into the map, neighbours past the last row / column repeat it, bilinear in
// the reference's operation order.  cm: the primitive's (Ht,Wt,3) map.
__device__ __forceinline__ float3 sample_cmap(const float* __restrict__ cm, int Ht, int Wt, float tx, float ty) {
  const float cx = fmaxf(0.f, fminf((float)(Wt - 1), tx));
  const float cy = fmaxf(0.f, fminf((float)(Ht - 1), ty));
  const int x0 = (int)cx, y0 = (int)cy;
  const int x1 = min(x0 + 1, Wt - 1), y1 = min(y0 + 1, Ht - 1);
  const float fx = cx - (float)x0, fy = cy - (float)y0;
  const float* p00 = cm + 3 * (y0 * Wt + x0);
  const float* p10 = cm + 3 * (y0 * Wt + x1);
  const float* p01 = cm + 3 * (y1 * Wt + x0);
  const float* p11 = cm + 3 * (y1 * Wt + x1);
  float r[3];
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const float c0 = __ldg(p00 + ch) * (1.f - fx) + __ldg(p10 + ch) * fx;
    const float c1 = __ldg(p01 + ch) * (1.f - fx) + __ldg(p11 + ch) * fx;
    r[ch] = c0 * (1.f - fy) + c1 * fy;
  }
  return make_float3(r[0], r[1], r[2]);
}

// ---------------------------------------------------------------------------
// Ballots of one staged chunk (bit j = entry base + j).
struct ChunkMasks {
  unsigned todo;     // entries the warp composites
  unsigned inside;   // footprint entirely inside the entry's cull square
  unsigned fast;     // ... and its texel-space box inside the template
  unsigned clear;    // clearance grid shows no fragment (skipped unless counting)
  unsigned miss;     // footprint misses the cull square
};

// CB: fragment colours blend a per-primitive colour map (cmap, (N,Ht,Wt,3))
// with weight cblend, (1 - cblend) sigmoid(c) + cblend c_o (tile_forward.cu:316-330).
#ifndef DBMP_PACKED_PAIRS
#define DBMP_PACKED_PAIRS 1
#endif


template <int TS, int NP, int KIND, bool CB = false>
struct TileWalker {
  using L = Layout<TS, NP>;
  static constexpr int NT = L::NT;
  static constexpr int NW = L::NW;
  static constexpr bool kGrid = KIND != ATLAS_F32;   // packed atlases carry a clearance grid
  static constexpr bool kQuad = KIND == ATLAS_F32_QUAD || KIND == ATLAS_F16_QUAD || KIND == ATLAS_BF16_QUAD;
  // Pixel-pair walk (2 pixels per thread, fixed colours).  Its staged record
  // holds the opacity and colours as duplicated pairs:
  //   [0] (mx, my, hw, hh)  [1] A  [2] (op, op, r, r)  [3] (g, g, b, b)  [4] (toff, goff, gext, -)
  // otherwise the PrimInfo record as is: [0] [1] A [2] (op, r, g, b) [3] (toff, goff, gext, -).
  static constexpr bool kPair = DBMP_PACKED_PAIRS && NP == 2 && !CB;
  static constexpr int kRec = kPair ? 5 : 4;
  using Rec = float4[kRec];

  // (op, r, g, b) and the atlas offset of a staged record.
  static __device__ __forceinline__ float4 rec_g2(const Rec& r) {
    if (kPair) {
      const float4 a = r[2], b = r[3];
      return make_float4(a.x, a.z, b.x, b.z);
    }
    return r[2];
  }
  static __device__ __forceinline__ int rec_toff(const Rec& r) { return __float_as_int(r[kRec - 1].x); }

  int warp, lw, lane, start, end;   // warp: index within the tile, lw: within the CTA
  const float* cmap = nullptr;
  float cblend = 0.f;

  // Fragment colour of pixel sample s for primitive id (g2.yzw = sigmoid(c)).
  __device__ __forceinline__ float3 frag_colour(const Geom& g, const float4& g2, int id, const Sample& s) const {
    if (!CB) return make_float3(g2.y, g2.z, g2.w);
    const float3 co = sample_cmap(cmap + (size_t)id * g.Ht * g.Wt * 3, g.Ht, g.Wt, s.tx, s.ty);
    const float k = 1.f - cblend;
    return make_float3(k * g2.y + cblend * co.x, k * g2.z + cblend * co.y, k * g2.w + cblend * co.z);
  }
  float pxf[NP], pyf[NP];
  bool valid[NP];
  float fx0, fx1, fy0, fy1, fcx, fcy;

  // tile: the CTA's tile; part: which group of warps of the tile the CTA runs
  // (a CTA holds kCtaWarps of the tile's NW warps).
  __device__ __forceinline__ void init(const Geom& g, int tile, int part, int cta_warps,
                                       const int* __restrict__ offs) {
    lw = threadIdx.x >> 5;
    warp = part * cta_warps + lw;
    lane = threadIdx.x & 31;
    const int tx = tile % g.tilesX, ty = tile / g.tilesX;
    start = __ldg(offs + tile);
    end = __ldg(offs + tile + 1);
    const int bx = px(tile, g, 0), by = py(tile, g, 0);
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      pxf[p] = (float)(bx + L::ox(p));
      pyf[p] = (float)(by + L::oy(p));
      valid[p] = bx + L::ox(p) < g.W && by + L::oy(p) < g.H;
    }
    fx0 = (float)(tx * TS + (warp % L::WPR) * L::FW);
    fx1 = fx0 + (float)(L::FW - 1);
    fy0 = (float)(ty * TS + (warp / L::WPR) * L::FH);
    fy1 = fy0 + (float)(L::FH - 1);
    fcx = fx0 + 0.5f * (float)(L::FW - 1);
    fcy = fy0 + 0.5f * (float)(L::FH - 1);
  }

  // Pixel coordinates of pixel p of this thread.
  __device__ __forceinline__ int px(int tile, const Geom& g, int p) const {
    return (tile % g.tilesX) * TS + (warp % L::WPR) * L::FW + (lane & 7) + L::ox(p);
  }
  __device__ __forceinline__ int py(int tile, const Geom& g, int p) const {
    return (tile / g.tilesX) * TS + (warp / L::WPR) * L::FH + (lane >> 3) + L::oy(p);
  }

  // Stages list positions [base, min(base + 32, stop)) into the warp's buffer
  // w (lane i: position base + i) and returns the chunk's ballots.  With
  // KEEP_CLEAR, entries the clearance grid rules out stay in `todo` (the
  // counting walk checks them).  Out-of-range primitive ids never yield a
  // fragment (tile_forward.cu:184-185).  my_id: this lane's primitive id.
  template <bool KEEP_CLEAR>
  __device__ __forceinline__ ChunkMasks stage(const Geom& g, const PrimInfo* __restrict__ prims,
                                              const int* __restrict__ idx, const unsigned char* __restrict__ grid,
                                              int base, int stop, Rec* w, int* my_id) {
    bool keep = false, inside = false, fast = false, clear = false, miss = false;
    int id = -1;
    __syncwarp();   // every lane is done with the previous chunk's records
    const int pos = base + lane;
    if (pos < stop) {
      id = __ldg(idx + pos);
      if (id >= 0 && id < g.N) {
        const float4* r = reinterpret_cast<const float4*>(prims + id);
        const float4 g0 = __ldg(r);
        miss = footprint_miss(g0, fx0, fx1, fy0, fy1);
        if (!miss) {
          const float4 q = __ldg(r + 3);
          const int toff = __float_as_int(q.x);
          if (toff != kNoFrag) {
            const float4 g1 = __ldg(r + 1);
            if (kGrid)
              clear = grid_clear(g, grid, g0, g1, __float_as_int(q.y), __float_as_int(q.z), fcx, fcy);
            keep = KEEP_CLEAR || !clear;
            if (keep) {
              inside = footprint_inside(g0, fx0, fx1, fy0, fy1);
              if (inside) {
                // texel box of the footprint: centre +- |A| (half extents), plus
                // 0.05 texel for the rounding of the per-pixel coordinates
                const float dx = fcx - g0.x, dy = fcy - g0.y;
                const float cx = fmaf(g1.x, dx, fmaf(g1.y, dy, g.hx));
                const float cy = fmaf(g1.z, dx, fmaf(g1.w, dy, g.hy));
                const float ex = fmaf(fabsf(g1.x), g.fhx, fmaf(fabsf(g1.y), g.fhy, 0.05f));
                const float ey = fmaf(fabsf(g1.z), g.fhx, fmaf(fabsf(g1.w), g.fhy, 0.05f));
                fast = cx - ex >= 0.f && cx + ex <= g.wm1 && cy - ey >= 0.f && cy + ey <= g.hm1;
              }
              float4 g2 = __ldg(r + 2);
              if (half_record(KIND)) {   // FP16 (alpha0, r) and (g, b) pairs
                const float2 ar = h2f(__float_as_uint(g2.x)), gb = h2f(__float_as_uint(g2.y));
                g2 = make_float4(ar.x, ar.y, gb.x, gb.y);
              }
              w[lane][0] = g0;
              w[lane][1] = g1;
              if (kPair) {
                w[lane][2] = make_float4(g2.x, g2.x, g2.y, g2.y);
                w[lane][3] = make_float4(g2.z, g2.z, g2.w, g2.w);
              } else {
                w[lane][2] = g2;
              }
              w[lane][kRec - 1] = q;
            }
          }
        }
      } else {
        id = -1;
      }
    }
    __syncwarp();   // the records are visible to every lane
    *my_id = id;
    ChunkMasks m;
    m.todo = __ballot_sync(kFull, keep);
    m.inside = __ballot_sync(kFull, inside);
    m.fast = __ballot_sync(kFull, fast);
    m.clear = KEEP_CLEAR ? __ballot_sync(kFull, clear) : 0u;
    m.miss = KEEP_CLEAR ? __ballot_sync(kFull, miss) : 0u;
    return m;
  }

  // Adds the warp's 8 per-primitive sums (acc, one set per lane) to dst[0..7]:
  // a recursive-halving reduction, 8 sums over 32 lanes in 9 shuffles, after
  // which lane l < 8 holds sum kidx and adds it in FP64.
  __device__ __forceinline__ void warp_add(float (&acc)[8], int kidx, double* __restrict__ dst) const {
    const bool b0 = lane & 1, b1 = lane & 2, b2 = lane & 4;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float send = b0 ? acc[k] : acc[k + 4];
      const float keep = b0 ? acc[k + 4] : acc[k];
      acc[k] = keep + __shfl_xor_sync(kFull, send, 1);
    }
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const float send = b1 ? acc[k] : acc[k + 2];
      const float keep = b1 ? acc[k + 2] : acc[k];
      acc[k] = keep + __shfl_xor_sync(kFull, send, 2);
    }
    {
      const float send = b2 ? acc[0] : acc[1];
      const float keep = b2 ? acc[1] : acc[0];
      acc[0] = keep + __shfl_xor_sync(kFull, send, 4);
    }
    acc[0] += __shfl_xor_sync(kFull, acc[0], 8);
    acc[0] += __shfl_xor_sync(kFull, acc[0], 16);
    if (lane < 8 && acc[0] != 0.f) atomicAdd(dst + kidx, (double)acc[0]);
  }

  // Phase 1 of a forward entry for a pixel pair: coordinates and texel loads.
  __device__ __forceinline__ void pair_issue(const Geom& g, const void* __restrict__ atlas, const Rec* w, int e,
                                             const ChunkMasks& cm, const bool (&live)[2], PairPre<KIND>& p) const {
    const int toff = rec_toff(w[e]);
    const float4 g0 = w[e][0];
    const float4 g1 = w[e][1];
    const bool inside = (cm.inside >> e) & 1u;
    if ((cm.fast >> e) & 1u) pair_prep<L, KIND, true>(g, atlas, toff, g0, g1, inside, pxf, pyf, live, p);
    else pair_prep<L, KIND, false>(g, atlas, toff, g0, g1, inside, pxf, pyf, live, p);
  }

  // Forward state of a pixel pair.
  struct PairFwd {
    float2 cr, cg, cb, t, tl;
    int lp0, lp1;
    bool live[2];
  };

  // Phase 2 of a forward entry: blend the loaded texels and composite.
  // Returns true when every pixel of the warp has stopped.
  __device__ __forceinline__ bool pair_composite(const Geom& g, const Rec* w, int e, int pos, const PairPre<KIND>& p,
                                                 PairFwd& f, bool vote = true) const {
    const float4 c0 = w[e][2];
    const float4 c1 = w[e][3];
    PairSample s;
    pair_unpack<KIND>(g, p, s);
    const float2 m = pair_blend<false, false>(g, s, nullptr, nullptr);
    // a pixel may have stopped since the loads were issued
    const bool f0 = s.ok0 && f.live[0] && m.x > 1e-6f, f1 = s.ok1 && f.live[1] && m.y > 1e-6f;
    float2 a = make_float2(f0 ? c0.x * m.x : 0.f, f1 ? c0.y * m.y : 0.f);
    const float2 wt = make_float2(f.t.x * a.x, f.t.y * a.y);
    f.cr = make_float2(fmaf(wt.x, c0.z, f.cr.x), fmaf(wt.y, c0.w, f.cr.y));
    f.cg = make_float2(fmaf(wt.x, c1.x, f.cg.x), fmaf(wt.y, c1.y, f.cg.y));
    f.cb = make_float2(fmaf(wt.x, c1.z, f.cb.x), fmaf(wt.y, c1.w, f.cb.y));
    f.tl.x = f0 ? f.t.x : f.tl.x;
    f.tl.y = f1 ? f.t.y : f.tl.y;
    f.lp0 = f0 ? pos : f.lp0;
    f.lp1 = f1 ? pos : f.lp1;
    // T (1 - a) as in forward(), saturated per pixel (no packed form)
    f.t.x = __saturatef(fmaf(-f.t.x, a.x, f.t.x));
    f.t.y = __saturatef(fmaf(-f.t.y, a.y, f.t.y));
    f.live[0] = f.live[0] && !(f.t.x < g.t_stop);
    f.live[1] = f.live[1] && !(f.t.y < g.t_stop);
    return vote && __all_sync(kFull, !f.live[0] && !f.live[1]);
  }

  // Forward walk of the pixel-pair form: the walk of forward() with both
  // pixels' sampling, blending and compositing as packed pairs.  Entries go
  // two at a time: the texel loads of both are issued before either is
  // composited, so their latencies overlap.
  __device__ __forceinline__ void forward_pair(const Geom& g, const PrimInfo* __restrict__ prims,
                                               const void* __restrict__ atlas, const int* __restrict__ idx, Rec* w,
                                               float (&C)[2][3], float (&T)[2], float (&Tl)[2], int (&lp)[2]) {
    const unsigned char* grid = static_cast<const unsigned char*>(atlas) + g.grid_off;
    PairFwd f;
    f.cr = f.cg = f.cb = make_float2(0.f, 0.f);
    f.t = f.tl = make_float2(1.f, 1.f);
    f.lp0 = f.lp1 = -1;
    f.live[0] = valid[0];
    f.live[1] = valid[1];
    bool warp_done = __all_sync(kFull, !f.live[0] && !f.live[1]);
    for (int base = start; base < end && !warp_done; base += kChunk) {
      int my_id;
      const ChunkMasks cm = stage<false>(g, prims, idx, grid, base, end, w, &my_id);
      unsigned todo = cm.todo;
      while (todo) {
        const int e1 = __ffs(todo) - 1;
        todo &= todo - 1;
        const bool two = todo != 0;
        const int e2 = two ? __ffs(todo) - 1 : e1;   // e1 again when it is the chunk's last
        todo &= todo - 1;
        PairPre<KIND> p1, p2;
        pair_issue(g, atlas, w, e1, cm, f.live, p1);
        pair_issue(g, atlas, w, e2, cm, f.live, p2);
        // one termination vote per pair: a pixel that stops at e1 has live
        // false, so e2 composites nothing for it
        if (pair_composite(g, w, e1, base - start + e1, p1, f, !two)) { warp_done = true; break; }
        if (two && pair_composite(g, w, e2, base - start + e2, p2, f)) { warp_done = true; break; }
      }
    }
    C[0][0] = f.cr.x; C[0][1] = f.cg.x; C[0][2] = f.cb.x;
    C[1][0] = f.cr.y; C[1][1] = f.cg.y; C[1][2] = f.cb.y;
    T[0] = f.t.x; T[1] = f.t.y;
    Tl[0] = f.tl.x; Tl[1] = f.tl.y;
    lp[0] = f.lp0; lp[1] = f.lp1;
  }

  // Reverse walk of the pixel-pair form (the walk of backward() with both
  // pixels' arithmetic as packed pairs; each per-primitive sum adds the two
  // pixels' terms before the warp reduction).
  __device__ __forceinline__ void backward_pair(const Geom& g, const PrimInfo* __restrict__ prims,
                                                const void* __restrict__ atlas, const int* __restrict__ idx, Rec* w,
                                                const float (&gC)[2][3], const float (&gA)[2], float (&Ts)[2],
                                                const int (&lp)[2], double* __restrict__ gacc) {
    const int warp_max = __reduce_max_sync(kFull, max(lp[0], lp[1]));
    if (warp_max < 0) return;
    const unsigned char* grid = static_cast<const unsigned char*>(atlas) + g.grid_off;
    const int kidx = 4 * (lane & 1) + 2 * ((lane >> 1) & 1) + ((lane >> 2) & 1);
    const float2 gcr = make_float2(gC[0][0], gC[1][0]), gcg = make_float2(gC[0][1], gC[1][1]),
                 gcb = make_float2(gC[0][2], gC[1][2]), ga = make_float2(gA[0], gA[1]);
    float2 h = make_float2(0.f, 0.f), bt = make_float2(1.f, 1.f), ts = make_float2(Ts[0], Ts[1]);
    for (int cb = (warp_max / kChunk) * kChunk; cb >= 0; cb -= kChunk) {
      int my_id;
      const ChunkMasks cm = stage<false>(g, prims, idx, grid, start + cb, start + warp_max + 1, w, &my_id);
      unsigned todo = cm.todo;
      while (todo) {
        const int e = 31 - __clz(todo);
        todo &= ~(1u << e);
        const int pos = cb + e;
        const int id = __shfl_sync(kFull, my_id, e);
        const float4 g0 = w[e][0];
        const float4 g1 = w[e][1];
        const float4 c0 = w[e][2];
        const float4 c1 = w[e][3];
        const int toff = rec_toff(w[e]);
        const bool live[2] = {pos <= lp[0], pos <= lp[1]};
        PairSample s;
        const bool inside = (cm.inside >> e) & 1u;
        if ((cm.fast >> e) & 1u) pair_sample<L, KIND, true>(g, atlas, toff, g0, g1, inside, pxf, pyf, live, s);
        else pair_sample<L, KIND, false>(g, atlas, toff, g0, g1, inside, pxf, pyf, live, s);
        float2 gx, gy;
        const float2 m = pair_blend<true>(g, s, &gx, &gy);
        const float2 tx = s.tx, ty = s.ty;
        const bool f0 = s.ok0 && m.x > 1e-6f, f1 = s.ok1 && m.y > 1e-6f;
        float2 a = make_float2(f0 ? c0.x * m.x : 0.f, f1 ? c0.y * m.y : 0.f);
        const float2 om = make_float2(__saturatef(1.f - a.x), __saturatef(1.f - a.y));
        // T entering this fragment (see backward())
        const float2 tk = make_float2((pos == lp[0]) ? ts.x : __fdividef(ts.x, om.x),
                                      (pos == lp[1]) ? ts.y : __fdividef(ts.y, om.y));
        ts = tk;
        const float2 col_r = make_float2(c0.z, c0.w), col_g = make_float2(c1.x, c1.y),
                     col_b = make_float2(c1.z, c1.w);
        const float2 gcc = make_float2(fmaf(gcr.x, col_r.x, fmaf(gcg.x, col_g.x, gcb.x * col_b.x)),
                                       fmaf(gcr.y, col_r.y, fmaf(gcg.y, col_g.y, gcb.y * col_b.y)));
        // dL/da and the mask-gradient terms: scalar for the quad layouts, packed
        // for the others (each measured faster on B200)
        float2 dlda, u, v;
        if (kQuad) {
          dlda = make_float2(tk.x * fmaf(ga.x, bt.x, gcc.x - h.x), tk.y * fmaf(ga.y, bt.y, gcc.y - h.y));
          u = make_float2(dlda.x * (f0 ? gx.x : 0.f), dlda.y * (f1 ? gx.y : 0.f));
          v = make_float2(dlda.x * (f0 ? gy.x : 0.f), dlda.y * (f1 ? gy.y : 0.f));
        } else {
          dlda = mul2(tk, fma2(ga, bt, sub2(g, gcc, h)));
          u = mul2(dlda, make_float2(f0 ? gx.x : 0.f, f1 ? gx.y : 0.f));
          v = mul2(dlda, make_float2(f0 ? gy.x : 0.f, f1 ? gy.y : 0.f));
        }
        const float2 ex = add2(tx, g.nhx), ey = add2(ty, g.nhy);
        const float2 wt = mul2(a, tk);
        float acc[8];
        acc[0] = u.x + u.y;
        acc[1] = v.x + v.y;
        {
          const float2 r = fma2(u, ex, mul2(v, ey));
          acc[2] = r.x + r.y;
        }
        {
          const float2 r = fma2(mul2(u, g.rxy2), ey, mul2(mul2(v, g.nryx2), ex));
          acc[3] = r.x + r.y;
        }
        acc[4] = fmaf(gcr.y, wt.y, gcr.x * wt.x);
        acc[5] = fmaf(gcg.y, wt.y, gcg.x * wt.x);
        acc[6] = fmaf(gcb.y, wt.y, gcb.x * wt.x);
        acc[7] = fmaf(dlda.y, a.y, dlda.x * a.x);
        h = make_float2(fmaf(om.x, h.x, a.x * gcc.x), fmaf(om.y, h.y, a.y * gcc.y));
        bt = make_float2(bt.x * om.x, bt.y * om.y);
        if (__any_sync(kFull, f0 || f1)) warp_add(acc, kidx, gacc + (size_t)id * 8);
      }
    }
    Ts[0] = ts.x;
    Ts[1] = ts.y;
  }

  // Forward walk.  STATS: counts (pixel, primitive) pairs that pass the cull
  // and fragments composited, both before termination, plus walk statistics;
  // it evaluates the clearance-grid test without skipping and counts the
  // warp entries it would skip and, among them, those with a fragment (a
  // correct grid gives 0).
  template <bool STATS = false>
  __device__ __forceinline__ void forward(const Geom& g, const PrimInfo* __restrict__ prims,
                                          const void* __restrict__ atlas, const int* __restrict__ idx,
                                          Rec* w,
                                          float (&C)[NP][3], float (&T)[NP], float (&Tl)[NP], int (&lp)[NP],
                                          unsigned long long* cnt = nullptr) {
    if constexpr (kPair && !STATS) {
      forward_pair(g, prims, atlas, idx, w, C, T, Tl, lp);
      return;
    }
    unsigned long long n_cand = 0, n_frag = 0, n_went = 0, n_slots = 0, n_miss = 0, n_empty = 0, n_clear = 0,
                       n_bad = 0;
    unsigned n_depth[NP];
    const unsigned char* grid = static_cast<const unsigned char*>(atlas) + g.grid_off;
    bool live[NP];
    bool all_done = true;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      C[p][0] = C[p][1] = C[p][2] = 0.f;
      T[p] = 1.f; Tl[p] = 1.f; lp[p] = -1;
      live[p] = valid[p];
      n_depth[p] = 0;
      all_done = all_done && !live[p];
    }
    bool warp_done = __all_sync(kFull, all_done);
    for (int base = start; base < end && !warp_done; base += kChunk) {
      int my_id;
      const ChunkMasks cm = stage<STATS>(g, prims, idx, grid, base, end, w, &my_id);
      unsigned todo = cm.todo;
      if (STATS) n_miss += __popc(cm.miss);
      while (todo) {
        const int e = __ffs(todo) - 1;
        todo &= todo - 1;
        const float4 g0 = w[e][0];
        const float4 g1 = w[e][1];
        const float4 g2 = rec_g2(w[e]);
        const int toff = rec_toff(w[e]);
        const int pos = base - start + e;
        const bool clear = (cm.clear >> e) & 1u;
        if (STATS) {
          ++n_went;
          n_clear += clear;
#pragma unroll
          for (int p = 0; p < NP; ++p) n_slots += __popc(__ballot_sync(kFull, live[p]));
        }
        Sample s[NP];
        float m[NP];
        entry_sample<NP, L, KIND>(g, atlas, toff, g0, g1, (cm.inside >> e) & 1u, (cm.fast >> e) & 1u, pxf, pyf,
                                  live, s);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          m[p] = blend<false>(s[p], nullptr, nullptr);
          if (STATS) {
            const bool c = live[p] && !(fabsf(pxf[p] - g0.x) > g0.z || fabsf(pyf[p] - g0.y) > g0.w);
            n_cand += c;
          }
        }
        if (STATS) {
          bool anyf = false;
#pragma unroll
          for (int p = 0; p < NP; ++p) anyf = anyf || (s[p].ok && m[p] > 1e-6f);
          anyf = __any_sync(kFull, anyf);
          n_empty += !anyf;
          n_bad += clear && anyf;
        }
        bool local_done = true;
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const bool frag = s[p].ok && m[p] > 1e-6f;
          if (STATS) { n_frag += frag; n_depth[p] += frag; }
          const float a = frag ? g2.x * m[p] : 0.f;
          const float wt = T[p] * a;
          if (CB) {
            const float3 col = frag_colour(g, g2, __shfl_sync(kFull, my_id, e), s[p]);
            C[p][0] = fmaf(wt, col.x, C[p][0]);
            C[p][1] = fmaf(wt, col.y, C[p][1]);
            C[p][2] = fmaf(wt, col.z, C[p][2]);
          } else {
            C[p][0] = fmaf(wt, g2.y, C[p][0]);
            C[p][1] = fmaf(wt, g2.z, C[p][1]);
            C[p][2] = fmaf(wt, g2.w, C[p][2]);
          }
          Tl[p] = frag ? T[p] : Tl[p];
          lp[p] = frag ? pos : lp[p];
          // T (1 - a); 0 when a > 1 (alpha_max > 1).  a >= 0 (alpha_max >= 0), so
          // T stays <= 1 and saturating equals max(., 0), NaN included.
          T[p] = __saturatef(fmaf(-T[p], a, T[p]));
          live[p] = live[p] && !(T[p] < g.t_stop);
          local_done = local_done && !live[p];
        }
        if (__all_sync(kFull, local_done)) { warp_done = true; break; }
      }
    }
    if (STATS) {
      atomicAdd(cnt + 0, n_cand);
      atomicAdd(cnt + 1, n_frag);
      unsigned dmax = 0;
#pragma unroll
      for (int p = 0; p < NP; ++p) dmax = max(dmax, n_depth[p]);
      dmax = __reduce_max_sync(kFull, dmax);
      if (lane == 0) {
        atomicAdd(cnt + 3, n_went);
        atomicAdd(cnt + 4, n_slots);
        atomicAdd(cnt + 5, n_miss);
        atomicMax(cnt + 6, (unsigned long long)dmax);
        atomicAdd(cnt + 7, n_empty);
        atomicAdd(cnt + 8, n_clear);
        atomicAdd(cnt + 9, n_bad);
      }
    }
  }

  // Reverse walk.  gC/gA: upstream gradients per pixel; Ts: on entry the T
  // entering each pixel's last contributor (lp).  Per entry the warp reduces
  // its per-primitive partial sums and lanes 0..7 add them to gacc (N,8) f64
  // (layout documented at finalize_kernel).
  __device__ __forceinline__ void backward(const Geom& g, const PrimInfo* __restrict__ prims,
                                           const void* __restrict__ atlas, const int* __restrict__ idx,
                                           Rec* w, const float (&gC)[NP][3], const float (&gA)[NP],
                                           float (&Ts)[NP], const int (&lp)[NP], double* __restrict__ gacc) {
    if constexpr (kPair) {
      backward_pair(g, prims, atlas, idx, w, gC, gA, Ts, lp, gacc);
      return;
    }
    int my_max = -1;
#pragma unroll
    for (int p = 0; p < NP; ++p) my_max = max(my_max, lp[p]);
    const int warp_max = __reduce_max_sync(kFull, my_max);
    if (warp_max < 0) return;
    const unsigned char* grid = static_cast<const unsigned char*>(atlas) + g.grid_off;
    // sum index that lane l < 8 holds after the recursive-halving reduction
    const int kidx = 4 * (lane & 1) + 2 * ((lane >> 1) & 1) + ((lane >> 2) & 1);

    // H = gC . R and B = prod(1 - a) over the fragments behind the current
    // one, where R is their colour composited from T = 1; both obey
    // X_{k-1} = (1 - a_k) X_k + a_k x_k, so dL/da_k = T_k (gC.c_k - H + gA B).
    float H[NP], B[NP];
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      H[p] = 0.f;
      B[p] = 1.f;
    }
    for (int cb = (warp_max / kChunk) * kChunk; cb >= 0; cb -= kChunk) {
      int my_id;
      const ChunkMasks cm = stage<false>(g, prims, idx, grid, start + cb, start + warp_max + 1, w, &my_id);
      unsigned todo = cm.todo;
      while (todo) {
        const int e = 31 - __clz(todo);
        todo &= ~(1u << e);
        const int pos = cb + e;
        const int id = __shfl_sync(kFull, my_id, e);
        const float4 g0 = w[e][0];
        const float4 g1 = w[e][1];
        const float4 g2 = rec_g2(w[e]);
        const int toff = rec_toff(w[e]);
        float acc[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = 0.f;
        bool any = false;
        bool live[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) live[p] = pos <= lp[p];
        Sample s[NP];
        float m[NP], gx[NP], gy[NP];
        entry_sample<NP, L, KIND>(g, atlas, toff, g0, g1, (cm.inside >> e) & 1u, (cm.fast >> e) & 1u, pxf, pyf,
                                  live, s);
#pragma unroll
        for (int p = 0; p < NP; ++p) m[p] = blend<true>(s[p], &gx[p], &gy[p]);
#pragma unroll
        for (int p = 0; p < NP; ++p) {
          const bool frag = s[p].ok && m[p] > 1e-6f;
          const float a = frag ? g2.x * m[p] : 0.f;
          const float om = __saturatef(1.f - a);   // max(1 - a, 0) for a >= 0
          // T entering this fragment: stored for the last contributor, else
          // undo the forward product (om >= t_stop > 0 for every earlier
          // fragment, so the fast division is well conditioned; om = 1 and
          // Ts is unchanged when there is no fragment).
          const float Tk = (pos == lp[p]) ? Ts[p] : __fdividef(Ts[p], om);
          Ts[p] = Tk;
          const float3 col = frag_colour(g, g2, id, s[p]);
          const float gCc = fmaf(gC[p][0], col.x, fmaf(gC[p][1], col.y, gC[p][2] * col.z));
          // a pixel without a fragment contributes nothing: a = 0 zeroes its colour
          // and opacity terms, and its mask gradient (from a redirected texel,
          // possibly NaN) is replaced by 0 rather than multiplied by 0
          const float dLda = Tk * (gCc - H[p] + gA[p] * B[p]);
          const float u = dLda * (frag ? gx[p] : 0.f), v = dLda * (frag ? gy[p] : 0.f);
          const float ex = s[p].tx - g.hx, ey = s[p].ty - g.hy;
          acc[0] += u;
          acc[1] += v;
          acc[2] = fmaf(u, ex, fmaf(v, ey, acc[2]));
          acc[3] = fmaf(u * g.rxy, ey, fmaf(-v * g.ryx, ex, acc[3]));
          const float wt = a * Tk;
          acc[4] = fmaf(gC[p][0], wt, acc[4]);
          acc[5] = fmaf(gC[p][1], wt, acc[5]);
          acc[6] = fmaf(gC[p][2], wt, acc[6]);
          acc[7] = fmaf(dLda, a, acc[7]);
          H[p] = fmaf(om, H[p], a * gCc);
          B[p] *= om;
          any = any || frag;
        }
        if (__any_sync(kFull, any)) warp_add(acc, kidx, gacc + (size_t)id * 8);
      }
    }
  }
};

// CTA shape of the walk kernels: a CTA runs kCtaWarps warps of one tile (the
// warps walk independently, so a tile may be split over several CTAs, which
// lets an SM refill as soon as a few warps finish); kParts CTAs per tile.
// Registers are bounded for a number of resident warps per SM, tuned on B200
// per atlas kind: 36 (56 registers a thread, a few bytes of spills) for the
// packed atlases, whose walk waits mostly on texel loads and gains from the
// extra warps; 32 (64 registers) for the reference layout and the
// colour-map walks.
#ifndef DBMP_CTA_WARPS
#define DBMP_CTA_WARPS 4
#endif
#ifndef DBMP_WARPS_PER_SM
#define DBMP_WARPS_PER_SM 36
#endif
#ifndef DBMP_WARPS_PER_SM_F32
#define DBMP_WARPS_PER_SM_F32 32
#endif
template <int TS> constexpr int kTileWarps() { return Layout<TS, DefaultNP<TS>::v>::NW; }
template <int TS> constexpr int kCtaWarps() {
  return kTileWarps<TS>() < DBMP_CTA_WARPS ? kTileWarps<TS>() : DBMP_CTA_WARPS;
}
template <int TS> constexpr int kParts() { return kTileWarps<TS>() / kCtaWarps<TS>(); }
template <int TS> constexpr int kThreadsOf() { return kCtaWarps<TS>() * 32; }
template <int TS, int KIND, bool CB = false> constexpr int kBlocksPerSM() {
  constexpr int w = (KIND == ATLAS_F32 || CB) ? DBMP_WARPS_PER_SM_F32 : DBMP_WARPS_PER_SM;
  return w / kCtaWarps<TS>() > 0 ? w / kCtaWarps<TS>() : 1;
}

// ---------------------------------------------------------------------------
template <int TS, int KIND, bool CB>
__global__ void __launch_bounds__(kThreadsOf<TS>(), kBlocksPerSM<TS, KIND, CB>()) forward_kernel(
    Geom g, const PrimInfo* __restrict__ prims, const void* __restrict__ atlas, const int* __restrict__ offs,
    const int* __restrict__ idx, float* __restrict__ out_color, float* __restrict__ out_alpha,
    float* __restrict__ T_last, int* __restrict__ last_pos, const float* __restrict__ cmap, float cblend,
    long long idx_stride, long long cmap_stride) {
  constexpr int NP = DefaultNP<TS>::v;
  using TW = TileWalker<TS, NP, KIND, CB>;
  __shared__ typename TW::Rec s_pi[kCtaWarps<TS>()][kChunk];
  // a batch of candidates is one grid over all their tiles: candidate b's
  // records, lists and images follow candidate b-1's
  const int gt = blockIdx.x / kParts<TS>(), part = blockIdx.x % kParts<TS>();
  const int b = gt / g.T, tile = gt - b * g.T;
  const size_t pix = (size_t)b * g.H * g.W;
  prims += (size_t)b * g.N;
  offs += (size_t)b * (g.T + 1);
  idx += (size_t)b * idx_stride;
  out_color += 3 * pix; out_alpha += pix; T_last += pix; last_pos += pix;
  TW tw;
  tw.cmap = CB ? cmap + (size_t)b * cmap_stride : cmap;
  tw.cblend = cblend;
  tw.init(g, tile, part, kCtaWarps<TS>(), offs);
  float C[NP][3], T[NP], Tl[NP];
  int lp[NP];
  tw.forward(g, prims, atlas, idx, s_pi[tw.lw], C, T, Tl, lp);
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    if (!tw.valid[p]) continue;
    const size_t q = (size_t)tw.py(tile, g, p) * g.W + tw.px(tile, g, p);
    out_color[3 * q + 0] = C[p][0];
    out_color[3 * q + 1] = C[p][1];
    out_color[3 * q + 2] = C[p][2];
    out_alpha[q] = 1.f - T[p];
    T_last[q] = Tl[p];
    last_pos[q] = lp[p];
  }
}

// Counting pass (diagnostics / roofline accounting): same walk as the
// forward, no outputs except the counters.
template <int TS, int KIND>
__global__ void __launch_bounds__(kThreadsOf<TS>()) count_kernel(Geom g, const PrimInfo* __restrict__ prims,
                                                                 const void* __restrict__ atlas,
                                                                 const int* __restrict__ offs,
                                                                 const int* __restrict__ idx,
                                                                 unsigned long long* __restrict__ cnt) {
  constexpr int NP = DefaultNP<TS>::v;
  using TW = TileWalker<TS, NP, KIND>;
  __shared__ typename TW::Rec s_pi[kCtaWarps<TS>()][kChunk];
  TW tw;
  const int tile = blockIdx.x / kParts<TS>(), part = blockIdx.x % kParts<TS>();
  tw.init(g, tile, part, kCtaWarps<TS>(), offs);
  float C[NP][3], T[NP], Tl[NP];
  int lp[NP];
  tw.template forward<true>(g, prims, atlas, idx, s_pi[tw.lw], C, T, Tl, lp, cnt);
  if (threadIdx.x == 0 && part == 0) atomicAdd(cnt + 2, (unsigned long long)(tw.end - tw.start));
}

template <int TS, int KIND, bool CB>
__global__ void __launch_bounds__(kThreadsOf<TS>(), kBlocksPerSM<TS, KIND, CB>()) backward_kernel(
    Geom g, const PrimInfo* __restrict__ prims, const void* __restrict__ atlas, const int* __restrict__ offs,
    const int* __restrict__ idx, const float* __restrict__ T_last, const int* __restrict__ last_pos,
    const float* __restrict__ grad_color, const float* __restrict__ grad_alpha, double* __restrict__ gacc,
    const float* __restrict__ cmap, float cblend, long long idx_stride, long long cmap_stride) {
  constexpr int NP = DefaultNP<TS>::v;
  using TW = TileWalker<TS, NP, KIND, CB>;
  __shared__ typename TW::Rec s_pi[kCtaWarps<TS>()][kChunk];
  const int gt = blockIdx.x / kParts<TS>(), part = blockIdx.x % kParts<TS>();
  const int b = gt / g.T, tile = gt - b * g.T;     // candidate and tile (see forward_kernel)
  const size_t pix = (size_t)b * g.H * g.W;
  prims += (size_t)b * g.N;
  offs += (size_t)b * (g.T + 1);
  idx += (size_t)b * idx_stride;
  T_last += pix; last_pos += pix; grad_color += 3 * pix;
  if (grad_alpha != nullptr) grad_alpha += pix;
  gacc += (size_t)b * g.N * 8;
  TW tw;
  tw.cmap = CB ? cmap + (size_t)b * cmap_stride : cmap;
  tw.cblend = cblend;
  tw.init(g, tile, part, kCtaWarps<TS>(), offs);
  float gC[NP][3], gA[NP], Ts[NP];
  int lp[NP];
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    if (tw.valid[p]) {
      const size_t q = (size_t)tw.py(tile, g, p) * g.W + tw.px(tile, g, p);
      gC[p][0] = grad_color[3 * q + 0];
      gC[p][1] = grad_color[3 * q + 1];
      gC[p][2] = grad_color[3 * q + 2];
      gA[p] = grad_alpha ? grad_alpha[q] : 0.f;
      Ts[p] = T_last[q];
      lp[p] = last_pos[q];
    } else {
      gC[p][0] = gC[p][1] = gC[p][2] = 0.f;
      gA[p] = 0.f; Ts[p] = 1.f; lp[p] = -1;
    }
  }
  tw.backward(g, prims, atlas, idx, s_pi[tw.lw], gC, gA, Ts, lp, gacc);
}

__device__ __forceinline__ double sigmoid_d(double x) {
  if (x >= 0.0) { const double z = exp(-x); return 1.0 / (1.0 + z); }
  const double z = exp(x);
  return z / (1.0 + z);
}

// Converts the accumulated per-primitive sums into the reference's gradient
// outputs (tile_backward.cu:255-343 chain rule, applied once per primitive).
// gacc[n] = { S dLda*gx, S dLda*gy, S dLda*(gx*ex + gy*ey),
//             S dLda*(gx*ey*hx/hy - gy*ex*hy/hx), S gC_r*a*T, S gC_g*a*T,
//             S gC_b*a*T, S dLda*a }  summed over the primitive's fragments,
// with (ex, ey) the texel coordinate minus (hx, hy) and gx, gy = d mask/d tex.
__global__ void finalize_kernel(Geom g, const float* __restrict__ radii, const float* __restrict__ rot,
                                const float* __restrict__ opac, const float* __restrict__ colors,
                                const double* __restrict__ gacc, float* __restrict__ g_means,
                                float* __restrict__ g_radii, float* __restrict__ g_rot, float* __restrict__ g_opac,
                                float* __restrict__ g_colors) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= g.N) return;
  const double* S = gacc + (size_t)n * 8;
  const float r = radii[n];
  const double rinv = (r > 1e-6f) ? 1.0 / (double)r : 1e6;
  double s, c;
  sincos((double)rot[n], &s, &c);
  const double sv = sigmoid_d((double)opac[n]);
  const double a0 = (double)g.alpha_max * sv;
  const double hx = g.hx, hy = g.hy;
  // A primitive without fragments has zero sums and zero gradients, also when
  // its rotation is not finite (the reference adds gradients per fragment): a
  // zero sum contributes 0 rather than NaN * 0.
  const double cx = S[0] != 0.0 ? c * hx * S[0] : 0.0, sx = S[0] != 0.0 ? s * hx * S[0] : 0.0;
  const double cy = S[1] != 0.0 ? c * hy * S[1] : 0.0, sy = S[1] != 0.0 ? s * hy * S[1] : 0.0;
  g_means[2 * n + 0] = (float)(a0 * rinv * (sy - cx));
  g_means[2 * n + 1] = (float)(a0 * rinv * (-sx - cy));
  g_radii[n] = (float)(-a0 * rinv * S[2]);
  g_rot[n] = (float)(a0 * S[3]);
  g_opac[n] = (float)((1.0 - sv) * S[7]);
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const double sc = sigmoid_d((double)colors[3 * n + ch]);
    g_colors[3 * n + ch] = (float)(sc * (1.0 - sc) * S[4 + ch]);
  }
}

// ---------------------------------------------------------------------------
// Fused forward + L2 loss + backward for image fitting.  The loss is the
// reference's mse_loss(rendered, target) (pydiffbmp/util/loss_functions.py:20-40)
// on rendered = C + (1 - A) * background (simple_tile_renderer.py:704-707):
//   dL/dC = 2 (rendered - target) / (3HW),  dL/dA = -sum_c dL/dC_c * bg_c.
// loss_out (f64, may be null) receives sum((rendered - target)^2) / (3HW):
// each warp leaves its partial in shared memory and the CTA's last warp to
// finish its forward walk adds the CTA's sum (no barrier between the walks).
template <int TS, int KIND>
__global__ void __launch_bounds__(kThreadsOf<TS>(), kBlocksPerSM<TS, KIND>()) fused_kernel(
    Geom g, const PrimInfo* __restrict__ prims, const void* __restrict__ atlas, const int* __restrict__ offs,
    const int* __restrict__ idx, const float* __restrict__ target, const float* __restrict__ background,
    float* __restrict__ out_image, double* __restrict__ gacc, double* __restrict__ loss_out,
    const int* __restrict__ skip_flag) {
  if (skip_flag != nullptr && *skip_flag != 0) return;   // binning overflowed: leave all state untouched
  constexpr int NP = DefaultNP<TS>::v;
  using TW = TileWalker<TS, NP, KIND>;
  __shared__ typename TW::Rec s_pi[kCtaWarps<TS>()][kChunk];
  __shared__ float s_loss[kCtaWarps<TS>()];
  __shared__ unsigned s_arrived;
  if (threadIdx.x == 0) s_arrived = 0u;
  __syncthreads();
  TW tw;
  const int tile = blockIdx.x / kParts<TS>(), part = blockIdx.x % kParts<TS>();
  tw.init(g, tile, part, kCtaWarps<TS>(), offs);
  float C[NP][3], T[NP], Tl[NP], gC[NP][3], gA[NP];
  int lp[NP];
  tw.forward(g, prims, atlas, idx, s_pi[tw.lw], C, T, Tl, lp);
  const float inv = 1.f / (3.f * (float)g.H * (float)g.W);
  float lsum = 0.f;
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    gA[p] = 0.f;
    gC[p][0] = gC[p][1] = gC[p][2] = 0.f;
    if (!tw.valid[p]) continue;
    const size_t q = (size_t)tw.py(tile, g, p) * g.W + tw.px(tile, g, p);
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      const float bg = background ? background[3 * q + ch] : 0.f;
      const float img = fmaf(T[p], bg, C[p][ch]);
      if (out_image) out_image[3 * q + ch] = img;
      const float d = img - target[3 * q + ch];
      lsum = fmaf(d, d, lsum);
      gC[p][ch] = 2.f * d * inv;
      gA[p] -= gC[p][ch] * bg;
    }
  }
  if (loss_out) {
    lsum += __shfl_xor_sync(kFull, lsum, 16);
    lsum += __shfl_xor_sync(kFull, lsum, 8);
    lsum += __shfl_xor_sync(kFull, lsum, 4);
    lsum += __shfl_xor_sync(kFull, lsum, 2);
    lsum += __shfl_xor_sync(kFull, lsum, 1);
    if (tw.lane == 0) {
      s_loss[tw.lw] = lsum;
      __threadfence_block();
      if (atomicAdd(&s_arrived, 1u) == (unsigned)(kCtaWarps<TS>() - 1)) {
        __threadfence_block();
        const volatile float* sl = s_loss;
        double t = 0.0;
        for (int w = 0; w < kCtaWarps<TS>(); ++w) t += sl[w];
        atomicAdd(loss_out, t * (double)inv);
      }
    }
  }
  tw.backward(g, prims, atlas, idx, s_pi[tw.lw], gC, gA, Tl, lp, gacc);
}

// ---------------------------------------------------------------------------
#define DBMP_KIND_SWITCH(kind, ...)                                                   \
  switch (kind) {                                                                     \
    case ATLAS_F32: { constexpr int KD = ATLAS_F32; __VA_ARGS__; } break;             \
    case ATLAS_F32_QUAD: { constexpr int KD = ATLAS_F32_QUAD; __VA_ARGS__; } break;   \
    case ATLAS_F16_QUAD: { constexpr int KD = ATLAS_F16_QUAD; __VA_ARGS__; } break;   \
    case ATLAS_BF16_QUAD: { constexpr int KD = ATLAS_BF16_QUAD; __VA_ARGS__; } break; \
    case ATLAS_F16_PAIR: { constexpr int KD = ATLAS_F16_PAIR; __VA_ARGS__; } break;   \
    case ATLAS_BF16_PAIR: { constexpr int KD = ATLAS_BF16_PAIR; __VA_ARGS__; } break; \
    default: set_error("unknown atlas kind %d", kind); return DBMP_ERR_INVALID;       \
  }

#define DBMP_TS_SWITCH(ts, ...)                                      \
  if ((ts) == 32) { constexpr int TSV = 32; __VA_ARGS__; }           \
  else if ((ts) == 16) { constexpr int TSV = 16; __VA_ARGS__; }      \
  else { set_error("tile_size %d is not supported (16 or 32)", ts); return DBMP_ERR_INVALID; }

// batch > 1: `batch` candidates of the same canvas in one grid, candidate b's
// records at prims + b N, lists at offs + b (T+1) / idx + b idx_stride,
// images at b H W (x3 for colour), colour maps at cmap + b cmap_stride.
int launch_forward_blend(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs,
                         const int* idx, float* color, float* alpha, float* T_last, int* last_pos, const float* cmap,
                         float cblend, cudaStream_t st, int batch, long long idx_stride, long long cmap_stride) {
  if (g.T == 0 || batch == 0) return DBMP_OK;
  const long long ctas = (long long)batch * g.T * kParts<32>();
  if (ctas > 0x7fffffffll) { set_error("forward: %d candidates x %d tiles exceed one grid", batch, g.T); return DBMP_ERR_INVALID; }
  if (cmap != nullptr && cblend > 0.f) {
    DBMP_TS_SWITCH(g.TS, DBMP_KIND_SWITCH(kind, (forward_kernel<TSV, KD, true>
                                                 <<<batch * g.T * kParts<TSV>(), kThreadsOf<TSV>(), 0, st>>>(
                                                     g, prims, atlas, offs, idx, color, alpha, T_last, last_pos,
                                                     cmap, cblend, idx_stride, cmap_stride))));
  } else {
    DBMP_TS_SWITCH(g.TS, DBMP_KIND_SWITCH(kind, (forward_kernel<TSV, KD, false>
                                                 <<<batch * g.T * kParts<TSV>(), kThreadsOf<TSV>(), 0, st>>>(
                                                     g, prims, atlas, offs, idx, color, alpha, T_last, last_pos,
                                                     nullptr, 0.f, idx_stride, 0))));
  }
  DBMP_CHECK_LAUNCH("forward_kernel");
  return DBMP_OK;
}

int launch_forward(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs,
                   const int* idx, float* color, float* alpha, float* T_last, int* last_pos, cudaStream_t st) {
  return launch_forward_blend(g, kind, prims, atlas, offs, idx, color, alpha, T_last, last_pos, nullptr, 0.f, st, 1,
                              0, 0);
}

int launch_count(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs, const int* idx,
                 unsigned long long* cnt, cudaStream_t st) {
  if (g.T == 0) return DBMP_OK;
  DBMP_TS_SWITCH(g.TS, DBMP_KIND_SWITCH(kind, (count_kernel<TSV, KD><<<g.T * kParts<TSV>(), kThreadsOf<TSV>(), 0, st>>>(
                                                   g, prims, atlas, offs, idx, cnt))));
  DBMP_CHECK_LAUNCH("count_kernel");
  return DBMP_OK;
}

int launch_backward_blend(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs,
                          const int* idx, const float* T_last, const int* last_pos, const float* grad_color,
                          const float* grad_alpha, double* gacc, const float* cmap, float cblend, cudaStream_t st,
                          int batch, long long idx_stride, long long cmap_stride) {
  if (g.T == 0 || batch == 0) return DBMP_OK;
  const long long ctas = (long long)batch * g.T * kParts<32>();
  if (ctas > 0x7fffffffll) { set_error("backward: %d candidates x %d tiles exceed one grid", batch, g.T); return DBMP_ERR_INVALID; }
  if (cmap != nullptr && cblend > 0.f) {
    DBMP_TS_SWITCH(g.TS, DBMP_KIND_SWITCH(kind, (backward_kernel<TSV, KD, true>
                                                 <<<batch * g.T * kParts<TSV>(), kThreadsOf<TSV>(), 0, st>>>(
                                                     g, prims, atlas, offs, idx, T_last, last_pos, grad_color,
                                                     grad_alpha, gacc, cmap, cblend, idx_stride, cmap_stride))));
  } else {
    DBMP_TS_SWITCH(g.TS, DBMP_KIND_SWITCH(kind, (backward_kernel<TSV, KD, false>
                                                 <<<batch * g.T * kParts<TSV>(), kThreadsOf<TSV>(), 0, st>>>(
                                                     g, prims, atlas, offs, idx, T_last, last_pos, grad_color,
                                                     grad_alpha, gacc, nullptr, 0.f, idx_stride, 0))));
  }
  DBMP_CHECK_LAUNCH("backward_kernel");
  return DBMP_OK;
}

int launch_backward(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs,
                    const int* idx, const float* T_last, const int* last_pos, const float* grad_color,
                    const float* grad_alpha, double* gacc, cudaStream_t st) {
  return launch_backward_blend(g, kind, prims, atlas, offs, idx, T_last, last_pos, grad_color, grad_alpha, gacc,
                               nullptr, 0.f, st, 1, 0, 0);
}

int launch_finalize(const Geom& g, const float* radii, const float* rot, const float* opac, const float* colors,
                    const double* gacc, float* gm, float* gr, float* grot, float* go, float* gc, cudaStream_t st) {
  if (g.N == 0) return DBMP_OK;
  finalize_kernel<<<(g.N + 255) / 256, 256, 0, st>>>(g, radii, rot, opac, colors, gacc, gm, gr, grot, go, gc);
  DBMP_CHECK_LAUNCH("finalize_kernel");
  return DBMP_OK;
}

int launch_fused(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs, const int* idx,
                 const float* target, const float* background, float* out_image, double* gacc, double* loss,
                 const int* skip_flag, cudaStream_t st) {
  if (g.T == 0) return DBMP_OK;
  DBMP_TS_SWITCH(g.TS, DBMP_KIND_SWITCH(kind, (fused_kernel<TSV, KD><<<g.T * kParts<TSV>(), kThreadsOf<TSV>(), 0, st>>>(
                                                   g, prims, atlas, offs, idx, target, background, out_image,
                                                   gacc, loss, skip_flag))));
  DBMP_CHECK_LAUNCH("fused_kernel");
  return DBMP_OK;
}

}  // namespace dbmp
