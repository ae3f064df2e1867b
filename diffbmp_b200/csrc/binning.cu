// Device binning: per-primitive preparation, primitive -> tile rectangles,
// then CSR tile lists built row by row without a sort: for each tile row a
// group of CTAs walks the primitives in index order, compacts those whose
// rectangle touches the group's tiles, and each warp counts (first pass) or
// writes (second pass) the entries of its own tile.  Lists therefore come out
// in ascending primitive order per tile, as the reference's per-tile nonzero()
// gives them, with no host round trip.
//
// This translation unit is compiled WITHOUT fast-math: the world-space bbox
// must reproduce the reference's float32 torch element-wise arithmetic
// (pydiffbmp/core/renderer/vector_renderer.py:214-250: torch.cos/torch.sin,
// then one rounding per multiply / add, no FMA) bit for bit.
#include <cub/cub.cuh>

#include "dbmp_internal.cuh"

namespace dbmp {

// ---------------------------------------------------------------------------
// Template bboxes (simple_tile_renderer.py:130-171): min/max texel column and
// row over texels > 1e-6, mapped with u = (col/(W-1))*2-1 in float32.  The
// map is monotone, so min/max of the integer indices give min/max of u.
__global__ void template_bbox_kernel(const float* __restrict__ tmpl, int Ht, int Wt,
                                     float* __restrict__ out) {
  const int p = blockIdx.x;
  const float* t = tmpl + (size_t)p * Ht * Wt;
  int mnx = INT_MAX, mxx = -1, mny = INT_MAX, mxy = -1;
  for (int i = threadIdx.x; i < Ht * Wt; i += blockDim.x) {
    if (t[i] > 1e-6f) {
      const int y = i / Wt, x = i - y * Wt;
      mnx = min(mnx, x); mxx = max(mxx, x); mny = min(mny, y); mxy = max(mxy, y);
    }
  }
  typedef cub::BlockReduce<int, 256> BR;
  __shared__ typename BR::TempStorage tmp;
  const int a = BR(tmp).Reduce(mnx, cub::Min()); __syncthreads();
  const int b = BR(tmp).Reduce(mxx, cub::Max()); __syncthreads();
  const int c = BR(tmp).Reduce(mny, cub::Min()); __syncthreads();
  const int d = BR(tmp).Reduce(mxy, cub::Max());
  if (threadIdx.x == 0) {
    if (b < 0) {
      out[4 * p + 0] = -1.f; out[4 * p + 1] = 1.f; out[4 * p + 2] = -1.f; out[4 * p + 3] = 1.f;
    } else {
      const float dw = (float)(Wt - 1), dh = (float)(Ht - 1);
      out[4 * p + 0] = __fsub_rn(__fmul_rn(__fdiv_rn((float)a, dw), 2.f), 1.f);
      out[4 * p + 1] = __fsub_rn(__fmul_rn(__fdiv_rn((float)b, dw), 2.f), 1.f);
      out[4 * p + 2] = __fsub_rn(__fmul_rn(__fdiv_rn((float)c, dh), 2.f), 1.f);
      out[4 * p + 3] = __fsub_rn(__fmul_rn(__fdiv_rn((float)d, dh), 2.f), 1.f);
    }
  }
}

// ---------------------------------------------------------------------------
// Atlas repacking into bilinear quads / pairs (precision form).  Each record
// holds a texel and the difference to its right neighbour, the difference
// taken against the stored (rounded) texel, so that stored texel + stored
// difference is the neighbour up to one rounding of the difference.
template <typename OutT>
__device__ __forceinline__ OutT to_storage(float v);
template <> __device__ __forceinline__ float to_storage<float>(float v) { return v; }
template <> __device__ __forceinline__ __half to_storage<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_storage<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }
__device__ __forceinline__ float from_storage(float v) { return v; }
__device__ __forceinline__ float from_storage(__half v) { return __half2float(v); }
__device__ __forceinline__ float from_storage(__nv_bfloat16 v) { return __bfloat162float(v); }

// Pair layout: (P, Ht+1, Wt) records of (t[y][x], t[y][x+1] - t[y][x]); row Ht is zero.
template <typename OutT>
__global__ void atlas_pair_kernel(const float* __restrict__ tmpl, int P, int Ht, int Wt, OutT* __restrict__ out) {
  const long long total = (long long)P * (Ht + 1) * Wt;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % Wt);
    const int y = (int)((i / Wt) % (Ht + 1));
    const long long p = i / ((long long)(Ht + 1) * Wt);
    const float* t = tmpl + (size_t)p * Ht * Wt;
    const float v0 = (y < Ht) ? t[(size_t)y * Wt + x] : 0.f;
    const float v1 = (y < Ht && x + 1 < Wt) ? t[(size_t)y * Wt + x + 1] : 0.f;
    const OutT s0 = to_storage<OutT>(v0);
    out[2 * i] = s0;
    out[2 * i + 1] = to_storage<OutT>(v1 - from_storage(s0));
  }
}

// Quad layout: (P, Ht, Wt) records of (t[y][x], t[y][x+1] - t[y][x], t[y+1][x],
// t[y+1][x+1] - t[y+1][x]); neighbours outside the template are 0.
template <typename OutT>
__global__ void atlas_pack_kernel(const float* __restrict__ tmpl, int P, int Ht, int Wt, OutT* __restrict__ out) {
  const long long total = (long long)P * Ht * Wt;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % Wt);
    const int y = (int)((i / Wt) % Ht);
    const float* t = tmpl + (i - (long long)y * Wt - x);
    const bool xr = x + 1 < Wt, yr = y + 1 < Ht;
    const float v00 = t[(size_t)y * Wt + x];
    const float v01 = xr ? t[(size_t)y * Wt + x + 1] : 0.f;
    const float v10 = yr ? t[(size_t)(y + 1) * Wt + x] : 0.f;
    const float v11 = (xr && yr) ? t[(size_t)(y + 1) * Wt + x + 1] : 0.f;
    OutT* o = out + 4 * i;
    const OutT s00 = to_storage<OutT>(v00), s10 = to_storage<OutT>(v10);
    o[0] = s00; o[1] = to_storage<OutT>(v01 - from_storage(s00));
    o[2] = s10; o[3] = to_storage<OutT>(v11 - from_storage(s10));
  }
}

// ---------------------------------------------------------------------------
// Per-primitive preparation.
__device__ __forceinline__ float nan_min(float a, float b) { return (isnan(a) || isnan(b)) ? __int_as_float(0x7fc00000) : fminf(a, b); }
__device__ __forceinline__ float nan_max(float a, float b) { return (isnan(a) || isnan(b)) ? __int_as_float(0x7fc00000) : fmaxf(a, b); }

// Tile columns hit by [bmin, bmax] under the reference's inclusive test
// !(bmax < tile_start || bmin > tile_end) with tile_end = min(start+ts, W)
// compared in float32 (vector_renderer.py:437-438).  NaN makes the test pass.
__device__ __forceinline__ int2 tile_span_content(float bmin, float bmax, int ts, int extent, int ntiles) {
  auto ts_start = [&](int t) { return (float)(t * ts); };
  auto ts_end = [&](int t) { return (float)min(t * ts + ts, extent); };
  int lo, hi;
  if (isnan(bmin)) lo = 0;
  else if (bmin > (float)extent) lo = ntiles;
  else if (bmin <= 0.f) lo = 0;
  else {
    lo = max(0, (int)floorf(bmin / (float)ts) - 2);
    while (lo < ntiles && bmin > ts_end(lo)) ++lo;
  }
  if (isnan(bmax)) hi = ntiles - 1;
  else if (bmax < 0.f) hi = -1;
  else if (bmax >= ts_start(ntiles - 1)) hi = ntiles - 1;
  else {
    hi = min(ntiles - 1, (int)floorf(bmax / (float)ts) + 2);
    while (hi >= 0 && bmax < ts_start(hi)) --hi;
  }
  return make_int2(lo, hi);
}

// Pixels p in [0, extent) that pass the kernel's square cull
// !(fabsf((float)p - m) > h) (tile_forward.cu:208), as a tile span.  The
// predicate is monotone in |p - m|, so the passing pixels form an interval.
__device__ __forceinline__ int2 tile_span_cull(float m, float h, int ts, int extent) {
  auto pass = [&](int p) { return !(fabsf((float)p - m) > h); };
  if (isnan(m) || isnan(h)) return make_int2(0, (extent - 1) / ts);
  if (h < 0.f) return make_int2(1, 0);
  const float lo_f = fminf(fmaxf(floorf(m - h) - 2.f, 0.f), (float)extent);
  const float hi_f = fminf(fmaxf(ceilf(m + h) + 2.f, -1.f), (float)(extent - 1));
  int a = (int)lo_f, b = (int)hi_f;
  while (a <= b && !pass(a)) ++a;
  while (b >= a && !pass(b)) --b;
  if (a > b) return make_int2(1, 0);
  return make_int2(a / ts, b / ts);
}

__global__ void prepare_kernel(Geom g, const float* __restrict__ means2D, const float* __restrict__ radii,
                               const float* __restrict__ rot, const float* __restrict__ opac,
                               const float* __restrict__ colors, const int* __restrict__ sel,
                               const float* __restrict__ tbbox, int bin_mode, PrimInfo* __restrict__ out,
                               int4* __restrict__ rects, int* __restrict__ diff, int span) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= g.N) return;
  const float mx = means2D[2 * n], my = means2D[2 * n + 1];
  const float r = radii[n], th = rot[n];
  const int tid = sel[n];
  const bool valid = tid >= 0 && tid < g.P;

  PrimInfo pi;
  pi.mx = mx; pi.my = my;
  // square cull half extents, in the reference's operation order (tile_forward.cu:198-205)
  const float maxd = fmaxf((float)g.Wt, (float)g.Ht);
  const float scale = __fdiv_rn(r, __fmul_rn(maxd, 0.5f));
  pi.hw = __fmul_rn(__fmul_rn((float)g.Wt, 0.5f), scale);
  pi.hh = __fmul_rn(__fmul_rn((float)g.Ht, 0.5f), scale);
  // inverse affine in double, rounded once (tile_forward.cu:250-264)
  const double rinv = (r > 1e-6f) ? 1.0 / (double)r : 1e6;
  double s, c;
  sincos((double)th, &s, &c);
  pi.a00 = (float)(c * rinv * (double)g.hx);
  pi.a01 = (float)(s * rinv * (double)g.hx);
  pi.a10 = (float)(-s * rinv * (double)g.hy);
  pi.a11 = (float)(c * rinv * (double)g.hy);
  pi.alpha0 = g.alpha_max * sigmoid_precise(opac[n]);
  pi.cr = sigmoid_precise(colors[3 * n + 0]);
  pi.cg = sigmoid_precise(colors[3 * n + 1]);
  pi.cb = sigmoid_precise(colors[3 * n + 2]);
  if (half_record(g.kind)) {   // the precision form stores opacity and colours in FP16
    const __half2 ar = __floats2half2_rn(pi.alpha0, pi.cr), gb = __floats2half2_rn(pi.cg, pi.cb);
    pi.alpha0 = __uint_as_float(*reinterpret_cast<const unsigned*>(&ar));
    pi.cr = __uint_as_float(*reinterpret_cast<const unsigned*>(&gb));
    pi.cg = pi.cb = 0.f;
  }
  const bool nan_geom = isnan(pi.a00) || isnan(pi.a01) || isnan(pi.a10) || isnan(pi.a11) || isnan(mx) || isnan(my);
  pi.toff = (!valid || nan_geom) ? kNoFrag : tid * template_records(g.kind, g.Ht, g.Wt);
  // clearance a warp footprint needs before the walk may skip it: the
  // footprint's texel-space half extent, plus the bilinear reach of 1 texel,
  // plus slack for the rounding of the per-pixel texel coordinates
  const float ex = fabsf(pi.a00) * g.fhx + fabsf(pi.a01) * g.fhy;
  const float ey = fabsf(pi.a10) * g.fhx + fabsf(pi.a11) * g.fhy;
  const float need = fmaxf(ex, ey) + 1.05f;
  pi.goff = valid ? tid * g.gGx * g.gGy : 0;
  pi.gext = (atlas_has_grid(g.kind) && need < (float)kGridCap) ? (int)ceilf(need) : kGridCap + 1;
  pi.pad = 0;
  out[n] = pi;

  if (rects == nullptr) return;
  int2 sx, sy;
  if (bin_mode == DBMP_BIN_CONTENT || bin_mode == DBMP_BIN_CONTENT_REF) {
    // vector_renderer.py:221-250 with the bbox of this primitive's template,
    // or, in the reference-exact mode, of template (N-1-n) % P as the
    // reference always takes it (vector_renderer.py:220-226)
    const int q = (bin_mode == DBMP_BIN_CONTENT_REF) ? (g.N - 1 - n) % g.P : (valid ? tid : 0);
    const float c32 = cosf(th), s32 = sinf(th);
    const float cu[4] = {tbbox[4 * q + 0], tbbox[4 * q + 1], tbbox[4 * q + 0], tbbox[4 * q + 1]};
    const float cv[4] = {tbbox[4 * q + 2], tbbox[4 * q + 2], tbbox[4 * q + 3], tbbox[4 * q + 3]};
    float xmn = 0.f, xmx = 0.f, ymn = 0.f, ymx = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float wx = __fadd_rn(mx, __fmul_rn(r, __fsub_rn(__fmul_rn(cu[k], c32), __fmul_rn(cv[k], s32))));
      const float wy = __fadd_rn(my, __fmul_rn(r, __fadd_rn(__fmul_rn(cu[k], s32), __fmul_rn(cv[k], c32))));
      if (k == 0) { xmn = xmx = wx; ymn = ymx = wy; }
      else { xmn = nan_min(xmn, wx); xmx = nan_max(xmx, wx); ymn = nan_min(ymn, wy); ymx = nan_max(ymx, wy); }
    }
    sx = tile_span_content(xmn, xmx, g.TS, g.W, g.tilesX);
    sy = tile_span_content(ymn, ymx, g.TS, g.H, g.tilesY);
  } else {
    if (valid) {
      sx = tile_span_cull(mx, pi.hw, g.TS, g.W);
      sy = tile_span_cull(my, pi.hh, g.TS, g.H);
    } else {
      sx = make_int2(1, 0); sy = make_int2(1, 0);
    }
  }
  rects[n] = make_int4(sx.x, sx.y, sy.x, sy.y);
  if (diff != nullptr && sx.x <= sx.y && sy.x <= sy.y) {
    // the rectangle's corners in its slice's 2-D difference array of
    // (tilesY+1) x (tilesX+1) counters; its 2-D prefix sum is the number of
    // the slice's rectangles covering each tile
    const int gw = g.tilesX + 1;
    int* d = diff + (size_t)(n / span) * (g.tilesY + 1) * gw;
    atomicAdd(d + sy.x * gw + sx.x, 1);
    atomicAdd(d + sy.x * gw + sx.y + 1, -1);
    atomicAdd(d + (sy.y + 1) * gw + sx.x, -1);
    atomicAdd(d + (sy.y + 1) * gw + sx.y + 1, 1);
  }
}

// Tile lists.  Counts: per primitive slice, prepare_kernel marks each
// rectangle's corners in a 2-D difference array and counts_kernel prefix-sums
// it into counts[t * S + slice], the number of the slice's rectangles covering
// tile t.  The exclusive scan of the counts is tile-major and slice-minor.
// Write: one CTA per (tile row, group of kBinGroup tiles, primitive slice),
// kBinTPW tiles per warp (warp w: tiles w + k kBinWarps of the group); the
// CTA walks the primitives of its slice in index order in chunks of
// kBinThreads, compacts those whose rectangle covers its row and overlaps its
// tile group, and each warp writes the ids of the compacted rectangles
// containing each of its tiles from offs[t * S + slice] on, so a tile's
// entries come out in ascending primitive order.  Two tiles per warp halve
// the per-tile share of the row filter, compaction and count scan (write
// pass 39.8 -> 29.4 us at 2048x2048, N=20000 on a B200).  The write pass also
// publishes tile_offsets, L and the overflow flag, and leaves the outputs
// untouched when L exceeds the capacity.
constexpr int kBinThreads = 512;
constexpr int kBinWarps = kBinThreads / 32;
constexpr int kBinTPW = 2;                       // tiles per warp
constexpr int kBinGroup = kBinTPW * kBinWarps;   // tiles per CTA

struct BinGrid {
  int groups;   // tile groups per row
  int slices;   // primitive slices
  int span;     // primitives per slice (multiple of kBinThreads)
  long long ctas;
};

// Enough slices to give every SM several CTAs, never a slice below one chunk.
static inline BinGrid bin_grid(int N, int tilesX, int tilesY) {
  BinGrid b;
  b.groups = (tilesX + kBinGroup - 1) / kBinGroup;
  const long long base = (long long)b.groups * tilesY;
  const int chunks = N > 0 ? (N + kBinThreads - 1) / kBinThreads : 1;
  const long long want = (148 * 8 + base - 1) / base;
  b.slices = (int)(want < chunks ? want : chunks);
  if (b.slices < 1) b.slices = 1;
  const int per = (chunks + b.slices - 1) / b.slices;
  b.span = per * kBinThreads;
  b.slices = N > 0 ? (N + b.span - 1) / b.span : 1;
  b.ctas = base * b.slices;
  return b;
}

// One CTA per slice: 2-D inclusive prefix sum of the slice's difference array
// (rows, then columns), written as counts[t * S + slice]; counts[T * S] = 0.
// SMEM: the array is staged in shared memory (it fits for canvases up to
// about 3500 x 3500 pixels at tile 32); otherwise it is scanned in place.
// Rows are scanned by whole warps (shuffle scans over 32-column chunks),
// columns by one thread each.
template <bool SMEM>
__global__ void __launch_bounds__(1024) counts_kernel(Geom g, BinGrid bg, int* __restrict__ diff,
                                                      long long* __restrict__ counts) {
  extern __shared__ int s_diff[];
  const int slice = blockIdx.x;
  const int gw = g.tilesX + 1;
  const int cells = (g.tilesY + 1) * gw;
  int* src = diff + (size_t)slice * cells;
  int* d = SMEM ? s_diff : src;
  if (SMEM) {
    for (int i = threadIdx.x; i < cells; i += blockDim.x) s_diff[i] = src[i];
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (int y = warp; y < g.tilesY; y += nwarps) {
    int carry = 0;
    for (int x0 = 0; x0 < g.tilesX; x0 += 32) {
      const int x = x0 + lane;
      int v = x < g.tilesX ? d[y * gw + x] : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
      }
      v += carry;
      if (x < g.tilesX) d[y * gw + x] = v;
      carry = __shfl_sync(0xffffffffu, v, 31);
    }
  }
  __syncthreads();
  for (int x = threadIdx.x; x < g.tilesX; x += blockDim.x) {
    long long acc = 0;
    for (int y = 0; y < g.tilesY; ++y) {
      acc += d[y * gw + x];
      counts[((long long)y * g.tilesX + x) * bg.slices + slice] = acc;
    }
  }
  if (slice == 0 && threadIdx.x == 0) counts[(long long)g.T * bg.slices] = 0;
}

__global__ void __launch_bounds__(kBinThreads, 3) bin_rows_kernel(Geom g, BinGrid bg,
                                                                  const int4* __restrict__ rects,
                                                                  const long long* __restrict__ offs, long long cap,
                                                                  int* __restrict__ indices,
                                                                  int* __restrict__ tile_offsets,
                                                                  int* __restrict__ total_out,
                                                                  int* __restrict__ overflow_out) {
  // Two compaction buffers: chunk c is compacted into buffer c & 1 while the
  // warps may still read chunk c - 1 from the other one, so one barrier per
  // chunk orders everything (see the loop).
  __shared__ int s_id[2][kBinThreads];
  __shared__ int2 s_xr[2][kBinThreads];   // the rectangle's tile columns x0, x1
  __shared__ int s_wcnt[2][kBinWarps];
  const int slice = blockIdx.x % bg.slices;
  const int rg = blockIdx.x / bg.slices;
  const int ty = rg / bg.groups;
  const int gx0 = (rg - ty * bg.groups) * kBinGroup, gx1 = min(gx0 + kBinGroup - 1, g.tilesX - 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long nslots = (long long)g.T * bg.slices;
  const unsigned lt = (1u << lane) - 1u;
  // this warp's tiles gx0 + warp + k kBinWarps: the column a rectangle must
  // reach (INT_MAX for a tile past the canvas, which no rectangle contains)
  // and the next write position of each
  int col[kBinTPW];
  long long cur[kBinTPW];
  {
    const long long L = offs[nslots];
    const bool first = blockIdx.x == 0 && threadIdx.x == 0;
    if (first) {
      if (total_out) *total_out = (int)min(L, (long long)INT_MAX);
      if (overflow_out) *overflow_out = (L > cap) ? 1 : 0;
    }
    if (L > cap) return;   // uniform over the CTA
    if (first) tile_offsets[g.T] = (int)L;
#pragma unroll
    for (int k = 0; k < kBinTPW; ++k) {
      const int tx = gx0 + warp + k * kBinWarps;
      col[k] = INT_MAX;
      cur[k] = 0;
      if (tx <= gx1) {
        const int t = ty * g.tilesX + tx;
        col[k] = tx;
        cur[k] = offs[(long long)t * bg.slices + slice];
        if (lane == 0 && slice == 0) tile_offsets[t] = (int)cur[k];
      }
    }
  }
  const int lo = slice * bg.span, hi = min(g.N, lo + bg.span);
  const int4 none = make_int4(1, 0, 1, 0);
  // a rectangle survives the CTA's test when it covers row ty and overlaps the tile group
  auto covers = [&](const int4& rc) { return rc.x <= rc.y && rc.z <= ty && ty <= rc.w && rc.x <= gx1 && rc.y >= gx0; };
  // chunk lo: test, count; the rectangles of the next chunk are loaded one chunk ahead
  int n = lo + (int)threadIdx.x;
  int4 rc = n < hi ? rects[n] : none;
  int4 rn = n + kBinThreads < hi ? rects[n + kBinThreads] : none;
  bool f = n < hi && covers(rc);
  unsigned b = __ballot_sync(0xffffffffu, f);
  if (lane == 0) s_wcnt[0][warp] = __popc(b);
  __syncthreads();
  int buf = 0;
  for (int base = lo; base < hi; base += kBinThreads, buf ^= 1) {
    // (1) compact chunk base into buffer buf (its counts were published before
    // the last barrier): lane w < kBinWarps scans the counts of warps 0..w
    int inc = lane < kBinWarps ? s_wcnt[buf][lane] : 0;
#pragma unroll
    for (int o = 1; o < kBinWarps; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += u;
    }
    const int total = __shfl_sync(0xffffffffu, inc, kBinWarps - 1);
    const int wbase = warp == 0 ? 0 : __shfl_sync(0xffffffffu, inc, warp - 1);
    if (f) {
      const int p = wbase + __popc(b & lt);
      s_id[buf][p] = n;
      s_xr[buf][p] = make_int2(rc.x, rc.y);
    }
    // (2) test and count the next chunk, and load the one after it
    n += kBinThreads;
    rc = rn;
    rn = n + kBinThreads < hi ? rects[n + kBinThreads] : none;
    f = n < hi && covers(rc);
    b = __ballot_sync(0xffffffffu, f);
    if (lane == 0) s_wcnt[buf ^ 1][warp] = __popc(b);
    // One barrier per chunk.  After it, buffer buf holds chunk base and
    // s_wcnt[buf ^ 1] the next chunk's counts.  The next iteration writes
    // buffer buf ^ 1, last read by this iteration's predecessor (before this
    // barrier), and s_wcnt[buf], last read in (1) above (before this barrier).
    __syncthreads();
    // (3) each warp writes the compacted rectangles that contain its tiles
    for (int j = lane; j < ((total + 31) & ~31); j += 32) {
      const int2 xr = j < total ? s_xr[buf][j] : make_int2(1, 0);
      const int id = j < total ? s_id[buf][j] : 0;
#pragma unroll
      for (int k = 0; k < kBinTPW; ++k) {
        const bool in = xr.x <= col[k] && col[k] <= xr.y;
        const unsigned m = __ballot_sync(0xffffffffu, in);
        if (in) indices[cur[k] + __popc(m & lt)] = id;
        cur[k] += __popc(m);
      }
    }
  }
}

// ---------------------------------------------------------------------------
struct BinWorkspace {
  int4* rects;         // N tile rectangles (x0, x1, y0, y1)
  long long* counts;   // T*S+1 entries per (tile, primitive slice)
  long long* offs;     // exclusive prefix of counts
  int* diff;           // S difference arrays of (tilesY+1) x (tilesX+1)
  size_t diff_bytes;
  void* cub_tmp;
  size_t cub_bytes;
  size_t total;
};

static inline size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

static BinWorkspace layout_ws(void* base, int N, int T, long long nslots, size_t diff_bytes, bool query,
                              size_t* needed) {
  BinWorkspace w{};
  size_t scan_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (long long*)nullptr, (long long*)nullptr, nslots + 1);
  w.cub_bytes = align_up(scan_bytes);
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += align_up(bytes); return o; };
  const size_t o_rects = take(sizeof(int4) * (size_t)(N > 0 ? N : 1));
  const size_t o_counts = take(sizeof(long long) * (size_t)(nslots + 1));
  const size_t o_offs = take(sizeof(long long) * (size_t)(nslots + 1));
  const size_t o_cub = take(w.cub_bytes);
  const size_t o_diff = take(diff_bytes);
  w.diff_bytes = diff_bytes;
  w.total = off;
  if (needed) *needed = off;
  if (!query) {
    char* b = static_cast<char*>(base);
    w.rects = reinterpret_cast<int4*>(b + o_rects);
    w.counts = reinterpret_cast<long long*>(b + o_counts);
    w.offs = reinterpret_cast<long long*>(b + o_offs);
    w.cub_tmp = b + o_cub;
    w.diff = reinterpret_cast<int*>(b + o_diff);
  }
  return w;
}

static inline size_t diff_bytes_of(const BinGrid& bg, int tilesX, int tilesY) {
  return sizeof(int) * (size_t)bg.slices * (tilesY + 1) * (tilesX + 1);
}

size_t bin_workspace_bytes(int N, int T, int tilesX, int tilesY, long long cap) {
  (void)cap;   // the row binning needs no scratch per list entry
  const BinGrid bg = bin_grid(N, tilesX, tilesY);
  size_t need = 0;
  layout_ws(nullptr, N, T, (long long)T * bg.slices, diff_bytes_of(bg, tilesX, tilesY), true, &need);
  return need;
}

int launch_template_bboxes(const float* tmpl, int P, int Ht, int Wt, float* out, cudaStream_t st) {
  if (P <= 0) return DBMP_OK;
  template_bbox_kernel<<<P, 256, 0, st>>>(tmpl, Ht, Wt, out);
  DBMP_CHECK_LAUNCH("template_bbox_kernel");
  return DBMP_OK;
}

size_t atlas_bytes(int P, int Ht, int Wt, int kind) {
  if (kind < ATLAS_F32 || kind > ATLAS_BF16_PAIR) return 0;
  if (!atlas_has_grid(kind)) return atlas_record_bytes(P, Ht, Wt, kind);
  int sx, sy, gx, gy;
  grid_shape(Wt, &sx, &gx);
  grid_shape(Ht, &sy, &gy);
  return atlas_grid_offset(P, Ht, Wt, kind) + (size_t)P * gx * gy;
}

// Clearance grid (layout in dbmp_internal.cuh), one CTA per (cell column,
// template).  Separable: per template row the x-distance from the column's
// range to the nearest support texel of that row, then per cell the minimum
// over rows of max(row distance, y-distance).  Texels further than kGridCap-1
// beyond the cell cannot lower a capped value and are not visited.
__global__ void atlas_grid_kernel(const float* __restrict__ tmpl, int Ht, int Wt, int gsx, int gsy, int Gx, int Gy,
                                  unsigned char* __restrict__ grid) {
  extern __shared__ unsigned char s_row[];   // Ht row distances
  const int ix = blockIdx.x, p = blockIdx.y;
  const float* t = tmpl + (size_t)p * Ht * Wt;
  const int lo = ix << gsx, hi = min((ix + 1) << gsx, Wt - 1);
  const int xa = max(0, lo - (kGridCap - 1)), xb = min(Wt - 1, hi + (kGridCap - 1));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  for (int y = warp; y < Ht; y += nwarps) {
    int best = kGridCap;
    const float* row = t + (size_t)y * Wt;
    for (int x = xa + lane; x <= xb; x += 32) {
      const float v = row[x];
      if (!(v <= kGridSupport)) best = min(best, max(0, max(lo - x, x - hi)));
    }
    best = __reduce_min_sync(0xffffffffu, best);
    if (lane == 0) s_row[y] = (unsigned char)best;
  }
  __syncthreads();
  for (int iy = threadIdx.x; iy < Gy; iy += blockDim.x) {
    const int ylo = iy << gsy, yhi = min((iy + 1) << gsy, Ht - 1);
    const int ya = max(0, ylo - (kGridCap - 1)), yb = min(Ht - 1, yhi + (kGridCap - 1));
    int best = kGridCap;
    for (int y = ya; y <= yb; ++y) best = min(best, max((int)s_row[y], max(0, max(ylo - y, y - yhi))));
    grid[((size_t)p * Gy + iy) * Gx + ix] = (unsigned char)best;
  }
}

int launch_atlas_grid(const float* tmpl, int P, int Ht, int Wt, int kind, void* out, cudaStream_t st) {
  int sx, sy, gx, gy;
  grid_shape(Wt, &sx, &gx);
  grid_shape(Ht, &sy, &gy);
  unsigned char* grid = static_cast<unsigned char*>(out) + atlas_grid_offset(P, Ht, Wt, kind);
  if (Ht > 48 * 1024) {   // row distances do not fit the shared buffer: clearance 0 never skips
    cudaError_t e = cudaMemsetAsync(grid, 0, (size_t)P * gx * gy, st);
    return e == cudaSuccess ? DBMP_OK : cuda_status(e, "cudaMemsetAsync(grid)");
  }
  atlas_grid_kernel<<<dim3(gx, P), 256, Ht, st>>>(tmpl, Ht, Wt, sx, sy, gx, gy, grid);
  DBMP_CHECK_LAUNCH("atlas_grid_kernel");
  return DBMP_OK;
}

int launch_atlas_pack(const float* tmpl, int P, int Ht, int Wt, int kind, void* out, cudaStream_t st) {
  const long long total = (long long)P * (Ht + 1) * Wt;
  if (total == 0) return DBMP_OK;
  const int blocks = (int)((total + 255) / 256 < 148 * 32 ? (total + 255) / 256 : 148 * 32);
  switch (kind) {
    case ATLAS_F16_PAIR: atlas_pair_kernel<__half><<<blocks, 256, 0, st>>>(tmpl, P, Ht, Wt, (__half*)out); break;
    case ATLAS_BF16_PAIR: atlas_pair_kernel<__nv_bfloat16><<<blocks, 256, 0, st>>>(tmpl, P, Ht, Wt, (__nv_bfloat16*)out); break;
    case ATLAS_F32_QUAD: atlas_pack_kernel<float><<<blocks, 256, 0, st>>>(tmpl, P, Ht, Wt, (float*)out); break;
    case ATLAS_F16_QUAD: atlas_pack_kernel<__half><<<blocks, 256, 0, st>>>(tmpl, P, Ht, Wt, (__half*)out); break;
    case ATLAS_BF16_QUAD: atlas_pack_kernel<__nv_bfloat16><<<blocks, 256, 0, st>>>(tmpl, P, Ht, Wt, (__nv_bfloat16*)out); break;
    default: set_error("dbmp_atlas_pack: kind %d is not a packed kind", kind); return DBMP_ERR_INVALID;
  }
  DBMP_CHECK_LAUNCH("atlas_pack_kernel");
  return launch_atlas_grid(tmpl, P, Ht, Wt, kind, out, st);
}

// Gaussian blur of the templates (pydiffbmp/util/utils.py:22-67,
// gaussian_blur, as vector_renderer.py:80-96 applies it to the atlas): a K x K
// kernel, K = 2 round(3 sigma) + 1, weights k[i] k[j] of the normalised 1-D
// Gaussian exp(-0.5 ((i - K/2) / sigma)^2), zero padding, same output size.
// One thread per output texel; the 1-D weights sit in shared memory.
__device__ __forceinline__ void blur_weights(float sigma, int K, float* s_k) {
  float sum = 0.f;
  for (int i = 0; i < K; ++i) {
    const float a = (float)(i - K / 2) / sigma;
    s_k[i] = expf(-0.5f * (a * a));
    sum += s_k[i];
  }
  for (int i = 0; i < K; ++i) s_k[i] /= sum;
}

__device__ __forceinline__ void blur_texels(const float* __restrict__ in, int P, int Ht, int Wt, int K,
                                            const float* s_k, float* __restrict__ out) {
  const long long total = (long long)P * Ht * Wt;
  const int h = K / 2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(t % Wt), y = (int)((t / Wt) % Ht);
    const float* src = in + (t - (long long)y * Wt - x);
    float acc = 0.f;
    for (int i = 0; i < K; ++i) {
      const int yy = y + i - h;
      if (yy < 0 || yy >= Ht) continue;
      for (int j = 0; j < K; ++j) {
        const int xx = x + j - h;
        if (xx < 0 || xx >= Wt) continue;
        acc = fmaf(s_k[i] * s_k[j], src[(size_t)yy * Wt + xx], acc);
      }
    }
    out[t] = acc;
  }
}

__global__ void template_blur_kernel(const float* __restrict__ in, int P, int Ht, int Wt, int K, float sigma,
                                     float* __restrict__ out) {
  extern __shared__ float s_k[];
  if (threadIdx.x == 0) blur_weights(sigma, K, s_k);
  __syncthreads();
  blur_texels(in, P, Ht, Wt, K, s_k, out);
}

// Kernel size of a blur sigma: 2 round(3 sigma) + 1 with Python's round (ties
// to even, as rint does).
__host__ __device__ inline int blur_kernel_size(double sigma) { return (int)(2.0 * rint(3.0 * sigma) + 1.0); }

// The blur of one fit iteration it = *step_count under a schedule
// (simple_tile_renderer.py:1015-1021): sigma in double as the reference's
// Python computes it, the kernel size from that double, the weights in float
// (gaussian_blur's float32 tensor arithmetic); sigma <= 0 copies.  The weight
// buffer holds kmax entries, the largest kernel of the schedule.
__global__ void template_blur_sched_kernel(const float* __restrict__ in, int P, int Ht, int Wt,
                                           dbmp_blur_schedule sched, const int* __restrict__ step_count, int kmax,
                                           float* __restrict__ out) {
  extern __shared__ float s_k[];
  __shared__ int s_K;
  if (threadIdx.x == 0) {
    double sigma = 0.0;
    if (sched.mode == 1) {
      sigma = (double)sched.sigma;
    } else if (sched.mode == 2) {
      const double progress = (double)*step_count / (double)sched.num_iterations;
      sigma = (double)sched.sigma_start * (1.0 - progress) + (double)sched.sigma_end * progress;
    }
    int K = sigma > 0.0 ? blur_kernel_size(sigma) : 0;
    if (K > kmax) K = kmax;      // cannot happen for a linear schedule between its two ends
    if (K > 0) blur_weights((float)sigma, K, s_k);
    s_K = K;
  }
  __syncthreads();
  const int K = s_K;
  if (K > 0) {
    blur_texels(in, P, Ht, Wt, K, s_k, out);
    return;
  }
  const long long total = (long long)P * Ht * Wt;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x)
    out[t] = in[t];
}

int launch_template_blur(const float* in, int P, int Ht, int Wt, float sigma, float* out, cudaStream_t st) {
  const long long total = (long long)P * Ht * Wt;
  if (total == 0) return DBMP_OK;
  if (!(sigma > 0.f)) {   // sigma <= 0 leaves the templates unchanged (utils.py:37-38)
    if (in == out) return DBMP_OK;
    cudaError_t e = cudaMemcpyAsync(out, in, sizeof(float) * (size_t)total, cudaMemcpyDeviceToDevice, st);
    return e == cudaSuccess ? DBMP_OK : cuda_status(e, "cudaMemcpyAsync(templates)");
  }
  const int K = blur_kernel_size((double)sigma);
  if (K > 4097) { set_error("dbmp_template_blur: sigma %g gives a kernel of %d texels", (double)sigma, K); return DBMP_ERR_INVALID; }
  const int blocks = (int)((total + 255) / 256 < 148 * 16 ? (total + 255) / 256 : 148 * 16);
  template_blur_kernel<<<blocks, 256, sizeof(float) * K, st>>>(in, P, Ht, Wt, K, sigma, out);
  DBMP_CHECK_LAUNCH("template_blur_kernel");
  return DBMP_OK;
}

int launch_template_blur_sched(const float* in, int P, int Ht, int Wt, const dbmp_blur_schedule* sched,
                               const int* step_count, float* out, cudaStream_t st) {
  const long long total = (long long)P * Ht * Wt;
  if (total == 0) return DBMP_OK;
  // largest kernel over the schedule: sigma is constant or linear between its ends
  double smax = 0.0;
  if (sched->mode == 1) smax = sched->sigma;
  if (sched->mode == 2) smax = sched->sigma_start > sched->sigma_end ? sched->sigma_start : sched->sigma_end;
  const int kmax = smax > 0.0 ? blur_kernel_size(smax) : 1;
  if (kmax > 4097) {
    set_error("dbmp_template_blur_scheduled: sigma %g gives a kernel of %d texels", smax, kmax);
    return DBMP_ERR_INVALID;
  }
  const int blocks = (int)((total + 255) / 256 < 148 * 16 ? (total + 255) / 256 : 148 * 16);
  template_blur_sched_kernel<<<blocks, 256, sizeof(float) * kmax, st>>>(in, P, Ht, Wt, *sched, step_count, kmax,
                                                                         out);
  DBMP_CHECK_LAUNCH("template_blur_sched_kernel");
  return DBMP_OK;
}

int launch_prepare(const Geom& g, const float* means2D, const float* radii, const float* rot, const float* opac,
                   const float* colors, const int* sel, PrimInfo* out, cudaStream_t st) {
  if (g.N == 0) return DBMP_OK;
  prepare_kernel<<<(g.N + 255) / 256, 256, 0, st>>>(g, means2D, radii, rot, opac, colors, sel, nullptr, 0,
                                                    out, nullptr, nullptr, 1);
  DBMP_CHECK_LAUNCH("prepare_kernel");
  return DBMP_OK;
}

int launch_bin(const Geom& g, int bin_mode, const float* means2D, const float* radii, const float* rot,
               const float* opac, const float* colors, const int* sel, const float* tbbox, PrimInfo* prim_info,
               int* tile_offsets, int* tile_indices, long long cap, int* total_out, int* overflow_out,
               void* ws, size_t ws_bytes, cudaStream_t st) {
  const BinGrid bg = bin_grid(g.N, g.tilesX, g.tilesY);
  const long long nslots = (long long)g.T * bg.slices;
  size_t need = 0;
  BinWorkspace w = layout_ws(ws, g.N, g.T, nslots, diff_bytes_of(bg, g.tilesX, g.tilesY), false, &need);
  if (ws_bytes < need) {
    set_error("dbmp_bin: workspace of %zu bytes is smaller than the %zu bytes required", ws_bytes, need);
    return DBMP_ERR_CAPACITY;
  }
  if (bg.ctas > 0x7fffffffll) { set_error("dbmp_bin: canvas and primitive count too large"); return DBMP_ERR_INVALID; }
  cudaError_t e = cudaMemsetAsync(w.diff, 0, w.diff_bytes, st);
  if (e != cudaSuccess) return cuda_status(e, "cudaMemsetAsync(diff)");
  if (g.N > 0) {
    prepare_kernel<<<(g.N + 255) / 256, 256, 0, st>>>(g, means2D, radii, rot, opac, colors, sel, tbbox, bin_mode,
                                                      prim_info, w.rects, w.diff, bg.span);
    DBMP_CHECK_LAUNCH("prepare_kernel");
  }
  const size_t cells_bytes = sizeof(int) * (size_t)(g.tilesY + 1) * (g.tilesX + 1);
  if (cells_bytes <= 48 * 1024) counts_kernel<true><<<bg.slices, 1024, cells_bytes, st>>>(g, bg, w.diff, w.counts);
  else counts_kernel<false><<<bg.slices, 1024, 0, st>>>(g, bg, w.diff, w.counts);
  DBMP_CHECK_LAUNCH("counts_kernel");
  size_t tmp = w.cub_bytes;
  e = cub::DeviceScan::ExclusiveSum(w.cub_tmp, tmp, w.counts, w.offs, nslots + 1, st);
  if (e != cudaSuccess) return cuda_status(e, "cub::DeviceScan::ExclusiveSum");
  const int grid = (int)bg.ctas;   // (tile row, tile group, primitive slice) triples
  bin_rows_kernel<<<grid, kBinThreads, 0, st>>>(g, bg, w.rects, w.offs, cap, tile_indices, tile_offsets, total_out,
                                                overflow_out);
  DBMP_CHECK_LAUNCH("bin_rows_kernel");
  return DBMP_OK;
}

}  // namespace dbmp
