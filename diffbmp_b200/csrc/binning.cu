// Device binning: per-primitive preparation, primitive -> tile rectangles,
// (tile, primitive) key emission and a stable radix sort by tile, producing
// the reference's CSR tile lists without any host round trip.
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
// Atlas repacking into bilinear quads (precision form).
template <typename OutT>
__device__ __forceinline__ OutT to_storage(float v);
template <> __device__ __forceinline__ float to_storage<float>(float v) { return v; }
template <> __device__ __forceinline__ __half to_storage<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 to_storage<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// Pair layout: (P, Ht+1, Wt) records of (t[y][x], t[y][x+1]); row Ht is zero.
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
    out[2 * i] = to_storage<OutT>(v0);
    out[2 * i + 1] = to_storage<OutT>(v1);
  }
}

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
    o[0] = to_storage<OutT>(v00); o[1] = to_storage<OutT>(v01);
    o[2] = to_storage<OutT>(v10); o[3] = to_storage<OutT>(v11);
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
                               int4* __restrict__ rects, long long* __restrict__ counts) {
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
  const bool nan_geom = isnan(pi.a00) || isnan(pi.a01) || isnan(pi.a10) || isnan(pi.a11) || isnan(mx) || isnan(my);
  pi.toff = !valid ? kNoFrag : (nan_geom ? kSolid : tid * template_records(g.kind, g.Ht, g.Wt));
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
  if (bin_mode == DBMP_BIN_CONTENT) {
    // vector_renderer.py:221-250 with the template of this primitive
    const int q = valid ? tid : 0;
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
  const long long w = max(0, sx.y - sx.x + 1), h = max(0, sy.y - sy.x + 1);
  rects[n] = make_int4(sx.x, sx.y, sy.x, sy.y);
  counts[n] = w * h;
}

// One warp per primitive writes (tile id, primitive id) for every tile of its
// rectangle, in row-major tile order, at its exclusive-scan offset.
__global__ void emit_kernel(Geom g, const int4* __restrict__ rects, const long long* __restrict__ offs,
                            long long cap, unsigned* __restrict__ keys, unsigned* __restrict__ vals) {
  const long long total = offs[g.N];
  if (total > cap) return;
  const int lane = threadIdx.x & 31;
  for (int n = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; n < g.N; n += (gridDim.x * blockDim.x) >> 5) {
    const long long o = offs[n], cnt = offs[n + 1] - o;
    if (cnt == 0) continue;
    const int4 rc = rects[n];
    const int w = rc.y - rc.x + 1;
    for (long long j = lane; j < cnt; j += 32) {
      const int dy = (int)(j / w), dx = (int)(j - (long long)dy * w);
      keys[o + j] = (unsigned)((rc.z + dy) * g.tilesX + rc.x + dx);
      vals[o + j] = (unsigned)n;
    }
  }
}

// Entries [L, cap) get the sentinel key T so they sort behind every tile.
__global__ void fill_tail_kernel(const long long* __restrict__ total_p, int N, long long cap, unsigned sentinel,
                                 unsigned* __restrict__ keys, unsigned* __restrict__ vals) {
  const long long L = total_p[N];
  if (L > cap) return;
  for (long long i = L + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < cap; i += (long long)gridDim.x * blockDim.x) {
    keys[i] = sentinel;
    vals[i] = 0u;
  }
}

// offsets[t] = first position whose sorted key >= t (t = 0..T).
__global__ void tile_offsets_kernel(const long long* __restrict__ total_p, int N, long long cap, int T,
                                    const unsigned* __restrict__ skeys, int* __restrict__ offsets,
                                    int* __restrict__ total_out, int* __restrict__ overflow_out) {
  const long long L = total_p[N];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    if (total_out) *total_out = (int)min(L, (long long)INT_MAX);
    if (overflow_out) *overflow_out = (L > cap) ? 1 : 0;
  }
  if (L > cap || t > T) return;
  long long lo = 0, hi = L;
  while (lo < hi) {
    const long long mid = (lo + hi) >> 1;
    if (skeys[mid] < (unsigned)t) lo = mid + 1; else hi = mid;
  }
  offsets[t] = (int)lo;
}

// ---------------------------------------------------------------------------
struct BinWorkspace {
  int4* rects;
  long long* counts;   // N+1
  long long* offs;     // N+1
  unsigned* keys_in;
  unsigned* vals_in;
  unsigned* keys_out;
  void* cub_tmp;
  size_t cub_bytes;
  size_t total;
};

static inline size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

static int key_bits(int T) {
  int bits = 0;
  while ((1u << bits) <= (unsigned)T && bits < 32) ++bits;
  return bits < 1 ? 1 : bits;
}

static BinWorkspace layout_ws(void* base, int N, int T, long long cap, bool query, size_t* needed) {
  BinWorkspace w{};
  size_t scan_bytes = 0, sort_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (long long*)nullptr, (long long*)nullptr, N + 1);
  if (cap > 0)
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (unsigned*)nullptr, (unsigned*)nullptr,
                                    (unsigned*)nullptr, (unsigned*)nullptr, (int)cap, 0, key_bits(T));
  w.cub_bytes = align_up(scan_bytes > sort_bytes ? scan_bytes : sort_bytes);
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off += align_up(bytes); return o; };
  const size_t o_rects = take(sizeof(int4) * (size_t)N);
  const size_t o_counts = take(sizeof(long long) * (size_t)(N + 1));
  const size_t o_offs = take(sizeof(long long) * (size_t)(N + 1));
  const size_t o_kin = take(sizeof(unsigned) * (size_t)cap);
  const size_t o_vin = take(sizeof(unsigned) * (size_t)cap);
  const size_t o_kout = take(sizeof(unsigned) * (size_t)cap);
  const size_t o_cub = take(w.cub_bytes);
  w.total = off;
  if (needed) *needed = off;
  if (!query) {
    char* b = static_cast<char*>(base);
    w.rects = reinterpret_cast<int4*>(b + o_rects);
    w.counts = reinterpret_cast<long long*>(b + o_counts);
    w.offs = reinterpret_cast<long long*>(b + o_offs);
    w.keys_in = reinterpret_cast<unsigned*>(b + o_kin);
    w.vals_in = reinterpret_cast<unsigned*>(b + o_vin);
    w.keys_out = reinterpret_cast<unsigned*>(b + o_kout);
    w.cub_tmp = b + o_cub;
  }
  return w;
}

size_t bin_workspace_bytes(int N, int T, long long cap) {
  size_t need = 0;
  layout_ws(nullptr, N, T, cap, true, &need);
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

int launch_prepare(const Geom& g, const float* means2D, const float* radii, const float* rot, const float* opac,
                   const float* colors, const int* sel, PrimInfo* out, cudaStream_t st) {
  if (g.N == 0) return DBMP_OK;
  prepare_kernel<<<(g.N + 255) / 256, 256, 0, st>>>(g, means2D, radii, rot, opac, colors, sel, nullptr, 0,
                                                    out, nullptr, nullptr);
  DBMP_CHECK_LAUNCH("prepare_kernel");
  return DBMP_OK;
}

int launch_bin(const Geom& g, int bin_mode, const float* means2D, const float* radii, const float* rot,
               const float* opac, const float* colors, const int* sel, const float* tbbox, PrimInfo* prim_info,
               int* tile_offsets, int* tile_indices, long long cap, int* total_out, int* overflow_out,
               void* ws, size_t ws_bytes, cudaStream_t st) {
  size_t need = 0;
  BinWorkspace w = layout_ws(ws, g.N, g.T, cap, false, &need);
  if (ws_bytes < need) {
    set_error("dbmp_bin: workspace of %zu bytes is smaller than the %zu bytes required", ws_bytes, need);
    return DBMP_ERR_CAPACITY;
  }
  const int N = g.N;
  cudaError_t e = cudaMemsetAsync(w.counts, 0, sizeof(long long) * (N + 1), st);
  if (e != cudaSuccess) return cuda_status(e, "cudaMemsetAsync(counts)");
  if (N > 0) {
    prepare_kernel<<<(N + 255) / 256, 256, 0, st>>>(g, means2D, radii, rot, opac, colors, sel, tbbox, bin_mode,
                                                    prim_info, w.rects, w.counts);
    DBMP_CHECK_LAUNCH("prepare_kernel");
  }
  size_t tmp = w.cub_bytes;
  e = cub::DeviceScan::ExclusiveSum(w.cub_tmp, tmp, w.counts, w.offs, N + 1, st);
  if (e != cudaSuccess) return cuda_status(e, "cub::DeviceScan::ExclusiveSum");
  if (cap > 0) {
    if (N > 0) {
      const int blocks = (N * 32 + 255) / 256 < 148 * 16 ? (N * 32 + 255) / 256 : 148 * 16;
      emit_kernel<<<blocks, 256, 0, st>>>(g, w.rects, w.offs, cap, w.keys_in, w.vals_in);
      DBMP_CHECK_LAUNCH("emit_kernel");
    }
    fill_tail_kernel<<<148 * 4, 256, 0, st>>>(w.offs, N, cap, (unsigned)g.T, w.keys_in, w.vals_in);
    DBMP_CHECK_LAUNCH("fill_tail_kernel");
    tmp = w.cub_bytes;
    e = cub::DeviceRadixSort::SortPairs(w.cub_tmp, tmp, w.keys_in, w.keys_out, w.vals_in,
                                        reinterpret_cast<unsigned*>(tile_indices), (int)cap, 0, key_bits(g.T), st);
    if (e != cudaSuccess) return cuda_status(e, "cub::DeviceRadixSort::SortPairs");
  }
  tile_offsets_kernel<<<(g.T + 1 + 255) / 256, 256, 0, st>>>(w.offs, N, cap, g.T, w.keys_out, tile_offsets,
                                                             total_out, overflow_out);
  DBMP_CHECK_LAUNCH("tile_offsets_kernel");
  return DBMP_OK;
}

}  // namespace dbmp
