// PSD layer export: one cropped uint8 RGBA layer per primitive.
//
// Replaces cuda_tile_rasterizer/cuda_kernels/psd_export_kernels.cu.  The
// reference launches N x (all 16x16 canvas tiles) blocks and has each thread
// loop over a canvas tile for its primitive, O(N*H*W) work for O(sum of crop
// areas) output.  Here a layout pass prefix-sums each layer's byte size and
// 16x16 block count on the device, and a persistent grid walks only the
// blocks of the crops, one pixel per thread, writing one uchar4 per pixel.
//
// The per-pixel arithmetic must give the reference's bytes exactly, and the
// reference builds it with --use_fast_math (setup_psd_export.py:69), so this
// file is compiled with --use_fast_math too and keeps each expression in the
// reference's operation order (psd_export_common.h:55-121,
// psd_export_kernels.cu:26-55,96-195).
#include <cstdint>

#include <mutex>

#include "dbmp_internal.cuh"

namespace dbmp {

constexpr int kPsdBlock = 16;

// Stage 1 (psd_export_kernels.cu:12-55): crop box [x0,x1) x [y0,y1) of each
// primitive's scaled square of half extent 1.5 r, clipped to the canvas; an
// empty box becomes (0,0,1,1).
__global__ void psd_bbox_kernel(const float* __restrict__ means2D, const float* __restrict__ radii, int N, int H,
                                int W, float scale, int* __restrict__ bbox, int* __restrict__ sizes) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const float x = means2D[n * 2 + 0] * scale;
  const float y = means2D[n * 2 + 1] * scale;
  const float r = radii[n] * scale;
  const float half_extent = r * 1.5f;
  const int x0 = max(0, (int)floorf(x - half_extent));
  const int y0 = max(0, (int)floorf(y - half_extent));
  const int x1 = min(W, (int)ceilf(x + half_extent));
  const int y1 = min(H, (int)ceilf(y + half_extent));
  int4 b = (x1 <= x0 || y1 <= y0) ? make_int4(0, 0, 1, 1) : make_int4(x0, y0, x1, y1);
  reinterpret_cast<int4*>(bbox)[n] = b;
  sizes[2 * n + 0] = b.z - b.x;
  sizes[2 * n + 1] = b.w - b.y;
}

// Layout: exclusive prefix sums of layer bytes (w*h*4) and of 16x16 blocks,
// in one CTA (the reference does the byte sum on the host,
// psd_export_uint8.py:70-77).  blk has N+1 entries; total_bytes is written.
__global__ void psd_layout_kernel(const int* __restrict__ sizes, int N, long long* __restrict__ layer_offsets,
                                  long long* __restrict__ blk, long long* __restrict__ total_bytes) {
  __shared__ long long s_b[1024], s_k[1024];
  const int t = threadIdx.x, nt = blockDim.x;
  const int per = (N + nt - 1) / nt;
  const int lo = min(N, t * per), hi = min(N, lo + per);
  long long sb = 0, sk = 0;
  for (int n = lo; n < hi; ++n) {
    const long long w = sizes[2 * n], h = sizes[2 * n + 1];
    sb += w * h * 4;
    sk += ((w + kPsdBlock - 1) / kPsdBlock) * ((h + kPsdBlock - 1) / kPsdBlock);
  }
  s_b[t] = sb; s_k[t] = sk;
  __syncthreads();
  for (int d = 1; d < nt; d <<= 1) {   // Hillis-Steele inclusive scan
    const long long vb = t >= d ? s_b[t - d] : 0, vk = t >= d ? s_k[t - d] : 0;
    __syncthreads();
    s_b[t] += vb; s_k[t] += vk;
    __syncthreads();
  }
  long long ob = s_b[t] - sb, ok = s_k[t] - sk;
  for (int n = lo; n < hi; ++n) {
    const long long w = sizes[2 * n], h = sizes[2 * n + 1];
    layer_offsets[n] = ob;
    blk[n] = ok;
    ob += w * h * 4;
    ok += ((w + kPsdBlock - 1) / kPsdBlock) * ((h + kPsdBlock - 1) / kPsdBlock);
  }
  if (t == nt - 1) {
    blk[N] = s_k[t];
    *total_bytes = s_b[t];
  }
}

// Template value at canvas pixel (px,py): psd_export_common.h:55-103 (u from
// (px - x) / r, hard zero when u_t < 0 or u_t >= W-1).
__device__ __forceinline__ float psd_template_value(const float* __restrict__ tmpl, int t_idx, int P, int Ht, int Wt,
                                                    int px, int py, float x, float y, float r, float cos_t,
                                                    float sin_t) {
  const float u_norm = ((float)px - x) / (r);
  const float v_norm = ((float)py - y) / (r);
  const float u_rot = cos_t * u_norm + sin_t * v_norm;
  const float v_rot = -sin_t * u_norm + cos_t * v_norm;
  const float u_t = (u_rot + 1.0f) * 0.5f * (Wt - 1);
  const float v_t = (v_rot + 1.0f) * 0.5f * (Ht - 1);
  if (u_t < 0.0f || u_t >= Wt - 1 || v_t < 0.0f || v_t >= Ht - 1) return 0.0f;
  if (t_idx < 0 || t_idx >= P) return 0.0f;   // the reference reads out of bounds here
  int u0 = (int)floorf(u_t);
  int v0 = (int)floorf(v_t);
  u0 = max(0, min(u0, Wt - 1));
  v0 = max(0, min(v0, Ht - 1));
  const float wu = u_t - u0;
  const float wv = v_t - v0;
  const float wu_inv = 1.0f - wu;
  const float wv_inv = 1.0f - wv;
  const float* t = tmpl + (size_t)t_idx * Ht * Wt;
  const float v00 = t[v0 * Wt + u0];
  const float v01 = t[v0 * Wt + u0 + 1];
  const float v10 = t[(v0 + 1) * Wt + u0];
  const float v11 = t[(v0 + 1) * Wt + u0 + 1];
  return wu_inv * wv_inv * v00 + wu * wv_inv * v01 + wu_inv * wv * v10 + wu * wv * v11;
}

// Clamped bilinear of a per-primitive RGB map (psd_export_common.h:124-196),
// used only with c_blend > 0.
__device__ __forceinline__ float3 psd_color_map(const float* __restrict__ cm, int map_h, int map_w, float x, float y,
                                                float radius, float rotation) {
  float r_inv = radius > 1e-6f ? (1.0f / radius) : 1e6f;
  float norm_x = x * r_inv;
  float norm_y = y * r_inv;
  float cos_theta = cosf(rotation);
  float sin_theta = sinf(rotation);
  float rot_x = cos_theta * norm_x + sin_theta * norm_y;
  float rot_y = -sin_theta * norm_x + cos_theta * norm_y;
  float coord_x = (rot_x + 1.0f) * 0.5f * (map_w - 1);
  float coord_y = (rot_y + 1.0f) * 0.5f * (map_h - 1);
  coord_x = fmaxf(0.0f, fminf(map_w - 1, coord_x));
  coord_y = fmaxf(0.0f, fminf(map_h - 1, coord_y));
  int x0 = (int)coord_x;
  int y0 = (int)coord_y;
  int x1 = min(x0 + 1, map_w - 1);
  int y1 = min(y0 + 1, map_h - 1);
  float fx = coord_x - x0;
  float fy = coord_y - y0;
  float3 out;
  float* o = &out.x;
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const float c00 = cm[3 * (y0 * map_w + x0) + ch], c01 = cm[3 * (y1 * map_w + x0) + ch];
    const float c10 = cm[3 * (y0 * map_w + x1) + ch], c11 = cm[3 * (y1 * map_w + x1) + ch];
    const float c0 = c00 * (1.0f - fx) + c10 * fx;
    const float c1 = c01 * (1.0f - fx) + c11 * fx;
    o[ch] = c0 * (1.0f - fy) + c1 * fy;
  }
  return out;
}

__device__ __forceinline__ uint8_t to_u8(float v) { return (uint8_t)fmaxf(0.0f, fminf(255.0f, v * 255.0f)); }

struct PsdArgs {
  int N, P, Ht, Wt;
  float scale, alpha_max, c_blend;
};

// Stage 2 (psd_export_kernels.cu:61-198): persistent grid over the 16x16
// blocks of all crops; block b belongs to the layer n with blk[n] <= b < blk[n+1].
// Everything that depends only on the layer -- its index (a binary search
// over blk), crop box, centre, radius, rotation with its cosine and sine,
// opacity and colour -- is computed once per block by one thread and shared
// through shared memory; each thread then computes one pixel with the
// reference's per-pixel operations on the same values, so the bytes are the
// ones a per-pixel evaluation gives.
struct PsdLayer {
  int4 bb;
  float x, y, r, theta, cos_t, sin_t, vis, cr, cg, cb;
  int n, t_idx;
  int bx, by;    // the block's first pixel within the crop
  long long off;
};

__global__ void __launch_bounds__(256) psd_layers_kernel(PsdArgs a, const float* __restrict__ means2D,
                                                         const float* __restrict__ radii,
                                                         const float* __restrict__ rot,
                                                         const float* __restrict__ colors,
                                                         const float* __restrict__ vis,
                                                         const float* __restrict__ tmpl, const int* __restrict__ sel,
                                                         const int* __restrict__ bbox,
                                                         const long long* __restrict__ layer_offsets,
                                                         const long long* __restrict__ blk,
                                                         const float* __restrict__ colors_orig,
                                                         uint8_t* __restrict__ out) {
  __shared__ PsdLayer s_l;
  const long long nblk = blk[a.N];
  const int lx = threadIdx.x & (kPsdBlock - 1), ly = threadIdx.x / kPsdBlock;
  for (long long b = blockIdx.x; b < nblk; b += gridDim.x) {
    __syncthreads();   // every thread is done with the previous block's layer
    if (threadIdx.x == 0) {
      int lo = 0, hi = a.N;   // largest n with blk[n] <= b
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (blk[mid] <= b) lo = mid; else hi = mid;
      }
      const int n = lo;
      PsdLayer L;
      L.n = n;
      L.bb = reinterpret_cast<const int4*>(bbox)[n];
      const int bx_n = (L.bb.z - L.bb.x + kPsdBlock - 1) / kPsdBlock;   // blocks per crop row
      const long long k = b - blk[n];
      L.bx = (int)(k % bx_n) * kPsdBlock;
      L.by = (int)(k / bx_n) * kPsdBlock;
      L.x = means2D[n * 2 + 0] * a.scale;
      L.y = means2D[n * 2 + 1] * a.scale;
      L.r = radii[n] * a.scale;
      L.theta = rot[n];
      L.cos_t = cosf(L.theta);
      L.sin_t = sinf(L.theta);
      L.vis = vis[n];
      L.cr = colors[n * 3 + 0];
      L.cg = colors[n * 3 + 1];
      L.cb = colors[n * 3 + 2];
      L.t_idx = sel[n];
      L.off = layer_offsets[n];
      s_l = L;
    }
    __syncthreads();
    const PsdLayer L = s_l;
    const int bw = L.bb.z - L.bb.x, bh = L.bb.w - L.bb.y;
    const int lpx = L.bx + lx, lpy = L.by + ly;
    if (lpx >= bw || lpy >= bh) continue;
    const int px = L.bb.x + lpx, py = L.bb.y + lpy;
    const float tv = psd_template_value(tmpl, L.t_idx, a.P, a.Ht, a.Wt, px, py, L.x, L.y, L.r, L.cos_t, L.sin_t);
    const float alpha_val = tv * L.vis * a.alpha_max;
    uchar4 px4 = make_uchar4(0, 0, 0, 0);
    if (!(alpha_val < 0.001f)) {
      float rgb_r = L.cr, rgb_g = L.cg, rgb_b = L.cb;
      if (colors_orig != nullptr && a.c_blend > 0.0f) {
        const float* cm = colors_orig + (size_t)L.n * a.Ht * a.Wt * 3;
        const float ux = L.x / a.scale, uy = L.y / a.scale;
        const float upx = (float)px / a.scale, upy = (float)py / a.scale;
        const float ur = L.r / a.scale;
        const float3 co = psd_color_map(cm, a.Ht, a.Wt, upx - ux, upy - uy, ur, L.theta);
        rgb_r = (1.0f - a.c_blend) * rgb_r + a.c_blend * co.x;
        rgb_g = (1.0f - a.c_blend) * rgb_g + a.c_blend * co.y;
        rgb_b = (1.0f - a.c_blend) * rgb_b + a.c_blend * co.z;
      }
      const float mask = tv > 0.0f ? 1.0f : 0.0f;
      px4 = make_uchar4(to_u8(mask * rgb_r), to_u8(mask * rgb_g), to_u8(mask * rgb_b), to_u8(alpha_val));
    }
    *reinterpret_cast<uchar4*>(out + L.off + ((long long)lpy * bw + lpx) * 4) = px4;
  }
}

// ---------------------------------------------------------------------------
// PSD file assembly: PackBits (RLE) channel data.
//
// The reference hands each cropped layer to psd-tools (PixelLayer.frompil,
// then PSDImage.save; psd_export_uint8.py:153-186, psd_exporter.py:468-501),
// which splits it into planes and RLE-compresses them row by row on the host.
// Here every (layer, channel, row) is encoded on the device.  Rows are taken
// 32 at a time: one CTA of 128 threads per group of 32 rows of a layer, one
// thread per (row, channel slot), so each thread runs a single encoder.  The
// CTA stages the group's uchar4 pixels through shared memory, 32 rows x 32
// pixels at a time (coalesced loads; a 33-word row pitch keeps the reads
// conflict-free: the four threads of a row read the same word).  In the
// write pass each thread keeps the bytes of its row in a 256-byte ring in
// shared memory, from which literal packets are written.
//
// Encoding rule (a valid PackBits stream; a packet never crosses a row):
//   - a maximal run of L >= 3 equal bytes becomes replicate packets
//     [1-k, v] of k = min(remaining, 128) bytes each; a one-byte remainder
//     becomes the literal packet [0, v];
//   - maximal runs of one or two bytes are gathered into literal segments,
//     written as packets [k-1, k bytes] of 128 bytes and a last shorter one.
// A literal segment that ends at a run of three or more is written as soon as
// the run reaches three bytes (the packets and their order are those of
// writing it when the run ends), so the bytes a pending literal segment needs
// are never more than 131 behind the current one and the ring suffices.
// The count pass writes each row's encoded size (at most w + ceil(w/128)
// bytes, so 16 bits suffice for w <= 30000, the PSD width limit) and each
// group's per-channel totals; the host plans where every channel block goes;
// the write pass re-encodes and stores.  Each store is checked against the
// planned extent of its row and the output size, so a plan that does not
// match the data can write wrong bytes but never out of bounds.
// ---------------------------------------------------------------------------

constexpr int kRleRows = 32;                  // rows per group (one CTA)
constexpr int kRleThreads = kRleRows * 4;     // one thread per (row, channel slot)
constexpr int kRlePitch = 33;                 // words per staged row (32 pixels + 1 pad)
constexpr int kRleRing = 256;                 // bytes of a thread's literal ring
constexpr int kRleRingPitch = kRleRing + 4;   // ring stride: threads of a warp hit distinct banks

struct RleArgs {
  const uint8_t* layers;        // packed RGBA crops, row-major per layer
  const int* sizes;             // (N,2) w, h
  const long long* layer_off;   // (N) byte offset of each crop
  const long long* group_base;  // (N+1) exclusive prefix of ceil(h/32)
  long long G;                  // number of row groups
  int N;
  unsigned order;               // byte index (0..3) of channel slot s in bits 8s..8s+1
  int width_limit;
  unsigned short* row_bytes;    // (G*32, 4) encoded size of each row's four channels
  int* group_tot;               // (G, 4) per-group totals (count pass)
  int* alpha_any;               // (N) 1 if a layer has a nonzero byte 3 (count pass; may be null)
  const long long* chan_off;    // (N, 4) channel block offsets in out, < 0 skips (write pass)
  const long long* group_dst;   // (G, 4) output offset of the group's first row (write pass)
  uint8_t* out;                 // (write pass)
  long long out_bytes;
};

// PackBits encoder of one channel row.  COUNT (WRITE false) only adds sizes;
// WRITE stores, reading literal bytes from the thread's ring (ring[x & 255] =
// byte x of the row).
template <bool WRITE>
struct RleChan {
  int prev, run, lit, lst;
  long long pos, lim;
  uint8_t* ring;
  uint8_t* out;

  __device__ __forceinline__ void put(unsigned v) {
    if (WRITE && pos < lim) out[pos] = (uint8_t)v;
    ++pos;
  }
  __device__ __forceinline__ void literal(int start, int k) {
    if (!WRITE) { pos += 1 + k; return; }
    put((unsigned)(k - 1));
    for (int j = 0; j < k; ++j) put(ring[(start + j) & (kRleRing - 1)]);
  }
  // Closes the run of `run` bytes equal to prev that ends before x = end.
  __device__ __forceinline__ void close(int end) {
    const int L = run;
    if (L >= 3) {
      // the pending literal segment went out when the run reached three bytes
      lst = end;
      if (!WRITE) { pos += 2 * ((L + 127) >> 7); return; }
      for (int rem = L; rem > 0; rem -= 128) {
        const int k = min(rem, 128);
        put(k >= 2 ? (unsigned)(1 - k) & 0xFFu : 0u);
        put((unsigned)prev);
      }
    } else {
      lit += L;
      if (lit >= 128) {
        literal(lst, 128);
        lst += 128;
        lit -= 128;
      }
    }
  }
  __device__ __forceinline__ void push(int v, int x) {
    if (v == prev) {
      if (++run == 3 && lit > 0) {   // this run will be replicate packets: the literals before it go now
        literal(lst, lit);
        lit = 0;
      }
      return;
    }
    close(x);
    prev = v;
    run = 1;
  }
  __device__ __forceinline__ void finish(int w) {
    close(w);
    if (lit > 0) literal(lst, lit);
  }
};

template <bool WRITE>
__global__ void __launch_bounds__(kRleThreads) psd_rle_kernel(RleArgs a) {
  __shared__ uint32_t stage[kRleRows * kRlePitch];
  __shared__ __align__(16) uint8_t ring[WRITE ? kRleThreads * kRleRingPitch : 16];
  __shared__ unsigned short s_planned[kRleRows * 4];
  __shared__ int s_tot[4];
  __shared__ int s_any;
  __shared__ int s_layer;
  const int t = threadIdx.x;
  const int row = t >> 2, slot = t & 3;          // the four threads of a row are adjacent lanes
  const int byte = (a.order >> (8 * slot)) & 3;   // which RGBA byte this thread's channel slot takes
  for (long long g = blockIdx.x; g < a.G; g += gridDim.x) {
    __syncthreads();   // the previous group is done with the shared buffers
    if (t == 0) {
      int lo = 0, hi = a.N;   // largest i with group_base[i] <= g
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (a.group_base[mid] <= g) lo = mid; else hi = mid;
      }
      s_layer = lo;
      s_any = 0;
    }
    if (t < 4) s_tot[t] = 0;
    __syncthreads();
    const int i = s_layer;
    const int w = a.sizes[2 * i], h = a.sizes[2 * i + 1];
    const long long off = a.layer_off[i];
    const bool ok = w >= 1 && w <= a.width_limit && h >= 1 && off >= 0 && (off & 3) == 0;
    const long long y0 = (g - a.group_base[i]) * kRleRows;
    const long long y = y0 + row;
    const bool active = ok && y < h;
    const uint8_t* base = a.layers + (ok ? off : 0);

    RleChan<WRITE> e;
    e.prev = -1; e.run = 0; e.lit = 0; e.lst = 0;
    e.pos = 0; e.lim = 0;
    e.ring = ring + (WRITE ? t * kRleRingPitch : 0);
    e.out = a.out;
    bool skip = !ok;   // CTA-uniform: depends on the layer only
    if (WRITE) {
      const unsigned short planned = (ok && active) ? a.row_bytes[(g * kRleRows + row) * 4 + slot] : 0;
      s_planned[row * 4 + slot] = planned;
      __syncthreads();
      long long pre = 0;   // exclusive prefix over the group's rows of this channel slot
      for (int r = 0; r < row; ++r) pre += s_planned[r * 4 + slot];
      const long long co = ok ? a.chan_off[4 * i + slot] : -1;
      const long long gd = ok ? a.group_dst[4 * g + slot] : -1;
      if (co >= 0 && gd >= 0) {
        e.pos = gd + pre;
        e.lim = min(e.pos + planned, a.out_bytes);
        if (active) {   // row byte count, big-endian, in the block's table; block header on row 0
          const long long tb = co + 2 + 2ll * y;
          if (tb + 1 < a.out_bytes) { a.out[tb] = (uint8_t)(planned >> 8); a.out[tb + 1] = (uint8_t)planned; }
          if (y == 0 && co + 1 < a.out_bytes) { a.out[co] = 0; a.out[co + 1] = 1; }
        }
      }
      skip = skip || (a.chan_off[4 * i] < 0 && a.chan_off[4 * i + 1] < 0 && a.chan_off[4 * i + 2] < 0 &&
                      a.chan_off[4 * i + 3] < 0);
    }

    unsigned any_alpha = 0;
    if (!skip) {
      for (int x0 = 0; x0 < w; x0 += 32) {
        __syncthreads();
        for (int k = t; k < kRleRows * 32; k += kRleThreads) {   // consecutive threads, consecutive pixels
          const int r = k >> 5, c = k & 31;
          uint32_t v = 0;
          if (y0 + r < h && x0 + c < w)
            v = *reinterpret_cast<const uint32_t*>(base + ((y0 + r) * (long long)w + x0 + c) * 4);
          stage[r * kRlePitch + c] = v;
        }
        __syncthreads();
        if (active) {
          const int n = min(32, w - x0);
          const uint32_t* src = stage + row * kRlePitch;
          for (int x = 0; x < n; ++x) {
            const uint32_t p = src[x];
            const int v = (p >> (8 * byte)) & 0xFF;
            any_alpha |= p >> 24;
            if (WRITE) e.ring[(x0 + x) & (kRleRing - 1)] = (uint8_t)v;
            e.push(v, x0 + x);
          }
        }
      }
      if (active) e.finish(w);
    }
    if (!WRITE) {
      const int c = active && !skip ? (int)e.pos : 0;
      a.row_bytes[(g * kRleRows + row) * 4 + slot] = (unsigned short)c;
      atomicAdd(&s_tot[slot], c);
      if (any_alpha != 0) s_any = 1;
      __syncthreads();
      if (t == 0) {
        reinterpret_cast<int4*>(a.group_tot)[g] = make_int4(s_tot[0], s_tot[1], s_tot[2], s_tot[3]);
        if (s_any && a.alpha_any) a.alpha_any[i] = 1;
      }
    }
  }
}

// CTAs of psd_rle_kernel<write> resident at once on the current device,
// computed once per (device, pass) under a lock (devices may differ).
static int rle_resident_ctas(bool write) {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static int resident[kMaxDevices][2] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 148;
  std::lock_guard<std::mutex> lock(mu);
  int& r = resident[dev][write ? 1 : 0];
  if (r == 0) {
    int per_sm = 0, sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (write) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, psd_rle_kernel<true>, kRleThreads, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, psd_rle_kernel<false>, kRleThreads, 0);
    r = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 148);
  }
  return r;
}

int launch_psd_rle(bool write, const uint8_t* layers, const int* sizes, const long long* layer_off,
                   const long long* group_base, int N, long long G, unsigned order, int width_limit,
                   unsigned short* row_bytes, int* group_tot, int* alpha_any, const long long* chan_off,
                   const long long* group_dst, uint8_t* out, long long out_bytes, cudaStream_t st) {
  if (G == 0 || N == 0) return DBMP_OK;
  const RleArgs a{layers, sizes, layer_off, group_base, G, N, order, width_limit, row_bytes, group_tot,
                  alpha_any, chan_off, group_dst, out, out_bytes};
  // persistent grid: as many CTAs as are resident at once, striding over the row groups
  const int resident = rle_resident_ctas(write);
  const long long ctas = G < resident ? G : resident;
  if (write) psd_rle_kernel<true><<<(int)ctas, kRleThreads, 0, st>>>(a);
  else psd_rle_kernel<false><<<(int)ctas, kRleThreads, 0, st>>>(a);
  DBMP_CHECK_LAUNCH("psd_rle_kernel");
  return DBMP_OK;
}

int launch_psd_bboxes(const float* means2D, const float* radii, int N, int H, int W, float scale, int* bbox,
                      int* sizes, cudaStream_t st) {
  if (N == 0) return DBMP_OK;
  psd_bbox_kernel<<<(N + 255) / 256, 256, 0, st>>>(means2D, radii, N, H, W, scale, bbox, sizes);
  DBMP_CHECK_LAUNCH("psd_bbox_kernel");
  return DBMP_OK;
}

int launch_psd_layout(const int* sizes, int N, long long* layer_offsets, long long* blk, long long* total,
                      cudaStream_t st) {
  psd_layout_kernel<<<1, 1024, 0, st>>>(sizes, N, layer_offsets, blk, total);
  DBMP_CHECK_LAUNCH("psd_layout_kernel");
  return DBMP_OK;
}

int launch_psd_layers(int N, int P, int Ht, int Wt, float scale, float alpha_max, float c_blend,
                      const float* means2D, const float* radii, const float* rot, const float* colors,
                      const float* vis, const float* tmpl, const int* sel, const int* bbox,
                      const long long* layer_offsets, const long long* blk, const float* colors_orig, uint8_t* out,
                      cudaStream_t st) {
  if (N == 0) return DBMP_OK;
  PsdArgs a{N, P, Ht, Wt, scale, alpha_max, c_blend};
  psd_layers_kernel<<<148 * 8, 256, 0, st>>>(a, means2D, radii, rot, colors, vis, tmpl, sel, bbox, layer_offsets,
                                             blk, colors_orig, out);
  DBMP_CHECK_LAUNCH("psd_layers_kernel");
  return DBMP_OK;
}

}  // namespace dbmp
