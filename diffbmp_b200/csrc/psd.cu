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
#include <type_traits>

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

// Template value at canvas pixel (px,py): psd_export_common.h:55-103, with
// each floating-point operation in the reference's order (the layers must be
// byte-identical under --use_fast_math).  The texel coordinate (sx, sy) comes
// from (px - x) / r rotated by theta; outside [0, W-1) x [0, H-1) the value is
// a hard zero.  After that test the cell (ix, iy) = floor(sx, sy) lies in
// [0, W-2] x [0, H-2] (a NaN coordinate converts to cell 0), so it needs no
// clamp, and the weights take the floors as floats, which equal the cell
// indices exactly.
__device__ __forceinline__ float psd_template_value(const float* __restrict__ tmpl, int t_idx, int P, int Ht, int Wt,
                                                    int px, int py, float x, float y, float r, float cos_t,
                                                    float sin_t) {
  const float qx = ((float)px - x) / (r);
  const float qy = ((float)py - y) / (r);
  const float ex = cos_t * qx + sin_t * qy;
  const float ey = -sin_t * qx + cos_t * qy;
  const float sx = (ex + 1.0f) * 0.5f * (Wt - 1);
  const float sy = (ey + 1.0f) * 0.5f * (Ht - 1);
  if (sx < 0.0f || sx >= Wt - 1 || sy < 0.0f || sy >= Ht - 1) return 0.0f;
  if (t_idx < 0 || t_idx >= P) return 0.0f;   // the reference reads out of bounds here
  const float flx = floorf(sx), fly = floorf(sy);
  const int ix = (int)flx, iy = (int)fly;
  const float fx = sx - flx;
  const float fy = sy - fly;
  const float gx = 1.0f - fx;
  const float gy = 1.0f - fy;
  const float* row = tmpl + (size_t)t_idx * Ht * Wt + iy * Wt + ix;
  const float s00 = row[0], s01 = row[1], s10 = row[Wt], s11 = row[Wt + 1];
  return gx * gy * s00 + fx * gy * s01 + gx * fy * s10 + fx * fy * s11;
}

// Clamped bilinear of a per-primitive RGB map (psd_export_common.h:124-196,
// operations in its order), used only with c_blend > 0: the coordinate is
// clamped into the map and the neighbours past the last row / column repeat it.
__device__ __forceinline__ float3 psd_color_map(const float* __restrict__ cm, int map_h, int map_w, float x, float y,
                                                float radius, float rotation) {
  const float inv = radius > 1e-6f ? (1.0f / radius) : 1e6f;
  const float qx = x * inv;
  const float qy = y * inv;
  const float ct = cosf(rotation);
  const float st = sinf(rotation);
  const float ex = ct * qx + st * qy;
  const float ey = -st * qx + ct * qy;
  float sx = (ex + 1.0f) * 0.5f * (map_w - 1);
  float sy = (ey + 1.0f) * 0.5f * (map_h - 1);
  sx = fmaxf(0.0f, fminf(map_w - 1, sx));
  sy = fmaxf(0.0f, fminf(map_h - 1, sy));
  const int ix = (int)sx, iy = (int)sy;
  const int jx = min(ix + 1, map_w - 1), jy = min(iy + 1, map_h - 1);
  const float fx = sx - ix;
  const float fy = sy - iy;
  float3 out;
  float* o = &out.x;
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const float a0 = cm[3 * (iy * map_w + ix) + ch], b0 = cm[3 * (jy * map_w + ix) + ch];
    const float a1 = cm[3 * (iy * map_w + jx) + ch], b1 = cm[3 * (jy * map_w + jx) + ch];
    const float top = a0 * (1.0f - fx) + a1 * fx;
    const float bot = b0 * (1.0f - fx) + b1 * fx;
    o[ch] = top * (1.0f - fy) + bot * fy;
  }
  return out;
}

__device__ __forceinline__ uint8_t to_u8(float v) { return (uint8_t)fmaxf(0.0f, fminf(255.0f, v * 255.0f)); }

struct PsdArgs {
  int N, P, Ht, Wt;
  float scale, alpha_max, c_blend;
};

// Stage 2 (psd_export_kernels.cu:61-198): the 16x16 blocks of all crops, block
// b of layer n for blk[n] <= b < blk[n+1].  Each warp takes a contiguous range
// of blocks and walks them in order, a whole block at a time: lane l owns
// column l % 16 and rows l / 16, l / 16 + 2, ... of the block (eight pixels;
// each half-warp stores 64 contiguous bytes of a row).  Lane 0 follows the
// layer index forward from block to block (a binary search only for the
// range's first block) and loads the layer's box, centre, radius, rotation
// with its cosine and sine, opacity and colour once per layer, broadcast to
// the lanes.  Each thread then computes its pixels with the reference's
// per-pixel operations on the same values, so the bytes are the ones a
// per-pixel evaluation gives.
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
  const long long nblk = blk[a.N];
  const int lane = threadIdx.x & 31;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const long long per = (nblk + nwarps - 1) / nwarps;
  const long long b0 = gw * per, b1 = min(b0 + per, nblk);
  const int lx = lane & (kPsdBlock - 1), ly0 = lane >> 4;   // this thread's column and first row in a block
  int n = -1;                      // the current layer (lane 0's bookkeeping, broadcast below)
  long long next = 0;              // blk[n + 1]
  int4 bb = make_int4(0, 0, 0, 0);
  float x = 0.f, y = 0.f, r = 0.f, theta = 0.f, cos_t = 0.f, sin_t = 0.f, vs = 0.f, cr = 0.f, cg = 0.f, cb = 0.f;
  int t_idx = 0, bx_n = 1;
  long long off = 0, first = 0;    // the layer's byte offset and first block
  int bx = 0, by = 0;              // the current block's first pixel within the crop
  for (long long b = b0; b < b1; ++b) {
    bool changed = false;
    if (lane == 0 && (n < 0 || b >= next)) {
      if (n < 0) {   // largest n with blk[n] <= b
        int lo = 0, hi = a.N;
        while (hi - lo > 1) {
          const int mid = (lo + hi) >> 1;
          if (blk[mid] <= b) lo = mid; else hi = mid;
        }
        n = lo;
      } else {
        while (blk[n + 1] <= b) ++n;   // empty crops have no blocks
      }
      next = blk[n + 1];
      changed = true;
    }
    if (__shfl_sync(0xffffffffu, changed, 0)) {
      if (lane == 0) {
        bb = reinterpret_cast<const int4*>(bbox)[n];
        x = means2D[n * 2 + 0] * a.scale;
        y = means2D[n * 2 + 1] * a.scale;
        r = radii[n] * a.scale;
        theta = rot[n];
        cos_t = cosf(theta);
        sin_t = sinf(theta);
        vs = vis[n];
        cr = colors[n * 3 + 0]; cg = colors[n * 3 + 1]; cb = colors[n * 3 + 2];
        t_idx = sel[n];
        off = layer_offsets[n];
        first = blk[n];
        bx_n = (bb.z - bb.x + kPsdBlock - 1) / kPsdBlock;
      }
      n = __shfl_sync(0xffffffffu, n, 0);
      bb.x = __shfl_sync(0xffffffffu, bb.x, 0); bb.y = __shfl_sync(0xffffffffu, bb.y, 0);
      bb.z = __shfl_sync(0xffffffffu, bb.z, 0); bb.w = __shfl_sync(0xffffffffu, bb.w, 0);
      x = __shfl_sync(0xffffffffu, x, 0); y = __shfl_sync(0xffffffffu, y, 0); r = __shfl_sync(0xffffffffu, r, 0);
      theta = __shfl_sync(0xffffffffu, theta, 0);
      cos_t = __shfl_sync(0xffffffffu, cos_t, 0); sin_t = __shfl_sync(0xffffffffu, sin_t, 0);
      vs = __shfl_sync(0xffffffffu, vs, 0);
      cr = __shfl_sync(0xffffffffu, cr, 0); cg = __shfl_sync(0xffffffffu, cg, 0); cb = __shfl_sync(0xffffffffu, cb, 0);
      t_idx = __shfl_sync(0xffffffffu, t_idx, 0);
      off = __shfl_sync(0xffffffffu, off, 0);
      first = __shfl_sync(0xffffffffu, first, 0);
      bx_n = __shfl_sync(0xffffffffu, bx_n, 0);
      const int k = (int)(b - first);   // block within the crop (a crop has < 2^31 blocks)
      bx = (k % bx_n) * kPsdBlock;
      by = (k / bx_n) * kPsdBlock;
    } else {                            // the next block of the same crop, row-major
      bx += kPsdBlock;
      if (bx >= bb.z - bb.x) { bx = 0; by += kPsdBlock; }
    }
    const int bw = bb.z - bb.x, bh = bb.w - bb.y;
    // Warp-uniform: true when the whole block maps outside the template
    // square [-1, 1) x [-1, 1) of the normalised frame (rotated (p - c) / r)
    // by a margin of 1e-3, far above the rounding of the per-pixel
    // coordinates; each of its pixels then takes the hard zero, and its bytes
    // are stored as zeros without the per-pixel arithmetic.  The map is affine,
    // so the block's four corner pixels bound it.  Only for finite inputs with
    // r > 1e-3: a non-finite coordinate or opacity can give nonzero bytes.
    bool outside = false;
    if (r > 1e-3f && isfinite(r) && isfinite(x) && isfinite(y) && isfinite(cos_t) && isfinite(sin_t) &&
        isfinite(vs) && isfinite(a.alpha_max)) {
      const float inv = 1.0f / r;
      const float qx0 = ((float)(bb.x + bx) - x) * inv, qx1 = ((float)(bb.x + bx + kPsdBlock - 1) - x) * inv;
      const float qy0 = ((float)(bb.y + by) - y) * inv, qy1 = ((float)(bb.y + by + kPsdBlock - 1) - y) * inv;
      const float ex00 = cos_t * qx0 + sin_t * qy0, ex10 = cos_t * qx1 + sin_t * qy0;
      const float ex01 = cos_t * qx0 + sin_t * qy1, ex11 = cos_t * qx1 + sin_t * qy1;
      const float ey00 = cos_t * qy0 - sin_t * qx0, ey10 = cos_t * qy0 - sin_t * qx1;
      const float ey01 = cos_t * qy1 - sin_t * qx0, ey11 = cos_t * qy1 - sin_t * qx1;
      const float m = 1e-3f;
      outside = fmaxf(fmaxf(ex00, ex10), fmaxf(ex01, ex11)) < -1.0f - m ||
                fminf(fminf(ex00, ex10), fminf(ex01, ex11)) > 1.0f + m ||
                fmaxf(fmaxf(ey00, ey10), fmaxf(ey01, ey11)) < -1.0f - m ||
                fminf(fminf(ey00, ey10), fminf(ey01, ey11)) > 1.0f + m;
    }
    const int lpx = bx + lx;
    if (lpx >= bw) continue;
    const int px = bb.x + lpx;
    const int rows = min(kPsdBlock, bh - by);   // rows of this block inside the crop
    if (outside) {
      for (int ly = ly0; ly < rows; ly += 2)
        *reinterpret_cast<uchar4*>(out + off + ((long long)(by + ly) * bw + lpx) * 4) = make_uchar4(0, 0, 0, 0);
      continue;
    }
    for (int ly = ly0; ly < rows; ly += 2) {
      const int lpy = by + ly;
      const int py = bb.y + lpy;
      // The column is hidden from the optimiser in every row, so no part of
      // the pixel's expression is hoisted out of the loop: a hoisted cos*u
      // lets the compiler fuse the other product instead, which changes the
      // fast-math rounding and, rarely, a byte against the reference kernel.
      int pxr = px;
      asm volatile("" : "+r"(pxr));
      const float tv = psd_template_value(tmpl, t_idx, a.P, a.Ht, a.Wt, pxr, py, x, y, r, cos_t, sin_t);
      const float alpha_val = tv * vs * a.alpha_max;
      uchar4 px4 = make_uchar4(0, 0, 0, 0);
      if (!(alpha_val < 0.001f)) {
        float rgb_r = cr, rgb_g = cg, rgb_b = cb;
        if (colors_orig != nullptr && a.c_blend > 0.0f) {
          const float* cm = colors_orig + (size_t)n * a.Ht * a.Wt * 3;
          const float ux = x / a.scale, uy = y / a.scale;
          const float upx = (float)pxr / a.scale, upy = (float)py / a.scale;
          const float ur = r / a.scale;
          const float3 co = psd_color_map(cm, a.Ht, a.Wt, upx - ux, upy - uy, ur, theta);
          rgb_r = (1.0f - a.c_blend) * rgb_r + a.c_blend * co.x;
          rgb_g = (1.0f - a.c_blend) * rgb_g + a.c_blend * co.y;
          rgb_b = (1.0f - a.c_blend) * rgb_b + a.c_blend * co.z;
        }
        const float mask = tv > 0.0f ? 1.0f : 0.0f;
        px4 = make_uchar4(to_u8(mask * rgb_r), to_u8(mask * rgb_g), to_u8(mask * rgb_b), to_u8(alpha_val));
      }
      *reinterpret_cast<uchar4*>(out + off + ((long long)lpy * bw + lpx) * 4) = px4;
    }
  }
}

// ---------------------------------------------------------------------------
// PSD file assembly: PackBits (RLE) channel data.
//
// The reference hands each cropped layer to psd-tools (PixelLayer.frompil,
// then PSDImage.save; psd_export_uint8.py:153-186, psd_exporter.py:468-501),
// which splits it into planes and RLE-compresses them row by row on the host.
// Here every (layer, channel, row) is encoded on the device.  Rows are taken
// 32 at a time, one warp per group of 32 rows of a layer and one lane per
// row; each lane runs four encoders at once, one per RGBA byte, on uchar4
// pixels that the warp stages through shared memory 32 rows x 32 pixels at a
// time (cp.async copies of coalesced row segments into two buffers, the next
// chunk in flight while the current one is encoded; conflict-free reads with
// a 36-word row pitch, four pixels per 16-byte read).
//
// Encoding rule (a valid PackBits stream; a packet never crosses a row):
//   - a maximal run of L >= 3 equal bytes becomes replicate packets
//     [1-k, v] of k = min(remaining, 128) bytes each; a one-byte remainder
//     becomes the literal packet [0, v];
//   - maximal runs of one or two bytes are gathered into literal segments,
//     written as packets [k-1, k bytes] of 128 bytes and a last shorter one.
// The count pass writes each row's encoded size (at most w + ceil(w/128)
// bytes, so 16 bits suffice for w <= 30000, the PSD width limit that the C
// ABI enforces on width_limit) and each
// group's per-channel totals; the host plans where every channel block goes;
// the write pass re-encodes and stores.  Each store is checked against the
// planned extent of its row and the output size, so a plan that does not
// match the data can write wrong bytes but never out of bounds.
// ---------------------------------------------------------------------------

constexpr int kRleWarps = 4;      // warps per CTA (two staging buffers of 32 x 36 words each)
// Words per staged row: 32 pixels + 4 pad.  Row starts 144 bytes apart keep
// the staging copies (32 consecutive words of a row) and each lane's 16-byte
// reads of its own row (8 lanes per phase on distinct 16-byte bank groups)
// free of bank conflicts.
constexpr int kRlePitch = 36;

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

// Four PackBits encoders of one row, counting output bytes only (count pass).
// A literal segment's headers are added when the segment closes, or when 128
// bytes are in.
struct RleCount {
  int prev[4], run[4], lit[4];
  long long pos[4];

  __device__ __forceinline__ void close(int s) {
    const int L = run[s];
    if (L >= 3) {
      if (lit[s] > 0) pos[s] += 1 + lit[s];
      lit[s] = 0;
      pos[s] += 2 * ((L + 127) >> 7);
    } else {
      lit[s] += L;
      if (lit[s] >= 128) {
        pos[s] += 129;
        lit[s] -= 128;
      }
    }
  }
  __device__ __forceinline__ void push(int s, int v) {
    if (v == prev[s]) { ++run[s]; return; }
    close(s);
    prev[s] = v;
    run[s] = 1;
  }
  __device__ __forceinline__ void finish(int s) {
    close(s);
    if (lit[s] > 0) pos[s] += 1 + lit[s];
  }
};

// Four PackBits encoders of one row that store their bytes (write pass).
// Positions are byte offsets within the row's output of each channel slot.
// A literal byte is stored as soon as its run closes (a run of one or two
// bytes), at its final place: a literal packet's header position is reserved
// when the packet opens and written when it closes (127 when 128 bytes are
// in, the count minus one at the end of the segment), so no byte of the crop
// is read twice.  (An earlier form re-read literal bytes from the crop when
// their segment closed: 23.3 against 14.9 ms at 2048x2048, N=20000.  The
// count pass keeps its own encoder: sharing this one took it from 8.0 to
// 14.1 ms.)
struct RleWrite {
  int prev[4], run[4], lit[4], pos[4], lim[4], hdr[4];
  uint8_t* dst[4];   // the row's first output byte of each slot

  __device__ __forceinline__ void store(int s, int p, unsigned v) {
    if (p < lim[s]) dst[s][p] = (uint8_t)v;
  }
  __device__ __forceinline__ void put(int s, unsigned v) {
    store(s, pos[s], v);
    ++pos[s];
  }
  // Appends one byte to the open literal segment.
  __device__ __forceinline__ void lit_byte(int s, unsigned v) {
    if ((lit[s] & 127) == 0) hdr[s] = pos[s]++;
    put(s, v);
    if ((++lit[s] & 127) == 0) store(s, hdr[s], 127u);
  }
  __device__ __forceinline__ void end_literal(int s) {
    if (lit[s] & 127) store(s, hdr[s], (unsigned)((lit[s] & 127) - 1));
    lit[s] = 0;
  }
  // Closes the run of run[s] bytes equal to prev[s].
  __device__ __forceinline__ void close(int s) {
    const int L = run[s];
    if (L >= 3) {
      end_literal(s);
      for (int rem = L; rem > 0; rem -= 128) {
        const int k = min(rem, 128);
        put(s, k >= 2 ? (unsigned)(1 - k) & 0xFFu : 0u);
        put(s, (unsigned)prev[s]);
      }
    } else {
      for (int j = 0; j < L; ++j) lit_byte(s, (unsigned)prev[s]);
    }
  }
  __device__ __forceinline__ void push(int s, int v) {
    if (v == prev[s]) { ++run[s]; return; }
    close(s);
    prev[s] = v;
    run[s] = 1;
  }
  __device__ __forceinline__ void finish(int s) {
    close(s);
    end_literal(s);
  }
};

// One 4-byte asynchronous copy from global to shared memory (cp.async); with
// valid false nothing is read and the word is zero-filled.
__device__ __forceinline__ void cp_async_word(uint32_t* dst, const void* src, bool valid) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory"); }

template <bool WRITE>
__global__ void __launch_bounds__(kRleWarps * 32) psd_rle_kernel(RleArgs a) {
  // Per warp, two staging buffers of 32 rows x 32 pixels: the copies of the
  // next 32 columns of the group's rows are in flight while the lanes encode
  // the current ones.
  __shared__ __align__(16) uint32_t stage[kRleWarps][2][32 * kRlePitch];
  const int lane = threadIdx.x & 31;
  uint32_t(*sm)[32 * kRlePitch] = stage[threadIdx.x >> 5];
  const long long nwarps = (long long)gridDim.x * kRleWarps;
  for (long long g = (long long)blockIdx.x * kRleWarps + (threadIdx.x >> 5); g < a.G; g += nwarps) {
    int lo = 0, hi = a.N;   // largest i with group_base[i] <= g
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (a.group_base[mid] <= g) lo = mid; else hi = mid;
    }
    const int i = lo;
    const int w = a.sizes[2 * i], h = a.sizes[2 * i + 1];
    const long long off = a.layer_off[i];
    const bool ok = w >= 1 && w <= a.width_limit && h >= 1 && off >= 0 && (off & 3) == 0;
    const long long y0 = (g - a.group_base[i]) * 32;
    const int y = (int)y0 + lane;
    const bool active = ok && y0 + lane < h;
    const uint8_t* base = a.layers + (ok ? off : 0);

    std::conditional_t<WRITE, RleWrite, RleCount> e;
    unsigned short planned[4] = {0, 0, 0, 0};
    bool skip = !ok;
#pragma unroll
    for (int s = 0; s < 4; ++s) e.pos[s] = 0;
    if constexpr (WRITE) {
#pragma unroll
      for (int s = 0; s < 4; ++s) { e.lim[s] = 0; e.hdr[s] = 0; e.dst[s] = a.out; }
      if (ok && active) {
        const ushort4 rb = reinterpret_cast<const ushort4*>(a.row_bytes)[g * 32 + lane];
        planned[0] = rb.x; planned[1] = rb.y; planned[2] = rb.z; planned[3] = rb.w;
      }
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        int pre = planned[s];   // exclusive prefix over the group's rows
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, pre, d);
          if (lane >= d) pre += t;
        }
        pre -= planned[s];
        const long long co = ok ? a.chan_off[4 * i + s] : -1;
        const long long gd = ok ? a.group_dst[4 * g + s] : -1;
        if (co >= 0 && gd >= 0) {   // otherwise every store of this slot is dropped
          const long long start = gd + pre;
          e.dst[s] = a.out + start;
          e.lim[s] = (int)max(0ll, min((long long)planned[s], a.out_bytes - start));
          if (active) {   // row byte count, big-endian, in the block's table; block header on row 0
            const long long t = co + 2 + 2ll * y;
            if (t + 1 < a.out_bytes) { a.out[t] = (uint8_t)(planned[s] >> 8); a.out[t + 1] = (uint8_t)planned[s]; }
            if (y == 0 && co + 1 < a.out_bytes) { a.out[co] = 0; a.out[co + 1] = 1; }
          }
        }
      }
      skip = skip || (a.chan_off[4 * i] < 0 && a.chan_off[4 * i + 1] < 0 && a.chan_off[4 * i + 2] < 0 &&
                      a.chan_off[4 * i + 3] < 0);
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) { e.prev[s] = -1; e.run[s] = 0; e.lit[s] = 0; }

    uint32_t any_alpha = 0;
    unsigned long long last = 1ull << 32;   // the previous pixel; no pixel equals the initial value
    int eq = 0;                             // pixels equal to it not yet added to the four runs
    if (!skip) {   // warp-uniform: skip depends on the layer only
      // columns x0 .. x0 + 31 of the group's 32 rows into buffer buf, one
      // coalesced 128-byte row segment per copy instruction of the warp
      auto stage_chunk = [&](int x0, uint32_t* buf) {
#pragma unroll 8
        for (int r = 0; r < 32; ++r) {
          const bool v = y0 + r < h && x0 + lane < w;
          cp_async_word(buf + r * kRlePitch + lane, v ? base + ((y0 + r) * (long long)w + x0 + lane) * 4 : base, v);
        }
        cp_async_commit();
      };
      __syncwarp();   // every lane is done with both buffers (previous group)
      stage_chunk(0, sm[0]);
      int cur = 0;
      for (int x0 = 0; x0 < w; x0 += 32, cur ^= 1) {
        if (x0 + 32 < w) {
          stage_chunk(x0 + 32, sm[cur ^ 1]);   // read by every lane in the previous iteration
          cp_async_wait<1>();
        } else {
          cp_async_wait<0>();
        }
        __syncwarp();   // the lanes' copies of this chunk are visible to the whole warp
        if (active) {
          const int n = min(32, w - x0);
          for (int x = 0; x < n; x += 4) {   // four pixels per 16-byte read
            const uint4 q = *reinterpret_cast<const uint4*>(&sm[cur][lane * kRlePitch + x]);
            // When all four bytes repeat, every run grows; such pixels are only
            // counted, and added to the four runs when the pixel changes.  Four
            // repeats are taken at once from one 16-byte read (2048x2048,
            // N=20000 on a B200: count pass 12.5 -> 6.2 ms, write pass 14.7 ->
            // 8.0 ms against a per-byte path on 4-byte reads).
            if (x + 4 <= n && (unsigned long long)q.x == last && q.y == q.x && q.z == q.x && q.w == q.x) {
              eq += 4;
              continue;
            }
            const int k = min(4, n - x);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              if (j >= k) break;
              const uint32_t p = j == 0 ? q.x : j == 1 ? q.y : j == 2 ? q.z : q.w;
              if ((unsigned long long)p == last) {
                ++eq;
                continue;
              }
#pragma unroll
              for (int s = 0; s < 4; ++s) e.run[s] += eq;
              eq = 0;
              last = p;
              any_alpha |= p & 0xFF000000u;
#pragma unroll
              for (int s = 0; s < 4; ++s) e.push(s, (p >> (8 * ((a.order >> (8 * s)) & 3))) & 0xFF);
            }
          }
        }
        __syncwarp();   // every lane is done with this buffer before the next iteration refills it
      }
      if (active) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          e.run[s] += eq;
          e.finish(s);
        }
      }
    }
    if (!WRITE) {
      int c[4];
#pragma unroll
      for (int s = 0; s < 4; ++s) c[s] = active && !skip ? (int)e.pos[s] : 0;
      reinterpret_cast<ushort4*>(a.row_bytes)[g * 32 + lane] =
          make_ushort4((unsigned short)c[0], (unsigned short)c[1], (unsigned short)c[2], (unsigned short)c[3]);
#pragma unroll
      for (int s = 0; s < 4; ++s) {
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) c[s] += __shfl_xor_sync(0xffffffffu, c[s], d);
      }
      if (lane == 0) reinterpret_cast<int4*>(a.group_tot)[g] = make_int4(c[0], c[1], c[2], c[3]);
      if (__any_sync(0xffffffffu, any_alpha != 0) && lane == 0 && a.alpha_any) a.alpha_any[i] = 1;
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
    if (write) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, psd_rle_kernel<true>, kRleWarps * 32, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, psd_rle_kernel<false>, kRleWarps * 32, 0);
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
  // Persistent grid: as many CTAs as are resident at once (the device's SMs x
  // the kernel's occupancy), so the grid-stride loop balances the row groups.
  const int resident = rle_resident_ctas(write);
  long long ctas = (G + kRleWarps - 1) / kRleWarps;
  if (ctas > resident) ctas = resident;
  if (write) psd_rle_kernel<true><<<(int)ctas, kRleWarps * 32, 0, st>>>(a);
  else psd_rle_kernel<false><<<(int)ctas, kRleWarps * 32, 0, st>>>(a);
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
