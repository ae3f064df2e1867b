// dbmp_oracle.cpp -- TEST INFRASTRUCTURE, not product code.
//
// A CPU restatement of DiffBMP's tile-rasterizer algorithm (reference project
// smhongok/diffbmp), used only as the checker by tests/, by
// __graft_entry__.smoke() and by bench.py's cpu_baseline / reference legs.
// The product path (diffbmp_b200) never links or calls this file.
//
// Precision: every per-pixel quantity is computed in double.  Binning is the
// exception: the reference bins with float32 torch element-wise ops, so the
// binning restatement below rounds to float32 after every operation, in the
// reference's order, to reproduce its tile lists bit for bit.
//
// Two sampling semantics are provided, because the reference has two
// implementations of the same renderer that differ at the template edge:
//   SEM_KERNEL  -- the CUDA kernels (cuda_tile_rasterizer/cuda_kernels/
//                  tile_forward.cu:182-391, tile_backward.cu:127-407,
//                  tile_common.h:175-239): square cull, hard zero outside
//                  [0,W-1], mask clamped to [0,1], fragments with mask<=1e-6
//                  dropped.
//   SEM_TORCH   -- the PyTorch per-tile path (pydiffbmp/core/renderer/
//                  simple_tile_renderer.py:1413-1445 with _generate_tile_masks
//                  :1459-1550 and vector_renderer.py:706-736): F.grid_sample
//                  with zero padding and align_corners=True (partial weights
//                  on the one-texel border), no cull, no clamp, no skip.
//                  sigmoid(c_blend) is taken as 0 (callers use c_blend<=-40).
// SEM_TORCH exists so that golden vectors produced by running the reference's
// Python code pin the shared geometry / compositing / gradient chain; the
// kernel-only differences are pinned by known-answer tests and by the
// reference's own CUDA kernels run on the GPU.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>
#include <atomic>
#include <thread>

namespace {

enum { SEM_KERNEL = 0, SEM_TORCH = 1 };

struct Scene {
  int H, W, ts;
  int N, P, Ht, Wt;
  const double* means2D;  // (N,2)
  const double* radii;    // (N)
  const double* rot;      // (N)
  const double* opac;     // (N) logits
  const double* colors;   // (N,3) logits
  const double* tmpl;     // (P,Ht,Wt)
  const int* sel;         // (N)
  double amax;
  int sem;
  double t_stop;          // 0 disables early termination (reference behaviour)
  double edge;            // boundary shift: > 0 widens the cull and the texel cut
                          // by `edge` (pixels / texels), < 0 narrows them, and
                          // the bilinear cell choice moves by 2 float32 ulps; tests
                          // use +-edge renders to find boundary-sensitive pixels
  const double* cmap = nullptr;   // (N,Ht,Wt,3) colour maps (colors_orig), or null
  double cblend = 0.0;            // colour-map blend weight (used when cmap && cblend > 0)
};

inline double sigmoid_d(double x) {
  // tile_common.h:125-133 (branch-stable form; exact in double either way)
  if (x >= 0) { double z = std::exp(-x); return 1.0 / (1.0 + z); }
  double z = std::exp(x);
  return z / (1.0 + z);
}

// Bilinear sample of one template at texel coordinate (x, y); value and
// d/dx, d/dy.  tile_common.h:201-239 (kernel) / F.grid_sample zeros+align_corners (torch).
inline double sample_tmpl(const double* t, int Ht, int Wt, double x, double y,
                          bool hard_cut, double* gx, double* gy, double edge = 0.0) {
  if (hard_cut) {
    if (x < -edge || x > (double)(Wt - 1) + edge || y < -edge || y > (double)(Ht - 1) + edge) {
      if (gx) { *gx = 0; *gy = 0; }
      return 0.0;
    }
  }
  // The bilinear cell is the one left of / above (x, y); its gradient jumps
  // across texel grid lines (the value does not), and a float32 texel
  // coordinate within its rounding of a line can fall on either side.  The
  // +-edge band runs therefore also move the cell choice by two float32 ulps
  // of the coordinate, so that both one-sided gradients of such points
  // appear in the band's spread.
  auto cell_shift = [&](double v) {
    if (edge == 0.0 || !std::isfinite(v)) return 0.0;
    const double ulp = std::ldexp(1.0, std::max(std::ilogb(std::max(std::fabs(v), 1.0)), -126) - 23);
    return std::copysign(2.0 * ulp, edge);
  };
  double fx = std::floor(x + cell_shift(x)), fy = std::floor(y + cell_shift(y));
  if (!std::isfinite(fx) || !std::isfinite(fy) || fx < -2.0 || fy < -2.0 ||
      fx > (double)Wt + 1.0 || fy > (double)Ht + 1.0) {
    if (gx) { *gx = 0; *gy = 0; }
    return 0.0;
  }
  int x0 = (int)fx, y0 = (int)fy;
  if (hard_cut) {  // reference clamps the base index (a no-op inside the cut)
    x0 = std::max(0, std::min(x0, Wt - 1));
    y0 = std::max(0, std::min(y0, Ht - 1));
  }
  double wx = x - x0, wy = y - y0;
  auto in = [&](int yy, int xx) { return xx >= 0 && xx < Wt && yy >= 0 && yy < Ht; };
  auto at = [&](int yy, int xx) { return in(yy, xx) ? (double)t[(size_t)yy * Wt + xx] : 0.0; };
  double v00 = at(y0, x0), v01 = at(y0, x0 + 1), v10 = at(y0 + 1, x0), v11 = at(y0 + 1, x0 + 1);
  double f = v00 * (1 - wx) * (1 - wy) + v01 * wx * (1 - wy) + v10 * (1 - wx) * wy + v11 * wx * wy;
  if (gx) {
    *gx = (v01 - v00) * (1 - wy) + (v11 - v10) * wy;
    *gy = (v10 - v00) * (1 - wx) + (v11 - v01) * wx;
  }
  return f;
}

// Colour map sample at texel coordinate (x, y), tile_forward.cu:17-89: the
// coordinate is clamped into the map, neighbours past the last row / column
// repeat it (not zero), bilinear weights.
inline void sample_cmap(const double* cm, int Ht, int Wt, double x, double y, double out[3]) {
  const double cx = std::max(0.0, std::min((double)(Wt - 1), x));
  const double cy = std::max(0.0, std::min((double)(Ht - 1), y));
  const int x0 = (int)cx, y0 = (int)cy;
  const int x1 = std::min(x0 + 1, Wt - 1), y1 = std::min(y0 + 1, Ht - 1);
  const double fx = cx - x0, fy = cy - y0;
  for (int ch = 0; ch < 3; ++ch) {
    const double c00 = cm[3 * ((size_t)y0 * Wt + x0) + ch], c10 = cm[3 * ((size_t)y0 * Wt + x1) + ch];
    const double c01 = cm[3 * ((size_t)y1 * Wt + x0) + ch], c11 = cm[3 * ((size_t)y1 * Wt + x1) + ch];
    const double c0 = c00 * (1 - fx) + c10 * fx, c1 = c01 * (1 - fx) + c11 * fx;
    out[ch] = c0 * (1 - fy) + c1 * fy;
  }
}

struct Frag {
  int n;            // primitive id
  double a;         // alpha
  double c[3];      // colour in [0,1] (blended with the colour map when enabled)
  double sc[3];     // sigmoid of the colour logits
  double m;         // mask
  double gx, gy;    // d mask / d texel coordinate
  double ex, ey;    // texel coordinate minus template half extent
  double T;         // transmittance entering this fragment
  double u, v;      // normalised template coordinates
  double cs, sn, rinv, sop;
};

// Evaluates one (pixel, primitive) pair.  Returns false when the pair yields
// no fragment.  tile_forward.cu:188-284 (kernel) / simple_tile_renderer.py:1413-1436 (torch).
inline bool eval_pair(const Scene& s, int n, int px, int py, Frag* f, bool* culled) {
  *culled = true;
  if (n < 0 || n >= s.N) return false;
  const double mx = s.means2D[2 * n], my = s.means2D[2 * n + 1];
  const double r = s.radii[n];
  const double dx = (double)px - mx, dy = (double)py - my;
  const int tid = s.sel[n];
  const bool valid = tid >= 0 && tid < s.P;
  if (s.sem == SEM_KERNEL) {
    if (valid) {
      const double maxd = std::max(s.Wt, s.Ht);
      const double scale = r / (maxd * 0.5);
      const double hw = s.Wt * 0.5 * scale, hh = s.Ht * 0.5 * scale;
      if (std::fabs(dx) > hw + s.edge || std::fabs(dy) > hh + s.edge) return false;
    } else {
      if (dx * dx + dy * dy > r * r) return false;
    }
  }
  *culled = false;
  if (!valid) return false;  // mask stays 0 -> no fragment
  double rinv = (s.sem == SEM_KERNEL) ? (r > 1e-6 ? 1.0 / r : 1e6) : 1.0 / r;
  const double phi = s.rot[n];
  const double cs = std::cos(phi), sn = std::sin(phi);
  const double ndx = dx * rinv, ndy = dy * rinv;
  const double u = cs * ndx + sn * ndy;
  const double v = -sn * ndx + cs * ndy;
  const double hx = 0.5 * (s.Wt - 1), hy = 0.5 * (s.Ht - 1);
  const double tx = (u + 1.0) * hx, ty = (v + 1.0) * hy;
  double gx = 0, gy = 0;
  const double* t = s.tmpl + (size_t)tid * s.Ht * s.Wt;
  double m = sample_tmpl(t, s.Ht, s.Wt, tx, ty, s.sem == SEM_KERNEL, &gx, &gy, s.edge);
  if (s.sem == SEM_KERNEL) {
    m = std::max(0.0, std::min(1.0, m));
    if (m <= 1e-6) return false;
  }
  const double sop = sigmoid_d(s.opac[n]);
  f->n = n;
  f->m = m;
  f->a = s.amax * sop * m;
  for (int ch = 0; ch < 3; ++ch) f->sc[ch] = f->c[ch] = sigmoid_d(s.colors[3 * n + ch]);
  if (s.sem == SEM_KERNEL && s.cmap != nullptr && s.cblend > 0.0) {
    // tile_forward.cu:316-330: (1 - c_blend) sigmoid(c) + c_blend c_o(x, y)
    double co[3];
    sample_cmap(s.cmap + (size_t)n * s.Ht * s.Wt * 3, s.Ht, s.Wt, tx, ty, co);
    for (int ch = 0; ch < 3; ++ch) f->c[ch] = (1.0 - s.cblend) * f->sc[ch] + s.cblend * co[ch];
  }
  f->gx = gx; f->gy = gy;
  f->ex = tx - hx; f->ey = ty - hy;
  f->u = u; f->v = v; f->cs = cs; f->sn = sn; f->rinv = rinv; f->sop = sop;
  return true;
}

struct PixStats {
  long long cand, frag, live;
  int depth;
};

// Walks one pixel's tile list front to back.  Fills frags (if non-null) with
// the fragments up to and including the last contributor.  tile_forward.cu:182-397.
inline void walk_pixel(const Scene& s, const int* list, int K, int px, int py,
                       double* C, double* Tfinal, double* Tlast, int* lastpos,
                       std::vector<Frag>* frags, std::vector<int>* fragpos, PixStats* st) {
  double T = 1.0;
  C[0] = C[1] = C[2] = 0.0;
  *Tlast = 1.0;
  *lastpos = -1;
  bool done = false;
  for (int kk = 0; kk < K; ++kk) {
    Frag f;
    bool culled;
    bool ok = eval_pair(s, list[kk], px, py, &f, &culled);
    if (!culled && st) st->cand++;
    if (!ok) continue;
    if (st) { st->frag++; st->depth++; }
    if (done) continue;  // counting only: past the termination point
    if (st) st->live++;
    f.T = T;
    for (int ch = 0; ch < 3; ++ch) C[ch] += T * f.a * f.c[ch];
    *Tlast = T;
    *lastpos = kk;
    if (frags) { frags->push_back(f); fragpos->push_back(kk); }
    if (s.sem == SEM_KERNEL) T *= std::max(1.0 - f.a, 0.0);
    else T *= (1.0 - f.a);
    if (s.t_stop > 0.0 && T < s.t_stop) {
      done = true;
      if (!st) break;
    }
  }
  *Tfinal = T;
}

// Runs fn(row, worker) for row in [0, rows) on `nthreads` host threads with
// dynamic row assignment.
template <class F>
void parallel_rows(int rows, int nthreads, F fn) {
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  nthreads = std::max(1, std::min(nthreads, rows));
  std::atomic<int> next{0};
  auto work = [&](int w) {
    for (int r = next.fetch_add(1); r < rows; r = next.fetch_add(1)) fn(r, w);
  };
  if (nthreads == 1) { work(0); return; }
  std::vector<std::thread> th;
  for (int w = 0; w < nthreads; ++w) th.emplace_back(work, w);
  for (auto& t : th) t.join();
}

inline int resolve_threads(int nthreads, int rows) {
  if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
  return std::max(1, std::min(nthreads, rows));
}

inline int tiles_x(const Scene& s) { return (s.W + s.ts - 1) / s.ts; }
inline int tiles_y(const Scene& s) { return (s.H + s.ts - 1) / s.ts; }

// ---------------------------------------------------------------------------
// float32 helpers for the bit-exact binning restatement
inline float nan_min(float a, float b) { return (std::isnan(a) || std::isnan(b)) ? std::numeric_limits<float>::quiet_NaN() : (a < b ? a : b); }
inline float nan_max(float a, float b) { return (std::isnan(a) || std::isnan(b)) ? std::numeric_limits<float>::quiet_NaN() : (a > b ? a : b); }

}  // namespace

extern "C" {

int orc_version() { return 3; }

// vector_renderer.py:151-192 _compute_primitive_bboxes: per template the
// bbox of texels > 1e-6 in normalised coordinates, float32 arithmetic.
int orc_template_bboxes(const float* S, int P, int Ht, int Wt, float* out4) {
  for (int p = 0; p < P; ++p) {
    const float* t = S + (size_t)p * Ht * Wt;
    bool any = false;
    float mnu = 0, mxu = 0, mnv = 0, mxv = 0;
    for (int yy = 0; yy < Ht; ++yy)
      for (int xx = 0; xx < Wt; ++xx) {
        if (!(t[(size_t)yy * Wt + xx] > 1e-6f)) continue;
        volatile float qu = (float)xx / (float)(Wt - 1);
        volatile float un = qu * 2.0f;
        volatile float u = un - 1.0f;
        volatile float qv = (float)yy / (float)(Ht - 1);
        volatile float vn = qv * 2.0f;
        volatile float v = vn - 1.0f;
        if (!any) { mnu = mxu = u; mnv = mxv = v; any = true; }
        mnu = std::min(mnu, (float)u); mxu = std::max(mxu, (float)u);
        mnv = std::min(mnv, (float)v); mxv = std::max(mxv, (float)v);
      }
    if (!any) { mnu = -1; mxu = 1; mnv = -1; mxv = 1; }
    out4[4 * p + 0] = mnu; out4[4 * p + 1] = mxu; out4[4 * p + 2] = mnv; out4[4 * p + 3] = mxv;
  }
  return 0;
}

// vector_renderer.py:194-252 _compute_primitive_world_bboxes in float32 with
// one rounding per torch op.  cos/sin are the correctly rounded float values.
int orc_world_bboxes(const float* means2D, const float* radii, const float* rot,
                     const int* bbox_sel, const float* tbbox, int N, int P, float* out4) {
  for (int n = 0; n < N; ++n) {
    const int q = bbox_sel[n];
    if (q < 0 || q >= P) return -1;
    const float x = means2D[2 * n], y = means2D[2 * n + 1], r = radii[n], th = rot[n];
    const float c = (float)std::cos((double)th), s = (float)std::sin((double)th);
    const float cu[4] = {tbbox[4 * q + 0], tbbox[4 * q + 1], tbbox[4 * q + 0], tbbox[4 * q + 1]};
    const float cv[4] = {tbbox[4 * q + 2], tbbox[4 * q + 2], tbbox[4 * q + 3], tbbox[4 * q + 3]};
    float xmn = 0, xmx = 0, ymn = 0, ymx = 0;
    for (int k = 0; k < 4; ++k) {
      volatile float a1 = cu[k] * c, a2 = cv[k] * s, a3 = a1 - a2, a4 = r * a3, wx = x + a4;
      volatile float b1 = cu[k] * s, b2 = cv[k] * c, b3 = b1 + b2, b4 = r * b3, wy = y + b4;
      if (k == 0) { xmn = xmx = wx; ymn = ymx = wy; }
      else { xmn = nan_min(xmn, wx); xmx = nan_max(xmx, wx); ymn = nan_min(ymn, wy); ymx = nan_max(ymx, wy); }
    }
    out4[4 * n + 0] = xmn; out4[4 * n + 1] = xmx; out4[4 * n + 2] = ymn; out4[4 * n + 3] = ymx;
  }
  return 0;
}

// Tile lists.  mode 0 (and 2, with the reference's bbox template choice):
// vector_renderer.py:401-444 _unified_primitive_assignment
// (world-bbox vs tile bounds, inclusive, float32 compare) followed by
// simple_tile_renderer.py:721-766 _convert_masks_to_mapping (tiles row-major,
// ascending primitive id).  mode 1: a tile holds a primitive iff some pixel of
// the tile passes the kernel's square cull (tile_forward.cu:194-210), i.e. the
// tight form of the reference's default all-primitives mapping
// (tile_rasterize.cu:171-194).  Writes offsets (T+1) and, if indices is
// non-null and cap is large enough, the indices.  Returns total L.
long long orc_bin(int H, int W, int ts, const float* means2D, const float* radii, const float* rot,
                  const int* sel, const float* tbbox, int N, int P, int Ht, int Wt, int mode,
                  int* offsets, int* indices, long long cap) {
  const int tX = (W + ts - 1) / ts, tY = (H + ts - 1) / ts, T = tX * tY;
  std::vector<float> wb((size_t)N * 4);
  std::vector<int> bsel(sel, sel + N);
  if (mode != 1) {
    // mode 2: the bbox template of primitive n is (N-1-n) % P whatever sel
    // says, as vector_renderer.py:220-226 takes it
    for (int n = 0; n < N; ++n) {
      if (mode == 2) bsel[n] = (N - 1 - n) % P;
      else if (bsel[n] < 0 || bsel[n] >= P) bsel[n] = 0;
    }
    orc_world_bboxes(means2D, radii, rot, bsel.data(), tbbox, N, P, wb.data());
  }
  // per-primitive tile-column / tile-row predicate
  auto colhit = [&](int n, int tx) -> bool {
    if (mode != 1) {
      const float xs = (float)(tx * ts), xe = (float)std::min(tx * ts + ts, W);
      return !((wb[4 * n + 1] < xs) || (wb[4 * n + 0] > xe));
    }
    const int q = sel[n];
    if (q < 0 || q >= P) return false;
    const float mx = means2D[2 * n], r = radii[n];
    const float maxd = (float)std::max(Wt, Ht);
    const float scale = r / (maxd * 0.5f);
    const float hw = ((float)Wt * 0.5f) * scale;
    const int a = tx * ts, b = std::min(tx * ts + ts, W) - 1;
    for (int px = a; px <= b; ++px) { volatile float d = (float)px - mx; if (!(std::fabs((float)d) > hw)) return true; }
    return false;
  };
  auto rowhit = [&](int n, int ty) -> bool {
    if (mode != 1) {
      const float ys = (float)(ty * ts), ye = (float)std::min(ty * ts + ts, H);
      return !((wb[4 * n + 3] < ys) || (wb[4 * n + 2] > ye));
    }
    const int q = sel[n];
    if (q < 0 || q >= P) return false;
    const float my = means2D[2 * n + 1], r = radii[n];
    const float maxd = (float)std::max(Wt, Ht);
    const float scale = r / (maxd * 0.5f);
    const float hh = ((float)Ht * 0.5f) * scale;
    const int a = ty * ts, b = std::min(ty * ts + ts, H) - 1;
    for (int py = a; py <= b; ++py) { volatile float d = (float)py - my; if (!(std::fabs((float)d) > hh)) return true; }
    return false;
  };
  std::vector<std::vector<char>> colm((size_t)N, std::vector<char>(tX)), rowm((size_t)N, std::vector<char>(tY));
  for (int n = 0; n < N; ++n) {
    for (int tx = 0; tx < tX; ++tx) colm[n][tx] = colhit(n, tx);
    for (int ty = 0; ty < tY; ++ty) rowm[n][ty] = rowhit(n, ty);
  }
  long long L = 0;
  offsets[0] = 0;
  for (int t = 0; t < T; ++t) {
    const int tx = t % tX, ty = t / tX;
    for (int n = 0; n < N; ++n) {
      if (colm[n][tx] && rowm[n][ty]) {
        if (indices && L < cap) indices[L] = n;
        ++L;
      }
    }
    offsets[t + 1] = (int)L;
  }
  return L;
}

// Forward render.  out_color (H,W,3) and out_alpha (H,W) in double; per pixel
// the transmittance entering the last contributor and its list position;
// stats[0..4] = candidates (pairs passing the cull), fragments, live
// fragments (walked before termination), max depth, list entries walked.
int orc_forward_cmap(int H, int W, int ts, int N, const double* means2D, const double* radii, const double* rot,
                     const double* opac, const double* colors, int P, int Ht, int Wt, const double* tmpl,
                     const int* sel, double amax, int sem, double t_stop, double edge,
                     const int* offsets, const int* indices,
                     double* out_color, double* out_alpha, double* T_last, int* last_pos, long long* stats,
                     int nthreads, const double* cmap, double cblend) {
  Scene s{H, W, ts, N, P, Ht, Wt, means2D, radii, rot, opac, colors, tmpl, sel, amax, sem, t_stop, edge};
  s.cmap = cmap;
  s.cblend = cblend;
  const int tX = tiles_x(s);
  const int nt = resolve_threads(nthreads, H);
  std::vector<long long> wc(nt, 0), wf(nt, 0), wl(nt, 0);
  std::vector<int> wd(nt, 0);
  parallel_rows(H, nt, [&](int py, int w) {
    long long& cand = wc[w]; long long& frag = wf[w]; long long& live = wl[w]; int& maxdepth = wd[w];
    for (int px = 0; px < W; ++px) {
      const int t = (py / ts) * tX + (px / ts);
      const int* list = indices + offsets[t];
      const int K = offsets[t + 1] - offsets[t];
      double C[3], Tf, Tl;
      int lp;
      PixStats st{0, 0, 0, 0};
      walk_pixel(s, list, K, px, py, C, &Tf, &Tl, &lp, nullptr, nullptr, &st);
      const size_t p = (size_t)py * W + px;
      for (int ch = 0; ch < 3; ++ch) out_color[3 * p + ch] = C[ch];
      out_alpha[p] = 1.0 - Tf;
      if (T_last) T_last[p] = Tl;
      if (last_pos) last_pos[p] = lp;
      cand += st.cand; frag += st.frag; live += st.live;
      maxdepth = std::max(maxdepth, st.depth);
    }
  });
  long long cand = 0, frag = 0, live = 0;
  int maxdepth = 0;
  for (int w = 0; w < nt; ++w) { cand += wc[w]; frag += wf[w]; live += wl[w]; maxdepth = std::max(maxdepth, wd[w]); }
  if (stats) { stats[0] = cand; stats[1] = frag; stats[2] = live; stats[3] = maxdepth; }
  return 0;
}

// Backward.  grads (N,8) in double, order: d means.x, d means.y, d radius,
// d rotation, d opacity-logit, d colour-logit r, g, b.
// SEM_KERNEL follows tile_backward.cu:212-343 literally (suffix S, back
// product B, 1/max(1-a,1e-6)); SEM_TORCH is the exact derivative of the
// torch composite (autograd through cumprod / grid_sample).
int orc_backward_cmap(int H, int W, int ts, int N, const double* means2D, const double* radii, const double* rot,
                      const double* opac, const double* colors, int P, int Ht, int Wt, const double* tmpl,
                      const int* sel, double amax, int sem, double t_stop, double edge,
                      const int* offsets, const int* indices,
                      const float* grad_color, const float* grad_alpha, double* grads, int nthreads,
                      const double* cmap, double cblend) {
  Scene s{H, W, ts, N, P, Ht, Wt, means2D, radii, rot, opac, colors, tmpl, sel, amax, sem, t_stop, edge};
  s.cmap = cmap;
  s.cblend = cblend;
  const int tX = tiles_x(s);
  const double hx = 0.5 * (Wt - 1), hy = 0.5 * (Ht - 1);
  const int nt = resolve_threads(nthreads, H);
  std::vector<std::vector<double>> acc(nt, std::vector<double>((size_t)N * 8, 0.0));
  parallel_rows(H, nt, [&](int py, int tid) {
    double* g = acc[tid].data();
    std::vector<Frag> fr;
    std::vector<int> fp;
    for (int px = 0; px < W; ++px) {
      const int t = (py / ts) * tX + (px / ts);
      const int* list = indices + offsets[t];
      const int K = offsets[t + 1] - offsets[t];
      fr.clear(); fp.clear();
      double C[3], Tf, Tl;
      int lp;
      walk_pixel(s, list, K, px, py, C, &Tf, &Tl, &lp, &fr, &fp, nullptr);
      const size_t p = (size_t)py * W + px;
      const double gC[3] = {grad_color[3 * p], grad_color[3 * p + 1], grad_color[3 * p + 2]};
      const double gA = grad_alpha ? grad_alpha[p] : 0.0;
      const int nf = (int)fr.size();
      // suffix quantities, walked back to front
      double S[3] = {0, 0, 0}, B = 1.0, R[3] = {0, 0, 0};
      for (int k = nf - 1; k >= 0; --k) {
        const Frag& f = fr[k];
        const int n = f.n;
        double* gn = g + (size_t)n * 8;
        double dLda;
        if (sem == SEM_KERNEL) {
          const double inv1m = 1.0 / std::max(1.0 - f.a, 1e-6);
          dLda = 0;
          for (int ch = 0; ch < 3; ++ch) dLda += gC[ch] * (f.T * f.c[ch] - S[ch] * inv1m);
          dLda += gA * (f.T * B);
        } else {
          dLda = 0;
          for (int ch = 0; ch < 3; ++ch) dLda += gC[ch] * (f.c[ch] - R[ch]);
          dLda += gA * B;
          dLda *= f.T;
        }
        // colour logits: gC a T sigma'(c), without a (1 - c_blend) factor, as
        // the reference computes it (tile_backward.cu:254-262); the colour
        // map's dependence on the geometry is not differentiated there either
        for (int ch = 0; ch < 3; ++ch) gn[5 + ch] += gC[ch] * f.a * f.T * f.sc[ch] * (1.0 - f.sc[ch]);
        const double sop = f.sop;
        gn[4] += dLda * amax * f.m * sop * (1.0 - sop);
        const double dLdm = dLda * amax * sop;
        const double dLdu = dLdm * f.gx * hx, dLdv = dLdm * f.gy * hy;
        const double c = f.cs, sn = f.sn, ir = f.rinv;
        gn[0] += dLdu * (-c * ir) + dLdv * (sn * ir);
        gn[1] += dLdu * (-sn * ir) + dLdv * (-c * ir);
        gn[2] += dLdu * (-f.u * ir) + dLdv * (-f.v * ir);
        gn[3] += dLdu * f.v + dLdv * (-f.u);
        // advance the suffix state past fragment k
        for (int ch = 0; ch < 3; ++ch) {
          S[ch] += f.c[ch] * f.a * f.T;
          R[ch] = f.c[ch] * f.a + (1.0 - f.a) * R[ch];
        }
        B *= (sem == SEM_KERNEL) ? std::max(1.0 - f.a, 0.0) : (1.0 - f.a);
      }
    }
  });
  for (size_t i = 0; i < (size_t)N * 8; ++i) {
    double v = 0;
    for (int t = 0; t < nt; ++t) v += acc[t][i];
    grads[i] = v;
  }
  return 0;
}

// PSD stage 1 (psd_export_kernels.cu:12-55), float32 arithmetic.
int orc_forward(int H, int W, int ts, int N, const double* means2D, const double* radii, const double* rot,
                const double* opac, const double* colors, int P, int Ht, int Wt, const double* tmpl,
                const int* sel, double amax, int sem, double t_stop, double edge,
                const int* offsets, const int* indices,
                double* out_color, double* out_alpha, double* T_last, int* last_pos, long long* stats,
                int nthreads) {
  return orc_forward_cmap(H, W, ts, N, means2D, radii, rot, opac, colors, P, Ht, Wt, tmpl, sel, amax, sem, t_stop,
                          edge, offsets, indices, out_color, out_alpha, T_last, last_pos, stats, nthreads, nullptr,
                          0.0);
}

int orc_backward(int H, int W, int ts, int N, const double* means2D, const double* radii, const double* rot,
                 const double* opac, const double* colors, int P, int Ht, int Wt, const double* tmpl,
                 const int* sel, double amax, int sem, double t_stop, double edge,
                 const int* offsets, const int* indices,
                 const float* grad_color, const float* grad_alpha, double* grads, int nthreads) {
  return orc_backward_cmap(H, W, ts, N, means2D, radii, rot, opac, colors, P, Ht, Wt, tmpl, sel, amax, sem, t_stop,
                           edge, offsets, indices, grad_color, grad_alpha, grads, nthreads, nullptr, 0.0);
}

int orc_psd_bboxes(const float* means2D, const float* radii, int N, int H, int W, float scale,
                   int* bbox, int* sizes) {
  for (int n = 0; n < N; ++n) {
    volatile float x = means2D[2 * n] * scale;
    volatile float y = means2D[2 * n + 1] * scale;
    volatile float r = radii[n] * scale;
    volatile float tr = r * 1.5f;
    volatile float x0f = x - tr, y0f = y - tr, x1f = x + tr, y1f = y + tr;
    int mnx = std::max(0, (int)std::floor((float)x0f));
    int mny = std::max(0, (int)std::floor((float)y0f));
    int mxx = std::min(W, (int)std::ceil((float)x1f));
    int mxy = std::min(H, (int)std::ceil((float)y1f));
    if (mxx <= mnx || mxy <= mny) {
      bbox[4 * n] = 0; bbox[4 * n + 1] = 0; bbox[4 * n + 2] = 1; bbox[4 * n + 3] = 1;
      sizes[2 * n] = 1; sizes[2 * n + 1] = 1;
    } else {
      bbox[4 * n] = mnx; bbox[4 * n + 1] = mny; bbox[4 * n + 2] = mxx; bbox[4 * n + 3] = mxy;
      sizes[2 * n] = mxx - mnx; sizes[2 * n + 1] = mxy - mny;
    }
  }
  return 0;
}

// PSD stage 2 (psd_export_kernels.cu:61-198, psd_export_common.h:55-121) in
// double.  colors/visibility are already sigmoid-ed.  `ambiguous` (same size
// as out, may be null) marks bytes whose value depends on float rounding:
// truncation within 0.05 of an integer step, the 0.001 alpha threshold, or a
// texel coordinate within 1e-3 of the sampling cut.
int orc_psd_layers(const float* means2D, const float* radii, const float* rot, const float* colors,
                   const float* vis, int P, int Ht, int Wt, const float* tmpl, const int* sel,
                   const int* bbox, const long long* offs, int N, float scale, float amax,
                   uint8_t* out, uint8_t* ambiguous) {
  const double hx = 0.5 * (Wt - 1), hy = 0.5 * (Ht - 1);
  for (int n = 0; n < N; ++n) {
    const int l = bbox[4 * n], t = bbox[4 * n + 1], rr = bbox[4 * n + 2], b = bbox[4 * n + 3];
    const int bw = rr - l;
    const double x = (double)means2D[2 * n] * scale, y = (double)means2D[2 * n + 1] * scale;
    const double r = (double)radii[n] * scale, th = rot[n];
    const double cs = std::cos(th), sn = std::sin(th);
    const int q = sel[n];
    for (int py = t; py < b; ++py)
      for (int px = l; px < rr; ++px) {
        const double un = (px - x) / r, vn = (py - y) / r;
        const double ur = cs * un + sn * vn, vr = -sn * un + cs * vn;
        const double ut = (ur + 1.0) * hx, vt = (vr + 1.0) * hy;
        double tv = 0.0;
        bool amb = false;
        if (std::fabs(ut) < 1e-3 || std::fabs(ut - (Wt - 1)) < 1e-3 || std::fabs(vt) < 1e-3 ||
            std::fabs(vt - (Ht - 1)) < 1e-3)
          amb = true;
        if (!(ut < 0.0 || ut >= Wt - 1 || vt < 0.0 || vt >= Ht - 1) && q >= 0 && q < P) {
          const float* tp = tmpl + (size_t)q * Ht * Wt;
          int u0 = (int)std::floor(ut), v0 = (int)std::floor(vt);
          u0 = std::max(0, std::min(u0, Wt - 1));
          v0 = std::max(0, std::min(v0, Ht - 1));
          const double wu = ut - u0, wv = vt - v0;
          tv = (1 - wu) * (1 - wv) * tp[(size_t)v0 * Wt + u0] + wu * (1 - wv) * tp[(size_t)v0 * Wt + u0 + 1] +
               (1 - wu) * wv * tp[(size_t)(v0 + 1) * Wt + u0] + wu * wv * tp[(size_t)(v0 + 1) * Wt + u0 + 1];
        }
        const double av = tv * vis[n] * amax;
        const size_t o = (size_t)offs[n] + ((size_t)(py - t) * bw + (px - l)) * 4;
        auto near_step = [](double v) {
          const double s = std::min(255.0, std::max(0.0, v * 255.0));
          return std::fabs(s - std::round(s)) < 0.05 && s > 0.5;
        };
        if (std::fabs(av - 0.001) < 1e-5) amb = true;
        if (av < 0.001) {
          out[o] = out[o + 1] = out[o + 2] = out[o + 3] = 0;
          if (ambiguous) for (int k = 0; k < 4; ++k) ambiguous[o + k] = amb;
          continue;
        }
        const double mask = tv > 0.0 ? 1.0 : 0.0;
        for (int ch = 0; ch < 3; ++ch) {
          const double v = mask * colors[3 * n + ch];
          out[o + ch] = (uint8_t)std::max(0.0, std::min(255.0, v * 255.0));
          if (ambiguous) ambiguous[o + ch] = amb || near_step(v);
        }
        out[o + 3] = (uint8_t)std::max(0.0, std::min(255.0, av * 255.0));
        if (ambiguous) ambiguous[o + 3] = amb || near_step(av);
      }
  }
  return 0;
}

// PackBits encoding of `rows` rows of `w` bytes: byte x of row y is
// src[y * row_pitch + x * stride], so one channel of an interleaved RGBA image
// is encoded in place.  Same rule as packbits_encode in oracle/psd_file.py
// (runs of >= 3 equal bytes -> replicate packets of <= 128 bytes, a one-byte
// remainder -> a one-byte literal; shorter runs gathered into literal packets
// of <= 128 bytes).  Writes the encodings back to back into out and each
// row's size into row_bytes; returns the total, or -1 if out_cap is too small.
long long orc_packbits_rows(const uint8_t* src, int rows, int w, long long row_pitch, int stride, uint8_t* out,
                            long long out_cap, int32_t* row_bytes) {
  long long pos = 0;
  auto put = [&](uint8_t v) { if (pos < out_cap) out[pos] = v; ++pos; };
  for (int y = 0; y < rows; ++y) {
    const uint8_t* r = src + (long long)y * row_pitch;
    const long long start = pos;
    int lit_start = 0, lit = 0;
    auto flush = [&]() {
      for (int k = 0; k < lit; k += 128) {
        const int n = std::min(128, lit - k);
        put((uint8_t)(n - 1));
        for (int j = 0; j < n; ++j) put(r[(long long)(lit_start + k + j) * stride]);
      }
      lit = 0;
    };
    int x = 0;
    while (x < w) {
      const uint8_t v = r[(long long)x * stride];
      int e = x + 1;
      while (e < w && r[(long long)e * stride] == v) ++e;
      const int L = e - x;
      if (L >= 3) {
        flush();
        for (int rem = L; rem > 0; rem -= 128) {
          const int k = std::min(rem, 128);
          put(k >= 2 ? (uint8_t)(1 - k) : (uint8_t)0);
          put(v);
        }
        lit_start = e;
      } else {
        if (lit == 0) lit_start = x;
        lit += L;
      }
      x = e;
    }
    flush();
    row_bytes[y] = (int32_t)(pos - start);
  }
  return pos <= out_cap ? pos : -1;
}

}  // extern "C"
