// Fused gradient chain + Adam + parameter clamp for image fitting.
//
// Replaces, in one launch, the reference optimiser step of
// pydiffbmp/core/renderer/simple_tile_renderer.py:961-968 (torch.optim.Adam
// with one parameter group per x, y, r, v, theta, c), :1125 (optimizer.step)
// and :1131 / :122-128 (_clamp_params_inplace: x in [0,W-1], y in [0,H-1],
// r in [2, min(H,W)//4]).  Gradients come as the raw per-primitive sums the
// raster kernels accumulate (see raster.cu finalize_kernel for the chain).
#include "dbmp_internal.cuh"

namespace dbmp {

__device__ __forceinline__ double sigmoid_dd(double x) {
  if (x >= 0.0) { const double z = exp(-x); return 1.0 / (1.0 + z); }
  const double z = exp(x);
  return z / (1.0 + z);
}

// One Adam update of parameter k of a primitive (torch.optim.Adam, single
// tensor form, in float32 like the reference's parameters): the step size
// lr_k * decay / (1 - beta1^t) and sqrt(1 - beta2^t) come precomputed.
__device__ __forceinline__ void adam_update(const AdamArgs& a, float step_size, float bc2s, float gk, float* m1,
                                            float* m2, float* p) {
  float mk = *m1, vk = *m2;
  mk = fmaf(1.f - a.beta1, gk - mk, mk);                 // exp_avg.lerp_(grad, 1-beta1)
  vk = fmaf(a.beta2, vk, (1.f - a.beta2) * gk * gk);     // exp_avg_sq.mul_(beta2).addcmul_(g, g, 1-beta2)
  *m1 = mk;
  *m2 = vk;
  const float denom = sqrtf(vk) / bc2s + a.eps;
  *p -= step_size * mk / denom;
}

// Work layout: the per-primitive chain and updates are split into three
// parameter groups, each run by whole warps over 32 consecutive primitives, so
// every warp takes one branch and a primitive's three groups run in parallel:
//   0: x, y        (sine and cosine of the rotation, 1/r, sigmoid(v))
//   1: r, theta, v (1/r, sigmoid(v))
//   2: the three colour logits (their sigmoids)
// A CTA holds the three group warps of kAdamBlocks blocks of 32 primitives
// (warp w: group w % 3, block w / 3).  Groups 0 and 1 both read r, theta and
// v, which group 1 updates, so every warp loads its inputs before a CTA
// barrier and updates after it.  The kernel is latency-bound (a few warps
// per SM at N = 20 K): splitting the chain shortens the longest thread.
constexpr int kAdamGroups = 3;
constexpr int kAdamBlocks = 2;
constexpr int kAdamThreads = 32 * kAdamGroups * kAdamBlocks;

__global__ void __launch_bounds__(kAdamThreads) adam_kernel(Geom g, AdamArgs a, const double* __restrict__ gacc,
                                                            float* __restrict__ means2D, float* __restrict__ radii,
                                                            float* __restrict__ rot, float* __restrict__ opac,
                                                            float* __restrict__ colors, float* __restrict__ m1,
                                                            float* __restrict__ m2, const int* __restrict__ step_count,
                                                            const int* __restrict__ skip_flag) {
  if (skip_flag != nullptr && *skip_flag != 0) return;
  // The step's scalars, once per CTA: thread k < 8 the step size of parameter
  // k, lr_k * gamma^(t-1) / (1 - beta1^t) in double as torch computes it
  // (torch.optim.lr_scheduler.ExponentialLR stepped after every optimizer
  // step, simple_tile_renderer.py:1128-1129), thread 8 sqrt(1 - beta2^t).
  __shared__ float s_step[8];
  __shared__ float s_bc2s;
  if (threadIdx.x < 9) {
    const int t = *step_count + 1;
    if (threadIdx.x < 8) {
      const double decay = a.gamma == 1.f ? 1.0 : pow((double)a.gamma, (double)(t - 1));
      const double bc1 = 1.0 - pow((double)a.beta1, (double)t);
      s_step[threadIdx.x] = (float)((double)a.lr[threadIdx.x] * decay / bc1);
    } else {
      s_bc2s = (float)sqrt(1.0 - pow((double)a.beta2, (double)t));
    }
  }
  const int warp = threadIdx.x >> 5;
  const int grp = warp % kAdamGroups;
  const int n = (blockIdx.x * kAdamBlocks + warp / kAdamGroups) * 32 + (threadIdx.x & 31);
  const bool live = n < g.N;
  // inputs of the chain, read before any warp of the CTA updates them
  float r = 0.f, th = 0.f, v = 0.f, c3[3] = {0.f, 0.f, 0.f};
  if (live) {
    if (grp == 2) {
#pragma unroll
      for (int ch = 0; ch < 3; ++ch) c3[ch] = colors[3 * n + ch];
    } else {
      r = radii[n];
      th = rot[n];
      v = opac[n];
    }
  }
  __syncthreads();
  if (!live) return;
  const float bc2s = s_bc2s;
  // gradient chain (as finalize_kernel): zero sums give zero gradients, also
  // for a non-finite rotation
  const double* S = gacc + (size_t)n * 8;
  float* M1 = m1 + (size_t)n * 8;
  float* M2 = m2 + (size_t)n * 8;
  if (grp == 2) {
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
      const double sc = sigmoid_dd((double)c3[ch]);
      const double gr = sc * (1.0 - sc) * S[4 + ch];
      adam_update(a, s_step[5 + ch], bc2s, (float)gr, M1 + 5 + ch, M2 + 5 + ch, colors + 3 * n + ch);
    }
    return;
  }
  const double sv = sigmoid_dd((double)v);
  const double a0 = (double)g.alpha_max * sv;
  const double rinv = (r > 1e-6f) ? 1.0 / (double)r : 1e6;
  if (grp == 0) {
    double s, c;
    sincos((double)th, &s, &c);
    const double hx = g.hx, hy = g.hy;
    const double cx = S[0] != 0.0 ? c * hx * S[0] : 0.0, sx = S[0] != 0.0 ? s * hx * S[0] : 0.0;
    const double cy = S[1] != 0.0 ? c * hy * S[1] : 0.0, sy = S[1] != 0.0 ? s * hy * S[1] : 0.0;
    const double gx = a0 * rinv * (sy - cx);
    const double gy = a0 * rinv * (-sx - cy);
    adam_update(a, s_step[0], bc2s, (float)gx, M1 + 0, M2 + 0, means2D + 2 * n);
    adam_update(a, s_step[1], bc2s, (float)gy, M1 + 1, M2 + 1, means2D + 2 * n + 1);
    if (a.clamp) {
      means2D[2 * n] = fminf(fmaxf(means2D[2 * n], 0.f), a.x_max);
      means2D[2 * n + 1] = fminf(fmaxf(means2D[2 * n + 1], 0.f), a.y_max);
    }
    return;
  }
  // grp == 1
  adam_update(a, s_step[2], bc2s, (float)(-a0 * rinv * S[2]), M1 + 2, M2 + 2, radii + n);
  adam_update(a, s_step[3], bc2s, (float)(a0 * S[3]), M1 + 3, M2 + 3, rot + n);
  adam_update(a, s_step[4], bc2s, (float)((1.0 - sv) * S[7]), M1 + 4, M2 + 4, opac + n);
  if (a.clamp) radii[n] = fminf(fmaxf(radii[n], a.r_min), a.r_max);
}

__global__ void step_increment_kernel(int* __restrict__ step_count, const int* __restrict__ skip_flag) {
  if (skip_flag != nullptr && *skip_flag != 0) return;
  *step_count += 1;
}

// ---------------------------------------------------------------------------
// Pruning (restart) of low-opacity primitives: the reference's do_prune
// (simple_tile_renderer.py:1007-1013 schedule, :1236-1270 selection and
// replacement) as one CTA.  Primitives with sigmoid(v) < threshold, in
// ascending index order, take consecutive rows of the replacement pool; a
// CTA-wide scan over chunks of kPruneThreads primitives gives each its rank.
constexpr int kPruneThreads = 1024;

__global__ void __launch_bounds__(kPruneThreads) prune_kernel(Geom g, PruneArgs a, const int* __restrict__ step_count,
                                                              const float* __restrict__ pool, int* __restrict__ state,
                                                              float* __restrict__ means2D, float* __restrict__ radii,
                                                              float* __restrict__ rot, float* __restrict__ opac,
                                                              float* __restrict__ colors,
                                                              const int* __restrict__ skip_flag) {
  __shared__ int s_warp[kPruneThreads / 32];
  __shared__ int s_total;
  if (skip_flag != nullptr && *skip_flag != 0) return;
  const int it = *step_count;
  // the reference's schedule (simple_tile_renderer.py:1007-1012); an iteration
  // replayed after an overflowed binning is not pruned a second time
  if (!(it != 0 && it % a.every == 0 && it < a.num_iterations - a.no_last && it > a.warmup) || state[1] == it)
    return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int base = state[0];
  int done = 0;
  for (int c = 0; c < g.N; c += kPruneThreads) {
    const int n = c + threadIdx.x;
    // torch.sigmoid in float32: 1 / (1 + exp(-v)); compared with the threshold as float32
    const bool low = n < g.N && (1.f / (1.f + expf(-opac[n]))) < a.threshold;
    const unsigned m = __ballot_sync(0xffffffffu, low);
    if (lane == 0) s_warp[warp] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
      int run = 0;
      for (int w = 0; w < kPruneThreads / 32; ++w) { const int v = s_warp[w]; s_warp[w] = run; run += v; }
      s_total = run;
    }
    __syncthreads();
    if (low) {
      const int rank = done + s_warp[warp] + __popc(m & ((1u << lane) - 1u));
      const float* r = pool + (size_t)((base + rank) % a.pool_rows) * 8;
      means2D[2 * n] = r[0];
      means2D[2 * n + 1] = r[1];
      radii[n] = r[2];
      rot[n] = r[3];
      opac[n] = r[4];
      colors[3 * n] = r[5];
      colors[3 * n + 1] = r[6];
      colors[3 * n + 2] = r[7];
    }
    done += s_total;
    __syncthreads();   // s_warp / s_total are rewritten by the next chunk
  }
  if (threadIdx.x == 0) {
    state[0] = (int)(((long long)base + done) % a.pool_rows);
    state[1] = it;
    state[2] = done;
    state[3] += done;
  }
}

int launch_prune(const Geom& g, const PruneArgs& a, const int* step_count, const float* pool, int* state,
                 float* means2D, float* radii, float* rot, float* opac, float* colors, const int* skip_flag,
                 cudaStream_t st) {
  if (g.N == 0) return DBMP_OK;
  prune_kernel<<<1, kPruneThreads, 0, st>>>(g, a, step_count, pool, state, means2D, radii, rot, opac, colors,
                                            skip_flag);
  DBMP_CHECK_LAUNCH("prune_kernel");
  return DBMP_OK;
}

int launch_adam(const Geom& g, const AdamArgs& a, const double* gacc, float* means2D, float* radii, float* rot,
                float* opac, float* colors, float* m1, float* m2, int* step_count, const int* skip_flag,
                cudaStream_t st) {
  if (g.N > 0) {
    const int ctas = (int)(((long long)g.N + 32 * kAdamBlocks - 1) / (32 * kAdamBlocks));
    adam_kernel<<<ctas, kAdamThreads, 0, st>>>(g, a, gacc, means2D, radii, rot, opac, colors, m1, m2, step_count,
                                               skip_flag);
    DBMP_CHECK_LAUNCH("adam_kernel");
  }
  step_increment_kernel<<<1, 1, 0, st>>>(step_count, skip_flag);
  DBMP_CHECK_LAUNCH("step_increment_kernel");
  return DBMP_OK;
}

}  // namespace dbmp
