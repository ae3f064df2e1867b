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

__global__ void adam_kernel(Geom g, AdamArgs a, const double* __restrict__ gacc, float* __restrict__ means2D,
                            float* __restrict__ radii, float* __restrict__ rot, float* __restrict__ opac,
                            float* __restrict__ colors, float* __restrict__ m1, float* __restrict__ m2,
                            const int* __restrict__ step_count, const int* __restrict__ skip_flag) {
  if (skip_flag != nullptr && *skip_flag != 0) return;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= g.N) return;
  const int t = *step_count + 1;
  // torch.optim.lr_scheduler.ExponentialLR stepped after every optimizer step:
  // the t-th step runs with lr * gamma^(t-1) (simple_tile_renderer.py:1128-1129)
  const double decay = a.gamma == 1.f ? 1.0 : pow((double)a.gamma, (double)(t - 1));
  const double bc1 = 1.0 - pow((double)a.beta1, (double)t);
  const double bc2s = sqrt(1.0 - pow((double)a.beta2, (double)t));
  // gradient chain (same as finalize_kernel)
  const double* S = gacc + (size_t)n * 8;
  const float r = radii[n];
  const double rinv = (r > 1e-6f) ? 1.0 / (double)r : 1e6;
  double s, c;
  sincos((double)rot[n], &s, &c);
  const double sv = sigmoid_dd((double)opac[n]);
  const double a0 = (double)g.alpha_max * sv;
  const double hx = g.hx, hy = g.hy;
  double grad[8];
  // zero sums give zero gradients also for a non-finite rotation (see finalize_kernel)
  const double cx = S[0] != 0.0 ? c * hx * S[0] : 0.0, sx = S[0] != 0.0 ? s * hx * S[0] : 0.0;
  const double cy = S[1] != 0.0 ? c * hy * S[1] : 0.0, sy = S[1] != 0.0 ? s * hy * S[1] : 0.0;
  grad[0] = a0 * rinv * (sy - cx);
  grad[1] = a0 * rinv * (-sx - cy);
  grad[2] = -a0 * rinv * S[2];
  grad[3] = a0 * S[3];
  grad[4] = (1.0 - sv) * S[7];
#pragma unroll
  for (int ch = 0; ch < 3; ++ch) {
    const double sc = sigmoid_dd((double)colors[3 * n + ch]);
    grad[5 + ch] = sc * (1.0 - sc) * S[4 + ch];
  }
  float* p[8] = {means2D + 2 * n, means2D + 2 * n + 1, radii + n, rot + n, opac + n,
                 colors + 3 * n, colors + 3 * n + 1, colors + 3 * n + 2};
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const float gk = (float)grad[k];
    float mk = m1[(size_t)n * 8 + k], vk = m2[(size_t)n * 8 + k];
    mk = fmaf(1.f - a.beta1, gk - mk, mk);                 // exp_avg.lerp_(grad, 1-beta1)
    vk = fmaf(a.beta2, vk, (1.f - a.beta2) * gk * gk);     // exp_avg_sq.mul_(beta2).addcmul_(g, g, 1-beta2)
    m1[(size_t)n * 8 + k] = mk;
    m2[(size_t)n * 8 + k] = vk;
    const float step_size = (float)((double)a.lr[k] * decay / bc1);
    const float denom = sqrtf(vk) / (float)bc2s + a.eps;
    *p[k] -= step_size * mk / denom;
  }
  if (a.clamp) {
    means2D[2 * n] = fminf(fmaxf(means2D[2 * n], 0.f), a.x_max);
    means2D[2 * n + 1] = fminf(fmaxf(means2D[2 * n + 1], 0.f), a.y_max);
    radii[n] = fminf(fmaxf(radii[n], a.r_min), a.r_max);
  }
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
    adam_kernel<<<(g.N + 255) / 256, 256, 0, st>>>(g, a, gacc, means2D, radii, rot, opac, colors, m1, m2,
                                                   step_count, skip_flag);
    DBMP_CHECK_LAUNCH("adam_kernel");
  }
  step_increment_kernel<<<1, 1, 0, st>>>(step_count, skip_flag);
  DBMP_CHECK_LAUNCH("step_increment_kernel");
  return DBMP_OK;
}

}  // namespace dbmp
