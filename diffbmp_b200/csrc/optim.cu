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

struct AdamArgs {
  float lr[8];            // per parameter: x, y, r, theta, v, c_r, c_g, c_b
  float beta1, beta2, eps;
  float x_max, y_max, r_min, r_max;
  int clamp;
};

__global__ void adam_kernel(Geom g, AdamArgs a, const double* __restrict__ gacc, float* __restrict__ means2D,
                            float* __restrict__ radii, float* __restrict__ rot, float* __restrict__ opac,
                            float* __restrict__ colors, float* __restrict__ m1, float* __restrict__ m2,
                            const int* __restrict__ step_count, const int* __restrict__ skip_flag) {
  if (skip_flag != nullptr && *skip_flag != 0) return;
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= g.N) return;
  const int t = *step_count + 1;
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
    const float step_size = (float)((double)a.lr[k] / bc1);
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
