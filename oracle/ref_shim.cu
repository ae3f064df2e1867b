// TEST INFRASTRUCTURE -- plain C entry points over the reference's own CUDA
// launchers (smhongok/diffbmp cuda_tile_rasterizer/cuda_kernels/tile_forward.h:6-11
// and tile_backward.h:6-14), compiled from the reference sources by
// oracle/Makefile into oracle/_ref/libref_raster.so.  Tests use it to compare
// the new kernels with the reference's on the GPU.  Caller-provided buffers
// replace the reference's TileRasterizer scratch (tile_rasterize.cu:50-207):
// caches must hold 5*H*W*K floats (+ slack) with K >= the deepest pixel.
#include <cuda_runtime.h>

#include "tile_backward.h"
#include "tile_forward.h"

extern "C" {

int ref_forward(int H, int W, int ts, float amax, int N, int P, int Ht, int Wt, int K,
                const float* means2D, const float* radii, const float* rot, const float* opac,
                const float* colors, const float* tmpl, const int* sel, int* offsets, int T1,
                int* indices, int L, float* out_color, float* out_alpha, float* caches, int* counts,
                float* sig) {
  const size_t HWK = (size_t)H * W * K;
  cudaMemset(caches, 0, 5 * HWK * sizeof(float));
  cudaMemset(counts, 0, (size_t)H * W * sizeof(int));
  cudaMemset(out_color, 0, (size_t)H * W * 3 * sizeof(float));
  cudaMemset(out_alpha, 0, (size_t)H * W * sizeof(float));
  CudaRasterizeTilesForwardKernel(
      InputTensors(means2D, radii, rot, opac, colors, nullptr, tmpl, sel, 0.0f),
      OutputTensors(out_color, out_alpha, nullptr, nullptr, nullptr, nullptr, nullptr),
      GlobalBuffers(caches, caches + HWK, caches + 2 * HWK, caches + 3 * HWK, caches + 4 * HWK, counts, sig,
                    sig + 4 * (size_t)N, offsets, indices, T1, L),
      TileConfig(H, W, ts, 0.0f, amax), PrimitiveConfig(N, P, Ht, Wt, K));
  return (int)cudaDeviceSynchronize();
}

int ref_backward(int H, int W, int ts, float amax, int N, int P, int Ht, int Wt, int K,
                 const float* means2D, const float* radii, const float* rot, const float* opac,
                 const float* colors, const float* tmpl, const int* sel, int* offsets, int T1,
                 int* indices, int L, const float* grad_color, const float* grad_alpha, float* caches,
                 int* counts, float* sig, float* g_means, float* g_radii, float* g_rot, float* g_opac,
                 float* g_colors) {
  const size_t HWK = (size_t)H * W * K;
  cudaMemset(g_means, 0, (size_t)N * 2 * sizeof(float));
  cudaMemset(g_radii, 0, (size_t)N * sizeof(float));
  cudaMemset(g_rot, 0, (size_t)N * sizeof(float));
  cudaMemset(g_opac, 0, (size_t)N * sizeof(float));
  cudaMemset(g_colors, 0, (size_t)N * 3 * sizeof(float));
  CudaRasterizeTilesBackwardKernel(
      grad_color, grad_alpha, InputTensors(means2D, radii, rot, opac, colors, nullptr, tmpl, sel, 0.0f),
      OutputTensors(nullptr, nullptr, g_means, g_radii, g_rot, g_opac, g_colors),
      GlobalBuffers(caches, caches + HWK, caches + 2 * HWK, caches + 3 * HWK, caches + 4 * HWK, counts, sig,
                    sig + 4 * (size_t)N, offsets, indices, T1, L),
      TileConfig(H, W, ts, 0.0f, amax), PrimitiveConfig(N, P, Ht, Wt, K),
      LearningRateConfig(0.1f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f));
  return (int)cudaDeviceSynchronize();
}

// The same with the colour-map blend (colors_orig (N,Ht,Wt,3), c_blend > 0,
// tile_forward.cu:316-330).
int ref_forward_cb(int H, int W, int ts, float amax, int N, int P, int Ht, int Wt, int K,
                   const float* means2D, const float* radii, const float* rot, const float* opac,
                   const float* colors, const float* colors_orig, float c_blend, const float* tmpl, const int* sel,
                   int* offsets, int T1, int* indices, int L, float* out_color, float* out_alpha, float* caches,
                   int* counts, float* sig) {
  const size_t HWK = (size_t)H * W * K;
  cudaMemset(caches, 0, 5 * HWK * sizeof(float));
  cudaMemset(counts, 0, (size_t)H * W * sizeof(int));
  cudaMemset(out_color, 0, (size_t)H * W * 3 * sizeof(float));
  cudaMemset(out_alpha, 0, (size_t)H * W * sizeof(float));
  CudaRasterizeTilesForwardKernel(
      InputTensors(means2D, radii, rot, opac, colors, colors_orig, tmpl, sel, c_blend),
      OutputTensors(out_color, out_alpha, nullptr, nullptr, nullptr, nullptr, nullptr),
      GlobalBuffers(caches, caches + HWK, caches + 2 * HWK, caches + 3 * HWK, caches + 4 * HWK, counts, sig,
                    sig + 4 * (size_t)N, offsets, indices, T1, L),
      TileConfig(H, W, ts, 0.0f, amax), PrimitiveConfig(N, P, Ht, Wt, K));
  return (int)cudaDeviceSynchronize();
}

int ref_backward_cb(int H, int W, int ts, float amax, int N, int P, int Ht, int Wt, int K,
                    const float* means2D, const float* radii, const float* rot, const float* opac,
                    const float* colors, const float* colors_orig, float c_blend, const float* tmpl,
                    const int* sel, int* offsets, int T1, int* indices, int L, const float* grad_color,
                    const float* grad_alpha, float* caches, int* counts, float* sig, float* g_means,
                    float* g_radii, float* g_rot, float* g_opac, float* g_colors) {
  const size_t HWK = (size_t)H * W * K;
  cudaMemset(g_means, 0, (size_t)N * 2 * sizeof(float));
  cudaMemset(g_radii, 0, (size_t)N * sizeof(float));
  cudaMemset(g_rot, 0, (size_t)N * sizeof(float));
  cudaMemset(g_opac, 0, (size_t)N * sizeof(float));
  cudaMemset(g_colors, 0, (size_t)N * 3 * sizeof(float));
  CudaRasterizeTilesBackwardKernel(
      grad_color, grad_alpha, InputTensors(means2D, radii, rot, opac, colors, colors_orig, tmpl, sel, c_blend),
      OutputTensors(nullptr, nullptr, g_means, g_radii, g_rot, g_opac, g_colors),
      GlobalBuffers(caches, caches + HWK, caches + 2 * HWK, caches + 3 * HWK, caches + 4 * HWK, counts, sig,
                    sig + 4 * (size_t)N, offsets, indices, T1, L),
      TileConfig(H, W, ts, 0.0f, amax), PrimitiveConfig(N, P, Ht, Wt, K),
      LearningRateConfig(0.1f, 1.f, 1.f, 1.f, 1.f, 1.f, 1.f));
  return (int)cudaDeviceSynchronize();
}

int ref_last_error(void) { return (int)cudaGetLastError(); }

}  // extern "C"
