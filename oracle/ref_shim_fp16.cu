// TEST / MEASUREMENT INFRASTRUCTURE -- plain C entry points over the
// reference's own all-half CUDA launchers (smhongok/diffbmp
// cuda_tile_rasterizer/cuda_kernels/tile_forward_fp16.h:9-14 and
// tile_backward_fp16.h:9-17), compiled from the reference sources by
// oracle/Makefile into oracle/_ref/libref_raster_fp16.so.  Used to time the
// reference's FP16 extension beside the new kernels.  Caller-provided buffers
// replace the reference's TileRasterizerFP16 scratch
// (tile_rasterize_fp16.cpp:59-143): caches hold 5*H*W*K halves with K >= the
// deepest pixel, sigma_inv / grad_sigma 4*N halves each.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "tile_backward_fp16.h"
#include "tile_forward_fp16.h"

extern "C" {

int ref_forward_fp16(int H, int W, int ts, float amax, int N, int P, int Ht, int Wt, int K,
                     const __half* means2D, const __half* radii, const __half* rot, const __half* opac,
                     const __half* colors, const __half* tmpl, const int* sel, int* offsets, int T1,
                     int* indices, int L, __half* out_color, __half* out_alpha, __half* caches, int* counts,
                     __half* sig) {
  const size_t HWK = (size_t)H * W * K;
  cudaMemset(caches, 0, 5 * HWK * sizeof(__half));
  cudaMemset(counts, 0, (size_t)H * W * sizeof(int));
  cudaMemset(out_color, 0, (size_t)H * W * 3 * sizeof(__half));
  cudaMemset(out_alpha, 0, (size_t)H * W * sizeof(__half));
  CudaRasterizeTilesForwardKernelFP16(
      InputTensorsFP16(means2D, radii, rot, opac, colors, nullptr, tmpl, sel, 0.0f),
      OutputTensorsFP16(out_color, out_alpha, nullptr, nullptr, nullptr, nullptr, nullptr),
      GlobalBuffersFP16(caches, caches + HWK, caches + 2 * HWK, caches + 3 * HWK, caches + 4 * HWK, counts, sig,
                        sig + 4 * (size_t)N, offsets, indices, T1, L),
      TileConfigFP16(H, W, ts, __float2half(0.0f), __float2half(amax)), PrimitiveConfigFP16(N, P, Ht, Wt, K));
  return (int)cudaDeviceSynchronize();
}

int ref_backward_fp16(int H, int W, int ts, float amax, int N, int P, int Ht, int Wt, int K,
                      const __half* means2D, const __half* radii, const __half* rot, const __half* opac,
                      const __half* colors, const __half* tmpl, const int* sel, int* offsets, int T1,
                      int* indices, int L, const __half* grad_color, const __half* grad_alpha, __half* caches,
                      int* counts, __half* sig, __half* g_means, __half* g_radii, __half* g_rot, __half* g_opac,
                      __half* g_colors) {
  const size_t HWK = (size_t)H * W * K;
  cudaMemset(g_means, 0, (size_t)N * 2 * sizeof(__half));
  cudaMemset(g_radii, 0, (size_t)N * sizeof(__half));
  cudaMemset(g_rot, 0, (size_t)N * sizeof(__half));
  cudaMemset(g_opac, 0, (size_t)N * sizeof(__half));
  cudaMemset(g_colors, 0, (size_t)N * 3 * sizeof(__half));
  const __half one = __float2half(1.0f);
  CudaRasterizeTilesBackwardKernelFP16(
      grad_color, grad_alpha, InputTensorsFP16(means2D, radii, rot, opac, colors, nullptr, tmpl, sel, 0.0f),
      OutputTensorsFP16(nullptr, nullptr, g_means, g_radii, g_rot, g_opac, g_colors),
      GlobalBuffersFP16(caches, caches + HWK, caches + 2 * HWK, caches + 3 * HWK, caches + 4 * HWK, counts, sig,
                        sig + 4 * (size_t)N, offsets, indices, T1, L),
      TileConfigFP16(H, W, ts, __float2half(0.0f), __float2half(amax)), PrimitiveConfigFP16(N, P, Ht, Wt, K),
      LearningRateConfigFP16(__float2half(0.1f), one, one, one, one, one, one));
  return (int)cudaDeviceSynchronize();
}

}  // extern "C"
