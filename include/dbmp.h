/*
 * dbmp.h -- C ABI of the DiffBMP B200 tile rasterizer (libdbmp.so).
 *
 * Plain pointers and sizes only: every array argument is a device pointer
 * (CUDA global memory of the current device) unless the comment says "host".
 * `stream` is a cudaStream_t passed as void*.  No entry point synchronises the
 * device or reads device memory from the host; all work is stream-ordered.
 * Every call returns a dbmp_status; on failure dbmp_last_error() describes it
 * (thread-local string).  There is no fallback path: a failed call leaves its
 * outputs undefined.
 *
 * Primitive parameters use the reference's layout and meaning
 * (smhongok/diffbmp, cuda_tile_rasterizer/ext.cpp:11-28):
 *   means2D (N,2) f32 pixel centres; radii (N) f32 half extent of the
 *   template square; rotations (N) f32 radians; opacities (N) f32 logits;
 *   colors (N,3) f32 logits; sel (N) i32 template id per primitive.
 * Tile lists use the reference's CSR form: offsets (T+1) i32 and indices (L)
 * i32, tiles row-major with tile_size x tile_size pixels, primitive ids
 * ascending within a tile (pydiffbmp/core/renderer/simple_tile_renderer.py:721-766).
 */
#ifndef DBMP_H
#define DBMP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  DBMP_OK = 0,
  DBMP_ERR_INVALID = 1,      /* bad argument (size, null pointer, unsupported tile size) */
  DBMP_ERR_CUDA = 2,         /* a CUDA runtime call or launch failed */
  DBMP_ERR_CAPACITY = 3,     /* caller buffer too small (see the entry point) */
  DBMP_ERR_UNSUPPORTED = 4   /* feature combination not built */
} dbmp_status;

/* Atlas storage kinds (dbmp_canvas.atlas_kind). */
#define DBMP_ATLAS_F32 0        /* (P,Ht,Wt) f32, the reference layout */
#define DBMP_ATLAS_F32_QUAD 1   /* (P,Ht,Wt,4) f32 bilinear quads, see dbmp_atlas_pack */
#define DBMP_ATLAS_F16_QUAD 2   /* (P,Ht,Wt,4) IEEE half quads */
#define DBMP_ATLAS_BF16_QUAD 3  /* (P,Ht,Wt,4) bfloat16 quads */
#define DBMP_ATLAS_F16_PAIR 4   /* (P,Ht+1,Wt,2) IEEE half horizontal pairs, see dbmp_atlas_pack */
#define DBMP_ATLAS_BF16_PAIR 5  /* (P,Ht+1,Wt,2) bfloat16 horizontal pairs */

/* Binning modes (dbmp_canvas.bin_mode). */
#define DBMP_BIN_CONTENT 0  /* world bbox of the template's texels > 1e-6:
                               pydiffbmp/core/renderer/vector_renderer.py:194-252,401-444 */
#define DBMP_BIN_CULL 1     /* square cull box: the tight equivalent of the
                               all-primitives default mapping of
                               cuda_tile_rasterizer/tile_rasterize.cu:171-194 */
#define DBMP_BIN_CONTENT_REF 2  /* as DBMP_BIN_CONTENT, but the content bbox of
                               primitive i is always that of template
                               (N-1-i) % P, whatever sel says, as the
                               reference's binning takes it
                               (vector_renderer.py:220-226).  Identical to
                               DBMP_BIN_CONTENT when sel is that default; with
                               another sel it reproduces the reference's lists,
                               which can miss tiles of a primitive whose
                               rendered template reaches beyond the bbox one. */

typedef struct {
  int32_t height, width;      /* canvas in pixels */
  int32_t tile_size;          /* 16 or 32 */
  int32_t num_prims;          /* N */
  int32_t num_templates;      /* P */
  int32_t tmpl_h, tmpl_w;     /* Ht, Wt */
  int32_t atlas_kind;         /* DBMP_ATLAS_* */
  int32_t bin_mode;           /* DBMP_BIN_* */
  float alpha_max;            /* alpha_upper_bound (finite, >= 0) */
  float t_stop;               /* early-termination transmittance, in [1e-30, 1) */
  int32_t reserved;
} dbmp_canvas;

const char* dbmp_last_error(void);
int dbmp_version(void);
/* Number of tiles of a canvas: ceil(H/ts)*ceil(W/ts). */
int dbmp_num_tiles(const dbmp_canvas* cv);

/* Per-template bbox of texels > 1e-6 in normalised [-1,1] coordinates,
 * (P,4) f32 [min_u, max_u, min_v, max_v]; (-1,1,-1,1) for an empty template.
 * Replaces SimpleTileRenderer._compute_primitive_bboxes
 * (pydiffbmp/core/renderer/simple_tile_renderer.py:130-171), bit-exact. */
int dbmp_template_bboxes(const float* templates, int P, int Ht, int Wt, float* out_bbox,
                         void* stream);

/* Gaussian blur of a (P,Ht,Wt) f32 atlas into out (same shape, not in
 * place): kernel size K = 2 round(3 sigma) + 1 (ties to even), weights the
 * outer product of the normalised 1-D Gaussian, zero padding; sigma <= 0
 * copies.  Replaces gaussian_blur (pydiffbmp/util/utils.py:22-67) as
 * VectorRenderer applies it to the templates it renders with
 * (pydiffbmp/core/renderer/vector_renderer.py:80-96); the content bboxes
 * stay those of the unblurred templates there (vector_renderer.py:103-104). */
int dbmp_template_blur(const float* templates, int P, int Ht, int Wt, float sigma, float* out,
                       void* stream);

/* Repacks a (P,Ht,Wt) f32 atlas into a storage kind of the precision form,
 * with each texel's right neighbour stored as a difference (the bilinear
 * blend then needs no subtraction):
 * *_QUAD: element (p,y,x) holds t[y][x], t[y][x+1] - t[y][x], t[y+1][x],
 *   t[y+1][x+1] - t[y+1][x]; out holds P*Ht*Wt*4 elements;
 * *_PAIR: element (p,y,x) holds t[y][x], t[y][x+1] - t[y][x] for y < Ht plus
 *   one zero row y = Ht; out holds P*(Ht+1)*Wt*2 elements.
 * Neighbours outside the template are 0; each difference is taken against
 * the stored (rounded) texel, then rounded to the storage type.  The texel
 * records are followed,
 * at the next 256-byte boundary, by a clearance grid: per template, cells of
 * 2^s x 2^t texels (s, t the smallest shifts giving at most 128 cells per
 * axis), one byte each, the L-infinity distance in texels (capped at 64) from
 * the cell to the nearest texel > 5e-7 or NaN.  The tile walk uses it to skip
 * warp footprints where a primitive's mask cannot pass the fragment test
 * mask > 1e-6.  dbmp_atlas_bytes gives the total size.  No reference
 * counterpart (storage format of the precision form). */
size_t dbmp_atlas_bytes(int P, int Ht, int Wt, int kind);
int dbmp_atlas_pack(const float* templates, int P, int Ht, int Wt, int kind, void* out, void* stream);

/* Scratch bytes that dbmp_bin needs (per primitive and per tile; the
 * capacity argument is accepted for compatibility and does not change it). */
size_t dbmp_bin_workspace_bytes(const dbmp_canvas* cv, long long capacity);
/* Bytes of the per-primitive record array written by dbmp_bin / dbmp_prepare. */
size_t dbmp_prim_info_bytes(int num_prims);

/* Per-primitive preparation only (for callers that supply their own tile
 * lists): fills prim_info (dbmp_prim_info_bytes(N) bytes, 16-byte aligned).
 * prim_info records atlas offsets for cv->atlas_kind: pass it only to calls
 * made with the same atlas_kind and template shape. */
int dbmp_prepare(const dbmp_canvas* cv, const float* means2D, const float* radii,
                 const float* rotations, const float* opacities, const float* colors,
                 const int32_t* sel, void* prim_info, void* stream);

/* Device binning: preparation + per-primitive tile rectangles -> CSR tile
 * lists, built per tile row in primitive order (no sort).  Writes prim_info,
 * tile_offsets (T+1),
 * tile_indices (first L of `capacity` entries) and *total_out (device int32,
 * = L).  When L > capacity the lists are not written, *total_out still holds
 * L and *overflow_out (device int32, may be null) is set to 1; call again with
 * capacity >= L.  capacity == 0 only counts.  tmpl_bbox is the output of
 * dbmp_template_bboxes (only read in the DBMP_BIN_CONTENT* modes).
 * Replaces VectorRenderer._unified_primitive_assignment
 * (pydiffbmp/core/renderer/vector_renderer.py:401-444) followed by
 * SimpleTileRenderer._convert_masks_to_mapping (simple_tile_renderer.py:721-766);
 * tile lists are bit-identical to the reference's in DBMP_BIN_CONTENT_REF
 * mode for any sel, and in DBMP_BIN_CONTENT mode for sel = (N-1-i) % P (the
 * renderer API's assignment, simple_tile_renderer.py:221-224). */
int dbmp_bin(const dbmp_canvas* cv, const float* means2D, const float* radii,
             const float* rotations, const float* opacities, const float* colors,
             const int32_t* sel, const float* tmpl_bbox, void* prim_info,
             int32_t* tile_offsets, int32_t* tile_indices, long long capacity,
             int32_t* total_out, int32_t* overflow_out, void* workspace, size_t workspace_bytes,
             void* stream);

/* Forward compositing.  out_color (H,W,3) f32 = sum_k T_k a_k c_k and
 * out_alpha (H,W) f32 = 1 - T_final, front to back over each tile's list,
 * stopping a pixel once T < t_stop.  Per pixel it also stores the
 * transmittance entering the last contributor (T_last, f32) and that
 * contributor's position in the tile list (last_pos, i32, -1 if none); the
 * backward recomputes everything else from these.
 * Replaces CudaRasterizeTilesForwardKernel
 * (cuda_tile_rasterizer/cuda_kernels/tile_forward.h:6-11) as called by
 * TileRasterizer::forward (cuda_tile_rasterizer/tile_rasterize.cu:297-498). */
int dbmp_forward(const dbmp_canvas* cv, const void* prim_info, const void* atlas,
                 const int32_t* tile_offsets, const int32_t* tile_indices,
                 float* out_color, float* out_alpha, float* T_last, int32_t* last_pos,
                 void* stream);

/* Backward.  Reverse traversal from each pixel's last contributor,
 * recovering T_k from T_last; per-primitive sums are warp/CTA reduced and
 * accumulated in grad_accum ((N,8) f64 scratch, zeroed by this call), then
 * converted, with the primitives' radii / rotations / opacity and colour
 * logits, into the reference's five gradient outputs (f32, overwritten):
 * grad_means2D (N,2), grad_radii (N), grad_rotations (N),
 * grad_opacities (N), grad_colors (N,3).  grad_alpha may be null.
 * Replaces CudaRasterizeTilesBackwardKernel
 * (cuda_tile_rasterizer/cuda_kernels/tile_backward.h:6-14) as called by
 * TileRasterizer::backward (cuda_tile_rasterizer/tile_rasterize.cu:638-780). */
int dbmp_backward(const dbmp_canvas* cv, const void* prim_info, const void* atlas,
                  const int32_t* tile_offsets, const int32_t* tile_indices,
                  const float* T_last, const int32_t* last_pos,
                  const float* grad_color, const float* grad_alpha,
                  const float* radii, const float* rotations, const float* opacities,
                  const float* colors, double* grad_accum,
                  float* grad_means2D, float* grad_radii, float* grad_rotations,
                  float* grad_opacities, float* grad_colors, void* stream);

/* dbmp_backward for callers that cannot allocate device memory (for example
 * a plug-in whose host owns the device allocator, or a frame loop that must
 * not allocate once running).  Same inputs, outputs and results as
 * dbmp_backward, but the (N,8) f64 gradient-sum scratch is a fixed array
 * inside this library's device module, so there is no grad_accum argument.
 * Limit: N <= dbmp_backward_noalloc_max_prims() (65536); larger N returns
 * DBMP_ERR_CAPACITY.  The array takes 4 MiB on every GPU that loads it
 * (under CUDA's default lazy module loading, at the first call of this entry
 * point on that GPU), until exit.  The first call on a device looks up the array's
 * device address with that device current, and a call after that device's
 * context changed (cudaDeviceReset) looks it up again: make the first call
 * on each device, and the first after a reset, before any stream capture.  All calls share the array (zeroed by each call), so calls that
 * overlap on the GPU race; serialise them.  No counterpart in the reference. */
int dbmp_backward_noalloc(const dbmp_canvas* cv, const void* prim_info, const void* atlas,
                          const int32_t* tile_offsets, const int32_t* tile_indices,
                          const float* T_last, const int32_t* last_pos,
                          const float* grad_color, const float* grad_alpha,
                          const float* radii, const float* rotations, const float* opacities,
                          const float* colors, float* grad_means2D, float* grad_radii,
                          float* grad_rotations, float* grad_opacities, float* grad_colors,
                          void* stream);
/* Largest N dbmp_backward_noalloc accepts. */
int dbmp_backward_noalloc_max_prims(void);

/* Forward / backward with colour-map blending (c_blend > 0): each fragment's
 * colour is (1 - c_blend) sigmoid(c) + c_blend c_o, where c_o is the
 * primitive's colour map colors_orig (N,Ht,Wt,3) f32 in [0,1] sampled at the
 * fragment's texel coordinate, clamped into the map and bilinear with
 * edge-repeating neighbours.  Replaces the colors_orig / c_blend branch of
 * tile_rasterize_forward_kernel (cuda_tile_rasterizer/cuda_kernels/
 * tile_forward.cu:17-89,316-330) and its backward (tile_backward.cu:228-270):
 * dL/dalpha uses the blended colour; the colour-logit gradient is
 * gC alpha T sigma'(c) without a (1 - c_blend) factor and the colour map's
 * dependence on the geometry is not differentiated, as in the reference.
 * c_blend = 0 or colors_orig = NULL is dbmp_forward / dbmp_backward.
 * c_blend must lie in [0, 1]. */
int dbmp_forward_blend(const dbmp_canvas* cv, const void* prim_info, const void* atlas,
                       const int32_t* tile_offsets, const int32_t* tile_indices,
                       const float* colors_orig, float c_blend, float* out_color, float* out_alpha,
                       float* T_last, int32_t* last_pos, void* stream);
int dbmp_backward_blend(const dbmp_canvas* cv, const void* prim_info, const void* atlas,
                        const int32_t* tile_offsets, const int32_t* tile_indices,
                        const float* colors_orig, float c_blend, const float* T_last,
                        const int32_t* last_pos, const float* grad_color, const float* grad_alpha,
                        const float* radii, const float* rotations, const float* opacities,
                        const float* colors, double* grad_accum, float* grad_means2D,
                        float* grad_radii, float* grad_rotations, float* grad_opacities,
                        float* grad_colors, void* stream);

/* Forward / backward of a batch of `batch` candidates of the same canvas,
 * atlas and template assignment in one launch: one grid over every
 * candidate's tiles, so a batch of small canvases fills the GPU.  Candidate b
 * has its records at prim_info + b*N (prepared per candidate, e.g. by dbmp_bin
 * into that slot), its lists at tile_offsets + b*(T+1) and tile_indices +
 * b*index_stride, its images at b*H*W (x3 for colour), its parameters at b*N
 * (x2 for means2D, x3 for colors), its gradient sums at grad_accum + b*N*8
 * and its colour maps at colors_orig + b*colors_orig_stride (stride 0: shared
 * maps).  Otherwise as dbmp_forward_blend / dbmp_backward_blend for each
 * candidate.  Replaces TileRasterizer::forward_batch / backward_batch
 * (cuda_tile_rasterizer/tile_rasterize.cu:500-636), which loop over the
 * candidates on the host. */
int dbmp_forward_batch(const dbmp_canvas* cv, int batch, const void* prim_info, const void* atlas,
                       const int32_t* tile_offsets, const int32_t* tile_indices, long long index_stride,
                       const float* colors_orig, long long colors_orig_stride, float c_blend, float* out_color,
                       float* out_alpha, float* T_last, int32_t* last_pos, void* stream);
int dbmp_backward_batch(const dbmp_canvas* cv, int batch, const void* prim_info, const void* atlas,
                        const int32_t* tile_offsets, const int32_t* tile_indices, long long index_stride,
                        const float* colors_orig, long long colors_orig_stride, float c_blend,
                        const float* T_last, const int32_t* last_pos, const float* grad_color,
                        const float* grad_alpha, const float* radii, const float* rotations,
                        const float* opacities, const float* colors, double* grad_accum,
                        float* grad_means2D, float* grad_radii, float* grad_rotations,
                        float* grad_opacities, float* grad_colors, void* stream);

/* Counting pass over the same walk as dbmp_forward (no image output):
 * counts[0] = (pixel, primitive) pairs that pass the square cull before the
 * pixel terminates, counts[1] = fragments composited, counts[2] = tile-list
 * entries (sum over tiles), counts[3] = (warp, entry) pairs a warp evaluated,
 * counts[4] = pixel slots still running summed over those pairs, counts[5] =
 * (warp, entry) pairs rejected by the warp-footprint test, counts[6] = the
 * largest number of fragments composited at one pixel, counts[7] = walked
 * (warp, entry) pairs without any fragment, counts[8] = walked pairs the
 * packed atlas's clearance grid skips, counts[9] = pairs the grid would skip
 * although they hold a fragment (0 unless the grid is wrong).  cv->t_stop may
 * be 0 here to count without termination (every fragment, as the reference
 * composites).  counts: 10 device u64, zeroed by the call.  Used for roofline
 * and memory accounting and to check the grid; no reference counterpart. */
int dbmp_count(const dbmp_canvas* cv, const void* prim_info, const void* atlas,
               const int32_t* tile_offsets, const int32_t* tile_indices,
               unsigned long long* counts, void* stream);

/* Fused forward + L2 loss + backward of one image-fitting iteration in one
 * launch: each warp composites its pixels of a tile, forms the reference
 * loss gradient of rendered = C + (1-A)*background against `target` for
 * them (mse_loss, pydiffbmp/util/loss_functions.py:20-40 on
 * simple_tile_renderer.py:704-707) and walks the same list back.  Zeroes and
 * fills grad_accum ((N,8) f64 raw per-primitive sums, consumed by
 * dbmp_adam_step) and *loss_out (device f64, mean squared error).
 * target / background (H,W,3) f32; background may be null (black);
 * out_image (H,W,3) f32 may be null.  If skip_flag (device int32, may be
 * null) is non-zero the call leaves every output untouched (used with
 * dbmp_bin's overflow flag).  Replaces the sequence forward kernel -> torch
 * loss -> backward kernel of simple_tile_renderer.py:1059-1074. */
int dbmp_fused_fwd_bwd(const dbmp_canvas* cv, const void* prim_info, const void* atlas,
                       const int32_t* tile_offsets, const int32_t* tile_indices,
                       const float* target, const float* background, float* out_image,
                       double* grad_accum, double* loss_out, const int32_t* skip_flag,
                       void* stream);

/* The reference's five gradient outputs from the raw per-primitive sums in
 * grad_accum ((N,8) f64, as left by dbmp_fused_fwd_bwd), for callers that
 * run their own optimiser after the fused step: grad_means2D (N,2),
 * grad_radii, grad_rotations, grad_opacities (N), grad_colors (N,3), f32,
 * overwritten, with the chain rule of dbmp_backward (the gradient-output
 * stage of TileRasterizer::backward, cuda_tile_rasterizer/tile_rasterize.cu:
 * 638-780, and tile_backward.cu:255-343). */
int dbmp_grads_from_accum(const dbmp_canvas* cv, const double* grad_accum, const float* radii,
                          const float* rotations, const float* opacities, const float* colors,
                          float* grad_means2D, float* grad_radii, float* grad_rotations,
                          float* grad_opacities, float* grad_colors, void* stream);

/* Optimiser settings of dbmp_adam_step: learning rate per parameter in the
 * order x, y, r, theta, opacity, colour r/g/b; Adam betas/eps; clamp bounds. */
typedef struct {
  float lr[8];
  float beta1, beta2, eps;
  float x_max, y_max, r_min, r_max;
  int32_t clamp;          /* 1: clamp x, y, r after the step */
  float lr_gamma;         /* ExponentialLR factor: the step after k completed
                             steps uses lr * lr_gamma^k (torch's
                             ExponentialLR stepped after every optimizer step,
                             simple_tile_renderer.py:970-973,1128-1129);
                             0 or 1: no decay */
} dbmp_adam_cfg;

/* In-place Adam step of every primitive parameter from the raw sums in
 * grad_accum (as left by dbmp_fused_fwd_bwd or dbmp_backward), followed by
 * the reference's parameter clamp.  adam_m / adam_v: (N,8) f32 moments;
 * step_count: device int32 of completed steps (incremented here).  If
 * skip_flag is non-zero nothing changes.  Replaces torch.optim.Adam.step +
 * _clamp_params_inplace (pydiffbmp/core/renderer/simple_tile_renderer.py:961-968,
 * 1125-1131, 122-128). */
int dbmp_adam_step(const dbmp_canvas* cv, const dbmp_adam_cfg* cfg, const double* grad_accum,
                   float* means2D, float* radii, float* rotations, float* opacities, float* colors,
                   float* adam_m, float* adam_v, int32_t* step_count, const int32_t* skip_flag,
                   void* stream);

/* Pruning (restart) of low-opacity primitives, the reference's do_prune
 * (simple_tile_renderer.py:1007-1013,1236-1270) on the device.  At iteration
 * it = *step_count (completed steps), when it != 0, it % every == 0,
 * it < num_iterations - no_prune_last and it > warmup, every primitive with
 * sigmoid(opacity) < threshold (float32 sigmoid, as torch.sigmoid) takes the
 * next row of `pool` ((pool_rows, 8) f32: x, y, r, theta, opacity logit,
 * colour logits r, g, b -- the replacement parameters an initializer drew,
 * used in ascending primitive order, cyclically); Adam moments are kept, as
 * in the reference.  state (4 device int32, zeroed by the caller before the
 * first step): [0] next pool row, [1] iteration of the last prune (a replayed
 * iteration is not pruned twice), [2] primitives replaced by the last prune,
 * [3] primitives replaced in total.  skip_flag as in dbmp_adam_step.  One
 * single-CTA launch; other iterations return at once. */
typedef struct {
  int32_t every;            /* prune_iterations */
  int32_t num_iterations;   /* iterations of the fit */
  int32_t no_prune_last;    /* no_prune_last_iterations */
  int32_t warmup;           /* no_prune_warmup_iterations */
  float threshold;          /* prune_threshold on sigmoid(opacity) */
  int32_t pool_rows;        /* rows of pool (>= 1) */
} dbmp_prune_cfg;
int dbmp_prune(const dbmp_canvas* cv, const dbmp_prune_cfg* cfg, const int32_t* step_count,
               const float* pool, int32_t* state, float* means2D, float* radii, float* rotations,
               float* opacities, float* colors, const int32_t* skip_flag, void* stream);

/* Blur schedule of the fit loop (simple_tile_renderer.py:975-979,1015-1021):
 * at iteration it = *step_count the templates are blurred with
 * mode 0: sigma 0 (unchanged); mode 1: `sigma` (do_gaussian_blur);
 * mode 2: sigma_start (1 - it/num_iterations) + sigma_end it/num_iterations
 * (do_adapt_gaussian_blur), evaluated in double as the reference does, then
 * as dbmp_template_blur (kernel size from the double sigma, weights in
 * float).  The reference's CPU path blurs its templates per iteration this
 * way (simple_tile_renderer.py:1499-1505); its CUDA path does not read the
 * per-iteration sigma at all (TileConfig.sigma, cuda_kernels/tile_common.h:28,
 * is unused by the kernels), which mode 0 reproduces. */
typedef struct {
  int32_t mode;
  float sigma, sigma_start, sigma_end;
  int32_t num_iterations;
} dbmp_blur_schedule;
int dbmp_template_blur_scheduled(const float* templates, int P, int Ht, int Wt,
                                 const dbmp_blur_schedule* sched, const int32_t* step_count, float* out,
                                 void* stream);

/* PSD stage 1: crop box per primitive, [x0,y0,x1,y1) of the square of half
 * extent 1.5*r*scale around means2D*scale, clipped to the HxW export canvas;
 * an empty box becomes (0,0,1,1).  out_bbox (N,4) i32 (16-byte aligned),
 * out_sizes (N,2) i32 = (w,h).  Bit-identical to the reference.  Replaces
 * launch_compute_bounding_boxes (cuda_tile_rasterizer/cuda_kernels/
 * psd_export_kernels.cu:206-231). */
int dbmp_psd_bboxes(const float* means2D, const float* radii, int N, int H, int W, float scale,
                    int32_t* out_bbox, int32_t* out_sizes, void* stream);

/* PSD layout: layer_offsets (N) i64 = exclusive sum of w*h*4 (byte offset of
 * each layer in the packed buffer), block_offsets (N+1) i64 = exclusive sum
 * of 16x16 blocks per layer (scratch for dbmp_psd_layers), *total_bytes
 * (device i64) = buffer size.  Replaces the host loop of
 * cuda_tile_rasterizer/psd_export_uint8.py:70-77. */
int dbmp_psd_layout(const int32_t* sizes, int N, int64_t* layer_offsets, int64_t* block_offsets,
                    int64_t* total_bytes, void* stream);

/* PSD stage 2: packed uint8 RGBA layers, layer n at byte layer_offsets[n],
 * row-major over its crop box.  colors / visibility are already sigmoid-ed;
 * colors_orig (N,Ht,Wt,3) f32 may be null (used only when c_blend > 0).  out
 * must be 4-byte aligned and hold *total_bytes.  Bytes are identical to the
 * reference's.  Replaces launch_generate_cropped_layers
 * (cuda_tile_rasterizer/cuda_kernels/psd_export_kernels.cu:233-273). */
int dbmp_psd_layers(const float* means2D, const float* radii, const float* rotations,
                    const float* colors, const float* visibility, const float* templates, int P, int Ht,
                    int Wt, const int32_t* sel, const int32_t* bbox, const int64_t* layer_offsets,
                    const int64_t* block_offsets, int N, float scale, float alpha_max, float c_blend,
                    const float* colors_orig, uint8_t* out, void* stream);

/* PSD file assembly, count pass: PackBits (RLE) sizes of every row of every
 * channel of N packed uint8 RGBA images (layer n at byte layer_offsets[n],
 * a multiple of 4, with (w,h) = sizes[n]; e.g. the output of dbmp_psd_layers).
 * Rows are taken in groups of 32 per layer: group_base (N+1) i64 is the
 * exclusive prefix sum of ceil(h/32) and num_groups = group_base[N].
 * channel_order gives, in byte s, which RGBA byte (0..3) is channel slot s
 * (0x02010003 = A,R,G,B as in layer records; 0x03020100 = R,G,B,A as in the
 * merged image).  Writes row_bytes ((num_groups*32, 4) u16, 8-byte aligned:
 * the encoded size of row 32*g+j of slot s at [(32*g + j)*4 + s], 0 past the
 * layer's last row), group_totals ((num_groups, 4) i32, 16-byte aligned) and,
 * if alpha_any is not null, alpha_any[n] = 1 for each layer with a nonzero
 * byte 3 (the caller zeroes it first).  Images wider than width_limit
 * (<= 30000, the PSD limit) are encoded as empty.  Replaces the per-layer
 * psd-tools calls of cuda_tile_rasterizer/psd_export_uint8.py:153-186
 * (PixelLayer.frompil, RLE compression at PSDImage.save,
 * pydiffbmp/util/psd_exporter.py:494-501). */
int dbmp_psd_rle_count(const uint8_t* layers, const int32_t* sizes, const int64_t* layer_offsets,
                       const int64_t* group_base, int N, long long num_groups, int channel_order, int width_limit,
                       uint16_t* row_bytes, int32_t* group_totals, int32_t* alpha_any, void* stream);

/* PSD file assembly, write pass: for each image n with channel_offsets
 * (N,4) i64 >= 0, writes slot s's PSD channel block at out +
 * channel_offsets[4n+s]: the compression word 1 (RLE), the h big-endian u16
 * row sizes and the rows' PackBits data, which starts for group g at
 * group_offsets[4g+s] (i64, (num_groups, 4)).  The caller plans both from
 * dbmp_psd_rle_count's outputs (block size = 2 + 2h + the slot's total).
 * Every store is bounded by its row's planned size and by out_bytes. */
int dbmp_psd_rle_write(const uint8_t* layers, const int32_t* sizes, const int64_t* layer_offsets,
                       const int64_t* group_base, int N, long long num_groups, int channel_order, int width_limit,
                       const uint16_t* row_bytes, const int64_t* channel_offsets, const int64_t* group_offsets,
                       uint8_t* out, long long out_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* DBMP_H */
