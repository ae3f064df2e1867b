// C ABI of libdbmp.so (declarations and contracts in include/dbmp.h).
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "dbmp_internal.cuh"

namespace dbmp {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int cuda_status(cudaError_t e, const char* what) {
  set_error("%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
  return DBMP_ERR_CUDA;
}

// launchers (binning.cu, raster.cu)
size_t bin_workspace_bytes(int N, int T, int tilesX, int tilesY, long long cap);
size_t atlas_bytes(int P, int Ht, int Wt, int kind);
int launch_template_bboxes(const float* tmpl, int P, int Ht, int Wt, float* out, cudaStream_t st);
int launch_template_blur(const float* in, int P, int Ht, int Wt, float sigma, float* out, cudaStream_t st);
int launch_atlas_pack(const float* tmpl, int P, int Ht, int Wt, int kind, void* out, cudaStream_t st);
int launch_prepare(const Geom& g, const float* means2D, const float* radii, const float* rot, const float* opac,
                   const float* colors, const int* sel, PrimInfo* out, cudaStream_t st);
int launch_bin(const Geom& g, int bin_mode, const float* means2D, const float* radii, const float* rot,
               const float* opac, const float* colors, const int* sel, const float* tbbox, PrimInfo* prim_info,
               int* tile_offsets, int* tile_indices, long long cap, int* total_out, int* overflow_out,
               void* ws, size_t ws_bytes, cudaStream_t st);
int launch_forward(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs,
                   const int* idx, float* color, float* alpha, float* T_last, int* last_pos, cudaStream_t st);
int launch_forward_blend(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs,
                         const int* idx, float* color, float* alpha, float* T_last, int* last_pos, const float* cmap,
                         float cblend, cudaStream_t st, int batch, long long idx_stride, long long cmap_stride);
int launch_backward_blend(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs,
                          const int* idx, const float* T_last, const int* last_pos, const float* grad_color,
                          const float* grad_alpha, double* gacc, const float* cmap, float cblend, cudaStream_t st,
                          int batch, long long idx_stride, long long cmap_stride);
int launch_count(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs, const int* idx,
                 unsigned long long* cnt, cudaStream_t st);
int launch_backward(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs,
                    const int* idx, const float* T_last, const int* last_pos, const float* grad_color,
                    const float* grad_alpha, double* gacc, cudaStream_t st);
int launch_finalize(const Geom& g, const float* radii, const float* rot, const float* opac, const float* colors,
                    const double* gacc, float* gm, float* gr, float* grot, float* go, float* gc, cudaStream_t st);
int launch_fused(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs, const int* idx,
                 const float* target, const float* background, float* out_image, double* gacc, double* loss,
                 const int* skip_flag, cudaStream_t st);
int launch_prune(const Geom& g, const PruneArgs& a, const int* step_count, const float* pool, int* state,
                 float* means2D, float* radii, float* rot, float* opac, float* colors, const int* skip_flag,
                 cudaStream_t st);
int launch_template_blur_sched(const float* in, int P, int Ht, int Wt, const dbmp_blur_schedule* sched,
                               const int* step_count, float* out, cudaStream_t st);
int launch_adam(const Geom& g, const AdamArgs& a, const double* gacc, float* means2D, float* radii, float* rot,
                float* opac, float* colors, float* m1, float* m2, int* step_count, const int* skip_flag,
                cudaStream_t st);

int launch_psd_bboxes(const float* means2D, const float* radii, int N, int H, int W, float scale, int* bbox,
                      int* sizes, cudaStream_t st);
int launch_psd_layout(const int* sizes, int N, long long* layer_offsets, long long* blk, long long* total,
                      cudaStream_t st);
int launch_psd_layers(int N, int P, int Ht, int Wt, float scale, float alpha_max, float c_blend,
                      const float* means2D, const float* radii, const float* rot, const float* colors,
                      const float* vis, const float* tmpl, const int* sel, const int* bbox,
                      const long long* layer_offsets, const long long* blk, const float* colors_orig, uint8_t* out,
                      cudaStream_t st);
int launch_psd_rle(bool write, const uint8_t* layers, const int* sizes, const long long* layer_off,
                   const long long* group_base, int N, long long G, unsigned order, int width_limit,
                   unsigned short* row_bytes, int* group_tot, int* alpha_any, const long long* chan_off,
                   const long long* group_dst, uint8_t* out, long long out_bytes, cudaStream_t st);

// Validates a canvas description and derives the launch geometry.
int make_geom(const dbmp_canvas* cv, Geom* g, const char* who) {
  if (!cv) { set_error("%s: canvas is null", who); return DBMP_ERR_INVALID; }
  if (cv->height <= 0 || cv->width <= 0) { set_error("%s: canvas %dx%d is empty", who, cv->height, cv->width); return DBMP_ERR_INVALID; }
  if (cv->tile_size != 16 && cv->tile_size != 32) { set_error("%s: tile_size %d is not supported (16 or 32)", who, cv->tile_size); return DBMP_ERR_INVALID; }
  if (cv->num_prims < 0) { set_error("%s: num_prims %d < 0", who, cv->num_prims); return DBMP_ERR_INVALID; }
  if (cv->num_templates <= 0 || cv->tmpl_h < 2 || cv->tmpl_w < 2) {
    set_error("%s: template atlas %dx%dx%d is invalid (need P>=1, Ht,Wt>=2)", who, cv->num_templates, cv->tmpl_h, cv->tmpl_w);
    return DBMP_ERR_INVALID;
  }
  if (cv->atlas_kind < DBMP_ATLAS_F32 || cv->atlas_kind > DBMP_ATLAS_BF16_PAIR) { set_error("%s: atlas_kind %d unknown", who, cv->atlas_kind); return DBMP_ERR_INVALID; }
  if (!(cv->alpha_max >= 0.f && cv->alpha_max < INFINITY)) { set_error("%s: alpha_max %g is not a finite value >= 0", who, (double)cv->alpha_max); return DBMP_ERR_INVALID; }
  if (half_record(cv->atlas_kind) && !(cv->alpha_max <= 65504.f)) {
    set_error("%s: alpha_max %g exceeds the FP16 range of the half / bfloat16 atlas kinds", who, (double)cv->alpha_max);
    return DBMP_ERR_INVALID;
  }
  if (!(cv->t_stop >= 1e-30f && cv->t_stop < 1.f)) { set_error("%s: t_stop %g outside [1e-30, 1)", who, (double)cv->t_stop); return DBMP_ERR_INVALID; }
  if ((long long)cv->height * cv->width > (1ll << 31) / 4) { set_error("%s: canvas too large", who); return DBMP_ERR_INVALID; }
  g->H = cv->height; g->W = cv->width; g->TS = cv->tile_size;
  g->tilesX = (cv->width + cv->tile_size - 1) / cv->tile_size;
  g->tilesY = (cv->height + cv->tile_size - 1) / cv->tile_size;
  g->T = g->tilesX * g->tilesY;
  g->N = cv->num_prims; g->P = cv->num_templates; g->Ht = cv->tmpl_h; g->Wt = cv->tmpl_w;
  g->hx = 0.5f * (float)(cv->tmpl_w - 1);
  g->hy = 0.5f * (float)(cv->tmpl_h - 1);
  g->rxy = g->hx / g->hy;
  g->ryx = g->hy / g->hx;
  g->k23 = make_float2(8388608.f, 8388608.f);
  g->m1 = make_float2(-1.f, -1.f);
  g->nhx = make_float2(-g->hx, -g->hx);
  g->nhy = make_float2(-g->hy, -g->hy);
  g->rxy2 = make_float2(g->rxy, g->rxy);
  g->nryx2 = make_float2(-g->ryx, -g->ryx);
  g->kbias = 0x4B000000u * (unsigned)(cv->tmpl_w + 1);
  g->wm1 = (float)(cv->tmpl_w - 1);
  g->hm1 = (float)(cv->tmpl_h - 1);
  g->kind = cv->atlas_kind;
  g->alpha_max = cv->alpha_max;
  g->t_stop = cv->t_stop;
  if (cv->tile_size == 32) {
    using L = Layout<32, DefaultNP<32>::v>;
    g->fhx = 0.5f * (float)(L::FW - 1); g->fhy = 0.5f * (float)(L::FH - 1);
  } else {
    using L = Layout<16, DefaultNP<16>::v>;
    g->fhx = 0.5f * (float)(L::FW - 1); g->fhy = 0.5f * (float)(L::FH - 1);
  }
  grid_shape(cv->tmpl_w, &g->gsx, &g->gGx);
  grid_shape(cv->tmpl_h, &g->gsy, &g->gGy);
  g->grid_off = (long long)atlas_grid_offset(g->P, g->Ht, g->Wt, g->kind);
  return DBMP_OK;
}

#define REQUIRE(cond, ...) \
  do { if (!(cond)) { set_error(__VA_ARGS__); return DBMP_ERR_INVALID; } } while (0)

}  // namespace dbmp

using namespace dbmp;

extern "C" {

const char* dbmp_last_error(void) { return g_err; }
int dbmp_version(void) { return 1; }

int dbmp_num_tiles(const dbmp_canvas* cv) {
  Geom g;
  if (make_geom(cv, &g, "dbmp_num_tiles") != DBMP_OK) return -1;
  return g.T;
}

size_t dbmp_prim_info_bytes(int num_prims) { return sizeof(PrimInfo) * (size_t)(num_prims > 0 ? num_prims : 0); }

int dbmp_template_bboxes(const float* templates, int P, int Ht, int Wt, float* out_bbox, void* stream) {
  REQUIRE(P >= 0 && Ht >= 2 && Wt >= 2, "dbmp_template_bboxes: bad atlas shape %dx%dx%d", P, Ht, Wt);
  REQUIRE(P == 0 || (templates && out_bbox), "dbmp_template_bboxes: null pointer");
  return launch_template_bboxes(templates, P, Ht, Wt, out_bbox, (cudaStream_t)stream);
}

int dbmp_template_blur(const float* templates, int P, int Ht, int Wt, float sigma, float* out, void* stream) {
  REQUIRE(P >= 0 && Ht >= 1 && Wt >= 1, "dbmp_template_blur: bad atlas shape %dx%dx%d", P, Ht, Wt);
  REQUIRE(P == 0 || (templates && out), "dbmp_template_blur: null pointer");
  REQUIRE(templates != out || !(sigma > 0.f), "dbmp_template_blur: in-place blur is not supported");
  return launch_template_blur(templates, P, Ht, Wt, sigma, out, (cudaStream_t)stream);
}

int dbmp_atlas_pack(const float* templates, int P, int Ht, int Wt, int kind, void* out, void* stream) {
  REQUIRE(P >= 0 && Ht >= 1 && Wt >= 1, "dbmp_atlas_pack: bad atlas shape %dx%dx%d", P, Ht, Wt);
  REQUIRE(P == 0 || (templates && out), "dbmp_atlas_pack: null pointer");
  return launch_atlas_pack(templates, P, Ht, Wt, kind, out, (cudaStream_t)stream);
}

size_t dbmp_atlas_bytes(int P, int Ht, int Wt, int kind) {
  if (P < 0 || Ht < 1 || Wt < 1) return 0;
  return atlas_bytes(P, Ht, Wt, kind);
}

size_t dbmp_bin_workspace_bytes(const dbmp_canvas* cv, long long capacity) {
  Geom g;
  if (make_geom(cv, &g, "dbmp_bin_workspace_bytes") != DBMP_OK) return 0;
  if (capacity < 0) capacity = 0;
  return bin_workspace_bytes(g.N, g.T, g.tilesX, g.tilesY, capacity);
}

int dbmp_prepare(const dbmp_canvas* cv, const float* means2D, const float* radii, const float* rotations,
                 const float* opacities, const float* colors, const int32_t* sel, void* prim_info, void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_prepare");
  if (rc) return rc;
  REQUIRE(g.N == 0 || (means2D && radii && rotations && opacities && colors && sel && prim_info),
          "dbmp_prepare: null pointer");
  REQUIRE(((uintptr_t)prim_info & 15) == 0, "dbmp_prepare: prim_info must be 16-byte aligned");
  return launch_prepare(g, means2D, radii, rotations, opacities, colors, sel, (PrimInfo*)prim_info,
                        (cudaStream_t)stream);
}

int dbmp_bin(const dbmp_canvas* cv, const float* means2D, const float* radii, const float* rotations,
             const float* opacities, const float* colors, const int32_t* sel, const float* tmpl_bbox,
             void* prim_info, int32_t* tile_offsets, int32_t* tile_indices, long long capacity,
             int32_t* total_out, int32_t* overflow_out, void* workspace, size_t workspace_bytes, void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_bin");
  if (rc) return rc;
  REQUIRE(cv->bin_mode == DBMP_BIN_CONTENT || cv->bin_mode == DBMP_BIN_CULL || cv->bin_mode == DBMP_BIN_CONTENT_REF,
          "dbmp_bin: bin_mode %d unknown", cv->bin_mode);
  REQUIRE(g.N == 0 || (means2D && radii && rotations && opacities && colors && sel && prim_info),
          "dbmp_bin: null pointer");
  REQUIRE(cv->bin_mode == DBMP_BIN_CULL || tmpl_bbox, "dbmp_bin: tmpl_bbox is required in the DBMP_BIN_CONTENT modes");
  REQUIRE(tile_offsets && total_out && workspace, "dbmp_bin: null output or workspace");
  REQUIRE(capacity >= 0 && capacity <= 0x7fffffffll, "dbmp_bin: capacity %lld outside [0, 2^31)", capacity);
  REQUIRE(capacity == 0 || tile_indices, "dbmp_bin: tile_indices is null");
  REQUIRE(((uintptr_t)prim_info & 15) == 0 && ((uintptr_t)workspace & 255) == 0,
          "dbmp_bin: prim_info must be 16-byte and workspace 256-byte aligned");
  return launch_bin(g, cv->bin_mode, means2D, radii, rotations, opacities, colors, sel, tmpl_bbox,
                    (PrimInfo*)prim_info, tile_offsets, tile_indices, capacity, total_out, overflow_out, workspace,
                    workspace_bytes, (cudaStream_t)stream);
}

int dbmp_forward(const dbmp_canvas* cv, const void* prim_info, const void* atlas, const int32_t* tile_offsets,
                 const int32_t* tile_indices, float* out_color, float* out_alpha, float* T_last, int32_t* last_pos,
                 void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_forward");
  if (rc) return rc;
  REQUIRE(atlas && tile_offsets && tile_indices && out_color && out_alpha && T_last && last_pos,
          "dbmp_forward: null pointer");
  REQUIRE(g.N == 0 || prim_info, "dbmp_forward: prim_info is null");
  return launch_forward(g, cv->atlas_kind, (const PrimInfo*)prim_info, atlas, tile_offsets, tile_indices, out_color,
                        out_alpha, T_last, last_pos, (cudaStream_t)stream);
}

int dbmp_backward(const dbmp_canvas* cv, const void* prim_info, const void* atlas, const int32_t* tile_offsets,
                  const int32_t* tile_indices, const float* T_last, const int32_t* last_pos, const float* grad_color,
                  const float* grad_alpha, const float* radii, const float* rotations, const float* opacities,
                  const float* colors, double* grad_accum, float* grad_means2D, float* grad_radii,
                  float* grad_rotations, float* grad_opacities, float* grad_colors, void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_backward");
  if (rc) return rc;
  REQUIRE(atlas && tile_offsets && tile_indices && T_last && last_pos && grad_color, "dbmp_backward: null input");
  REQUIRE(g.N == 0 || (prim_info && radii && rotations && opacities && colors), "dbmp_backward: null parameter");
  REQUIRE(g.N == 0 || (grad_accum && grad_means2D && grad_radii && grad_rotations && grad_opacities && grad_colors),
          "dbmp_backward: null output");
  cudaStream_t st = (cudaStream_t)stream;
  if (g.N > 0) {
    cudaError_t e = cudaMemsetAsync(grad_accum, 0, sizeof(double) * 8 * (size_t)g.N, st);
    if (e != cudaSuccess) return cuda_status(e, "cudaMemsetAsync(grad_accum)");
  }
  rc = launch_backward(g, cv->atlas_kind, (const PrimInfo*)prim_info, atlas, tile_offsets, tile_indices, T_last,
                       last_pos, grad_color, grad_alpha, grad_accum, st);
  if (rc) return rc;
  return launch_finalize(g, radii, rotations, opacities, colors, grad_accum, grad_means2D, grad_radii,
                         grad_rotations, grad_opacities, grad_colors, st);
}

int dbmp_grads_from_accum(const dbmp_canvas* cv, const double* grad_accum, const float* radii,
                          const float* rotations, const float* opacities, const float* colors, float* grad_means2D,
                          float* grad_radii, float* grad_rotations, float* grad_opacities, float* grad_colors,
                          void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_grads_from_accum");
  if (rc) return rc;
  REQUIRE(g.N == 0 || (grad_accum && radii && rotations && opacities && colors), "dbmp_grads_from_accum: null input");
  REQUIRE(g.N == 0 || (grad_means2D && grad_radii && grad_rotations && grad_opacities && grad_colors),
          "dbmp_grads_from_accum: null output");
  return launch_finalize(g, radii, rotations, opacities, colors, grad_accum, grad_means2D, grad_radii,
                         grad_rotations, grad_opacities, grad_colors, (cudaStream_t)stream);
}

int dbmp_forward_blend(const dbmp_canvas* cv, const void* prim_info, const void* atlas, const int32_t* tile_offsets,
                       const int32_t* tile_indices, const float* colors_orig, float c_blend, float* out_color,
                       float* out_alpha, float* T_last, int32_t* last_pos, void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_forward_blend");
  if (rc) return rc;
  REQUIRE(atlas && tile_offsets && tile_indices && out_color && out_alpha && T_last && last_pos,
          "dbmp_forward_blend: null pointer");
  REQUIRE(g.N == 0 || prim_info, "dbmp_forward_blend: prim_info is null");
  REQUIRE(c_blend >= 0.f && c_blend <= 1.f, "dbmp_forward_blend: c_blend %g outside [0, 1]", (double)c_blend);
  REQUIRE(c_blend == 0.f || g.N == 0 || colors_orig, "dbmp_forward_blend: colors_orig is null with c_blend > 0");
  return launch_forward_blend(g, cv->atlas_kind, (const PrimInfo*)prim_info, atlas, tile_offsets, tile_indices,
                              out_color, out_alpha, T_last, last_pos, colors_orig, c_blend, (cudaStream_t)stream, 1,
                              0, 0);
}

int dbmp_backward_blend(const dbmp_canvas* cv, const void* prim_info, const void* atlas, const int32_t* tile_offsets,
                        const int32_t* tile_indices, const float* colors_orig, float c_blend, const float* T_last,
                        const int32_t* last_pos, const float* grad_color, const float* grad_alpha,
                        const float* radii, const float* rotations, const float* opacities, const float* colors,
                        double* grad_accum, float* grad_means2D, float* grad_radii, float* grad_rotations,
                        float* grad_opacities, float* grad_colors, void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_backward_blend");
  if (rc) return rc;
  REQUIRE(atlas && tile_offsets && tile_indices && T_last && last_pos && grad_color,
          "dbmp_backward_blend: null input");
  REQUIRE(g.N == 0 || (prim_info && radii && rotations && opacities && colors), "dbmp_backward_blend: null parameter");
  REQUIRE(g.N == 0 || (grad_accum && grad_means2D && grad_radii && grad_rotations && grad_opacities && grad_colors),
          "dbmp_backward_blend: null output");
  REQUIRE(c_blend >= 0.f && c_blend <= 1.f, "dbmp_backward_blend: c_blend %g outside [0, 1]", (double)c_blend);
  REQUIRE(c_blend == 0.f || g.N == 0 || colors_orig, "dbmp_backward_blend: colors_orig is null with c_blend > 0");
  cudaStream_t st = (cudaStream_t)stream;
  if (g.N > 0) {
    cudaError_t e = cudaMemsetAsync(grad_accum, 0, sizeof(double) * 8 * (size_t)g.N, st);
    if (e != cudaSuccess) return cuda_status(e, "cudaMemsetAsync(grad_accum)");
  }
  rc = launch_backward_blend(g, cv->atlas_kind, (const PrimInfo*)prim_info, atlas, tile_offsets, tile_indices,
                             T_last, last_pos, grad_color, grad_alpha, grad_accum, colors_orig, c_blend, st, 1, 0, 0);
  if (rc) return rc;
  return launch_finalize(g, radii, rotations, opacities, colors, grad_accum, grad_means2D, grad_radii,
                         grad_rotations, grad_opacities, grad_colors, st);
}

int dbmp_forward_batch(const dbmp_canvas* cv, int batch, const void* prim_info, const void* atlas,
                       const int32_t* tile_offsets, const int32_t* tile_indices, long long index_stride,
                       const float* colors_orig, long long colors_orig_stride, float c_blend, float* out_color,
                       float* out_alpha, float* T_last, int32_t* last_pos, void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_forward_batch");
  if (rc) return rc;
  REQUIRE(batch >= 0, "dbmp_forward_batch: batch %d < 0", batch);
  REQUIRE(index_stride >= 0 && colors_orig_stride >= 0, "dbmp_forward_batch: negative stride");
  REQUIRE(batch == 0 || (atlas && tile_offsets && tile_indices && out_color && out_alpha && T_last && last_pos),
          "dbmp_forward_batch: null pointer");
  REQUIRE(batch == 0 || g.N == 0 || prim_info, "dbmp_forward_batch: prim_info is null");
  REQUIRE(c_blend >= 0.f && c_blend <= 1.f, "dbmp_forward_batch: c_blend %g outside [0, 1]", (double)c_blend);
  REQUIRE(c_blend == 0.f || g.N == 0 || colors_orig, "dbmp_forward_batch: colors_orig is null with c_blend > 0");
  REQUIRE(((uintptr_t)prim_info & 15) == 0, "dbmp_forward_batch: prim_info must be 16-byte aligned");
  return launch_forward_blend(g, cv->atlas_kind, (const PrimInfo*)prim_info, atlas, tile_offsets, tile_indices,
                              out_color, out_alpha, T_last, last_pos, colors_orig, c_blend, (cudaStream_t)stream,
                              batch, index_stride, colors_orig_stride);
}

int dbmp_backward_batch(const dbmp_canvas* cv, int batch, const void* prim_info, const void* atlas,
                        const int32_t* tile_offsets, const int32_t* tile_indices, long long index_stride,
                        const float* colors_orig, long long colors_orig_stride, float c_blend, const float* T_last,
                        const int32_t* last_pos, const float* grad_color, const float* grad_alpha,
                        const float* radii, const float* rotations, const float* opacities, const float* colors,
                        double* grad_accum, float* grad_means2D, float* grad_radii, float* grad_rotations,
                        float* grad_opacities, float* grad_colors, void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_backward_batch");
  if (rc) return rc;
  REQUIRE(batch >= 0, "dbmp_backward_batch: batch %d < 0", batch);
  REQUIRE(index_stride >= 0 && colors_orig_stride >= 0, "dbmp_backward_batch: negative stride");
  REQUIRE(batch == 0 || (atlas && tile_offsets && tile_indices && T_last && last_pos && grad_color),
          "dbmp_backward_batch: null input");
  const bool work = batch > 0 && g.N > 0;
  REQUIRE(!work || (prim_info && radii && rotations && opacities && colors), "dbmp_backward_batch: null parameter");
  REQUIRE(!work || (grad_accum && grad_means2D && grad_radii && grad_rotations && grad_opacities && grad_colors),
          "dbmp_backward_batch: null output");
  REQUIRE(c_blend >= 0.f && c_blend <= 1.f, "dbmp_backward_batch: c_blend %g outside [0, 1]", (double)c_blend);
  REQUIRE(c_blend == 0.f || g.N == 0 || colors_orig, "dbmp_backward_batch: colors_orig is null with c_blend > 0");
  if (!work) return DBMP_OK;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(grad_accum, 0, sizeof(double) * 8 * (size_t)g.N * batch, st);
  if (e != cudaSuccess) return cuda_status(e, "cudaMemsetAsync(grad_accum)");
  rc = launch_backward_blend(g, cv->atlas_kind, (const PrimInfo*)prim_info, atlas, tile_offsets, tile_indices,
                             T_last, last_pos, grad_color, grad_alpha, grad_accum, colors_orig, c_blend, st, batch,
                             index_stride, colors_orig_stride);
  if (rc) return rc;
  // the chain rule is per primitive: the batch's (B, N) primitives are one flat array
  Geom gb = g;
  gb.N = g.N * batch;
  return launch_finalize(gb, radii, rotations, opacities, colors, grad_accum, grad_means2D, grad_radii,
                         grad_rotations, grad_opacities, grad_colors, st);
}

int dbmp_count(const dbmp_canvas* cv, const void* prim_info, const void* atlas, const int32_t* tile_offsets,
               const int32_t* tile_indices, unsigned long long* counts, void* stream) {
  Geom g;
  // t_stop = 0 is allowed here: counting without termination (every fragment)
  dbmp_canvas c2 = cv ? *cv : dbmp_canvas{};
  const bool no_stop = cv && cv->t_stop == 0.f;
  if (no_stop) c2.t_stop = 0.5f;
  int rc = make_geom(cv ? &c2 : nullptr, &g, "dbmp_count");
  if (rc) return rc;
  if (no_stop) g.t_stop = 0.f;
  REQUIRE(atlas && tile_offsets && tile_indices && counts, "dbmp_count: null pointer");
  REQUIRE(g.N == 0 || prim_info, "dbmp_count: prim_info is null");
  cudaError_t e = cudaMemsetAsync(counts, 0, 10 * sizeof(unsigned long long), (cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_status(e, "cudaMemsetAsync(counts)");
  return launch_count(g, cv->atlas_kind, (const PrimInfo*)prim_info, atlas, tile_offsets, tile_indices, counts,
                      (cudaStream_t)stream);
}

int dbmp_fused_fwd_bwd(const dbmp_canvas* cv, const void* prim_info, const void* atlas, const int32_t* tile_offsets,
                       const int32_t* tile_indices, const float* target, const float* background, float* out_image,
                       double* grad_accum, double* loss_out, const int32_t* skip_flag, void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_fused_fwd_bwd");
  if (rc) return rc;
  REQUIRE(atlas && tile_offsets && tile_indices && target && loss_out, "dbmp_fused_fwd_bwd: null input");
  REQUIRE(g.N == 0 || (prim_info && grad_accum), "dbmp_fused_fwd_bwd: null prim_info / grad_accum");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(loss_out, 0, sizeof(double), st);
  if (e == cudaSuccess && g.N > 0) e = cudaMemsetAsync(grad_accum, 0, sizeof(double) * 8 * (size_t)g.N, st);
  if (e != cudaSuccess) return cuda_status(e, "cudaMemsetAsync(fused outputs)");
  return launch_fused(g, cv->atlas_kind, (const PrimInfo*)prim_info, atlas, tile_offsets, tile_indices, target,
                      background, out_image, grad_accum, loss_out, skip_flag, st);
}

int dbmp_adam_step(const dbmp_canvas* cv, const dbmp_adam_cfg* cfg, const double* grad_accum, float* means2D,
                   float* radii, float* rotations, float* opacities, float* colors, float* adam_m, float* adam_v,
                   int32_t* step_count, const int32_t* skip_flag, void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_adam_step");
  if (rc) return rc;
  REQUIRE(cfg && step_count, "dbmp_adam_step: null cfg / step_count");
  REQUIRE(g.N == 0 || (grad_accum && means2D && radii && rotations && opacities && colors && adam_m && adam_v),
          "dbmp_adam_step: null pointer");
  REQUIRE(cfg->beta1 >= 0.f && cfg->beta1 < 1.f && cfg->beta2 >= 0.f && cfg->beta2 < 1.f && cfg->eps > 0.f,
          "dbmp_adam_step: betas must be in [0,1) and eps > 0");
  AdamArgs a;
  for (int k = 0; k < 8; ++k) a.lr[k] = cfg->lr[k];
  a.beta1 = cfg->beta1; a.beta2 = cfg->beta2; a.eps = cfg->eps;
  a.x_max = cfg->x_max; a.y_max = cfg->y_max; a.r_min = cfg->r_min; a.r_max = cfg->r_max;
  a.clamp = cfg->clamp;
  a.gamma = (cfg->lr_gamma == 0.f) ? 1.f : cfg->lr_gamma;
  REQUIRE(a.gamma > 0.f && a.gamma <= 1e6f, "dbmp_adam_step: lr_gamma %g must be positive", (double)cfg->lr_gamma);
  return launch_adam(g, a, grad_accum, means2D, radii, rotations, opacities, colors, adam_m, adam_v, step_count,
                     skip_flag, (cudaStream_t)stream);
}

int dbmp_prune(const dbmp_canvas* cv, const dbmp_prune_cfg* cfg, const int32_t* step_count, const float* pool,
               int32_t* state, float* means2D, float* radii, float* rotations, float* opacities, float* colors,
               const int32_t* skip_flag, void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_prune");
  if (rc) return rc;
  REQUIRE(cfg && step_count && state, "dbmp_prune: null cfg / step_count / state");
  REQUIRE(cfg->every >= 1 && cfg->pool_rows >= 1, "dbmp_prune: every (%d) and pool_rows (%d) must be >= 1",
          cfg->every, cfg->pool_rows);
  REQUIRE(g.N == 0 || (pool && means2D && radii && rotations && opacities && colors), "dbmp_prune: null pointer");
  PruneArgs a{cfg->every, cfg->num_iterations, cfg->no_prune_last, cfg->warmup, cfg->threshold, cfg->pool_rows};
  return launch_prune(g, a, step_count, pool, state, means2D, radii, rotations, opacities, colors, skip_flag,
                      (cudaStream_t)stream);
}

int dbmp_template_blur_scheduled(const float* templates, int P, int Ht, int Wt, const dbmp_blur_schedule* sched,
                                 const int32_t* step_count, float* out, void* stream) {
  REQUIRE(P >= 0 && Ht >= 1 && Wt >= 1, "dbmp_template_blur_scheduled: bad atlas shape %dx%dx%d", P, Ht, Wt);
  REQUIRE(sched && step_count, "dbmp_template_blur_scheduled: null schedule / step_count");
  REQUIRE(P == 0 || (templates && out && templates != out), "dbmp_template_blur_scheduled: null or in-place buffers");
  REQUIRE(sched->mode >= 0 && sched->mode <= 2, "dbmp_template_blur_scheduled: mode %d unknown", sched->mode);
  REQUIRE(sched->mode != 2 || sched->num_iterations >= 1, "dbmp_template_blur_scheduled: num_iterations must be >= 1");
  return launch_template_blur_sched(templates, P, Ht, Wt, sched, step_count, out, (cudaStream_t)stream);
}

int dbmp_psd_bboxes(const float* means2D, const float* radii, int N, int H, int W, float scale, int32_t* out_bbox,
                    int32_t* out_sizes, void* stream) {
  REQUIRE(N >= 0 && H > 0 && W > 0, "dbmp_psd_bboxes: bad sizes N=%d H=%d W=%d", N, H, W);
  REQUIRE(N == 0 || (means2D && radii && out_bbox && out_sizes), "dbmp_psd_bboxes: null pointer");
  REQUIRE(((uintptr_t)out_bbox & 15) == 0, "dbmp_psd_bboxes: out_bbox must be 16-byte aligned");
  return launch_psd_bboxes(means2D, radii, N, H, W, scale, out_bbox, out_sizes, (cudaStream_t)stream);
}

int dbmp_psd_layout(const int32_t* sizes, int N, int64_t* layer_offsets, int64_t* block_offsets,
                    int64_t* total_bytes, void* stream) {
  REQUIRE(N >= 0, "dbmp_psd_layout: N=%d", N);
  REQUIRE(block_offsets && total_bytes && (N == 0 || (sizes && layer_offsets)), "dbmp_psd_layout: null pointer");
  return launch_psd_layout(sizes, N, (long long*)layer_offsets, (long long*)block_offsets, (long long*)total_bytes,
                           (cudaStream_t)stream);
}

int dbmp_psd_layers(const float* means2D, const float* radii, const float* rotations, const float* colors,
                    const float* visibility, const float* templates, int P, int Ht, int Wt, const int32_t* sel,
                    const int32_t* bbox, const int64_t* layer_offsets, const int64_t* block_offsets, int N,
                    float scale, float alpha_max, float c_blend, const float* colors_orig, uint8_t* out,
                    void* stream) {
  REQUIRE(N >= 0 && P > 0 && Ht >= 2 && Wt >= 2, "dbmp_psd_layers: bad sizes N=%d P=%d Ht=%d Wt=%d", N, P, Ht, Wt);
  REQUIRE(N == 0 || (means2D && radii && rotations && colors && visibility && templates && sel && bbox &&
                     layer_offsets && block_offsets && out), "dbmp_psd_layers: null pointer");
  REQUIRE(((uintptr_t)bbox & 15) == 0 && ((uintptr_t)out & 3) == 0,
          "dbmp_psd_layers: bbox must be 16-byte and out 4-byte aligned");
  return launch_psd_layers(N, P, Ht, Wt, scale, alpha_max, c_blend, means2D, radii, rotations, colors, visibility,
                           templates, sel, bbox, (const long long*)layer_offsets, (const long long*)block_offsets,
                           colors_orig, out, (cudaStream_t)stream);
}

static int check_psd_rle(const char* who, const uint8_t* layers, const int32_t* sizes, const int64_t* layer_offsets,
                         const int64_t* group_base, int N, long long num_groups, int channel_order,
                         int width_limit, const uint16_t* row_bytes) {
  REQUIRE(N >= 0 && num_groups >= 0, "%s: N=%d num_groups=%lld", who, N, num_groups);
  REQUIRE(width_limit >= 1 && width_limit <= 30000, "%s: width_limit %d outside [1, 30000] (PSD limit)", who,
          width_limit);
  REQUIRE(((unsigned)channel_order & ~0x03030303u) == 0, "%s: channel_order 0x%08x: each byte must be 0..3", who,
          (unsigned)channel_order);
  if (N == 0 || num_groups == 0) return DBMP_OK;
  REQUIRE(layers && sizes && layer_offsets && group_base && row_bytes, "%s: null pointer", who);
  REQUIRE(((uintptr_t)layers & 3) == 0 && ((uintptr_t)sizes & 3) == 0 && ((uintptr_t)row_bytes & 7) == 0,
          "%s: layers and sizes must be 4-byte and row_bytes 8-byte aligned", who);
  return DBMP_OK;
}

int dbmp_psd_rle_count(const uint8_t* layers, const int32_t* sizes, const int64_t* layer_offsets,
                       const int64_t* group_base, int N, long long num_groups, int channel_order, int width_limit,
                       uint16_t* row_bytes, int32_t* group_totals, int32_t* alpha_any, void* stream) {
  int rc = check_psd_rle("dbmp_psd_rle_count", layers, sizes, layer_offsets, group_base, N, num_groups,
                         channel_order, width_limit, row_bytes);
  if (rc != DBMP_OK) return rc;
  if (N == 0 || num_groups == 0) return DBMP_OK;
  REQUIRE(group_totals && ((uintptr_t)group_totals & 15) == 0,
          "dbmp_psd_rle_count: group_totals must be non-null and 16-byte aligned");
  return launch_psd_rle(false, layers, sizes, (const long long*)layer_offsets, (const long long*)group_base, N,
                        num_groups, (unsigned)channel_order, width_limit, (unsigned short*)row_bytes, group_totals,
                        alpha_any, nullptr, nullptr, nullptr, 0, (cudaStream_t)stream);
}

int dbmp_psd_rle_write(const uint8_t* layers, const int32_t* sizes, const int64_t* layer_offsets,
                       const int64_t* group_base, int N, long long num_groups, int channel_order, int width_limit,
                       const uint16_t* row_bytes, const int64_t* channel_offsets, const int64_t* group_offsets,
                       uint8_t* out, long long out_bytes, void* stream) {
  int rc = check_psd_rle("dbmp_psd_rle_write", layers, sizes, layer_offsets, group_base, N, num_groups,
                         channel_order, width_limit, row_bytes);
  if (rc != DBMP_OK) return rc;
  REQUIRE(out_bytes >= 0, "dbmp_psd_rle_write: out_bytes %lld < 0", out_bytes);
  if (N == 0 || num_groups == 0) return DBMP_OK;
  REQUIRE(channel_offsets && group_offsets && (out || out_bytes == 0), "dbmp_psd_rle_write: null pointer");
  return launch_psd_rle(true, layers, sizes, (const long long*)layer_offsets, (const long long*)group_base, N,
                        num_groups, (unsigned)channel_order, width_limit, (unsigned short*)row_bytes, nullptr,
                        nullptr, (const long long*)channel_offsets, (const long long*)group_offsets, out, out_bytes,
                        (cudaStream_t)stream);
}

}  // extern "C"
