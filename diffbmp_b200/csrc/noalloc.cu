// dbmp_backward_noalloc: the backward for callers that cannot allocate device
// memory.
//
// Some host applications do not own the device allocator: a compositor or
// renderer plug-in whose host hands it buffers but forbids cudaMalloc, or a
// frame loop that must not allocate once running.  dbmp_backward needs a
// caller-provided (N,8) f64 scratch for the per-primitive gradient sums; this
// entry point instead keeps that scratch in a fixed array of this library's
// device module, so the caller passes only inputs and outputs.
//
// The array holds kNoAllocMaxPrims primitives (4 MiB of device memory on
// every GPU that loads the library, held until the process exits).  Its device
// address is looked up on the first call made with a device current, and again
// whenever that device's context has changed since (a cudaDeviceReset reloads
// the module, which can move the array); make the first call on each device
// before any stream capture.  Every call shares the one array and zeroes it
// before use: calls that overlap on the GPU (on different streams, or from
// different host threads) race and must be serialised by the caller.
#include <cuda.h>

#include <mutex>

#include "dbmp_internal.cuh"

namespace dbmp {

constexpr int kNoAllocMaxPrims = 65536;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_accum[(size_t)kNoAllocMaxPrims * 8];

int make_geom(const dbmp_canvas* cv, Geom* g, const char* who);
int launch_backward(const Geom& g, int kind, const PrimInfo* prims, const void* atlas, const int* offs,
                    const int* idx, const float* T_last, const int* last_pos, const float* grad_color,
                    const float* grad_alpha, double* gacc, cudaStream_t st);
int launch_finalize(const Geom& g, const float* radii, const float* rot, const float* opac, const float* colors,
                    const double* gacc, float* gm, float* gr, float* grot, float* go, float* gc, cudaStream_t st);

// Unique id of the calling thread's current CUDA context (0 if none or if the
// driver does not provide it).  The driver entry points are taken through the
// runtime, so the library needs no link-time dependency on the driver library.
static unsigned long long current_context_id() {
  using GetCurrentFn = CUresult (*)(CUcontext*);
  using GetIdFn = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrentFn>(p);
    p = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetIdFn>(p);
  });
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx != nullptr &&
      get_id(ctx, &id) == CUDA_SUCCESS)
    return id;
  return 0;
}

// Device address of g_noalloc_accum on the current device (host code must not
// use the symbol itself: on the host it is only a stand-in, not a device
// address).  Cached per device together with the id of the context it was
// looked up in; a different context (or an unknown one) looks it up again.
static int noalloc_scratch(double** out) {
  static std::mutex mu;
  static double* addr[kMaxDevices] = {};
  static unsigned long long ctx_of[kMaxDevices] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, "dbmp_backward_noalloc: cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("dbmp_backward_noalloc: device %d beyond the %d supported", dev, kMaxDevices);
    return DBMP_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(mu);
  const unsigned long long ctx = current_context_id();
  if (addr[dev] == nullptr || ctx == 0 || ctx != ctx_of[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_accum);   // also makes the device's context current
    if (e != cudaSuccess) return cuda_status(e, "dbmp_backward_noalloc: cudaGetSymbolAddress");
    addr[dev] = static_cast<double*>(p);
    ctx_of[dev] = current_context_id();
  }
  *out = addr[dev];
  return DBMP_OK;
}

}  // namespace dbmp

using namespace dbmp;

extern "C" int dbmp_backward_noalloc_max_prims(void) { return kNoAllocMaxPrims; }

extern "C" int dbmp_backward_noalloc(const dbmp_canvas* cv, const void* prim_info, const void* atlas,
                                     const int32_t* tile_offsets, const int32_t* tile_indices,
                                     const float* T_last, const int32_t* last_pos, const float* grad_color,
                                     const float* grad_alpha, const float* radii, const float* rotations,
                                     const float* opacities, const float* colors, float* grad_means2D,
                                     float* grad_radii, float* grad_rotations, float* grad_opacities,
                                     float* grad_colors, void* stream) {
  Geom g;
  int rc = make_geom(cv, &g, "dbmp_backward_noalloc");
  if (rc) return rc;
  if (g.N > kNoAllocMaxPrims) {
    set_error("dbmp_backward_noalloc: %d primitives exceed the fixed scratch of %d; use dbmp_backward with "
              "caller-allocated scratch", g.N, kNoAllocMaxPrims);
    return DBMP_ERR_CAPACITY;
  }
  if (!(atlas && tile_offsets && tile_indices && T_last && last_pos && grad_color)) {
    set_error("dbmp_backward_noalloc: null input");
    return DBMP_ERR_INVALID;
  }
  if (g.N > 0 && !(prim_info && radii && rotations && opacities && colors && grad_means2D && grad_radii &&
                   grad_rotations && grad_opacities && grad_colors)) {
    set_error("dbmp_backward_noalloc: null parameter or output");
    return DBMP_ERR_INVALID;
  }
  double* scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (g.N > 0) {
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(double) * 8 * (size_t)g.N, st);
    if (e != cudaSuccess) return cuda_status(e, "dbmp_backward_noalloc: cudaMemsetAsync");
  }
  rc = launch_backward(g, cv->atlas_kind, (const PrimInfo*)prim_info, atlas, tile_offsets, tile_indices, T_last,
                       last_pos, grad_color, grad_alpha, scratch, st);
  if (rc) return rc;
  return launch_finalize(g, radii, rotations, opacities, colors, scratch, grad_means2D, grad_radii, grad_rotations,
                         grad_opacities, grad_colors, st);
}
