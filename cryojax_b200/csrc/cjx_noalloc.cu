// cjx_slice_ctf_forward_noalloc: the resize path of cjx_slice_ctf_forward
// for callers that cannot allocate device memory, because the host runtime
// that calls them owns every allocation (an XLA custom call with no scratch
// allocator, a real-time pipeline that forbids cudaMalloc after start-up) or
// because they run where allocating is not allowed.  The scratch lives in a
// fixed array inside this library, so the caller passes only inputs and
// outputs.
//
// Limits and sharing:
//  - the array holds CJX_NOALLOC_SCRATCH_BYTES (32 MiB); every GPU that loads
//    the library keeps it until the process exits;
//  - every call on a device uses the same array, so calls that overlap on
//    the GPU (different streams, or different host threads) race and must be
//    serialised by the caller;
//  - nothing in the array needs to start at zero: each call writes every
//    element it later reads, and later calls overwrite what earlier ones left.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "cjx_common.cuh"

namespace cjx {

int make_geom(const cjx_slice_desc* d, SliceGeom* g);
bool needs_resize(const SliceGeom& g);
size_t workspace_per_image(const SliceGeom& g);
int check_alignment(uint32_t flags, const void* grid, const void* out);
int launch_forward(const SliceGeom& g, const float2* grid, const cjx_image_params* params, const int32_t* order,
                   int64_t n_images, float2* out, void* workspace, int64_t chunk, cudaStream_t stream,
                   const Tuning& tn);

static __device__ __align__(256) unsigned char g_noalloc_scratch[CJX_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mutex;
static void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device.  Looked up once
// per device (the host-side symbol is only a stand-in, never a device
// address) and cached for the life of the process.  The cache does not
// survive a reset of the device's primary context (cudaDeviceReset, or the
// context being destroyed and re-created): after one, the library reloads on
// that device and the cached address no longer names the array, so a process
// that resets a device must not call this entry point on it again.
static int noalloc_scratch(void** ptr) {
  int dev = 0;
  if (int e = check_cuda(cudaGetDevice(&dev), "cudaGetDevice")) return e;
  if (dev < 0 || dev >= kMaxDevices) return fail(CJX_ERR_UNSUPPORTED, "device index beyond the 64 supported");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    if (int e = check_cuda(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)")) return e;
    g_noalloc_ptr[dev] = p;
  }
  *ptr = g_noalloc_ptr[dev];
  return CJX_OK;
}

}  // namespace cjx

using namespace cjx;

extern "C" int cjx_slice_ctf_forward_noalloc(const cjx_slice_desc* desc, const void* grid,
                                             const cjx_image_params* params, const int32_t* order,
                                             int64_t n_images, void* out, void* stream) {
  SliceGeom g;
  if (int e = make_geom(desc, &g)) return e;
  if (n_images < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "n_images < 0");
  if (n_images == 0) return CJX_OK;
  if (!grid || !params || !out) return fail(CJX_ERR_INVALID_ARGUMENT, "grid, params and out must be non-NULL");
  if (int e = check_alignment(g.flags, grid, out)) return e;
  if (!needs_resize(g))  // the fused no-resize kernel uses no scratch
    return launch_forward(g, static_cast<const float2*>(grid), params, order, n_images,
                          static_cast<float2*>(out), nullptr, 0, static_cast<cudaStream_t>(stream), current_tuning());
  const size_t per = workspace_per_image(g);
  if (per > CJX_NOALLOC_SCRATCH_BYTES)
    return fail(CJX_ERR_UNSUPPORTED, "one image needs more scratch than CJX_NOALLOC_SCRATCH_BYTES");
  int64_t chunk = (int64_t)(CJX_NOALLOC_SCRATCH_BYTES / per);
  if (desc->images_per_chunk > 0) {
    if ((size_t)desc->images_per_chunk * per > CJX_NOALLOC_SCRATCH_BYTES)
      return fail(CJX_ERR_UNSUPPORTED, "images_per_chunk needs more scratch than CJX_NOALLOC_SCRATCH_BYTES");
    chunk = desc->images_per_chunk;
  }
  chunk = std::min<int64_t>(std::min<int64_t>(chunk, n_images), 65535);
  void* scratch = nullptr;
  if (int e = noalloc_scratch(&scratch)) return e;
  return launch_forward(g, static_cast<const float2*>(grid), params, order, n_images, static_cast<float2*>(out),
                        scratch, chunk, static_cast<cudaStream_t>(stream), current_tuning());
}
