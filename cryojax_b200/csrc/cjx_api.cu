// extern "C" entry points of libcryojax_b200 (declared in include/cryojax_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "cjx_common.cuh"

namespace cjx {

int make_geom(const cjx_slice_desc* d, SliceGeom* g);
bool needs_resize(const SliceGeom& g);
size_t workspace_per_image(const SliceGeom& g);
int check_alignment(uint32_t flags, const void* grid, const void* out);
int64_t default_chunk(const SliceGeom& g, int64_t n_images);
int launch_forward(const SliceGeom& g, const float2* grid, const cjx_image_params* params, const int32_t* order,
                   int64_t n_images, float2* out, void* workspace, int64_t chunk, cudaStream_t stream,
                   const Tuning& tn);
int64_t tuning_get(int key);
size_t search_candidate_bytes(const SliceGeom& g, size_t per_image_fwd);
size_t search_workspace_bytes(const SliceGeom& g, size_t per_fwd, int64_t chunk, int64_t n_images);
int launch_search(const SliceGeom& g, size_t per_fwd, int64_t chunk, const float2* grid,
                  const cjx_image_params* image_params, const double* rot, const int32_t* candidates,
                  int64_t n_images, int K, const float2* obs, float* scores, float* best_score, int32_t* best_orient,
                  void* workspace, cudaStream_t stream, const Tuning& tn);
int launch_loss_grad(const SliceGeom& g, const float2* grid, const cjx_image_params* params, const int32_t* order,
                     int64_t n_images, const float2* obs, double* grads, float2* grad_grid, float2* acc,
                     void* workspace, int64_t chunk, cudaStream_t stream, const Tuning& tn);
size_t loss_accumulator_bytes(int n);
int tuning_set(int key, int64_t value);
int launch_read_probe(const void* buf, size_t bytes, int passes, void* sink, cudaStream_t stream);
size_t bricked_elements(int n);
int launch_brick_volume(int n, const float2* grid, float2* bricked, cudaStream_t stream);
int launch_brick_volume_pairs(int n, const float2* grid, float4* out, cudaStream_t stream);
size_t spline_workspace_elements(int n);
int launch_render_gaussians(const cjx_render_desc* d, const float* positions, const float* amplitudes,
                            const float* variances, int64_t n_atoms, float* grid, cudaStream_t stream);
int launch_spline_coefficients(int n, const float2* grid, float2* coef, float2* work, cudaStream_t stream);

static thread_local std::string g_last_error;

void set_last_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return CJX_OK;
  return fail(CJX_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

static int64_t chunk_for(const SliceGeom& g, const cjx_slice_desc* d, int64_t n_images) {
  if (d->images_per_chunk > 0) return std::min<int64_t>(d->images_per_chunk, std::max<int64_t>(n_images, 1));
  return default_chunk(g, n_images);
}

// The kernels read a grid with 8-byte loads (16-byte loads in the x-pair
// layout) and write complex64 outputs with 8-byte stores: reject pointers
// that would fault those accesses.
int check_alignment(uint32_t flags, const void* grid, const void* out) {
  const uintptr_t g = reinterpret_cast<uintptr_t>(grid), o = reinterpret_cast<uintptr_t>(out);
  if ((flags & CJX_GRID_BRICKED_PAIRS) && (g & 15))
    return fail(CJX_ERR_INVALID_ARGUMENT, "an x-pair grid must be 16-byte aligned");
  if (g & 7) return fail(CJX_ERR_INVALID_ARGUMENT, "grid must be 8-byte aligned");
  if (o & 7) return fail(CJX_ERR_INVALID_ARGUMENT, "the output array must be 8-byte aligned");
  return CJX_OK;
}

}  // namespace cjx

using namespace cjx;

extern "C" {

int cjx_get_version(void) { return CJX_ABI_VERSION; }

const char* cjx_get_last_error(void) { return g_last_error.c_str(); }

int cjx_slice_ctf_workspace_size(const cjx_slice_desc* desc, int64_t n_images, size_t* bytes) {
  if (!bytes) return fail(CJX_ERR_INVALID_ARGUMENT, "bytes is NULL");
  if (n_images < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "n_images < 0");
  SliceGeom g;
  if (int e = make_geom(desc, &g)) return e;
  *bytes = (needs_resize(g) && n_images > 0) ? (size_t)chunk_for(g, desc, n_images) * workspace_per_image(g) : 0;
  return CJX_OK;
}

int cjx_slice_ctf_forward(const cjx_slice_desc* desc, const void* grid, const cjx_image_params* params,
                          const int32_t* order, int64_t n_images, void* out, void* workspace, size_t workspace_bytes,
                          void* stream) {
  SliceGeom g;
  if (int e = make_geom(desc, &g)) return e;
  if (n_images < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "n_images < 0");
  if (n_images == 0) return CJX_OK;
  if (!grid || !params || !out) return fail(CJX_ERR_INVALID_ARGUMENT, "grid, params and out must be non-NULL");
  if (int e = check_alignment(g.flags, grid, out)) return e;
  int64_t chunk = 0;
  if (needs_resize(g)) {
    chunk = chunk_for(g, desc, n_images);
    const size_t need = (size_t)chunk * workspace_per_image(g);
    if (!workspace || workspace_bytes < need)
      return fail(CJX_ERR_WORKSPACE, "workspace smaller than cjx_slice_ctf_workspace_size()");
  }
  return launch_forward(g, static_cast<const float2*>(grid), params, order, n_images, static_cast<float2*>(out),
                        workspace, chunk, static_cast<cudaStream_t>(stream), current_tuning());
}

int cjx_slice_ctf_forward_filtered(const cjx_slice_desc* desc, const void* grid, const cjx_image_params* params,
                                   const int32_t* order, int64_t n_images, const float* filter, void* out,
                                   void* workspace, size_t workspace_bytes, void* stream) {
  SliceGeom g;
  if (int e = make_geom(desc, &g)) return e;
  if (n_images < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "n_images < 0");
  if (n_images == 0) return CJX_OK;
  if (!grid || !params || !out) return fail(CJX_ERR_INVALID_ARGUMENT, "grid, params and out must be non-NULL");
  if (int e = check_alignment(g.flags, grid, out)) return e;
  g.filter = filter;
  int64_t chunk = 0;
  if (needs_resize(g)) {
    chunk = chunk_for(g, desc, n_images);
    if (!workspace || workspace_bytes < (size_t)chunk * workspace_per_image(g))
      return fail(CJX_ERR_WORKSPACE, "workspace smaller than cjx_slice_ctf_workspace_size()");
  }
  return launch_forward(g, static_cast<const float2*>(grid), params, order, n_images, static_cast<float2*>(out),
                        workspace, chunk, static_cast<cudaStream_t>(stream), current_tuning());
}

static int group_plan(const cjx_slice_group& gr, SliceGeom* g, int64_t* chunk, size_t* need) {
  if (int e = make_geom(&gr.desc, g)) return e;
  if (gr.n_images < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "group n_images < 0");
  const bool resize = needs_resize(*g) && gr.n_images > 0;  // an empty group needs no scratch
  *chunk = resize ? chunk_for(*g, &gr.desc, gr.n_images) : 0;
  *need = resize ? (size_t)*chunk * workspace_per_image(*g) : 0;
  return CJX_OK;
}

int cjx_slice_ctf_multi_workspace_size(const cjx_slice_group* groups, int n_groups, size_t* bytes) {
  if (!bytes || (!groups && n_groups > 0) || n_groups < 0)
    return fail(CJX_ERR_INVALID_ARGUMENT, "need groups, n_groups >= 0 and bytes");
  size_t mx = 0;
  for (int i = 0; i < n_groups; ++i) {
    SliceGeom g;
    int64_t chunk;
    size_t need;
    if (int e = group_plan(groups[i], &g, &chunk, &need)) return e;
    mx = std::max(mx, need);
  }
  *bytes = mx;
  return CJX_OK;
}

int cjx_slice_ctf_forward_multi(const cjx_slice_group* groups, int n_groups, void* workspace,
                                size_t workspace_bytes, void* stream) {
  if ((!groups && n_groups > 0) || n_groups < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "need groups, n_groups >= 0");
  // validate every group before launching anything
  for (int i = 0; i < n_groups; ++i) {
    const cjx_slice_group& gr = groups[i];
    SliceGeom g;
    int64_t chunk;
    size_t need;
    if (int e = group_plan(gr, &g, &chunk, &need)) return e;
    if (gr.n_images > 0 && (!gr.grid || !gr.params || !gr.out))
      return fail(CJX_ERR_INVALID_ARGUMENT, "group grid, params and out must be non-NULL");
    if (gr.n_images > 0)
      if (int e = check_alignment(g.flags, gr.grid, gr.out)) return e;
    if (need && (!workspace || workspace_bytes < need))
      return fail(CJX_ERR_WORKSPACE, "workspace smaller than cjx_slice_ctf_multi_workspace_size()");
    if (gr.tuning_valid) {
      if (gr.gather_ilp != 1 && gr.gather_ilp != 2 && gr.gather_ilp != 4)
        return fail(CJX_ERR_INVALID_ARGUMENT, "group gather_ilp must be 1, 2 or 4");
      if (gr.gather_tile < 0 || gr.gather_tile > 3)
        return fail(CJX_ERR_INVALID_ARGUMENT, "group gather_tile must be 0, 1, 2 or 3");
    }
  }
  const Tuning base = current_tuning();
  if (base.multi_waves && n_groups <= kMaxWaveGroups) {
    // every group on the fused register-FFT path with one grid layout: one launch per pass for all of them
    WaveInput in[kMaxWaveGroups];
    int n_in = 0;
    bool eligible = true;
    const uint32_t layout_bits = CJX_GRID_BRICKED | CJX_GRID_BRICKED_PAIRS;
    uint32_t layout = 0;
    for (int i = 0; i < n_groups && eligible; ++i) {
      const cjx_slice_group& gr = groups[i];
      if (gr.n_images == 0) continue;
      SliceGeom g;
      int64_t chunk;
      size_t need;
      group_plan(gr, &g, &chunk, &need);
      if (n_in == 0) layout = g.flags & layout_bits;
      eligible = wave_eligible(g, base) && (g.flags & layout_bits) == layout;
      in[n_in++] = WaveInput{g, static_cast<const float2*>(gr.grid), gr.params, gr.order,
                             static_cast<float2*>(gr.out), gr.n_images};
    }
    int64_t per_wave[kMaxWaveGroups];
    if (eligible && n_in > 0 && plan_waves(in, n_in, workspace_bytes, per_wave) > 0)
      return launch_forward_waves(in, n_in, workspace, workspace_bytes, static_cast<cudaStream_t>(stream), base);
  }
  for (int i = 0; i < n_groups; ++i) {
    const cjx_slice_group& gr = groups[i];
    if (gr.n_images == 0) continue;
    SliceGeom g;
    int64_t chunk;
    size_t need;
    group_plan(gr, &g, &chunk, &need);
    Tuning tn = base;
    if (gr.tuning_valid) {
      if (gr.desc.flags & CJX_GRID_SPLINE)
        tn.spline_ilp = gr.gather_ilp;
      else
        tn.ilp = gr.gather_ilp;
      tn.tile = gr.gather_tile;
    }
    if (int e = launch_forward(g, static_cast<const float2*>(gr.grid), gr.params, gr.order, gr.n_images,
                               static_cast<float2*>(gr.out), workspace, chunk, static_cast<cudaStream_t>(stream), tn))
      return e;
  }
  return CJX_OK;
}

int cjx_bricked_volume_size(int n, size_t* bytes) {
  if (!bytes) return fail(CJX_ERR_INVALID_ARGUMENT, "bytes is NULL");
  if (n < 2 || n > CJX_MAX_SIDE + 2) return fail(CJX_ERR_UNSUPPORTED, "n must be in [2, CJX_MAX_SIDE + 2]");
  *bytes = bricked_elements(n) * sizeof(float2);
  return CJX_OK;
}

int cjx_brick_volume(int n, const void* grid, void* bricked, void* stream) {
  if (n < 2 || n > CJX_MAX_SIDE + 2) return fail(CJX_ERR_UNSUPPORTED, "n must be in [2, CJX_MAX_SIDE + 2]");
  if (!grid || !bricked) return fail(CJX_ERR_INVALID_ARGUMENT, "grid and bricked must be non-NULL");
  if (grid == bricked) return fail(CJX_ERR_INVALID_ARGUMENT, "grid and bricked must not alias");
  return launch_brick_volume(n, static_cast<const float2*>(grid), static_cast<float2*>(bricked),
                             static_cast<cudaStream_t>(stream));
}

int cjx_brick_volume_pairs(int n, const void* grid, void* pairs, void* stream) {
  if (n < 2 || n > CJX_MAX_SIDE + 2) return fail(CJX_ERR_UNSUPPORTED, "n must be in [2, CJX_MAX_SIDE + 2]");
  if (!grid || !pairs) return fail(CJX_ERR_INVALID_ARGUMENT, "grid and pairs must be non-NULL");
  if (grid == pairs) return fail(CJX_ERR_INVALID_ARGUMENT, "grid and pairs must not alias");
  return launch_brick_volume_pairs(n, static_cast<const float2*>(grid), static_cast<float4*>(pairs),
                                   static_cast<cudaStream_t>(stream));
}

int cjx_spline_coefficients_workspace_size(int n, size_t* bytes) {
  if (!bytes) return fail(CJX_ERR_INVALID_ARGUMENT, "bytes is NULL");
  if (n < 4 || n > CJX_MAX_SIDE) return fail(CJX_ERR_UNSUPPORTED, "n must be in [4, CJX_MAX_SIDE]");
  *bytes = spline_workspace_elements(n) * sizeof(float2);
  return CJX_OK;
}

int cjx_spline_coefficients(int n, const void* grid, void* coefficients, void* workspace, size_t workspace_bytes,
                            void* stream) {
  if (n < 4 || n > CJX_MAX_SIDE) return fail(CJX_ERR_UNSUPPORTED, "n must be in [4, CJX_MAX_SIDE]");
  if (!grid || !coefficients) return fail(CJX_ERR_INVALID_ARGUMENT, "grid and coefficients must be non-NULL");
  if (grid == coefficients) return fail(CJX_ERR_INVALID_ARGUMENT, "grid and coefficients must not alias");
  if (!workspace || workspace_bytes < spline_workspace_elements(n) * sizeof(float2))
    return fail(CJX_ERR_WORKSPACE, "workspace smaller than cjx_spline_coefficients_workspace_size()");
  return launch_spline_coefficients(n, static_cast<const float2*>(grid), static_cast<float2*>(coefficients),
                                    static_cast<float2*>(workspace), static_cast<cudaStream_t>(stream));
}

int cjx_render_gaussians(const cjx_render_desc* desc, const float* positions, const float* amplitudes,
                         const float* variances, int64_t n_atoms, float* grid, void* stream) {
  if (!desc) return fail(CJX_ERR_INVALID_ARGUMENT, "desc is NULL");
  if (desc->nz < 1 || desc->ny < 1 || desc->nx < 1 || desc->nz > 4096 || desc->ny > 4096 || desc->nx > 4096)
    return fail(CJX_ERR_INVALID_ARGUMENT, "grid sides must be in [1, 4096]");
  if (desc->n_gaussians < 1 || desc->n_gaussians > CJX_RENDER_MAX_GAUSSIANS)
    return fail(CJX_ERR_INVALID_ARGUMENT, "n_gaussians must be in [1, CJX_RENDER_MAX_GAUSSIANS]");
  if (!(desc->voxel_size > 0.f) || desc->cutoff_sigmas < 0.f)
    return fail(CJX_ERR_INVALID_ARGUMENT, "need voxel_size > 0 and cutoff_sigmas >= 0");
  if (desc->flags & ~CJX_RENDER_ACCUMULATE) return fail(CJX_ERR_INVALID_ARGUMENT, "unknown flag bits");
  if (n_atoms < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "n_atoms < 0");
  if (!grid) return fail(CJX_ERR_INVALID_ARGUMENT, "grid must be non-NULL");
  if (n_atoms > 0 && (!positions || !amplitudes || !variances))
    return fail(CJX_ERR_INVALID_ARGUMENT, "positions, amplitudes and variances must be non-NULL");
  return launch_render_gaussians(desc, positions, amplitudes, variances, n_atoms, grid,
                                 static_cast<cudaStream_t>(stream));
}

int cjx_slice_ctf_loss_workspace_size(const cjx_slice_desc* desc, int64_t n_images, size_t* bytes) {
  if (!bytes) return fail(CJX_ERR_INVALID_ARGUMENT, "bytes is NULL");
  if (n_images < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "n_images < 0");
  SliceGeom g;
  if (int e = make_geom(desc, &g)) return e;
  if (!needs_resize(g)) return fail(CJX_ERR_UNSUPPORTED, "loss gradient needs the resize path ((Py, Px) != (N, N))");
  if ((g.flags & CJX_EWALD_SPHERE) && !(g.flags & CJX_APPLY_CTF))
    return fail(CJX_ERR_UNSUPPORTED, "loss gradient on the Ewald sphere needs the contrast transfer (CJX_APPLY_CTF)");
  const size_t acc = (g.flags & CJX_GRID_SPLINE) ? 0 : loss_accumulator_bytes(g.n);
  *bytes = n_images > 0 ? (size_t)chunk_for(g, desc, n_images) * workspace_per_image(g) + acc : 0;
  return CJX_OK;
}

int cjx_slice_ctf_loss_grad(const cjx_slice_desc* desc, const void* grid, const cjx_image_params* params,
                            const int32_t* order, int64_t n_images, const void* observed, double* image_grads,
                            void* grid_grad, void* workspace, size_t workspace_bytes, void* stream) {
  SliceGeom g;
  if (int e = make_geom(desc, &g)) return e;
  if (n_images < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "n_images < 0");
  if (n_images == 0) return CJX_OK;
  if (!needs_resize(g)) return fail(CJX_ERR_UNSUPPORTED, "loss gradient needs the resize path ((Py, Px) != (N, N))");
  if ((g.flags & CJX_EWALD_SPHERE) && !(g.flags & CJX_APPLY_CTF))
    return fail(CJX_ERR_UNSUPPORTED, "loss gradient on the Ewald sphere needs the contrast transfer (CJX_APPLY_CTF)");
  if (!grid || !params || !observed || !image_grads)
    return fail(CJX_ERR_INVALID_ARGUMENT, "grid, params, observed and image_grads must be non-NULL");
  if (int e = check_alignment(g.flags, grid, observed)) return e;
  if (reinterpret_cast<uintptr_t>(grid_grad) & 7) return fail(CJX_ERR_INVALID_ARGUMENT, "grid_grad must be 8-byte aligned");
  const int64_t chunk = chunk_for(g, desc, n_images);
  const size_t scratch = (size_t)chunk * workspace_per_image(g);
  if (!workspace || workspace_bytes < scratch)
    return fail(CJX_ERR_WORKSPACE, "workspace smaller than cjx_slice_ctf_loss_workspace_size()");
  // the grid scatter's bricked accumulator, when the workspace has room for it (voxel grids)
  float2* acc = nullptr;
  if (grid_grad && !(g.flags & CJX_GRID_SPLINE) && workspace_bytes >= scratch + loss_accumulator_bytes(g.n)) {
    const uintptr_t a = (reinterpret_cast<uintptr_t>(workspace) + scratch + 255) & ~(uintptr_t)255;
    acc = reinterpret_cast<float2*>(a);
  }
  return launch_loss_grad(g, static_cast<const float2*>(grid), params, order, n_images,
                          static_cast<const float2*>(observed), image_grads, static_cast<float2*>(grid_grad), acc,
                          workspace, chunk, static_cast<cudaStream_t>(stream), current_tuning());
}

static int search_plan(const cjx_search_desc* d, SliceGeom* g, int* K, int64_t* chunk, size_t* bytes) {
  if (!d) return fail(CJX_ERR_INVALID_ARGUMENT, "desc is NULL");
  if (int e = make_geom(&d->slice, g)) return e;
  if (!needs_resize(*g)) return fail(CJX_ERR_UNSUPPORTED, "search needs the resize path ((Py, Px) != (N, N))");
  if ((g->flags & CJX_EWALD_SPHERE) && !(g->flags & CJX_APPLY_CTF))
    return fail(CJX_ERR_UNSUPPORTED, "search on the Ewald sphere needs the contrast transfer (CJX_APPLY_CTF)");
  if (d->n_images < 0 || d->n_orientations < 1 || d->candidates_per_image < 0)
    return fail(CJX_ERR_INVALID_ARGUMENT, "need n_images >= 0, n_orientations >= 1, candidates_per_image >= 0");
  if (d->n_orientations > 2147483647LL) return fail(CJX_ERR_UNSUPPORTED, "too many orientations");
  *K = d->candidates_per_image ? d->candidates_per_image : (int)d->n_orientations;
  const size_t per = search_candidate_bytes(*g, workspace_per_image(*g));
  int64_t c = (int64_t)((size_t)tuning_get(CJX_TUNE_CHUNK_BYTES) / per);
  const int64_t total = std::max<int64_t>(1, d->n_images * (int64_t)*K);
  c = std::max<int64_t>(1, std::min<int64_t>(std::min<int64_t>(c, 65535), total));
  if (d->slice.images_per_chunk > 0) c = std::min<int64_t>(d->slice.images_per_chunk, total);
  *chunk = c;
  *bytes = search_workspace_bytes(*g, workspace_per_image(*g), c, std::max<int64_t>(d->n_images, 1));
  return CJX_OK;
}

int cjx_search_workspace_size(const cjx_search_desc* desc, size_t* bytes) {
  if (!bytes) return fail(CJX_ERR_INVALID_ARGUMENT, "bytes is NULL");
  SliceGeom g;
  int K;
  int64_t chunk;
  return search_plan(desc, &g, &K, &chunk, bytes);
}

int cjx_search(const cjx_search_desc* desc, const void* grid, const cjx_image_params* image_params,
               const double* rotations, const int32_t* candidates, const void* observed, float* scores,
               float* best_score, int32_t* best_orientation, void* workspace, size_t workspace_bytes, void* stream) {
  SliceGeom g;
  int K;
  int64_t chunk;
  size_t need;
  if (int e = search_plan(desc, &g, &K, &chunk, &need)) return e;
  if (desc->n_images == 0) return CJX_OK;
  if (!grid || !image_params || !rotations || !observed)
    return fail(CJX_ERR_INVALID_ARGUMENT, "grid, image_params, rotations and observed must be non-NULL");
  if (int e = check_alignment(g.flags, grid, observed)) return e;
  if (!workspace || workspace_bytes < need) return fail(CJX_ERR_WORKSPACE, "workspace smaller than cjx_search_workspace_size()");
  return launch_search(g, workspace_per_image(g), chunk, static_cast<const float2*>(grid), image_params, rotations,
                       candidates, desc->n_images, K, static_cast<const float2*>(observed), scores, best_score,
                       best_orientation, workspace, static_cast<cudaStream_t>(stream), current_tuning());
}

int cjx_tuning_set(int key, int64_t value) { return tuning_set(key, value); }

int cjx_tuning_get(int key, int64_t* value) {
  if (!value) return fail(CJX_ERR_INVALID_ARGUMENT, "value is NULL");
  const int64_t v = tuning_get(key);
  if (v < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "unknown tuning key");
  *value = v;
  return CJX_OK;
}

int cjx_probe_read_bandwidth(const void* buf, size_t bytes, int passes, void* sink, void* stream) {
  if (!buf || !sink || bytes < 16 || passes < 1)
    return fail(CJX_ERR_INVALID_ARGUMENT, "need buf, sink, bytes >= 16, passes >= 1");
  return launch_read_probe(buf, bytes, passes, sink, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
