// Gaussian-mixture rendering to a real-space voxel grid (sm_100a).
//
// cryojax/simulator/_volume_rendering/gaussian_rendering.py:196-336
// (GaussianMixtureRenderFn): voxel (z, y, x) holds
//   sum over atoms and their Gaussians g of  a_g / (2 dx)^3 * Ix * Iy * Iz,
//   Ix = erf(s_g (L_x - p_x + dx)) - erf(s_g (L_x - p_x)),  s_g = 1 / sqrt(2 var_g)
// (the reference's 2 pi / sqrt(B) with B = 8 pi^2 var), L the voxel's left
// edge (i - D/2) dx - dx/2.  The reference evaluates every voxel against
// every atom (a matmul per z-plane); here each atom is splatted: one CTA
// per atom computes its per-axis integrals over the window where its
// Gaussians exceed cutoff standard deviations (plus one voxel), in 64-voxel
// sub-boxes staged in shared memory, and adds each voxel's sum with a
// fire-and-forget float atomic.  Outside the window every axis integral is
// below erfc(cutoff / sqrt 2) (about 3e-12 at the default 7).
#include <algorithm>

#include "cjx_common.cuh"
#include "cjx_profile.cuh"

namespace cjx {

constexpr int kRenderChunk = 64;  // sub-box side staged in shared memory
constexpr int kRenderThreads = 128;

struct RenderGeom {
  int nz, ny, nx, g;
  float dx, cutoff;
};

// G (Gaussians per atom) is a template parameter so the per-Gaussian
// constants and the hoisted y * z products stay in registers.  The splat
// gives each warp whole (z, y) rows of the sub-box and its lanes the x
// positions: one integer division per row, G multiply-adds per voxel.
template <int G>
__global__ void __launch_bounds__(kRenderThreads)
    k_render_gaussians(const float* __restrict__ positions, const float* __restrict__ amplitudes,
                       const float* __restrict__ variances, int64_t n_atoms, float* __restrict__ grid, RenderGeom rg) {
  __shared__ float ix[G][kRenderChunk];
  __shared__ float iy[G][kRenderChunk];
  __shared__ float iz[G][kRenderChunk];
  const float dx = rg.dx;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, n_warps = blockDim.x >> 5;
  for (int64_t atom = blockIdx.x; atom < n_atoms; atom += gridDim.x) {
    const float p[3] = {positions[3 * atom], positions[3 * atom + 1], positions[3 * atom + 2]};
    float s[G], pref[G];
    float var_max = 0.f;
#pragma unroll
    for (int g = 0; g < G; ++g) {
      const float v = variances[atom * G + g];
      var_max = fmaxf(var_max, v);
      s[g] = rsqrtf(2.0f * v);
      pref[g] = amplitudes[atom * G + g] / (8.0f * dx * dx * dx);
    }
    const float reach = rg.cutoff * sqrtf(var_max) + dx;
    // voxel index windows per axis (x, y, z)
    const int dims[3] = {rg.nx, rg.ny, rg.nz};
    int lo[3], hi[3];
    bool empty = false;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      // clamped in floating point first, so atoms far outside (or NaN) convert safely: lo in [0, D], hi in [-1, D-1]
      const float half = (float)(dims[a] / 2);
      const float flo = floorf((p[a] - reach) / dx + half), fhi = ceilf((p[a] + reach) / dx + half);
      lo[a] = (int)fmaxf(0.f, fminf(flo, (float)dims[a]));
      hi[a] = (int)fminf((float)(dims[a] - 1), fmaxf(fhi, -1.f));
      empty = empty || hi[a] < lo[a];
    }
    if (empty) continue;
    for (int z0 = lo[2]; z0 <= hi[2]; z0 += kRenderChunk) {
      const int wz = min(kRenderChunk, hi[2] - z0 + 1);
      for (int y0 = lo[1]; y0 <= hi[1]; y0 += kRenderChunk) {
        const int wy = min(kRenderChunk, hi[1] - y0 + 1);
        for (int x0 = lo[0]; x0 <= hi[0]; x0 += kRenderChunk) {
          const int wx = min(kRenderChunk, hi[0] - x0 + 1);
          __syncthreads();  // the previous sub-box's integrals are no longer read
          for (int e = threadIdx.x; e < 3 * kRenderChunk; e += blockDim.x) {
            const int a = e / kRenderChunk, i = e % kRenderChunk;
            const int w = a == 0 ? wx : (a == 1 ? wy : wz);
            if (i >= w) continue;
            const int idx = (a == 0 ? x0 : (a == 1 ? y0 : z0)) + i;
            const float d = (float)(idx - dims[a] / 2) * dx - 0.5f * dx - p[a];
#pragma unroll
            for (int g = 0; g < G; ++g) {
              float v = erff(s[g] * (d + dx)) - erff(s[g] * d);
              if (a == 0) v *= pref[g];
              (a == 0 ? ix : (a == 1 ? iy : iz))[g][i] = v;
            }
          }
          __syncthreads();
          for (int zy = warp; zy < wz * wy; zy += n_warps) {
            const int z = zy / wy, y = zy - z * wy;
            float cyz[G];
#pragma unroll
            for (int g = 0; g < G; ++g) cyz[g] = iy[g][y] * iz[g][z];
            float* row = grid + ((size_t)(z0 + z) * rg.ny + (y0 + y)) * rg.nx + x0;
            for (int x = lane; x < wx; x += 32) {
              float v = 0.f;
#pragma unroll
              for (int g = 0; g < G; ++g) v = fmaf(ix[g][x], cyz[g], v);
              atomicAdd(row + x, v);
            }
          }
        }
      }
    }
  }
}

int launch_render_gaussians(const cjx_render_desc* d, const float* positions, const float* amplitudes,
                            const float* variances, int64_t n_atoms, float* grid, cudaStream_t stream) {
  const size_t bytes = sizeof(float) * (size_t)d->nz * d->ny * d->nx;
  if (!(d->flags & CJX_RENDER_ACCUMULATE))
    if (int e = check_cuda(cudaMemsetAsync(grid, 0, bytes, stream), "cudaMemsetAsync")) return e;
  if (n_atoms == 0) return CJX_OK;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  RenderGeom rg{d->nz, d->ny, d->nx, d->n_gaussians, d->voxel_size, d->cutoff_sigmas > 0.f ? d->cutoff_sigmas : 7.f};
  const int blocks = (int)std::min<int64_t>(n_atoms, (int64_t)sms * 16);
  prof_begin(stream);
  switch (rg.g) {
#define CJX_RENDER_CASE(G)                                                                                        \
  case G:                                                                                                         \
    k_render_gaussians<G><<<blocks, kRenderThreads, 0, stream>>>(positions, amplitudes, variances, n_atoms, grid, \
                                                                 rg);                                            \
    break;
    CJX_RENDER_CASE(1) CJX_RENDER_CASE(2) CJX_RENDER_CASE(3) CJX_RENDER_CASE(4)
    CJX_RENDER_CASE(5) CJX_RENDER_CASE(6) CJX_RENDER_CASE(7) CJX_RENDER_CASE(8)
#undef CJX_RENDER_CASE
    default:
      return fail(CJX_ERR_INVALID_ARGUMENT, "n_gaussians must be in [1, CJX_RENDER_MAX_GAUSSIANS]");
  }
  prof_end("k_render_gaussians", stream);
  return check_cuda(cudaGetLastError(), "k_render_gaussians launch");
}

}  // namespace cjx
