// Orientation search: simulate every candidate (image, orientation) pair
// with the image's own CTF and score it against the observed image by
// normalised cross-correlation, keeping each image's best orientation.
//
// This is the reference's plain grid search: run_grid_search with
// MinimumSearchMethod evaluates fn(grid_point) = a full simulate for every
// orientation, reduced with a running argmin
// (cryojax/jax_util/_grid_search/search_loop.py:24-158,
// search_method.py:237-265); the score is the zero-mean, unit-variance
// real-space dot product (cryojax/ndimage/_normalize.py:11-28).  In Fourier
// space, with A, B the rfft half-planes (Hermitian-fixed columns kx = 0 and
// kx = Px/2), DC excluded and Parseval weights w (1 on those columns, 2
// elsewhere):
//   NCC = sum w Re(conj(B) A) / sqrt(sum w |A|^2 * sum w |B|^2).
#include <algorithm>
#include <mutex>

#include "cjx_common.cuh"
#include "cjx_profile.cuh"

namespace cjx {

int launch_forward_to_t2(const SliceGeom& g, const float2* grid, const cjx_image_params* params, const int32_t* order,
                         int64_t k0, int cnt, float2* t1, float2* t2, float2* hb, cudaStream_t stream,
                         const Tuning& tn);

// Candidate c = (image c / K, slot c % K); orientation = candidates[c] or slot.
__global__ void k_build_candidates(const cjx_image_params* __restrict__ image_params, const double* __restrict__ rot,
                                   const int32_t* __restrict__ candidates, int64_t c0, int cnt, int K,
                                   cjx_image_params* __restrict__ cparams, int32_t* __restrict__ cimg,
                                   int32_t* __restrict__ corient) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)cnt * 32;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(e >> 5), f = (int)(e & 31);
    const int64_t c = c0 + k;
    const int64_t img = c / K;
    const int32_t t = candidates ? candidates[c] : (int32_t)(c % K);
    const double* src = reinterpret_cast<const double*>(image_params + img);
    double v = src[f];
    if (f < 9) v = rot[(int64_t)t * 9 + f];
    reinterpret_cast<double*>(cparams + k)[f] = v;
    if (f == 0) {
      cimg[k] = (int32_t)img;
      corient[k] = t;
    }
  }
}

// Sum over the half-plane (DC excluded) of w |O|^2 for each observed image.
__global__ void k_fourier_power(const float2* __restrict__ obs, float* __restrict__ oo, int py, int px) {
  const int pxh = px / 2 + 1;
  const float2* o = obs + (size_t)blockIdx.x * py * pxh;
  float acc = 0.f;
  for (int e = threadIdx.x; e < py * pxh; e += blockDim.x) {
    const int i = e / pxh, j = e - i * pxh;
    if (i == 0 && j == 0) continue;
    const float w = (j == 0 || ((px % 2 == 0) && j == px / 2)) ? 1.f : 2.f;
    const float2 v = o[e];
    acc += w * (v.x * v.x + v.y * v.y);
  }
  __shared__ float red[32];
  for (int s = 16; s > 0; s >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    oo[blockIdx.x] = t;
  }
}

// Pass C for scoring: column FFT, epilogue (CTF, ...), then the two NCC sums
// instead of storing the image.
template <int R>
__global__ void __launch_bounds__(kWarps * 32)
    k_colfft_score_reg(const float2* __restrict__ t2, const cjx_image_params* __restrict__ cparams,
                       const int32_t* __restrict__ cimg, const float2* __restrict__ obs, float* __restrict__ sums,
                       SliceGeom g, float norm) {
  constexpr int py = 32 * R;
  constexpr int stride = pad16(py) + 1;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  __shared__ float red[kWarps][2];
  __shared__ ImageConsts sc;
  float2* tab = smem;
  float2* row_phase = smem + py;  // exp(-2 pi i qy(i) ty)
  float2* bufs = smem + 2 * py;
  float2* obuf = bufs + kWarps * stride;
  const int j0 = blockIdx.x * kWarps;
  const int ncols = min(kWarps, g.pxh - j0);
  const int k = blockIdx.y;
  const int64_t img = cimg[k];
  const float2* src = t2 + (size_t)k * py * g.ld2 + j0;
  const float2* ocol = obs + (size_t)img * py * g.pxh + j0;
  // staging as in the forward column pass: thread t moves column t % kWarps,
  // rows t / kWarps + 32 q, loads issued before the table copy
  static_assert(kWarps * 32 == 256, "the staging map assumes 256 threads");
  const int sj = threadIdx.x % kWarps, sm0 = threadIdx.x / kWarps;
  float2 st[R], so[R];
  if (sj < ncols) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      st[q] = src[(size_t)(sm0 + 32 * q) * g.ld2 + sj];
      so[q] = ocol[(size_t)(sm0 + 32 * q) * g.pxh + sj];
    }
  }
  build_reg_twiddles(tab, py);
  build_w32(w32);
  if (sj < ncols) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      bufs[sj * stride + pad16(sm0 + 32 * q)] = st[q];
      obuf[sj * stride + pad16(sm0 + 32 * q)] = so[q];
    }
  }
  if (threadIdx.x == 0) sc = load_image_consts(cparams + k, norm, g.py, g.px);
  __syncthreads();
  // R <= 8 keeps a register copy (cheaper at 128^2, where registers are not
  // scarce); larger R reads the shared copy where used (keeps 4 CTAs per SM)
  const ImageConsts c_reg = sc;
  const ImageConsts& c = (R <= 8) ? c_reg : sc;
  if (g.flags & CJX_APPLY_TRANSLATION)
    for (int i = threadIdx.x; i < py; i += blockDim.x) row_phase[i] = phase_factor((double)fft_index(i, py) * c.qy_step * c.ty);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float num = 0.f, den = 0.f;
  if (warp < ncols) {
    float2* buf = bufs + warp * stride;
    const float2* ob = obuf + warp * stride;
    const LaneTwiddles lt = make_lane_twiddles(w32, lane);
    const int bl = brev5(lane);
    const int j = j0 + warp;
    float2 x[R];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) x[n1] = buf[pad16(32 * n1 + bl)];
    warp_fft_reg<R, -1>(x, tab, lt, lane);
    const ColumnEpilogue ce = column_epilogue(j, g.flags, c);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) {
      const int i = k1 + R * lane;
      buf[pad16(i)] = apply_column_epilogue(x[k1], i, j, py, g.px, g.flags, c, ce, row_phase);
    }
    __syncwarp();
    const bool self_col = (j == 0) || ((g.px % 2 == 0) && j == g.px / 2);
    const float w = self_col ? 1.f : 2.f;
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) {
      const int i = k1 + R * lane;
      if (i == 0 && j == 0) continue;
      float2 f = buf[pad16(i)];
      if (self_col) {
        const float2 fm = buf[pad16(i == 0 ? 0 : py - i)];
        f = make_float2(0.5f * (f.x + fm.x), 0.5f * (f.y - fm.y));
      }
      const float2 o = ob[pad16(i)];
      num += w * (o.x * f.x + o.y * f.y);
      den += w * (f.x * f.x + f.y * f.y);
    }
  }
  for (int s = 16; s > 0; s >>= 1) {
    num += __shfl_xor_sync(0xffffffffu, num, s);
    den += __shfl_xor_sync(0xffffffffu, den, s);
  }
  if (lane == 0) {
    red[warp][0] = num;
    red[warp][1] = den;
  }
  __syncthreads();
  if (threadIdx.x < 2) {  // per-block partials: the finalize pass sums them in a fixed order
    float t = 0.f;
    for (int w = 0; w < kWarps; ++w) t += red[w][threadIdx.x];
    sums[((size_t)k * gridDim.x + blockIdx.x) * 2 + threadIdx.x] = t;
  }
}

// Pass C for scoring on the Ewald sphere: each warp transforms a column x of
// the full object spectrum and its mirror (Px - x) mod Px, forms the
// contrast that pairs +q with -q (ewald_column_epilogue, the forward's
// k_ewald_colfft_reg epilogue), then accumulates the two NCC sums against
// the observed rfft image exactly as k_colfft_score_reg does.
template <int R>
__global__ void __launch_bounds__(kWarps * 32)
    k_ewald_colfft_score_reg(const float2* __restrict__ t2, const cjx_image_params* __restrict__ cparams,
                             const int32_t* __restrict__ cimg, const float2* __restrict__ obs,
                             float* __restrict__ sums, SliceGeom g, float norm) {
  constexpr int py = 32 * R;
  constexpr int stride = pad16(py) + 1;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  __shared__ float red[kWarps][2];
  __shared__ ImageConsts sc;
  float2* tab = smem;
  float2* row_phase = smem + py;               // exp(-2 pi i qy(i) ty)
  float2* bufs = smem + 2 * py;                // own columns [0, kWarps), mirrors [kWarps, 2 kWarps)
  float2* obuf = bufs + 2 * kWarps * stride;   // observed columns
  const int px = g.px;
  const int j0 = blockIdx.x * kWarps;
  const int ncols = min(kWarps, g.pxh - j0);
  const int k = blockIdx.y;
  const int64_t img = cimg[k];
  const float2* src = t2 + (size_t)k * py * g.ld2;
  const float2* ocol = obs + (size_t)img * py * g.pxh + j0;
  build_reg_twiddles(tab, py);
  build_w32(w32);
  for (int e = threadIdx.x; e < py * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) {
      bufs[jj * stride + pad16(m)] = src[(size_t)m * g.ld2 + j0 + jj];
      bufs[(kWarps + jj) * stride + pad16(m)] = src[(size_t)m * g.ld2 + (px - j0 - jj) % px];
      obuf[jj * stride + pad16(m)] = ocol[(size_t)m * g.pxh + jj];
    }
  }
  if (threadIdx.x == 0) sc = load_image_consts(cparams + k, norm, g.py, g.px);
  __syncthreads();
  const ImageConsts& c = sc;
  if (g.flags & CJX_APPLY_TRANSLATION)
    for (int i = threadIdx.x; i < py; i += blockDim.x) row_phase[i] = phase_factor((double)fft_index(i, py) * c.qy_step * c.ty);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float num = 0.f, den = 0.f;
  if (warp < ncols) {
    const LaneTwiddles lt = make_lane_twiddles(w32, lane);
    const int bl = brev5(lane);
    float2* A = bufs + warp * stride;
    float2* B = bufs + (kWarps + warp) * stride;
    const float2* ob = obuf + warp * stride;
    float2 x[R];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) x[n1] = A[pad16(32 * n1 + bl)];
    warp_fft_reg<R, -1>(x, tab, lt, lane);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) A[pad16(k1 + R * lane)] = x[k1];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) x[n1] = B[pad16(32 * n1 + bl)];
    warp_fft_reg<R, -1>(x, tab, lt, lane);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) B[pad16(k1 + R * lane)] = x[k1];
    __syncwarp();
    const int j = j0 + warp;
    const ColumnEpilogue ce = column_epilogue(j, g.flags, c);
    for (int i = lane; i < py; i += 32)  // row i is read and written by this lane only
      A[pad16(i)] = ewald_column_epilogue(A[pad16(i)], B[pad16((py - i) % py)], i, j, py, px, g.flags, c, ce,
                                          row_phase);
    __syncwarp();
    const bool self_col = (j == 0) || ((px % 2 == 0) && j == px / 2);
    const float w = self_col ? 1.f : 2.f;
    for (int i = lane; i < py; i += 32) {
      if (i == 0 && j == 0) continue;
      float2 f = A[pad16(i)];
      if (self_col) {
        const float2 fm = A[pad16(i == 0 ? 0 : py - i)];
        f = make_float2(0.5f * (f.x + fm.x), 0.5f * (f.y - fm.y));
      }
      const float2 o = ob[pad16(i)];
      num += w * (o.x * f.x + o.y * f.y);
      den += w * (f.x * f.x + f.y * f.y);
    }
  }
  for (int s = 16; s > 0; s >>= 1) {
    num += __shfl_xor_sync(0xffffffffu, num, s);
    den += __shfl_xor_sync(0xffffffffu, den, s);
  }
  if (lane == 0) {
    red[warp][0] = num;
    red[warp][1] = den;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    float t = 0.f;
    for (int w = 0; w < kWarps; ++w) t += red[w][threadIdx.x];
    sums[((size_t)k * gridDim.x + blockIdx.x) * 2 + threadIdx.x] = t;
  }
}

// Orderable 64-bit key: score (monotone bits) in the high word, and the
// complement of the orientation index in the low word (ties -> lowest index).
__device__ __forceinline__ unsigned long long score_key(float s, int32_t orient) {
  unsigned int u = __float_as_uint(s);
  u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
  return ((unsigned long long)u << 32) | (unsigned long long)(0xFFFFFFFFu - (unsigned int)orient);
}

__global__ void k_finalize_scores(const float* __restrict__ sums, int nparts, const int32_t* __restrict__ cimg,
                                  const int32_t* __restrict__ corient, const float* __restrict__ oo,
                                  float* __restrict__ scores, unsigned long long* __restrict__ best, int64_t c0,
                                  int cnt) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= cnt) return;
  const int32_t img = cimg[k];
  float num = 0.f, den = 0.f;
  for (int p = 0; p < nparts; ++p) {
    num += sums[((size_t)k * nparts + p) * 2];
    den += sums[((size_t)k * nparts + p) * 2 + 1];
  }
  const float o2 = oo[img];
  const float s = (den > 0.f && o2 > 0.f) ? num * rsqrtf(den * o2) : 0.f;
  if (scores) scores[c0 + k] = s;
  atomicMax(&best[img], score_key(s, corient[k]));
}

__global__ void k_init_best(unsigned long long* best, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    best[i] = 0ull;
}

__global__ void k_unpack_best(const unsigned long long* __restrict__ best, float* __restrict__ best_score,
                              int32_t* __restrict__ best_orient, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long b = best[i];
    unsigned int u = (unsigned int)(b >> 32);
    u = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
    if (best_score) best_score[i] = __uint_as_float(u);
    if (best_orient) best_orient[i] = (int32_t)(0xFFFFFFFFu - (unsigned int)(b & 0xFFFFFFFFull));
  }
}

// Once per device (function attributes belong to each device's context);
// the outcome of that first attempt is returned to every later call.
static cudaError_t search_smem_attrs() {
  static PerDeviceOnce once;
  return once.run([] {
    cudaError_t err = cudaSuccess;
#define CJX_SA(R)                                                                                              \
  if (err == cudaSuccess)                                                                                      \
    err = cudaFuncSetAttribute(k_colfft_score_reg<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024); \
  if (err == cudaSuccess)                                                                                      \
    err = cudaFuncSetAttribute(k_ewald_colfft_score_reg<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    CJX_SA(1) CJX_SA(2) CJX_SA(3) CJX_SA(4) CJX_SA(5) CJX_SA(6) CJX_SA(8) CJX_SA(10) CJX_SA(12) CJX_SA(16)
#undef CJX_SA
    return err;
  });
}

// Workspace: per candidate the forward intermediates + a params record,
// image / orientation ids and two sums; per image the power of O and the
// packed best key.
static int score_parts(const SliceGeom& g) { return (g.pxh + kWarps - 1) / kWarps; }

size_t search_candidate_bytes(const SliceGeom& g, size_t per_image_fwd) {
  return per_image_fwd + sizeof(cjx_image_params) + 2 * sizeof(int32_t) + 2 * sizeof(float) * score_parts(g);
}

int launch_search(const SliceGeom& g, size_t per_fwd, int64_t chunk, const float2* grid,
                  const cjx_image_params* image_params, const double* rot, const int32_t* candidates,
                  int64_t n_images, int K, const float2* obs, float* scores, float* best_score, int32_t* best_orient,
                  void* workspace, cudaStream_t stream, const Tuning& tn) {
  const int rpy = reg_fft_radix(g.py);
  if (!rpy) return fail(CJX_ERR_UNSUPPORTED, "search needs Py = 32 R with R in {1-6, 8, 10, 12, 16}");
  if (cudaError_t e = search_smem_attrs()) return check_cuda(e, "cudaFuncSetAttribute");
  // carve the workspace (each piece 256-byte aligned)
  auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
  char* p = static_cast<char*>(workspace);
  float2* t1 = reinterpret_cast<float2*>(p);
  float2* t2 = t1 + (size_t)chunk * g.py * g.ld1;
  float2* hb = t2 + (size_t)chunk * g.py * g.ld2;
  p += align((size_t)chunk * per_fwd);
  cjx_image_params* cparams = reinterpret_cast<cjx_image_params*>(p);
  p += align((size_t)chunk * sizeof(cjx_image_params));
  int32_t* cimg = reinterpret_cast<int32_t*>(p);
  p += align((size_t)chunk * sizeof(int32_t));
  int32_t* corient = reinterpret_cast<int32_t*>(p);
  p += align((size_t)chunk * sizeof(int32_t));
  float* sums = reinterpret_cast<float*>(p);
  const int nparts = score_parts(g);
  p += align((size_t)chunk * nparts * 2 * sizeof(float));
  float* oo = reinterpret_cast<float*>(p);
  p += align((size_t)n_images * sizeof(float));
  unsigned long long* best = reinterpret_cast<unsigned long long*>(p);

  const float norm = (float)(1.0 / ((double)g.n * (double)g.n));
  const size_t s_score = sizeof(float2) * (size_t)(2 * g.py + 2 * kWarps * (pad16(g.py) + 1));
  const size_t s_ewald = sizeof(float2) * (size_t)(2 * g.py + 3 * kWarps * (pad16(g.py) + 1));
  prof_begin(stream);
  k_fourier_power<<<(unsigned)n_images, 256, 0, stream>>>(obs, oo, g.py, g.px);
  prof_end("k_fourier_power", stream);
  k_init_best<<<64, 256, 0, stream>>>(best, n_images);
  const int64_t total = n_images * (int64_t)K;
  for (int64_t c0 = 0; c0 < total; c0 += chunk) {
    const int cnt = (int)std::min<int64_t>(chunk, total - c0);
    prof_begin(stream);
    k_build_candidates<<<std::min(1024, (cnt * 32 + 255) / 256), 256, 0, stream>>>(
        image_params, rot, candidates, c0, cnt, K, cparams, cimg, corient);
    prof_end("k_build_candidates", stream);
    if (int e = launch_forward_to_t2(g, grid, cparams, nullptr, 0, cnt, t1, t2, hb, stream, tn)) return e;
    prof_begin(stream);
    const dim3 gs(nparts, cnt);
    if (g.flags & CJX_EWALD_SPHERE) {
      switch (rpy) {
#define CJX_S_CASE(R)                                                                                                  \
  case R:                                                                                                              \
    k_ewald_colfft_score_reg<R><<<gs, kWarps * 32, s_ewald, stream>>>(t2, cparams, cimg, obs, sums, g, norm); break;
        CJX_S_CASE(1) CJX_S_CASE(2) CJX_S_CASE(3) CJX_S_CASE(4) CJX_S_CASE(5)
        CJX_S_CASE(6) CJX_S_CASE(8) CJX_S_CASE(10) CJX_S_CASE(12) CJX_S_CASE(16)
#undef CJX_S_CASE
      }
    } else {
      switch (rpy) {
#define CJX_S_CASE(R) \
  case R: k_colfft_score_reg<R><<<gs, kWarps * 32, s_score, stream>>>(t2, cparams, cimg, obs, sums, g, norm); break;
        CJX_S_CASE(1) CJX_S_CASE(2) CJX_S_CASE(3) CJX_S_CASE(4) CJX_S_CASE(5)
        CJX_S_CASE(6) CJX_S_CASE(8) CJX_S_CASE(10) CJX_S_CASE(12) CJX_S_CASE(16)
#undef CJX_S_CASE
      }
    }
    prof_end("k_colfft_score", stream);
    prof_begin(stream);
    k_finalize_scores<<<(cnt + 255) / 256, 256, 0, stream>>>(sums, nparts, cimg, corient, oo, scores, best, c0, cnt);
    prof_end("k_finalize_scores", stream);
  }
  k_unpack_best<<<64, 256, 0, stream>>>(best, best_score, best_orient, n_images);
  return check_cuda(cudaGetLastError(), "search launch");
}

size_t search_workspace_bytes(const SliceGeom& g, size_t per_fwd, int64_t chunk, int64_t n_images) {
  auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
  return align((size_t)chunk * per_fwd) + align((size_t)chunk * sizeof(cjx_image_params)) +
         2 * align((size_t)chunk * sizeof(int32_t)) + align((size_t)chunk * score_parts(g) * 2 * sizeof(float)) +
         align((size_t)n_images * sizeof(float)) + align((size_t)n_images * sizeof(unsigned long long));
}

}  // namespace cjx
