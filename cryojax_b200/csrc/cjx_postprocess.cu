// Real-space output and post-processing of simulated images (sm_100a).
//
// AbstractImageModel.postprocess (cryojax/simulator/_image_model/base_image_model.py:107-158)
// after the Fourier image: irfftn (cryojax/ndimage/_fft.py:57-77: inverse
// real FFT, then fftshift) -> centre crop to the image shape
// (cryojax/ndimage/_edges.py:15-62) -> normalise ((x - mean) / std, the
// population std) -> mask (times a real-space array); and the reference's
// rfftn of real-space images (ifftshift, then rfft2; cryojax/ndimage/_fft.py:80-99),
// used on observed images and on masked images whose Fourier form is wanted.
//
// irfft2, three passes per chunk of images:
//   1 k_pp_colifft: per column kx of the half plane a Py-point inverse FFT
//     (columns kx = 0 and, for even Px, kx = Px/2 made Hermitian in ky first:
//     the part of them an inverse real FFT keeps) into the workspace T;
//   2 k_pp_rows_c2r: two rows of T at a time, Hermitian-extended and packed as
//     A + iB, one Px-point inverse FFT gives both real rows; the fftshift and
//     the crop are an index map on the rows read and the columns written; the
//     mask multiplies here unless the image is normalised, and the per-image
//     sums for the normalisation are accumulated in double;
//   3 k_pp_normalize (only with CJX_PP_NORMALIZE): (x - mean) / std, then the mask.
// rfft2, two passes, in place in the output: k_pp_rows_r2c (two real rows as
// one complex FFT, split into their half spectra) and k_pp_colfft.
// The transforms are the library's shared-memory Stockham warp FFTs, so every
// size up to CJX_MAX_SIDE works.
#include <algorithm>

#include "cjx_common.cuh"
#include "cjx_profile.cuh"

namespace cjx {

namespace {

// Result buffer of warp_fft: a after an even number of Stockham stages, b otherwise.
inline int fft_result_offset(const FftPlan& p, int n) { return (p.nstages == 0 || (p.nstages & 1)) ? n : 0; }

// Pass 1 of irfft2: column inverse FFTs of the half plane.
__global__ void __launch_bounds__(kWarps * 32)
    k_pp_colifft(const float2* __restrict__ in, float2* __restrict__ t, int py, int px, FftPlan plan, int res_off) {
  extern __shared__ float2 smem[];
  const int pxh = px / 2 + 1;
  const int stride = 2 * py + 2;
  float2* tw = smem;
  float2* bufs = smem + py;
  build_twiddles(tw, py);
  const int j0 = blockIdx.x * kWarps;
  const int ncols = min(kWarps, pxh - j0);
  const float2* src = in + (size_t)blockIdx.y * py * pxh + j0;
  for (int e = threadIdx.x; e < py * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) bufs[jj * stride + m] = src[(size_t)m * pxh + jj];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < ncols) {
    float2* a = bufs + warp * stride;
    const int j = j0 + warp;
    if (j == 0 || ((px % 2 == 0) && j == px / 2)) {
      // (S[v] + conj(S[-v])) / 2: the pairs (v, -v) are disjoint across lanes
      for (int i = lane; i <= py / 2; i += 32) {
        const int i2 = (i == 0) ? 0 : py - i;
        const float2 x = a[i], y = a[i2];
        const float2 sv = make_float2(0.5f * (x.x + y.x), 0.5f * (x.y - y.y));
        a[i] = sv;
        a[i2] = cconj(sv);
      }
      __syncwarp();
    }
    warp_fft<+1>(a, a + py, plan, tw, lane);
  }
  __syncthreads();
  float2* dst = t + (size_t)blockIdx.y * py * pxh + j0;
  for (int e = threadIdx.x; e < py * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) dst[(size_t)m * pxh + jj] = bufs[jj * stride + res_off + m];
  }
}

// Pass 2 of irfft2: rows (two per warp) -> fftshift -> crop -> scale (-> mask) -> float32 output,
// plus the per-image sum and sum of squares (double) when stats != NULL.
__global__ void __launch_bounds__(kWarps * 32)
    k_pp_rows_c2r(const float2* __restrict__ t, float* __restrict__ out, int py, int px, int h, int w,
                  const float* __restrict__ mask, double* __restrict__ stats, FftPlan plan) {
  extern __shared__ float2 smem[];
  const int pxh = px / 2 + 1;
  float2* tw = smem;
  float2* bufs = smem + px;
  build_twiddles(tw, px);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r0 = 2 * (blockIdx.x * kWarps + warp);
  if (r0 >= h) return;
  const bool has_b = r0 + 1 < h;
  // output row r of the crop is row (r + y0 + py - py/2) mod py of the unshifted inverse transform
  const int y0 = py / 2 - h / 2, x0 = px / 2 - w / 2;
  const int sa = (r0 + y0 + py - py / 2) % py;
  const int sb = (r0 + 1 + y0 + py - py / 2) % py;
  const float2* rowA = t + ((size_t)blockIdx.y * py + sa) * pxh;
  const float2* rowB = t + ((size_t)blockIdx.y * py + sb) * pxh;
  float2* a = bufs + warp * (2 * px + 2);
  float2* b = a + px;
  // z = A + iB on the Hermitian extension; DC and (even Px) Nyquist bins keep their real parts only
  for (int k = lane; k <= px / 2; k += 32) {
    const float2 A = rowA[k];
    const float2 B = has_b ? rowB[k] : make_float2(0.f, 0.f);
    if (k == 0 || ((px % 2 == 0) && k == px / 2)) {
      a[k] = make_float2(A.x, B.x);
    } else {
      a[k] = make_float2(A.x - B.y, A.y + B.x);
      a[px - k] = make_float2(A.x + B.y, B.x - A.y);
    }
  }
  __syncwarp();
  const float2* z = warp_fft<+1>(a, b, plan, tw, lane);
  const float scale = (float)(1.0 / ((double)py * (double)px));
  const bool fuse_mask = mask && !stats;
  float* oa = out + ((size_t)blockIdx.y * h + r0) * w;
  double s = 0.0, ss = 0.0;
  for (int c = lane; c < w; c += 32) {
    const float2 v = z[(c + x0 + px - px / 2) % px];
    float va = v.x * scale, vb = v.y * scale;
    s += (double)va;
    ss += (double)va * (double)va;
    if (has_b) {
      s += (double)vb;
      ss += (double)vb * (double)vb;
    }
    if (fuse_mask) {
      va *= __ldg(mask + (size_t)r0 * w + c);
      if (has_b) vb *= __ldg(mask + (size_t)(r0 + 1) * w + c);
    }
    oa[c] = va;
    if (has_b) oa[w + c] = vb;
  }
  if (stats) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      ss += __shfl_xor_sync(0xffffffffu, ss, o);
    }
    if (lane == 0) {
      atomicAdd(stats + 2 * blockIdx.y, s);
      atomicAdd(stats + 2 * blockIdx.y + 1, ss);
    }
  }
}

// Pass 3 of irfft2 (normalisation): (x - mean) / std with the population std, then the optional mask.
// One image per blockIdx.y: its mean and 1 / std come once per thread from the double sums.
__global__ void k_pp_normalize(float* __restrict__ out, int hw, const double* __restrict__ stats,
                               const float* __restrict__ mask) {
  const int64_t img = blockIdx.y;
  const double mean_d = stats[2 * img] / hw;
  const double var = fmax(stats[2 * img + 1] / hw - mean_d * mean_d, 0.0);
  const float mean = (float)mean_d, istd = (float)(1.0 / sqrt(var));
  float* o = out + img * hw;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < hw; p += gridDim.x * blockDim.x) {
    float v = (o[p] - mean) * istd;
    if (mask) v *= __ldg(mask + p);
    o[p] = v;
  }
}

// rfft2 pass 1: rows (two per warp) of ifftshift(image) as one complex FFT, split into the half spectra.
__global__ void __launch_bounds__(kWarps * 32)
    k_pp_rows_r2c(const float* __restrict__ image, float2* __restrict__ out, int py, int px, FftPlan plan) {
  extern __shared__ float2 smem[];
  const int pxh = px / 2 + 1;
  float2* tw = smem;
  float2* bufs = smem + px;
  build_twiddles(tw, px);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ra = 2 * (blockIdx.x * kWarps + warp);
  if (ra >= py) return;
  const bool has_b = ra + 1 < py;
  // ifftshift: transform row i / column j read image row (i + py/2) mod py / column (j + px/2) mod px
  const float* xa = image + ((size_t)blockIdx.y * py + (ra + py / 2) % py) * px;
  const float* xb = image + ((size_t)blockIdx.y * py + (ra + 1 + py / 2) % py) * px;
  float2* a = bufs + warp * (2 * px + 2);
  float2* b = a + px;
  for (int j = lane; j < px; j += 32) {
    const int c = (j + px / 2) % px;
    a[j] = make_float2(xa[c], has_b ? xb[c] : 0.f);
  }
  __syncwarp();
  const float2* Z = warp_fft<-1>(a, b, plan, tw, lane);
  float2* oa = out + ((size_t)blockIdx.y * py + ra) * pxh;
  for (int k = lane; k < pxh; k += 32) {
    const float2 Zk = Z[k];
    const float2 Zm = Z[(px - k) % px];
    oa[k] = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
    if (has_b) oa[pxh + k] = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
  }
}

// rfft2 pass 2: column forward FFTs, in place (each CTA owns its columns).
__global__ void __launch_bounds__(kWarps * 32)
    k_pp_colfft(float2* __restrict__ data, int py, int px, FftPlan plan, int res_off) {
  extern __shared__ float2 smem[];
  const int pxh = px / 2 + 1;
  const int stride = 2 * py + 2;
  float2* tw = smem;
  float2* bufs = smem + py;
  build_twiddles(tw, py);
  const int j0 = blockIdx.x * kWarps;
  const int ncols = min(kWarps, pxh - j0);
  float2* col0 = data + (size_t)blockIdx.y * py * pxh + j0;
  for (int e = threadIdx.x; e < py * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) bufs[jj * stride + m] = col0[(size_t)m * pxh + jj];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < ncols) warp_fft<-1>(bufs + warp * stride, bufs + warp * stride + py, plan, tw, lane);
  __syncthreads();
  for (int e = threadIdx.x; e < py * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) col0[(size_t)m * pxh + jj] = bufs[jj * stride + res_off + m];
  }
}

// rfft2 with the register FFTs when Px and Py are 32 R (R in 1-6, 8, 10, 12,
// 16): compile-time twiddle tables copied once per CTA instead of double
// sin / cos per CTA, shuffles instead of the Stockham stages' shared-memory
// passes.  Same two passes as above.
template <int R>
__global__ void __launch_bounds__(kWarps * 32)
    k_pp_rows_r2c_reg(const float* __restrict__ image, float2* __restrict__ out, int py) {
  constexpr int n = 32 * R;  // Px
  constexpr int stride = pad16(n - 1) + 1;
  constexpr int pxh = n / 2 + 1;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  float2* tab = smem;
  float2* bufs = smem + n;
  build_reg_twiddles(tab, n);
  build_w32(w32);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ra = 2 * (blockIdx.x * kWarps + warp);
  if (ra >= py) return;
  const bool has_b = ra + 1 < py;
  // ifftshift: transform row i / column j read image row (i + py/2) mod py / column (j + n/2) mod n
  const float* xa = image + ((size_t)blockIdx.y * py + (ra + py / 2) % py) * n;
  const float* xb = image + ((size_t)blockIdx.y * py + (ra + 1 + py / 2) % py) * n;
  const int bl = brev5(lane);
  float2 z[R];
#pragma unroll
  for (int n1 = 0; n1 < R; ++n1) {
    const int c = (32 * n1 + bl + n / 2) % n;
    z[n1] = make_float2(xa[c], has_b ? xb[c] : 0.f);
  }
  const LaneTwiddles lt = make_lane_twiddles(w32, lane);
  warp_fft_reg<R, -1>(z, tab, lt, lane);
  float2* buf = bufs + warp * stride;
#pragma unroll
  for (int k1 = 0; k1 < R; ++k1) buf[pad16(k1 + R * lane)] = z[k1];
  __syncwarp();
  float2* oa = out + ((size_t)blockIdx.y * py + ra) * pxh;
  for (int k = lane; k < pxh; k += 32) {
    const float2 Zk = buf[pad16(k)];
    const float2 Zm = buf[pad16((n - k) % n)];
    oa[k] = make_float2(0.5f * (Zk.x + Zm.x), 0.5f * (Zk.y - Zm.y));
    if (has_b) oa[pxh + k] = make_float2(0.5f * (Zk.y + Zm.y), -0.5f * (Zk.x - Zm.x));
  }
}

template <int R>
__global__ void __launch_bounds__(kWarps * 32) k_pp_colfft_reg(float2* __restrict__ data, int px) {
  constexpr int n = 32 * R;  // Py
  constexpr int stride = pad16(n - 1) + 1;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  const int pxh = px / 2 + 1;
  float2* tab = smem;
  float2* bufs = smem + n;
  build_reg_twiddles(tab, n);
  build_w32(w32);
  const int j0 = blockIdx.x * kWarps;
  const int ncols = min(kWarps, pxh - j0);
  float2* col0 = data + (size_t)blockIdx.y * n * pxh + j0;
  for (int e = threadIdx.x; e < n * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) bufs[jj * stride + pad16(m)] = col0[(size_t)m * pxh + jj];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < ncols) {
    float2* buf = bufs + warp * stride;
    const int bl = brev5(lane);
    float2 x[R];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) x[n1] = buf[pad16(32 * n1 + bl)];
    const LaneTwiddles lt = make_lane_twiddles(w32, lane);
    warp_fft_reg<R, -1>(x, tab, lt, lane);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) buf[pad16(k1 + R * lane)] = x[k1];
  }
  __syncthreads();
  for (int e = threadIdx.x; e < n * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) col0[(size_t)m * pxh + jj] = bufs[jj * stride + pad16(m)];
  }
}

size_t smem_reg(int n) { return sizeof(float2) * (size_t)(n + kWarps * (pad16(n - 1) + 1)); }

// irfft2 passes 1 and 2 on the register FFTs (Py, Px = 32 R): the column
// inverse FFTs with the self-conjugate columns' Hermitian fix, and two rows
// per warp as one complex inverse FFT of their Hermitian extensions, then
// the same fftshift, crop, scale, statistics and mask as k_pp_rows_c2r.
template <int R>
__global__ void __launch_bounds__(kWarps * 32)
    k_pp_colifft_reg(const float2* __restrict__ in, float2* __restrict__ t, int px) {
  constexpr int n = 32 * R;  // Py
  constexpr int stride = pad16(n - 1) + 1;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  const int pxh = px / 2 + 1;
  float2* tab = smem;
  float2* bufs = smem + n;
  build_reg_twiddles(tab, n);
  build_w32(w32);
  const int j0 = blockIdx.x * kWarps;
  const int ncols = min(kWarps, pxh - j0);
  const float2* src = in + (size_t)blockIdx.y * n * pxh + j0;
  for (int e = threadIdx.x; e < n * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) bufs[jj * stride + pad16(m)] = src[(size_t)m * pxh + jj];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < ncols) {
    float2* buf = bufs + warp * stride;
    const int j = j0 + warp;
    if (j == 0 || ((px % 2 == 0) && j == px / 2)) {
      // (S[v] + conj(S[-v])) / 2: the pairs (v, -v) are disjoint across lanes
      for (int i = lane; i <= n / 2; i += 32) {
        const int i2 = (i == 0) ? 0 : n - i;
        const float2 x = buf[pad16(i)], y = buf[pad16(i2)];
        const float2 sv = make_float2(0.5f * (x.x + y.x), 0.5f * (x.y - y.y));
        buf[pad16(i)] = sv;
        buf[pad16(i2)] = cconj(sv);
      }
      __syncwarp();
    }
    const int bl = brev5(lane);
    float2 x[R];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) x[n1] = buf[pad16(32 * n1 + bl)];
    const LaneTwiddles lt = make_lane_twiddles(w32, lane);
    warp_fft_reg<R, +1>(x, tab, lt, lane);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) buf[pad16(k1 + R * lane)] = x[k1];
  }
  __syncthreads();
  float2* dst = t + (size_t)blockIdx.y * n * pxh + j0;
  for (int e = threadIdx.x; e < n * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) dst[(size_t)m * pxh + jj] = bufs[jj * stride + pad16(m)];
  }
}

template <int R>
__global__ void __launch_bounds__(kWarps * 32)
    k_pp_rows_c2r_reg(const float2* __restrict__ t, float* __restrict__ out, int py, int h, int w,
                      const float* __restrict__ mask, double* __restrict__ stats) {
  constexpr int n = 32 * R;  // Px
  constexpr int stride = pad16(n - 1) + 1;
  constexpr int hx = n / 2, pxh = n / 2 + 1;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  float2* tab = smem;
  float2* bufs = smem + n;
  build_reg_twiddles(tab, n);
  build_w32(w32);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r0 = 2 * (blockIdx.x * kWarps + warp);
  if (r0 >= h) return;
  const bool has_b = r0 + 1 < h;
  // output row r of the crop is row (r + y0 + py - py/2) mod py of the unshifted inverse transform
  const int y0 = py / 2 - h / 2, x0 = hx - w / 2;
  const int sa = (r0 + y0 + py - py / 2) % py;
  const int sb = (r0 + 1 + y0 + py - py / 2) % py;
  const float2* rowA = t + ((size_t)blockIdx.y * py + sa) * pxh;
  const float2* rowB = t + ((size_t)blockIdx.y * py + sb) * pxh;
  // z = A + iB on the Hermitian extension, in the lane's bit-reversed input order; the DC and Nyquist
  // bins keep their real parts only
  const int bl = brev5(lane);
  float2 z[R];
#pragma unroll
  for (int n1 = 0; n1 < R; ++n1) {
    const int k = 32 * n1 + bl;
    if (k == 0 || k == hx) {
      const float2 A = rowA[k], B = has_b ? rowB[k] : make_float2(0.f, 0.f);
      z[n1] = make_float2(A.x, B.x);
    } else if (k < hx) {
      const float2 A = rowA[k], B = has_b ? rowB[k] : make_float2(0.f, 0.f);
      z[n1] = make_float2(A.x - B.y, A.y + B.x);
    } else {
      const float2 A = rowA[n - k], B = has_b ? rowB[n - k] : make_float2(0.f, 0.f);
      z[n1] = make_float2(A.x + B.y, B.x - A.y);
    }
  }
  const LaneTwiddles lt = make_lane_twiddles(w32, lane);
  warp_fft_reg<R, +1>(z, tab, lt, lane);
  float2* buf = bufs + warp * stride;
#pragma unroll
  for (int k1 = 0; k1 < R; ++k1) buf[pad16(k1 + R * lane)] = z[k1];
  __syncwarp();
  const float scale = (float)(1.0 / ((double)py * (double)n));
  const bool fuse_mask = mask && !stats;
  float* oa = out + ((size_t)blockIdx.y * h + r0) * w;
  double s = 0.0, ss = 0.0;
  for (int c = lane; c < w; c += 32) {
    const float2 v = buf[pad16((c + x0 + n - hx) % n)];
    float va = v.x * scale, vb = v.y * scale;
    s += (double)va;
    ss += (double)va * (double)va;
    if (has_b) {
      s += (double)vb;
      ss += (double)vb * (double)vb;
    }
    if (fuse_mask) {
      va *= __ldg(mask + (size_t)r0 * w + c);
      if (has_b) vb *= __ldg(mask + (size_t)(r0 + 1) * w + c);
    }
    oa[c] = va;
    if (has_b) oa[w + c] = vb;
  }
  if (stats) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s += __shfl_xor_sync(0xffffffffu, s, o);
      ss += __shfl_xor_sync(0xffffffffu, ss, o);
    }
    if (lane == 0) {
      atomicAdd(stats + 2 * blockIdx.y, s);
      atomicAdd(stats + 2 * blockIdx.y + 1, ss);
    }
  }
}



size_t smem_cols(int py) { return sizeof(float2) * (size_t)(py + kWarps * (2 * py + 2)); }
size_t smem_rows(int px) { return sizeof(float2) * (size_t)(px + kWarps * (2 * px + 2)); }

int ensure_pp_smem() {
  static PerDeviceOnce once;
  const cudaError_t e = once.run([] {
    const int kMax = 227 * 1024;
    cudaError_t r = cudaFuncSetAttribute(k_pp_colifft, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(k_pp_rows_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(k_pp_rows_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax);
    if (r == cudaSuccess) r = cudaFuncSetAttribute(k_pp_colfft, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax);
    return r;
  });
  return e == cudaSuccess ? CJX_OK : check_cuda(e, "cudaFuncSetAttribute (post-processing kernels)");
}

int check_shape(int64_t n, int py, int px) {
  if (n < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "n < 0");
  if (py < 1 || px < 2) return fail(CJX_ERR_INVALID_ARGUMENT, "need py >= 1 and px >= 2");
  if (py > CJX_MAX_SIDE || px > CJX_MAX_SIDE) return fail(CJX_ERR_UNSUPPORTED, "image sides are limited to CJX_MAX_SIDE");
  if (smem_cols(py) > 227 * 1024 || smem_rows(px) > 227 * 1024)
    return fail(CJX_ERR_UNSUPPORTED, "post-processing shared-memory footprint exceeds 227 KB");
  return CJX_OK;
}

size_t pp_bytes_per_image(int py, int px) { return sizeof(float2) * (size_t)py * (px / 2 + 1) + 2 * sizeof(double); }

}  // namespace

}  // namespace cjx

using namespace cjx;

extern "C" int cjx_postprocess_workspace_size(int64_t n_images, int py, int px, size_t* bytes) {
  if (!bytes) return fail(CJX_ERR_INVALID_ARGUMENT, "bytes is NULL");
  if (int e = check_shape(n_images, py, px)) return e;
  *bytes = (size_t)n_images * pp_bytes_per_image(py, px);
  return CJX_OK;
}

extern "C" int cjx_postprocess_real(int64_t n_images, int py, int px, int h, int w, uint32_t flags,
                                    const void* fourier, const float* mask, float* out, void* workspace,
                                    size_t workspace_bytes, void* stream) {
  if (int e = check_shape(n_images, py, px)) return e;
  if (h < 1 || w < 1 || h > py || w > px)
    return fail(CJX_ERR_INVALID_ARGUMENT, "the image shape (h, w) must fit inside the padded shape (py, px)");
  if (flags & ~CJX_PP_NORMALIZE) return fail(CJX_ERR_INVALID_ARGUMENT, "unknown post-processing flag bits");
  if (n_images == 0) return CJX_OK;
  if (!fourier || !out || !workspace)
    return fail(CJX_ERR_INVALID_ARGUMENT, "fourier, out and workspace must be non-NULL");
  const size_t per = pp_bytes_per_image(py, px);
  if (workspace_bytes < per) return fail(CJX_ERR_WORKSPACE, "workspace smaller than one image's need");
  if (int e = ensure_pp_smem()) return e;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int64_t chunk = std::min<int64_t>({(int64_t)(workspace_bytes / per), n_images, 65535});
  const bool normalize = (flags & CJX_PP_NORMALIZE) != 0;
  const int pxh = px / 2 + 1;
  float2* t = static_cast<float2*>(workspace);
  double* stats = reinterpret_cast<double*>(static_cast<char*>(workspace) + (size_t)chunk * py * pxh * sizeof(float2));
  const FftPlan plan_y = make_fft_plan(py), plan_x = make_fft_plan(px);
  const int rx = reg_fft_radix(px), ry = reg_fft_radix(py);  // register FFTs when both are 32 R
  for (int64_t k0 = 0; k0 < n_images; k0 += chunk) {
    const int cnt = (int)std::min<int64_t>(chunk, n_images - k0);
    const float2* src = static_cast<const float2*>(fourier) + (size_t)k0 * py * pxh;
    float* dst = out + (size_t)k0 * h * w;
    const dim3 gcol((pxh + kWarps - 1) / kWarps, cnt), grow((h + 2 * kWarps - 1) / (2 * kWarps), cnt);
    prof_begin(s);
    if (ry && rx) {
      switch (ry) {
#define CJX_PPCI(R) \
  case R: k_pp_colifft_reg<R><<<gcol, kWarps * 32, smem_reg(py), s>>>(src, t, px); break;
        CJX_PPCI(1) CJX_PPCI(2) CJX_PPCI(3) CJX_PPCI(4) CJX_PPCI(5) CJX_PPCI(6) CJX_PPCI(8) CJX_PPCI(10)
        CJX_PPCI(12) CJX_PPCI(16)
#undef CJX_PPCI
      }
    } else {
      k_pp_colifft<<<gcol, kWarps * 32, smem_cols(py), s>>>(src, t, py, px, plan_y, fft_result_offset(plan_y, py));
    }
    prof_end("k_pp_colifft", s);
    if (normalize) {
      if (int e = check_cuda(cudaMemsetAsync(stats, 0, sizeof(double) * 2 * cnt, s), "cudaMemsetAsync")) return e;
    }
    double* st = normalize ? stats : nullptr;
    prof_begin(s);
    if (ry && rx) {
      switch (rx) {
#define CJX_PPRC(R) \
  case R: k_pp_rows_c2r_reg<R><<<grow, kWarps * 32, smem_reg(px), s>>>(t, dst, py, h, w, mask, st); break;
        CJX_PPRC(1) CJX_PPRC(2) CJX_PPRC(3) CJX_PPRC(4) CJX_PPRC(5) CJX_PPRC(6) CJX_PPRC(8) CJX_PPRC(10)
        CJX_PPRC(12) CJX_PPRC(16)
#undef CJX_PPRC
      }
    } else {
      k_pp_rows_c2r<<<grow, kWarps * 32, smem_rows(px), s>>>(t, dst, py, px, h, w, mask, st, plan_x);
    }
    prof_end("k_pp_rows_c2r", s);
    if (normalize) {
      prof_begin(s);
      const int bx = std::min((h * w + 255) / 256, 32);
      k_pp_normalize<<<dim3(bx, cnt), 256, 0, s>>>(dst, h * w, stats, mask);
      prof_end("k_pp_normalize", s);
    }
  }
  return check_cuda(cudaGetLastError(), "post-processing launch");
}

extern "C" int cjx_rfft2(int64_t n_images, int py, int px, const float* image, void* out, void* stream) {
  if (int e = check_shape(n_images, py, px)) return e;
  if (n_images == 0) return CJX_OK;
  if (!image || !out) return fail(CJX_ERR_INVALID_ARGUMENT, "image and out must be non-NULL");
  if (int e = ensure_pp_smem()) return e;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int pxh = px / 2 + 1;
  const int rx = reg_fft_radix(px), ry = reg_fft_radix(py);
  if (rx && ry) {
    for (int64_t k0 = 0; k0 < n_images; k0 += 65535) {
      const int cnt = (int)std::min<int64_t>(65535, n_images - k0);
      float2* o = static_cast<float2*>(out) + (size_t)k0 * py * pxh;
      const float* im = image + (size_t)k0 * py * px;
      prof_begin(s);
      switch (rx) {
#define CJX_PPR(R)                                                                                          \
  case R:                                                                                                   \
    k_pp_rows_r2c_reg<R><<<dim3((py + 2 * kWarps - 1) / (2 * kWarps), cnt), kWarps * 32, smem_reg(px), s>>>( \
        im, o, py);                                                                                         \
    break;
        CJX_PPR(1) CJX_PPR(2) CJX_PPR(3) CJX_PPR(4) CJX_PPR(5) CJX_PPR(6) CJX_PPR(8) CJX_PPR(10) CJX_PPR(12) CJX_PPR(16)
#undef CJX_PPR
      }
      prof_end("k_pp_rows_r2c", s);
      prof_begin(s);
      switch (ry) {
#define CJX_PPC(R)                                                                                                 \
  case R:                                                                                                          \
    k_pp_colfft_reg<R><<<dim3((pxh + kWarps - 1) / kWarps, cnt), kWarps * 32, smem_reg(py), s>>>(o, px);           \
    break;
        CJX_PPC(1) CJX_PPC(2) CJX_PPC(3) CJX_PPC(4) CJX_PPC(5) CJX_PPC(6) CJX_PPC(8) CJX_PPC(10) CJX_PPC(12) CJX_PPC(16)
#undef CJX_PPC
      }
      prof_end("k_pp_colfft", s);
    }
    return check_cuda(cudaGetLastError(), "rfft2 launch");
  }
  const FftPlan plan_y = make_fft_plan(py), plan_x = make_fft_plan(px);
  for (int64_t k0 = 0; k0 < n_images; k0 += 65535) {
    const int cnt = (int)std::min<int64_t>(65535, n_images - k0);
    float2* o = static_cast<float2*>(out) + (size_t)k0 * py * pxh;
    prof_begin(s);
    k_pp_rows_r2c<<<dim3((py + 2 * kWarps - 1) / (2 * kWarps), cnt), kWarps * 32, smem_rows(px), s>>>(
        image + (size_t)k0 * py * px, o, py, px, plan_x);
    prof_end("k_pp_rows_r2c", s);
    prof_begin(s);
    k_pp_colfft<<<dim3((pxh + kWarps - 1) / kWarps, cnt), kWarps * 32, smem_cols(py), s>>>(
        o, py, px, plan_y, fft_result_offset(plan_y, py));
    prof_end("k_pp_colfft", s);
  }
  return check_cuda(cudaGetLastError(), "rfft2 launch");
}
