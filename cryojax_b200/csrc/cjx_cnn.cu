// Pose-proposal network kernels (everything except the GEMMs, which run on
// the tensor cores through launch_gemm): input noise + normalisation,
// im2col / col2im for 3x3 stride-2 convolutions in NHWC BF16, BF16
// transposes, ReLU masks, column sums (bias gradients), softmax cross
// entropy with neighbour label smoothing, AdamW with BF16 weight copies,
// and top-k direction proposals expanded to in-plane candidates.
// No counterpart in the reference (its pose search has no network).
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "cjx_common.cuh"
#include "cjx_profile.cuh"

namespace cjx {

using bf16 = __nv_bfloat16;

static unsigned grid_for(int64_t n, int threads, int64_t cap = 148 * 32) {
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(cap, (n + threads - 1) / threads));
}

__device__ __forceinline__ float block_sum(float v, float* red) {
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  float t = 0.f;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  return t;
}

// Counter-based standard normal draw: SplitMix64 (Steele, Lea, Flood,
// "Fast splittable pseudorandom number generators", OOPSLA 2014) of
// (seed, image, pixel) gives two 24-bit uniforms; Box-Muller maps them to
// one normal variate.
__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ float normal_draw(uint64_t seed, int64_t image, int64_t pixel) {
  const uint64_t h = splitmix64(seed ^ splitmix64((uint64_t)image * 0x100000001B3ull + (uint64_t)pixel));
  const float u1 = ((float)(h >> 40) + 0.5f) * (1.0f / 16777216.0f);  // (0, 1)
  const float u2 = (float)((h >> 16) & 0xFFFFFF) * (1.0f / 16777216.0f);
  float s, c;
  sincospif(2.0f * u2, &s, &c);
  return sqrtf(-2.0f * logf(u1)) * c;
}

// out[b] = normalise(img[src_b] + sigma_b * noise), sigma_b^2 = var(img[src_b]) / snr
// (snr <= 0: no noise).  normalise = zero mean, unit standard deviation
// (population), written as BF16 [b][h][w][1].  src_b = index ? index[b] : b.
__global__ void k_noisy_normalize(const float* __restrict__ img, const int64_t* __restrict__ index, int hw,
                                  float snr, uint64_t seed, bf16* __restrict__ out) {
  __shared__ float red[32];
  const int64_t src = index ? index[blockIdx.x] : blockIdx.x;
  const float* x = img + (size_t)src * hw;
  float sigma = 0.f;
  if (snr > 0.f) {
    float s = 0.f;
    for (int i = threadIdx.x; i < hw; i += blockDim.x) s += x[i];
    const float mean = block_sum(s, red) / hw;
    float v = 0.f;
    for (int i = threadIdx.x; i < hw; i += blockDim.x) {
      const float d = x[i] - mean;
      v += d * d;
    }
    sigma = sqrtf(block_sum(v, red) / hw / snr);
  }
  float s = 0.f;
  for (int i = threadIdx.x; i < hw; i += blockDim.x) s += x[i] + (sigma > 0.f ? sigma * normal_draw(seed, src, i) : 0.f);
  const float mean = block_sum(s, red) / hw;
  float v = 0.f;
  for (int i = threadIdx.x; i < hw; i += blockDim.x) {
    const float d = x[i] + (sigma > 0.f ? sigma * normal_draw(seed, src, i) : 0.f) - mean;
    v += d * d;
  }
  const float var = block_sum(v, red) / hw;
  const float inv = var > 0.f ? rsqrtf(var) : 1.f;
  bf16* o = out + (size_t)blockIdx.x * hw;
  for (int i = threadIdx.x; i < hw; i += blockDim.x)
    o[i] = __float2bfloat16_rn((x[i] + (sigma > 0.f ? sigma * normal_draw(seed, src, i) : 0.f) - mean) * inv);
}

// Area-weighted downsampling: output pixel (i, j) of an h x w image is the
// mean of the input over [i H/h, (i+1) H/h) x [j W/w, (j+1) W/w), input
// pixels weighted by their overlap.
__device__ __forceinline__ float overlap(float a0, float a1, int p) {
  return fmaxf(0.f, fminf(a1, (float)(p + 1)) - fmaxf(a0, (float)p));
}

__global__ void k_area_downsample(const float* __restrict__ src, int H, int W, float* __restrict__ dst, int h, int w,
                                  int64_t n) {
  const float fy = (float)H / h, fx = (float)W / w;
  const float inv = 1.f / (fy * fx);
  const int64_t total = n * h * w;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int j = (int)(e % w);
    const int64_t t = e / w;
    const int i = (int)(t % h);
    const int64_t b = t / h;
    const float y0 = i * fy, y1 = (i + 1) * fy, x0 = j * fx, x1 = (j + 1) * fx;
    const float* s = src + (size_t)b * H * W;
    float acc = 0.f;
    for (int y = (int)floorf(y0); y < min(H, (int)ceilf(y1)); ++y) {
      const float wy = overlap(y0, y1, y);
      for (int x = (int)floorf(x0); x < min(W, (int)ceilf(x1)); ++x) acc += wy * overlap(x0, x1, x) * s[(size_t)y * W + x];
    }
    dst[e] = acc * inv;
  }
}

// col[p][k] for a 3x3, stride-2, pad-1 convolution of x [B][H][W][C]:
// p = (b Ho + oy) Wo + ox, k = (3 ky + kx) C + c, zero in [9C, ldk).
template <bool VEC>
__global__ void k_im2col_s2(const bf16* __restrict__ x, int B, int H, int W, int C, bf16* __restrict__ col,
                            int ldk) {
  const int Ho = H / 2, Wo = W / 2;
  const int gpr = ldk / 8;
  const int64_t total = (int64_t)B * Ho * Wo * gpr;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = e / gpr;
    const int k0 = (int)(e - p * gpr) * 8;
    const int ox = (int)(p % Wo);
    const int64_t t = p / Wo;
    const int oy = (int)(t % Ho);
    const int b = (int)(t / Ho);
    uint4 v = make_uint4(0, 0, 0, 0);
    if (VEC) {
      const int tap = k0 / C, c0 = k0 - tap * C;
      if (tap < 9) {
        const int iy = 2 * oy + tap / 3 - 1, ix = 2 * ox + tap % 3 - 1;
        if (iy >= 0 && ix >= 0 && iy < H && ix < W)
          v = *reinterpret_cast<const uint4*>(x + (((size_t)b * H + iy) * W + ix) * C + c0);
      }
    } else {
      bf16 h[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int k = k0 + j;
        h[j] = __float2bfloat16_rn(0.f);
        const int tap = k / C;
        if (tap < 9) {
          const int c = k - tap * C;
          const int iy = 2 * oy + tap / 3 - 1, ix = 2 * ox + tap % 3 - 1;
          if (iy >= 0 && ix >= 0 && iy < H && ix < W) h[j] = x[(((size_t)b * H + iy) * W + ix) * C + c];
        }
      }
      v = *reinterpret_cast<const uint4*>(h);
    }
    *reinterpret_cast<uint4*>(col + p * ldk + k0) = v;
  }
}

// First layer at inference: 3x3 stride-2 convolution of a one-channel BF16
// image (zero padding 1) into COUT channels, + bias, ReLU, BF16 NHWC out,
// with no im2col matrix: what im2col + the tensor-core GEMM compute for
// that layer (weights w [COUT][ldk], tap k = 3 dy + dx), one output pixel
// per thread.  BF16 products are exact in FP32; the 9 taps are summed in
// tap order, then the bias is added, as the GEMM epilogue adds it.
template <int COUT>
__global__ void __launch_bounds__(256, 4)
    k_conv0_s2(const bf16* __restrict__ x, int B, int H, int W, const bf16* __restrict__ w, int ldk,
               const float* __restrict__ bias, bf16* __restrict__ y) {
  __shared__ float ws[9][COUT];
  __shared__ float bs[COUT];
  for (int e = threadIdx.x; e < 9 * COUT; e += blockDim.x) ws[e / COUT][e % COUT] = __bfloat162float(w[(e % COUT) * ldk + e / COUT]);
  for (int c = threadIdx.x; c < COUT; c += blockDim.x) bs[c] = bias ? bias[c] : 0.f;
  __syncthreads();
  const int Ho = H / 2, Wo = W / 2;
  const int64_t total = (int64_t)B * Ho * Wo;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < total; p += (int64_t)gridDim.x * blockDim.x) {
    const int ox = (int)(p % Wo);
    const int64_t t = p / Wo;
    const int oy = (int)(t % Ho);
    const int64_t b = t / Ho;
    float in[9];
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int iy = 2 * oy + tap / 3 - 1, ix = 2 * ox + tap % 3 - 1;
      in[tap] = (iy >= 0 && ix >= 0 && iy < H && ix < W) ? __bfloat162float(x[((size_t)b * H + iy) * W + ix]) : 0.f;
    }
    uint4* dst = reinterpret_cast<uint4*>(y + (size_t)p * COUT);
#pragma unroll 1
    for (int c8 = 0; c8 < COUT / 8; ++c8) {
      __align__(16) bf16 o[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int c = 8 * c8 + q;
        float acc = 0.f;
#pragma unroll
        for (int tap = 0; tap < 9; ++tap) acc = fmaf(in[tap], ws[tap][c], acc);
        o[q] = __float2bfloat16_rn(fmaxf(acc + bs[c], 0.f));
      }
      dst[c8] = *reinterpret_cast<const uint4*>(o);
    }
  }
}

// D (16 x 8, FP32) += A (16 x 16, BF16) B (16 x 8, BF16) on the tensor cores.
__device__ __forceinline__ void mma16816_bf16(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                              uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// A later layer at inference without the im2col matrix (implicit GEMM):
// y (BF16 NHWC [B][H/2][W/2][64 NG]) = ReLU(conv3x3_s2(x) + bias) for x
// (BF16 NHWC [B][H][W][CIN], zero padding 1) and weights w [64 NG][ldk]
// with k = (3 ky + kx) CIN + c, the im2col order.  Each warp takes 16 output
// pixels x 64 channels; a CTA's 8 warps cover 8 / NG pixel tiles x NG
// channel groups.  A K step is one tap's 32 channels: lane (g, t) loads
// channels [8 t, 8 t + 8) of the tap for pixels g and g + 8 and of the
// weights for channels g of each 8-wide column tile, and the step's two
// m16n8k16 products take them as k = {2t, 2t+1, 2t+8, 2t+9}: the same
// relabelling for both operands, so the sums are the convolution's.  BF16
// products, FP32 accumulation, then bias, ReLU and BF16 as the GEMM's
// epilogue.
template <int CIN, int NG>
__global__ void __launch_bounds__(256)
    k_conv_s2_mma(const bf16* __restrict__ x, int B, int H, int W, const bf16* __restrict__ w, int ldk,
                  const float* __restrict__ bias, bf16* __restrict__ y) {
  static_assert(CIN % 32 == 0, "one K step is 32 channels of one tap");
  constexpr int COUT = 64 * NG;
  constexpr int MT = 8 / NG;  // pixel tiles of 16 per CTA
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int Ho = H / 2, Wo = W / 2;
  const int64_t total = (int64_t)B * Ho * Wo;
  const int64_t p0 = (int64_t)blockIdx.x * (16 * MT) + 16 * (warp % MT);
  const int n0 = 64 * (warp / MT);
  // this lane's two output pixels (g and g + 8 of the warp's tile)
  int oy[2], ox[2];
  int64_t ob[2];
  bool live[2];
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int64_t p = p0 + g + 8 * h;
    live[h] = p < total;
    const int64_t pp = live[h] ? p : 0;
    ox[h] = (int)(pp % Wo);
    oy[h] = (int)((pp / Wo) % Ho);
    ob[h] = pp / ((int64_t)Wo * Ho);
  }
  float acc[8][4];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  const uint4 z = make_uint4(0u, 0u, 0u, 0u);
#pragma unroll 1
  for (int tap = 0; tap < 9; ++tap) {
    const int ky = tap / 3, kx = tap % 3;
    const bf16* src[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int iy = 2 * oy[h] + ky - 1, ix = 2 * ox[h] + kx - 1;
      src[h] = (live[h] && iy >= 0 && ix >= 0 && iy < H && ix < W) ? x + ((ob[h] * H + iy) * W + ix) * CIN : nullptr;
    }
#pragma unroll 1
    for (int c0 = 0; c0 < CIN; c0 += 32) {
      const uint4 al = src[0] ? *reinterpret_cast<const uint4*>(src[0] + c0 + 8 * t) : z;
      const uint4 ah = src[1] ? *reinterpret_cast<const uint4*>(src[1] + c0 + 8 * t) : z;
      const int k = tap * CIN + c0 + 8 * t;
      uint4 b[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = __ldg(reinterpret_cast<const uint4*>(w + (size_t)(n0 + 8 * j + g) * ldk + k));
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        mma16816_bf16(acc[j], al.x, ah.x, al.y, ah.y, b[j].x, b[j].y);
        mma16816_bf16(acc[j], al.z, ah.z, al.w, ah.w, b[j].z, b[j].w);
      }
    }
  }
  // accumulator (pixel g / g + 8, channel 8 j + 2 t / + 1): bias, ReLU, BF16 pairs
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (!live[h]) continue;
    bf16* dst = y + (size_t)(p0 + g + 8 * h) * COUT + n0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = 8 * j + 2 * t;
      const float b0 = bias ? bias[n0 + c] : 0.f, b1 = bias ? bias[n0 + c + 1] : 0.f;
      __nv_bfloat162 v;
      v.x = __float2bfloat16_rn(fmaxf(acc[j][2 * h] + b0, 0.f));
      v.y = __float2bfloat16_rn(fmaxf(acc[j][2 * h + 1] + b1, 0.f));
      *reinterpret_cast<__nv_bfloat162*>(dst + c) = v;
    }
  }
}

// dx[b][y][x][c] = sum over the taps that read (y, x) of dcol[p][k], times
// (act > 0) when act is given (ReLU of the layer that produced x).
__global__ void k_col2im_s2(const float* __restrict__ dcol, int ldk, const bf16* __restrict__ act, int B, int H,
                            int W, int C, bf16* __restrict__ dx) {
  const int Ho = H / 2, Wo = W / 2;
  const int64_t total = (int64_t)B * H * W * C;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    if (act && !(__bfloat162float(act[e]) > 0.f)) {
      dx[e] = __float2bfloat16_rn(0.f);
      continue;
    }
    const int c = (int)(e % C);
    int64_t t = e / C;
    const int xx = (int)(t % W);
    t /= W;
    const int y = (int)(t % H);
    const int b = (int)(t / H);
    float s = 0.f;
#pragma unroll
    for (int ky = 0; ky < 3; ++ky) {
      const int ty = y + 1 - ky;
      if (ty < 0 || (ty & 1) || (ty >> 1) >= Ho) continue;
#pragma unroll
      for (int kx = 0; kx < 3; ++kx) {
        const int tx = xx + 1 - kx;
        if (tx < 0 || (tx & 1) || (tx >> 1) >= Wo) continue;
        s += dcol[(((size_t)b * Ho + (ty >> 1)) * Wo + (tx >> 1)) * ldk + (3 * ky + kx) * C + c];
      }
    }
    dx[e] = __float2bfloat16_rn(s);
  }
}

template <typename Tin>
__device__ __forceinline__ float to_f(Tin v);
template <>
__device__ __forceinline__ float to_f<float>(float v) { return v; }
template <>
__device__ __forceinline__ float to_f<bf16>(bf16 v) { return __bfloat162float(v); }

// out[c][r] = in[r][c] (to BF16), 32 x 32 tiles through shared memory.
template <typename Tin>
__global__ void k_transpose_to_bf16(const Tin* __restrict__ in, int64_t rows, int64_t cols, int64_t ldi,
                                    bf16* __restrict__ out, int64_t ldo) {
  __shared__ float tile[32][33];
  const int64_t c0 = (int64_t)blockIdx.x * 32, r0 = (int64_t)blockIdx.y * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int64_t r = r0 + j, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[j][threadIdx.x] = to_f<Tin>(in[r * ldi + c]);
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int64_t c = c0 + j, r = r0 + threadIdx.x;
    if (c < cols && r < rows) out[c * ldo + r] = __float2bfloat16_rn(tile[threadIdx.x][j]);
  }
}

__global__ void k_relu_mask(const float* __restrict__ g, const bf16* __restrict__ act, int64_t n,
                            bf16* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn((act == nullptr || __bfloat162float(act[i]) > 0.f) ? g[i] : 0.f);
}

// out[c] += sum_r x[r][c]; block (32 x 8) per 32 columns x a chunk of rows.
template <typename Tin>
__global__ void k_colsum(const Tin* __restrict__ x, int64_t rows, int64_t cols, int64_t ld, int64_t rows_per_block,
                         float* __restrict__ out) {
  __shared__ float red[8][33];
  const int64_t c = (int64_t)blockIdx.x * 32 + threadIdx.x;
  const int64_t r0 = (int64_t)blockIdx.y * rows_per_block, r1 = min(rows, r0 + rows_per_block);
  float s = 0.f;
  if (c < cols)
    for (int64_t r = r0 + threadIdx.y; r < r1; r += 8) s += to_f<Tin>(x[r * ld + c]);
  red[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && c < cols) {
    float t = 0.f;
    for (int j = 0; j < 8; ++j) t += red[j][threadIdx.x];
    atomicAdd(out + c, t);
  }
}

// One warp per row: softmax cross entropy against the target
// (1 - eps) at the label + eps / n_nb at each of its n_nb neighbours
// (eps / C everywhere when n_nb == 0).  loss[r] = -sum t log p;
// dlogits[r][j] = (p_j - t_j) * grad_scale as BF16 (when non-NULL).
__global__ void k_softmax_xent(const float* __restrict__ logits, int64_t B, int C, const int32_t* __restrict__ labels,
                               const int32_t* __restrict__ nb, int n_nb, float eps, float grad_scale,
                               float* __restrict__ loss, bf16* __restrict__ dlogits) {
  const int64_t r = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= B) return;
  const float* l = logits + r * C;
  float m = -INFINITY;
  for (int j = lane; j < C; j += 32) m = fmaxf(m, l[j]);
  for (int s = 16; s > 0; s >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, s));
  float z = 0.f;
  for (int j = lane; j < C; j += 32) z += expf(l[j] - m);
  for (int s = 16; s > 0; s >>= 1) z += __shfl_xor_sync(0xffffffffu, z, s);
  const float logz = m + logf(z);
  const int lab = labels[r];
  const int32_t* nbr = (nb && n_nb > 0) ? nb + (size_t)lab * n_nb : nullptr;
  // target t_j = (1 - eps) [j == lab] + (eps / n_nb per listed neighbour, or eps / C for every j)
  const float w_nb = nbr ? eps / n_nb : eps / C;
  if (lane == 0 && loss) {
    float t = (1.f - eps) * (logz - l[lab]);
    if (nbr) {
      for (int q = 0; q < n_nb; ++q) t += w_nb * (logz - l[nbr[q]]);
    } else if (eps > 0.f) {
      float sum_l = 0.f;
      for (int j = 0; j < C; ++j) sum_l += logz - l[j];
      t += w_nb * sum_l;
    }
    loss[r] = t;
  }
  if (dlogits) {
    for (int j = lane; j < C; j += 32) {
      float t = (j == lab) ? 1.f - eps : 0.f;
      if (nbr) {
        for (int q = 0; q < n_nb; ++q) t += (nbr[q] == j) ? w_nb : 0.f;
      } else {
        t += w_nb;
      }
      dlogits[r * C + j] = __float2bfloat16_rn((expf(l[j] - logz) - t) * grad_scale);
    }
  }
}

constexpr int kMaxParamSegments = 24;
struct ParamSegments {
  cjx_param_segment s[kMaxParamSegments];
  int n;
};

// AdamW over the flat FP32 parameter vector; weight segments also refresh
// their BF16 copies W [cols][ldk] (element (k, o) at o * ldk + k) and
// Wt [rows][cols] (at k * cols + o), where the FP32 master is [rows][cols].
__global__ void k_adamw(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                        float* __restrict__ v, int64_t n, ParamSegments segs, float lr, float b1, float b2,
                        float eps, float wd, float bc1, float bc2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    int si = 0;
    while (si + 1 < segs.n && i >= segs.s[si + 1].offset) ++si;
    const cjx_param_segment& sg = segs.s[si];
    const float decay = sg.weight_decay ? wd : 0.f;
    const float pi = p[i] - lr * ((mi / bc1) / (sqrtf(vi / bc2) + eps) + decay * p[i]);
    p[i] = pi;
    if (sg.cols > 0 && i >= sg.offset && i < sg.offset + sg.count) {
      const int64_t e = i - sg.offset;
      const int64_t k = e / sg.cols, o = e - k * sg.cols;
      const bf16 h = __float2bfloat16_rn(pi);
      if (sg.w_bf16) static_cast<bf16*>(sg.w_bf16)[o * sg.ldk + k] = h;
      if (sg.wt_bf16) static_cast<bf16*>(sg.wt_bf16)[k * sg.cols + o] = h;
    }
  }
}

// One warp per row: the k largest logits (ties -> lower index), then
// candidates[r][t * n_inplane + a] = dirs[r][t] * n_inplane + a.
__global__ void k_topk_candidates(const float* __restrict__ logits, int64_t B, int C, int k, int n_inplane,
                                  int32_t* __restrict__ dirs, int32_t* __restrict__ cand) {
  const int64_t r = blockIdx.x * (int64_t)(blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (r >= B) return;
  float v[32];
#pragma unroll
  for (int i = 0; i < 32; ++i) {
    const int j = lane + 32 * i;
    v[i] = j < C ? logits[r * C + j] : -INFINITY;
  }
  for (int t = 0; t < k; ++t) {
    float bv = -INFINITY;
    int bj = 0x7fffffff;
#pragma unroll
    for (int i = 0; i < 32; ++i) {
      const int j = lane + 32 * i;
      if (j < C && (v[i] > bv || (v[i] == bv && j < bj))) {
        bv = v[i];
        bj = j;
      }
    }
    for (int s = 16; s > 0; s >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, bv, s);
      const int oj = __shfl_xor_sync(0xffffffffu, bj, s);
      if (ov > bv || (ov == bv && oj < bj)) {
        bv = ov;
        bj = oj;
      }
    }
    if (bj == 0x7fffffff) bj = t;  // fewer finite logits than k (NaN rows): any distinct index
    if ((bj & 31) == lane) {
#pragma unroll
      for (int i = 0; i < 32; ++i)
        if (lane + 32 * i == bj) v[i] = -INFINITY;
    }
    if (dirs && lane == 0) dirs[r * k + t] = bj;
    if (cand)
      for (int a = lane; a < n_inplane; a += 32) cand[(r * k + t) * n_inplane + a] = bj * n_inplane + a;
  }
}

}  // namespace cjx

// ---- C-ABI -------------------------------------------------------------------

using cjx::bf16;

extern "C" {

int cjx_cnn_noisy_normalize(const float* images, const int64_t* index, int64_t n, int h, int w, float snr,
                            uint64_t seed, void* out, void* stream) {
  if (n < 0 || h < 1 || w < 1) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "bad image batch shape");
  if (n == 0) return CJX_OK;
  if (!images || !out) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "images and out must be non-NULL");
  if (n > 2147483647LL) return cjx::fail(CJX_ERR_UNSUPPORTED, "too many images");
  cjx::prof_begin(static_cast<cudaStream_t>(stream));
  cjx::k_noisy_normalize<<<(unsigned)n, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      images, index, h * w, snr, seed, static_cast<bf16*>(out));
  cjx::prof_end("k_noisy_normalize", static_cast<cudaStream_t>(stream));
  return cjx::check_cuda(cudaGetLastError(), "noisy_normalize launch");
}

int cjx_area_downsample(const float* src, int64_t n, int H, int W, float* dst, int h, int w, void* stream) {
  if (n < 0 || h < 1 || w < 1 || H < h || W < w)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "area_downsample needs 1 <= h <= H and 1 <= w <= W");
  if (n == 0) return CJX_OK;
  if (!src || !dst) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "src and dst must be non-NULL");
  cjx::k_area_downsample<<<cjx::grid_for(n * h * w, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      src, H, W, dst, h, w, n);
  return cjx::check_cuda(cudaGetLastError(), "area_downsample launch");
}

int cjx_cnn_im2col(const void* x, int64_t B, int H, int W, int C, void* col, int64_t ldk, void* stream) {
  if (B < 0 || H < 2 || W < 2 || (H & 1) || (W & 1) || C < 1 || ldk < 9 * C || (ldk % 8))
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "im2col needs even H, W >= 2, C >= 1, ldk >= 9C, ldk % 8 == 0");
  if (B == 0) return CJX_OK;
  if (!x || !col) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "x and col must be non-NULL");
  const int64_t total = B * (H / 2) * (W / 2) * (ldk / 8);
  auto st = static_cast<cudaStream_t>(stream);
  if (C % 8 == 0)
    cjx::k_im2col_s2<true><<<cjx::grid_for(total, 256), 256, 0, st>>>(static_cast<const bf16*>(x), (int)B, H, W, C,
                                                                      static_cast<bf16*>(col), (int)ldk);
  else
    cjx::k_im2col_s2<false><<<cjx::grid_for(total, 256), 256, 0, st>>>(static_cast<const bf16*>(x), (int)B, H, W, C,
                                                                       static_cast<bf16*>(col), (int)ldk);
  return cjx::check_cuda(cudaGetLastError(), "im2col launch");
}

int cjx_cnn_conv0(const void* x, int64_t B, int H, int W, const void* w, int64_t ldk, int cout, const float* bias,
                  void* y, void* stream) {
  if (B < 0 || H < 2 || W < 2 || (H & 1) || (W & 1) || ldk < 9 || cout != 32)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "cnn_conv0 needs even H, W >= 2, ldk >= 9 and cout = 32");
  if (B == 0) return CJX_OK;
  if (!x || !w || !y) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "x, w and y must be non-NULL");
  if (reinterpret_cast<uintptr_t>(y) % 16) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "y must be 16-byte aligned");
  const int64_t total = B * (H / 2) * (W / 2);
  cjx::prof_begin(static_cast<cudaStream_t>(stream));
  cjx::k_conv0_s2<32><<<cjx::grid_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const bf16*>(x), (int)B, H, W, static_cast<const bf16*>(w), (int)ldk, bias, static_cast<bf16*>(y));
  cjx::prof_end("k_conv0_s2", static_cast<cudaStream_t>(stream));
  return cjx::check_cuda(cudaGetLastError(), "cnn_conv0 launch");
}

int cjx_cnn_conv_s2(const void* x, int64_t B, int H, int W, int C, const void* w, int64_t ldk, int cout,
                    const float* bias, void* y, void* stream) {
  if (B < 0 || H < 2 || W < 2 || (H & 1) || (W & 1) || ldk < 9 * C || (ldk % 8))
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "cnn_conv_s2 needs even H, W >= 2, ldk >= 9 C, ldk % 8 == 0");
  if (B == 0) return CJX_OK;
  if (!x || !w || !y) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "x, w and y must be non-NULL");
  for (const void* ptr : {x, w})
    if (reinterpret_cast<uintptr_t>(ptr) % 16)
      return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "cnn_conv_s2: x and w must be 16-byte aligned");
  if (reinterpret_cast<uintptr_t>(y) % 4) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "y must be 4-byte aligned");
  const int64_t total = B * (H / 2) * (W / 2);
  auto st = static_cast<cudaStream_t>(stream);
  const bf16* xb = static_cast<const bf16*>(x);
  const bf16* wb = static_cast<const bf16*>(w);
  bf16* yb = static_cast<bf16*>(y);
#define CJX_CONV_CASE(CI, NG)                                                                                      \
  if (C == CI && cout == 64 * NG) {                                                                                \
    const int64_t ctas = (total + 16 * (8 / NG) - 1) / (16 * (8 / NG));                                            \
    if (ctas > 2147483647LL) return cjx::fail(CJX_ERR_UNSUPPORTED, "cnn_conv_s2: too many pixels");             \
    cjx::prof_begin(st);                                                                                          \
    cjx::k_conv_s2_mma<CI, NG><<<(unsigned)ctas, 256, 0, st>>>(xb, (int)B, H, W, wb, (int)ldk, bias, yb);          \
    cjx::prof_end("k_conv_s2_mma", st);                                                                           \
    return cjx::check_cuda(cudaGetLastError(), "cnn_conv_s2 launch");                                             \
  }
  CJX_CONV_CASE(32, 1) CJX_CONV_CASE(64, 2) CJX_CONV_CASE(128, 2) CJX_CONV_CASE(128, 4) CJX_CONV_CASE(256, 4)
#undef CJX_CONV_CASE
  return cjx::fail(CJX_ERR_UNSUPPORTED, "cnn_conv_s2: (C, cout) must be (32, 64), (64, 128), (128, 128), "
                                        "(128, 256) or (256, 256)");
}

int cjx_cnn_col2im(const float* dcol, int64_t ldk, const void* act, int64_t B, int H, int W, int C, void* dx,
                   void* stream) {
  if (B < 0 || H < 2 || W < 2 || (H & 1) || (W & 1) || C < 1 || ldk < 9 * C)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "col2im needs even H, W >= 2, C >= 1, ldk >= 9C");
  if (B == 0) return CJX_OK;
  if (!dcol || !dx) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "dcol and dx must be non-NULL");
  const int64_t total = B * H * W * C;
  cjx::k_col2im_s2<<<cjx::grid_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      dcol, (int)ldk, static_cast<const bf16*>(act), (int)B, H, W, C, static_cast<bf16*>(dx));
  return cjx::check_cuda(cudaGetLastError(), "col2im launch");
}

int cjx_transpose_to_bf16(const void* in, int in_is_bf16, int64_t rows, int64_t cols, int64_t ld_in, void* out,
                          int64_t ld_out, void* stream) {
  if (rows < 0 || cols < 0 || ld_in < cols || ld_out < rows)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "transpose needs ld_in >= cols, ld_out >= rows");
  if (rows == 0 || cols == 0) return CJX_OK;
  if (!in || !out) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "in and out must be non-NULL");
  if ((rows + 31) / 32 > 65535) return cjx::fail(CJX_ERR_UNSUPPORTED, "transpose: too many rows");
  const dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32));
  auto st = static_cast<cudaStream_t>(stream);
  if (in_is_bf16)
    cjx::k_transpose_to_bf16<bf16><<<grid, dim3(32, 8), 0, st>>>(static_cast<const bf16*>(in), rows, cols, ld_in,
                                                                 static_cast<bf16*>(out), ld_out);
  else
    cjx::k_transpose_to_bf16<float><<<grid, dim3(32, 8), 0, st>>>(static_cast<const float*>(in), rows, cols, ld_in,
                                                                  static_cast<bf16*>(out), ld_out);
  return cjx::check_cuda(cudaGetLastError(), "transpose launch");
}

int cjx_relu_mask(const float* grad, const void* act, int64_t n, void* out, void* stream) {
  if (n < 0) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "n < 0");
  if (n == 0) return CJX_OK;
  if (!grad || !out) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "grad and out must be non-NULL");
  cjx::k_relu_mask<<<cjx::grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      grad, static_cast<const bf16*>(act), n, static_cast<bf16*>(out));
  return cjx::check_cuda(cudaGetLastError(), "relu_mask launch");
}

int cjx_colsum(const void* x, int x_is_bf16, int64_t rows, int64_t cols, int64_t ld, float* out, void* stream) {
  if (rows < 0 || cols < 0 || ld < cols) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "colsum needs ld >= cols");
  if (rows == 0 || cols == 0) return CJX_OK;
  if (!x || !out) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "x and out must be non-NULL");
  const int64_t col_blocks = (cols + 31) / 32;
  const int64_t row_blocks = std::min<int64_t>(std::max<int64_t>(1, 1184 / col_blocks), (rows + 255) / 256);
  const int64_t rpb = (rows + row_blocks - 1) / row_blocks;
  const dim3 grid((unsigned)col_blocks, (unsigned)((rows + rpb - 1) / rpb));
  auto st = static_cast<cudaStream_t>(stream);
  if (x_is_bf16)
    cjx::k_colsum<bf16><<<grid, dim3(32, 8), 0, st>>>(static_cast<const bf16*>(x), rows, cols, ld, rpb, out);
  else
    cjx::k_colsum<float><<<grid, dim3(32, 8), 0, st>>>(static_cast<const float*>(x), rows, cols, ld, rpb, out);
  return cjx::check_cuda(cudaGetLastError(), "colsum launch");
}

int cjx_softmax_xent(const float* logits, int64_t B, int C, const int32_t* labels, const int32_t* neighbours,
                     int n_neighbours, float smoothing, float grad_scale, float* loss, void* dlogits, void* stream) {
  if (B < 0 || C < 1 || n_neighbours < 0 || smoothing < 0.f || smoothing > 1.f)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "softmax_xent: bad sizes or smoothing");
  if (B == 0) return CJX_OK;
  if (!logits || !labels) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "logits and labels must be non-NULL");
  const unsigned blocks = (unsigned)((B + 7) / 8);
  cjx::k_softmax_xent<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      logits, B, C, labels, neighbours, neighbours ? n_neighbours : 0, smoothing, grad_scale, loss,
      static_cast<bf16*>(dlogits));
  return cjx::check_cuda(cudaGetLastError(), "softmax_xent launch");
}

int cjx_adamw(float* params, const float* grads, float* m, float* v, int64_t n, const cjx_param_segment* segments,
              int n_segments, float lr, float beta1, float beta2, float eps, float weight_decay, int64_t step,
              void* stream) {
  if (n < 0 || n_segments < 1 || n_segments > cjx::kMaxParamSegments || step < 1)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "adamw: need n >= 0, 1..24 segments, step >= 1");
  if (n == 0) return CJX_OK;
  if (!params || !grads || !m || !v || !segments)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "adamw: NULL pointer");
  cjx::ParamSegments segs{};
  segs.n = n_segments;
  for (int i = 0; i < n_segments; ++i) {
    segs.s[i] = segments[i];
    const cjx_param_segment& s = segments[i];
    if (s.offset < 0 || s.count < 0 || s.offset + s.count > n || (i > 0 && s.offset < segments[i - 1].offset) ||
        (s.cols > 0 && (s.count % s.cols || s.ldk < s.count / s.cols)))
      return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "adamw: bad parameter segment");
  }
  if (segments[0].offset != 0) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "adamw: first segment must start at 0");
  const float bc1 = 1.f - powf(beta1, (float)step), bc2 = 1.f - powf(beta2, (float)step);
  cjx::k_adamw<<<cjx::grid_for(n, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      params, grads, m, v, n, segs, lr, beta1, beta2, eps, weight_decay, bc1, bc2);
  return cjx::check_cuda(cudaGetLastError(), "adamw launch");
}

int cjx_topk_candidates(const float* logits, int64_t B, int C, int k, int n_inplane, int32_t* dirs,
                        int32_t* candidates, void* stream) {
  if (B < 0 || C < 1 || C > 1024 || k < 1 || k > C || n_inplane < 1)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "topk: need 1 <= k <= C <= 1024, n_inplane >= 1");
  if (B == 0) return CJX_OK;
  if (!logits) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "logits must be non-NULL");
  cjx::prof_begin(static_cast<cudaStream_t>(stream));
  cjx::k_topk_candidates<<<(unsigned)((B + 7) / 8), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      logits, B, C, k, n_inplane, dirs, candidates);
  cjx::prof_end("k_topk_candidates", static_cast<cudaStream_t>(stream));
  return cjx::check_cuda(cudaGetLastError(), "topk launch");
}

}  // extern "C"
