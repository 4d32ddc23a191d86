// Template-sharing exhaustive search: the NCC of every (image, orientation)
// pair from two tensor-core GEMMs instead of one simulation per pair.
//
// The simulated image of orientation t for image b is F = m_b * S_t, with
// S_t the CTF-free central slice (resized, Hermitian-fixed columns) and m_b
// the image's multiplier (scale, CTF, envelope, translation phase, Nyquist
// zeroing; real and even in ky on the self-conjugate columns, so it
// commutes with their Hermitian fix).  With Parseval weights w (0 at DC, 1
// on the self-conjugate columns kx = 0 and kx = Px/2, 2 elsewhere):
//   num(b, t) = sum w Re(conj(O_b) m_b S_t) = sum Y_b . S_t,  Y_b = w conj(m_b) O_b
//   den(b, t) = sum w |m_b|^2 |S_t|^2      = sum Z_b |S_t|^2, Z_b = w |m_b|^2
//   NCC = num / sqrt(den * sum w |O_b|^2)
// so num is a GEMM over K = 2 Py (Px/2+1) interleaved (re, im) values and
// den one over K = Py (Px/2+1).  Rows are stored in FP16 after a per-row
// scale to unit RMS (the scales cancel in the NCC except for the image's).
// No counterpart in the reference: its grid search simulates every pair.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "cjx_common.cuh"
#include "cjx_profile.cuh"

namespace cjx {

__device__ __forceinline__ float block_sum_f(float v, float* red) {
  for (int s = 16; s > 0; s >>= 1) v += __shfl_xor_sync(0xffffffffu, v, s);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  float t = 0.f;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  return t;
}

__device__ __forceinline__ bool self_conj_col(int j, int px) { return j == 0 || ((px % 2 == 0) && j == px / 2); }

// Hermitian fix of the self-conjugate columns: (S(i) + conj S(-i)) / 2.
__device__ __forceinline__ float2 sym_value(const float2* img, int i, int j, int py, int px, int pxh) {
  float2 v = img[(size_t)i * pxh + j];
  if (self_conj_col(j, px)) {
    const float2 m = img[(size_t)((py - i) % py) * pxh + j];
    v = make_float2(0.5f * (v.x + m.x), 0.5f * (v.y - m.y));
  }
  return v;
}

// Per template (block): S16 row = s (re, im) of the Hermitian-fixed slice,
// P16 row = s^2 |S|^2, with s = sqrt(Py pxh / sum |S|^2).
__global__ void k_pack_templates(const float2* __restrict__ img, int py, int px, __half* __restrict__ s16,
                                 __half* __restrict__ p16) {
  __shared__ float red[32];
  const int pxh = px / 2 + 1;
  const int kp = py * pxh;
  const float2* a = img + (size_t)blockIdx.x * kp;
  float acc = 0.f;
  for (int e = threadIdx.x; e < kp; e += blockDim.x) {
    const float2 v = sym_value(a, e / pxh, e % pxh, py, px, pxh);
    acc += v.x * v.x + v.y * v.y;
  }
  const float tot = block_sum_f(acc, red);
  const float s = tot > 0.f ? sqrtf((float)kp / tot) : 0.f;
  __half2* so = reinterpret_cast<__half2*>(s16 + (size_t)blockIdx.x * 2 * kp);
  __half* po = p16 + (size_t)blockIdx.x * kp;
  for (int e = threadIdx.x; e < kp; e += blockDim.x) {
    const float2 v = sym_value(a, e / pxh, e % pxh, py, px, pxh);
    so[e] = __floats2half2_rn(s * v.x, s * v.y);
    po[e] = __float2half_rn(s * s * (v.x * v.x + v.y * v.y));
  }
}

// Per observed image (block): Y16 = (w conj(m) O) / yinv, Z16 = (w |m|^2) / zinv
// with yinv, zinv the rows' RMS, and oo = sum w |O|^2.
__global__ void k_pack_observed(const float2* __restrict__ obs, const cjx_image_params* __restrict__ params, int py,
                                int px, uint32_t flags, __half* __restrict__ y16, __half* __restrict__ z16,
                                float* __restrict__ oo, float* __restrict__ yinv, float* __restrict__ zinv) {
  __shared__ float red[32];
  const int pxh = px / 2 + 1;
  const int kp = py * pxh;
  const float2* o = obs + (size_t)blockIdx.x * kp;
  const ImageConsts c = load_image_consts(params + blockIdx.x, 1.0f, py, px);
  float ay = 0.f, az = 0.f, ao = 0.f;
  for (int e = threadIdx.x; e < kp; e += blockDim.x) {
    const int i = e / pxh, j = e - (e / pxh) * pxh;
    const float w = (i == 0 && j == 0) ? 0.f : (self_conj_col(j, px) ? 1.f : 2.f);
    const float2 m = apply_epilogue(make_float2(1.f, 0.f), i, j, py, px, flags, c);
    const float2 v = o[e];
    const float yx = w * (m.x * v.x + m.y * v.y), yy = w * (m.x * v.y - m.y * v.x);
    const float z = w * (m.x * m.x + m.y * m.y);
    ay += yx * yx + yy * yy;
    az += z * z;
    ao += w * (v.x * v.x + v.y * v.y);
  }
  const float ty = block_sum_f(ay, red), tz = block_sum_f(az, red), to = block_sum_f(ao, red);
  const float ry = ty > 0.f ? sqrtf(ty / (2.f * kp)) : 1.f, rz = tz > 0.f ? sqrtf(tz / kp) : 1.f;
  if (threadIdx.x == 0) {
    oo[blockIdx.x] = to;
    yinv[blockIdx.x] = ry;
    zinv[blockIdx.x] = rz;
  }
  __half2* yo = reinterpret_cast<__half2*>(y16 + (size_t)blockIdx.x * 2 * kp);
  __half* zo = z16 + (size_t)blockIdx.x * kp;
  const float sy = 1.f / ry, sz = 1.f / rz;
  for (int e = threadIdx.x; e < kp; e += blockDim.x) {
    const int i = e / pxh, j = e - (e / pxh) * pxh;
    const float w = (i == 0 && j == 0) ? 0.f : (self_conj_col(j, px) ? 1.f : 2.f);
    const float2 m = apply_epilogue(make_float2(1.f, 0.f), i, j, py, px, flags, c);
    const float2 v = o[e];
    yo[e] = __floats2half2_rn(sy * w * (m.x * v.x + m.y * v.y), sy * w * (m.x * v.y - m.y * v.x));
    zo[e] = __float2half_rn(sz * w * (m.x * m.x + m.y * m.y));
  }
}

// Most candidates per image that the top-m selection and the FP32 re-ranking take.
constexpr int kTopMMax = 16;

// Per observed image (block): the same NCC terms in FP32 and unscaled,
//   y32 = w conj(m) O (complex), z32 = w |m|^2, oo = sum w |O|^2,
// for the re-ranking against the FP32 template bank (k_ncc_rerank32).
__global__ void k_pack_observed32(const float2* __restrict__ obs, const cjx_image_params* __restrict__ params,
                                  int py, int px, uint32_t flags, float2* __restrict__ y32, float* __restrict__ z32,
                                  float* __restrict__ oo) {
  __shared__ float red[32];
  const int pxh = px / 2 + 1;
  const int kp = py * pxh;
  const float2* o = obs + (size_t)blockIdx.x * kp;
  float2* yo = y32 + (size_t)blockIdx.x * kp;
  float* zo = z32 + (size_t)blockIdx.x * kp;
  const ImageConsts c = load_image_consts(params + blockIdx.x, 1.0f, py, px);
  float ao = 0.f;
  for (int e = threadIdx.x; e < kp; e += blockDim.x) {
    const int i = e / pxh, j = e - (e / pxh) * pxh;
    const float w = (i == 0 && j == 0) ? 0.f : (self_conj_col(j, px) ? 1.f : 2.f);
    const float2 m = apply_epilogue(make_float2(1.f, 0.f), i, j, py, px, flags, c);
    const float2 v = o[e];
    yo[e] = make_float2(w * (m.x * v.x + m.y * v.y), w * (m.x * v.y - m.y * v.x));
    zo[e] = w * (m.x * m.x + m.y * m.y);
    ao += w * (v.x * v.x + v.y * v.y);
  }
  const float to = block_sum_f(ao, red);
  if (threadIdx.x == 0) oo[blockIdx.x] = to;
}

// Per observed image (block of 256; warp r takes candidates r, r + 8, ..):
// FP32 NCC against each of its m candidate templates, read from the FP32
// bank of CTF-free slices [T][Py][Px/2+1] with the self-conjugate columns
// Hermitian-fixed as in the FP16 rows:
//   num = sum y32 . S, den = sum z32 |S|^2, NCC = num / sqrt(den oo)
// (0 when den or oo is 0; -inf for a candidate index outside [0, T)).  The
// best (ties -> lower template index) -> best_score[b], best_orient[b];
// every candidate's NCC -> scores[b][r] when scores is not NULL.
__global__ void __launch_bounds__(256)
    k_ncc_rerank32(const float2* __restrict__ bank, int py, int px, int64_t T, const float2* __restrict__ y32,
                   const float* __restrict__ z32, const float* __restrict__ oo, const int32_t* __restrict__ cand,
                   int m, float* __restrict__ scores, float* __restrict__ best_score,
                   int32_t* __restrict__ best_orient) {
  __shared__ float sc[kTopMMax];
  const int64_t b = blockIdx.x;
  const int pxh = px / 2 + 1;
  const int kp = py * pxh;
  const float2* yb = y32 + b * kp;
  const float* zb = z32 + b * kp;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = warp; r < m; r += (int)(blockDim.x >> 5)) {
    const int32_t t = cand[b * m + r];
    float s = -INFINITY;
    if (t >= 0 && (int64_t)t < T) {
      const float2* S = bank + (size_t)t * kp;
      float num = 0.f, den = 0.f;
#pragma unroll 4
      for (int e = lane; e < kp; e += 32) {  // unrolled so that several rows' loads are in flight
        const int i = e / pxh, j = e - i * pxh;
        const float2 v = sym_value(S, i, j, py, px, pxh);
        const float2 y = yb[e];
        num = fmaf(v.x, y.x, fmaf(v.y, y.y, num));
        den = fmaf(zb[e], v.x * v.x + v.y * v.y, den);
      }
      for (int o = 16; o > 0; o >>= 1) {
        num += __shfl_xor_sync(0xffffffffu, num, o);
        den += __shfl_xor_sync(0xffffffffu, den, o);
      }
      const float o2 = oo[b];
      s = (den > 0.f && o2 > 0.f) ? (float)((double)num / sqrt((double)den * (double)o2)) : 0.f;
    }
    if (lane == 0) sc[r] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float bv = -INFINITY;
    int32_t bi = m > 0 ? cand[b * m] : 0;
    for (int r = 0; r < m; ++r) {
      const int32_t t = cand[b * m + r];
      if (sc[r] > bv || (sc[r] == bv && t < bi)) {
        bv = sc[r];
        bi = t;
      }
    }
    best_score[b] = bv;
    best_orient[b] = bi;
  }
  if (scores && threadIdx.x < m) scores[b * m + threadIdx.x] = sc[threadIdx.x];
}

// Per image row (block): NCC over the T templates and its argmax (ties ->
// lowest index); optional scores out.
__global__ void k_ncc_argmax(const float* __restrict__ num, const float* __restrict__ den, int64_t ld,
                             int64_t T, const float* __restrict__ oo, const float* __restrict__ yinv,
                             const float* __restrict__ zinv, int64_t t0, float* __restrict__ scores,
                             int64_t ld_scores, float* __restrict__ best_score, int32_t* __restrict__ best_orient,
                             int accumulate_best) {
  __shared__ float sv[32];
  __shared__ int64_t si[32];
  const int64_t b = blockIdx.x;
  const float yr = yinv[b], zr = zinv[b], o2 = oo[b];
  float bv = -INFINITY;
  int64_t bi = INT64_MAX;
  for (int64_t t = threadIdx.x; t < T; t += blockDim.x) {
    const float n = num[b * ld + t] * yr, d = den[b * ld + t] * zr;
    const float s = (d > 0.f && o2 > 0.f) ? n * rsqrtf(d * o2) : 0.f;
    if (scores) scores[b * ld_scores + t0 + t] = s;
    if (s > bv) {  // t increases per thread: strict ">" keeps the lowest index
      bv = s;
      bi = t0 + t;
    }
  }
  for (int s = 16; s > 0; s >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, bv, s);
    const int64_t oi = __shfl_xor_sync(0xffffffffu, bi, s);
    if (ov > bv || (ov == bv && oi < bi)) {
      bv = ov;
      bi = oi;
    }
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sv[w] = bv;
    si[w] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
      if (sv[k] > bv || (sv[k] == bv && si[k] < bi)) {
        bv = sv[k];
        bi = si[k];
      }
    if (bi == INT64_MAX) bi = t0;
    if (!accumulate_best || bv > best_score[b] || (bv == best_score[b] && bi < best_orient[b])) {
      best_score[b] = bv;
      best_orient[b] = (int32_t)bi;
    }
  }
}

// Per image row (block of 256): the m <= 16 highest NCCs over the T
// templates (descending; ties -> lower index) -> idx_out[b][0..m).  Each
// thread keeps a sorted list of its best m, the block merges the lists in
// shared memory and one warp selects the final m.

__device__ __forceinline__ bool key_gt(float a, int32_t ia, float b, int32_t ib) {
  return a > b || (a == b && ia < ib);
}

__global__ void __launch_bounds__(256)
    k_ncc_topm(const float* __restrict__ num, const float* __restrict__ den, int64_t ld, int64_t T,
               const float* __restrict__ oo, const float* __restrict__ yinv, const float* __restrict__ zinv, int m,
               int32_t* __restrict__ idx_out) {
  __shared__ float sv[256 * kTopMMax];
  __shared__ int32_t si[256 * kTopMMax];
  const int64_t b = blockIdx.x;
  const float yr = yinv[b], zr = zinv[b], o2 = oo[b];
  float v[kTopMMax];
  int32_t ix[kTopMMax];
#pragma unroll
  for (int k = 0; k < kTopMMax; ++k) {
    v[k] = -INFINITY;
    ix[k] = INT32_MAX;
  }
  for (int64_t t = threadIdx.x; t < T; t += blockDim.x) {
    const float n = num[b * ld + t] * yr, d = den[b * ld + t] * zr;
    const float s = (d > 0.f && o2 > 0.f) ? n * rsqrtf(d * o2) : 0.f;
    if (!key_gt(s, (int32_t)t, v[m - 1], ix[m - 1])) continue;
    // insert into the sorted list (registers: unrolled compare-and-shift)
    float cs = s;
    int32_t ci = (int32_t)t;
#pragma unroll
    for (int k = 0; k < kTopMMax; ++k) {
      if (k < m && key_gt(cs, ci, v[k], ix[k])) {
        const float tv = v[k];
        const int32_t ti = ix[k];
        v[k] = cs;
        ix[k] = ci;
        cs = tv;
        ci = ti;
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kTopMMax; ++k) {
    sv[threadIdx.x * kTopMMax + k] = k < m ? v[k] : -INFINITY;
    si[threadIdx.x * kTopMMax + k] = k < m ? ix[k] : INT32_MAX;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    for (int r = 0; r < m; ++r) {
      float bv = -INFINITY;
      int32_t bi = INT32_MAX;
      int bp = -1;
      for (int p = lane; p < 256 * kTopMMax; p += 32) {
        if (key_gt(sv[p], si[p], bv, bi)) {
          bv = sv[p];
          bi = si[p];
          bp = p;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
        const int32_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
        const int op = __shfl_xor_sync(0xffffffffu, bp, o);
        if (key_gt(ov, oi, bv, bi)) {
          bv = ov;
          bi = oi;
          bp = op;
        }
      }
      if (lane == 0) {
        idx_out[b * m + r] = (bi == INT32_MAX) ? r : bi;
        if (bp >= 0) sv[bp] = -INFINITY;
        if (bp >= 0) si[bp] = INT32_MAX;
      }
      __syncwarp();
    }
  }
}

// ---------------------------------------------------------------------------
// Candidate blocks of the learned search: each image's proposed directions
// against the shared template rows, without simulating anything.
// ---------------------------------------------------------------------------
// Counting sort of the (image, slot) pairs by proposed direction, so the CTAs
// that read one direction's n_inplane template rows run together and find
// them in L2.  cursor: [n_dir + 1] ints (zeroed, then counts, then offsets);
// directions outside [0, n_dir) go to the last bin.
__device__ __forceinline__ int dir_bin(int d, int n_dir) { return (unsigned)d < (unsigned)n_dir ? d : n_dir; }

__global__ void k_dir_count(const int32_t* __restrict__ dirs, int64_t pairs, int n_dir, int* __restrict__ cursor) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < pairs; p += (int64_t)gridDim.x * blockDim.x)
    atomicAdd(cursor + dir_bin(dirs[p], n_dir), 1);
}

// exclusive prefix sum of cursor[0..bins) in place (one block of 1024 threads)
__global__ void k_dir_scan(int* __restrict__ cursor, int bins) {
  __shared__ int part[1024];
  const int per = (bins + 1023) / 1024;
  const int lo = threadIdx.x * per, hi = min(lo + per, bins);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += cursor[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (int i = lo; i < hi; ++i) {
    const int c = cursor[i];
    cursor[i] = run;
    run += c;
  }
}

__global__ void k_dir_scatter(const int32_t* __restrict__ dirs, int64_t pairs, int n_dir, int* __restrict__ cursor,
                              int32_t* __restrict__ sorted) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < pairs; p += (int64_t)gridDim.x * blockDim.x)
    sorted[atomicAdd(cursor + dir_bin(dirs[p], n_dir), 1)] = (int32_t)p;
}

// Tiles of the (image, slot) pairs in direction order: for each bin d in
// [0, n_dir] (n_dir = directions outside the grid) its first pair start[d]
// and its tiles of up to kTilePairs pairs, numbered from tile_start[d];
// start[n_dir + 1] = pairs, tile_start[n_dir + 1] = the tile count.  One
// block of 1024 threads; `cursor` holds the bins' exclusive offsets.
constexpr int kTilePairs = 16;

__global__ void k_dir_tiles(const int* __restrict__ cursor, int n_dir, int pairs, int* __restrict__ start,
                            int* __restrict__ tile_start) {
  __shared__ int part[1024];
  const int bins = n_dir + 1;
  const int per = (bins + 1023) / 1024;
  const int lo = threadIdx.x * per, hi = min(lo + per, bins);
  int s = 0;
  for (int d = lo; d < hi; ++d) {
    const int next = d + 1 < bins ? cursor[d + 1] : pairs;
    start[d] = cursor[d];
    s += (next - cursor[d] + kTilePairs - 1) / kTilePairs;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (int d = lo; d < hi; ++d) {
    const int next = d + 1 < bins ? cursor[d + 1] : pairs;
    tile_start[d] = run;
    run += (next - cursor[d] + kTilePairs - 1) / kTilePairs;
  }
  if (threadIdx.x == 1023) {
    start[bins] = pairs;
    tile_start[bins] = part[1023];
  }
}

// D (16 x 8, FP32) += A (16 x 16, FP16) B (16 x 8, FP16) on the tensor cores.
__device__ __forceinline__ void mma16816(float (&c)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Templates per pass of the tile kernel: kNTiles tensor-core column tiles of 8.
constexpr int kNTiles = 6;

// One warp's share of a tile's dot products: rows lo / hi (the tile's pairs
// g and g + 8 of this lane's group, NULL when the tile has no such pair)
// against the templates tmpl[j] (template of column g of column tile j,
// NULL past n_inplane), over the warp's K steps.  A K step is 32 halves:
// lane (g, t) loads halves [8 t, 8 t + 8) of the step from each row, and the
// two m16n8k16 products of the step take halves {8t, 8t+1, 8t+2, 8t+3} and
// {8t+4, .., 8t+7} as their k = {2t, 2t+1, 2t+8, 2t+9}: the same relabelling
// of k for both operands, so the sums are the dot products.
__device__ __forceinline__ void tile_dots(const uint4* lo, const uint4* hi, const uint4* const (&tmpl)[kNTiles],
                                          int64_t vrow, int warp, int t, float (&acc)[kNTiles][4]) {
  const int64_t steps = (vrow + 3) / 4;
  for (int64_t st = warp; st < steps; st += 8) {
    const int64_t v = 4 * st + t;
    const bool in = v < vrow;
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    const uint4 al = (in && lo) ? __ldg(lo + v) : z;
    const uint4 ah = (in && hi) ? __ldg(hi + v) : z;
    uint4 b[kNTiles];
#pragma unroll
    for (int j = 0; j < kNTiles; ++j) b[j] = (in && tmpl[j]) ? __ldg(tmpl[j] + v) : z;
#pragma unroll
    for (int j = 0; j < kNTiles; ++j) {
      mma16816(acc[j], al.x, ah.x, al.y, ah.y, b[j].x, b[j].y);
      mma16816(acc[j], al.z, ah.z, al.w, ah.w, b[j].z, b[j].w);
    }
  }
}

// One CTA per tile: up to 16 (image, slot) pairs that proposed direction d,
// against d's n_inplane templates t = d n_inplane + a:
//   num[b][k n_inplane + a] = y16[b] . s16[t]   (K = 2 kp)
//   den[b][k n_inplane + a] = z16[b] . p16[t]   (K = kp)
// FP16 operands, FP32 accumulation on the tensor cores (mma.sync m16n8k16);
// each template row is read once per tile instead of once per pair.  The
// 8 warps split K; their partial sums meet in shared memory.
__global__ void __launch_bounds__(256, 2)
    k_ncc_dir_tiles(const uint4* __restrict__ y16, const uint4* __restrict__ z16, const uint4* __restrict__ s16,
                    const uint4* __restrict__ p16, int64_t kp, const int32_t* __restrict__ sorted,
                    const int* __restrict__ start, const int* __restrict__ tile_start, int kd, int n_dir,
                    int n_inplane, float* __restrict__ num, float* __restrict__ den) {
  __shared__ float red[8][kTilePairs][kNTiles * 8];
  __shared__ int64_t out0[kTilePairs];
  __shared__ int64_t img[kTilePairs];
  const int tile = blockIdx.x;
  if (tile >= tile_start[n_dir + 1]) return;
  // the bin holding this tile: the largest d with tile_start[d] <= tile (empty bins share their
  // successor's value, so the largest is the non-empty one)
  int lo_d = 0, hi_d = n_dir;
  while (lo_d < hi_d) {
    const int mid = (lo_d + hi_d + 1) >> 1;
    if (tile_start[mid] <= tile) lo_d = mid;
    else hi_d = mid - 1;
  }
  const int d = lo_d;
  const int p0 = start[d] + (tile - tile_start[d]) * kTilePairs;
  const int np = min(kTilePairs, start[d + 1] - p0);
  if (threadIdx.x < kTilePairs) {
    const int r = threadIdx.x;
    const int pair = r < np ? sorted[p0 + r] : 0;
    img[r] = pair / kd;
    out0[r] = (int64_t)(pair / kd) * kd * n_inplane + (int64_t)(pair % kd) * n_inplane;
  }
  __syncthreads();
  if (d >= n_dir) {  // no such direction: zero sums, which score 0
    for (int e = threadIdx.x; e < np * n_inplane; e += blockDim.x) {
      num[out0[e / n_inplane] + e % n_inplane] = 0.f;
      den[out0[e / n_inplane] + e % n_inplane] = 0.f;
    }
    return;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int64_t vn = 2 * kp / 8, vd = kp / 8;  // 16-byte vectors per row
  for (int a0 = 0; a0 < n_inplane; a0 += kNTiles * 8) {
#pragma unroll 1
    for (int part = 0; part < 2; ++part) {  // numerators, then denominators
      const uint4* rows = part ? z16 : y16;
      const uint4* bank = part ? p16 : s16;
      const int64_t vrow = part ? vd : vn;
      const uint4* lo = g < np ? rows + img[g] * vrow : nullptr;
      const uint4* hi = g + 8 < np ? rows + img[g + 8] * vrow : nullptr;
      const uint4* tmpl[kNTiles];
#pragma unroll
      for (int j = 0; j < kNTiles; ++j) {
        const int a = a0 + 8 * j + g;
        tmpl[j] = a < n_inplane ? bank + ((int64_t)d * n_inplane + a) * vrow : nullptr;
      }
      float acc[kNTiles][4];
#pragma unroll
      for (int j = 0; j < kNTiles; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
      tile_dots(lo, hi, tmpl, vrow, warp, t, acc);
      // accumulator (row g / g + 8, column 2t / 2t + 1) of column tile j
#pragma unroll
      for (int j = 0; j < kNTiles; ++j) {
        red[warp][g][8 * j + 2 * t] = acc[j][0];
        red[warp][g][8 * j + 2 * t + 1] = acc[j][1];
        red[warp][g + 8][8 * j + 2 * t] = acc[j][2];
        red[warp][g + 8][8 * j + 2 * t + 1] = acc[j][3];
      }
      __syncthreads();
      float* out = part ? den : num;
      for (int e = threadIdx.x; e < kTilePairs * kNTiles * 8; e += blockDim.x) {
        const int r = e / (kNTiles * 8), c = e % (kNTiles * 8);
        if (r < np && a0 + c < n_inplane) {
          float s = 0.f;
#pragma unroll
          for (int w = 0; w < 8; ++w) s += red[w][r][c];
          out[out0[r] + a0 + c] = s;
        }
      }
      __syncthreads();
    }
  }
}

}  // namespace cjx

extern "C" {

int cjx_pack_templates(const void* images, int64_t n, int py, int px, void* s16, void* p16, void* stream) {
  if (n < 0 || py < 2 || px < 2) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "pack_templates: bad shape");
  if (n == 0) return CJX_OK;
  if (!images || !s16 || !p16) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "pack_templates: NULL pointer");
  if (n > 2147483647LL) return cjx::fail(CJX_ERR_UNSUPPORTED, "pack_templates: too many templates");
  cjx::k_pack_templates<<<(unsigned)n, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(images), py, px, static_cast<__half*>(s16), static_cast<__half*>(p16));
  return cjx::check_cuda(cudaGetLastError(), "pack_templates launch");
}

int cjx_pack_observed(const void* observed, const cjx_image_params* params, int64_t n, int py, int px, int flags,
                      void* y16, void* z16, float* oo, float* yinv, float* zinv, void* stream) {
  if (n < 0 || py < 2 || px < 2) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "pack_observed: bad shape");
  if (n == 0) return CJX_OK;
  if (!observed || !params || !y16 || !z16 || !oo || !yinv || !zinv)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "pack_observed: NULL pointer");
  if (n > 2147483647LL) return cjx::fail(CJX_ERR_UNSUPPORTED, "pack_observed: too many images");
  cjx::prof_begin(static_cast<cudaStream_t>(stream));
  cjx::k_pack_observed<<<(unsigned)n, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(observed), params, py, px, (uint32_t)flags, static_cast<__half*>(y16),
      static_cast<__half*>(z16), oo, yinv, zinv);
  cjx::prof_end("k_pack_observed", static_cast<cudaStream_t>(stream));
  return cjx::check_cuda(cudaGetLastError(), "pack_observed launch");
}

int cjx_pack_observed32(const void* observed, const cjx_image_params* params, int64_t n, int py, int px, int flags,
                        void* y32, float* z32, float* oo, void* stream) {
  if (n < 0 || py < 2 || px < 2) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "pack_observed32: bad shape");
  if (n == 0) return CJX_OK;
  if (!observed || !params || !y32 || !z32 || !oo)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "pack_observed32: NULL pointer");
  if (n > 2147483647LL) return cjx::fail(CJX_ERR_UNSUPPORTED, "pack_observed32: too many images");
  cjx::prof_begin(static_cast<cudaStream_t>(stream));
  cjx::k_pack_observed32<<<(unsigned)n, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(observed), params, py, px, (uint32_t)flags, static_cast<float2*>(y32), z32, oo);
  cjx::prof_end("k_pack_observed32", static_cast<cudaStream_t>(stream));
  return cjx::check_cuda(cudaGetLastError(), "pack_observed32 launch");
}

int cjx_ncc_rerank32(const void* bank, int py, int px, int64_t T, const void* y32, const float* z32, const float* oo,
                     int64_t n, const int32_t* candidates, int m, float* scores, float* best_score,
                     int32_t* best_orientation, void* stream) {
  if (n < 0 || py < 2 || px < 2 || T < 1 || m < 1 || m > cjx::kTopMMax)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_rerank32: need 1 <= m <= 16, T >= 1 and a valid shape");
  if (n == 0) return CJX_OK;
  if (!bank || !y32 || !z32 || !oo || !candidates || !best_score || !best_orientation)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_rerank32: NULL pointer");
  if (n > 2147483647LL) return cjx::fail(CJX_ERR_UNSUPPORTED, "ncc_rerank32: too many images");
  for (const void* ptr : {bank, y32})
    if (reinterpret_cast<uintptr_t>(ptr) % 8)
      return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_rerank32: complex arrays must be 8-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cjx::prof_begin(s);
  cjx::k_ncc_rerank32<<<(unsigned)n, 256, 0, s>>>(static_cast<const float2*>(bank), py, px, T,
                                                  static_cast<const float2*>(y32), z32, oo, candidates, m, scores,
                                                  best_score, best_orientation);
  cjx::prof_end("k_ncc_rerank32", s);
  return cjx::check_cuda(cudaGetLastError(), "ncc_rerank32 launch");
}

int cjx_ncc_argmax(const float* num, const float* den, int64_t ld, int64_t n, int64_t T, const float* oo,
                   const float* yinv, const float* zinv, int64_t t0, float* scores, int64_t ld_scores,
                   float* best_score, int32_t* best_orientation, int accumulate_best, void* stream) {
  if (n < 0 || T < 1 || ld < T || t0 < 0 || t0 + T > 2147483647LL)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_argmax: bad sizes");
  if (n == 0) return CJX_OK;
  if (!num || !den || !oo || !yinv || !zinv || !best_score || !best_orientation)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_argmax: NULL pointer");
  cjx::prof_begin(static_cast<cudaStream_t>(stream));
  cjx::k_ncc_argmax<<<(unsigned)n, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      num, den, ld, T, oo, yinv, zinv, t0, scores, ld_scores, best_score, best_orientation, accumulate_best);
  cjx::prof_end("k_ncc_argmax", static_cast<cudaStream_t>(stream));
  return cjx::check_cuda(cudaGetLastError(), "ncc_argmax launch");
}

int cjx_ncc_topk(const float* num, const float* den, int64_t ld, int64_t n, int64_t T, const float* oo,
                 const float* yinv, const float* zinv, int k, int32_t* indices, void* stream) {
  if (n < 0 || T < 1 || ld < T || T > 2147483647LL || k < 1 || k > cjx::kTopMMax || k > T)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_topk: need 1 <= k <= min(16, T), ld >= T");
  if (n == 0) return CJX_OK;
  if (!num || !den || !oo || !yinv || !zinv || !indices)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_topk: NULL pointer");
  cjx::prof_begin(static_cast<cudaStream_t>(stream));
  cjx::k_ncc_topm<<<(unsigned)n, 256, 0, static_cast<cudaStream_t>(stream)>>>(num, den, ld, T, oo, yinv, zinv, k,
                                                                            indices);
  cjx::prof_end("k_ncc_topm", static_cast<cudaStream_t>(stream));
  return cjx::check_cuda(cudaGetLastError(), "ncc_topk launch");
}


// cursor [n_dir + 1], start [n_dir + 2], tile_start [n_dir + 2], sorted pairs [n kd]
static size_t ncc_directions_workspace_bytes(int64_t n, int kd, int n_dir) {
  return sizeof(int) * (3 * ((size_t)n_dir + 2) + (size_t)n * kd);
}

int cjx_ncc_directions_workspace_size(int64_t n, int kd, int n_dir, size_t* bytes) {
  if (!bytes) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "bytes is NULL");
  if (n < 0 || kd < 1 || n_dir < 1) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_directions: bad sizes");
  *bytes = ncc_directions_workspace_bytes(n, kd, n_dir);
  return CJX_OK;
}

int cjx_ncc_directions(const void* y16, const void* z16, const void* s16, const void* p16, int64_t n, int64_t kp,
                       const int32_t* dirs, int kd, int n_dir, int n_inplane, float* num, float* den,
                       void* workspace, size_t workspace_bytes, void* stream) {
  if (n < 0 || kp < 8 || kp % 8 || kd < 1 || n_dir < 1 || n_inplane < 1)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT,
                     "ncc_directions: need kp a positive multiple of 8 and kd, n_dir, n_inplane >= 1");
  if (n * (int64_t)kd > 2147483647LL) return cjx::fail(CJX_ERR_UNSUPPORTED, "ncc_directions: too many pairs");
  if (n == 0) return CJX_OK;
  if (!y16 || !z16 || !s16 || !p16 || !dirs || !num || !den || !workspace)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_directions: NULL pointer");
  if (workspace_bytes < ncc_directions_workspace_bytes(n, kd, n_dir))
    return cjx::fail(CJX_ERR_WORKSPACE, "ncc_directions: workspace smaller than cjx_ncc_directions_workspace_size");
  for (const void* ptr : {y16, z16, s16, p16})
    if (reinterpret_cast<uintptr_t>(ptr) % 16)
      return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_directions: rows must be 16-byte aligned");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int* cursor = static_cast<int*>(workspace);
  int* start = cursor + n_dir + 2;
  int* tile_start = start + n_dir + 2;
  int32_t* sorted = tile_start + n_dir + 2;
  const int64_t pairs = n * kd;
  if (int e = cjx::check_cuda(cudaMemsetAsync(cursor, 0, sizeof(int) * ((size_t)n_dir + 1), s), "cudaMemsetAsync"))
    return e;
  const int blocks = (int)std::min<int64_t>((pairs + 255) / 256, 1184);
  cjx::prof_begin(s);
  cjx::k_dir_count<<<blocks, 256, 0, s>>>(dirs, pairs, n_dir, cursor);
  cjx::k_dir_scan<<<1, 1024, 0, s>>>(cursor, n_dir + 1);
  cjx::k_dir_tiles<<<1, 1024, 0, s>>>(cursor, n_dir, (int)pairs, start, tile_start);
  cjx::k_dir_scatter<<<blocks, 256, 0, s>>>(dirs, pairs, n_dir, cursor, sorted);
  cjx::prof_end("k_dir_sort", s);
  // every bin has at most pairs_d / 16 + 1 tiles: a grid of pairs / 16 + n_dir + 1 CTAs covers them
  const int64_t max_tiles = pairs / cjx::kTilePairs + n_dir + 1;
  cjx::prof_begin(s);
  cjx::k_ncc_dir_tiles<<<(unsigned)max_tiles, 256, 0, s>>>(
      static_cast<const uint4*>(y16), static_cast<const uint4*>(z16), static_cast<const uint4*>(s16),
      static_cast<const uint4*>(p16), kp, sorted, start, tile_start, kd, n_dir, n_inplane, num, den);
  cjx::prof_end("k_ncc_directions", s);
  return cjx::check_cuda(cudaGetLastError(), "ncc_directions launch");
}

}  // extern "C"
