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
constexpr int kTopMMax = 16;

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

// FP32 dot product of 8 halves at a time
__device__ __forceinline__ float dot8(uint4 a, uint4 b, float acc) {
  const __half2* ha = reinterpret_cast<const __half2*>(&a);
  const __half2* hb = reinterpret_cast<const __half2*>(&b);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float2 fa = __half22float2(ha[q]), fb = __half22float2(hb[q]);
    acc = fmaf(fa.x, fb.x, acc);
    acc = fmaf(fa.y, fb.y, acc);
  }
  return acc;
}

// One CTA per (image b, slot k) pair (in direction order): for a in
// [0, n_inplane), template t = dirs[b][k] n_inplane + a,
//   num[b][k n_inplane + a] = y16[b] . s16[t]   (K = 2 kp)
//   den[b][k n_inplane + a] = z16[b] . p16[t]   (K = kp)
// Each warp takes 3 templates at a time, so one load of the image's row
// serves three template rows.  Rows are 16-byte aligned (kp % 8 == 0).
constexpr int kDirTemplatesPerPass = 3;

__global__ void __launch_bounds__(256)
    k_ncc_directions(const uint4* __restrict__ y16, const uint4* __restrict__ z16, const uint4* __restrict__ s16,
                     const uint4* __restrict__ p16, int64_t kp, const int32_t* __restrict__ dirs,
                     const int32_t* __restrict__ sorted, int kd, int n_dir, int n_inplane, float* __restrict__ num,
                     float* __restrict__ den) {
  const int32_t pair = sorted[blockIdx.x];
  const int64_t b = pair / kd;
  const int k = pair % kd;
  const int d = dirs[pair];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t out0 = b * (int64_t)kd * n_inplane + (int64_t)k * n_inplane;
  if ((unsigned)d >= (unsigned)n_dir) {  // no such direction: zero sums, which score 0
    for (int a = threadIdx.x; a < n_inplane; a += blockDim.x) {
      num[out0 + a] = 0.f;
      den[out0 + a] = 0.f;
    }
    return;
  }
  const int64_t vn = 2 * kp / 8, vd = kp / 8;  // 16-byte vectors per row
  const uint4* yb = y16 + b * vn;
  const uint4* zb = z16 + b * vd;
  for (int a0 = warp * kDirTemplatesPerPass; a0 < n_inplane; a0 += 8 * kDirTemplatesPerPass) {
    float accn[kDirTemplatesPerPass], accd[kDirTemplatesPerPass];
    const uint4* srow[kDirTemplatesPerPass];
    const uint4* prow[kDirTemplatesPerPass];
#pragma unroll
    for (int q = 0; q < kDirTemplatesPerPass; ++q) {
      accn[q] = accd[q] = 0.f;
      const int a = min(a0 + q, n_inplane - 1);  // a tail pass recomputes the last template, stored once
      const int64_t t = (int64_t)d * n_inplane + a;
      srow[q] = s16 + t * vn;
      prow[q] = p16 + t * vd;
    }
    for (int64_t i = lane; i < vn; i += 32) {
      const uint4 yv = __ldg(yb + i);
#pragma unroll
      for (int q = 0; q < kDirTemplatesPerPass; ++q) accn[q] = dot8(yv, __ldg(srow[q] + i), accn[q]);
    }
    for (int64_t i = lane; i < vd; i += 32) {
      const uint4 zv = __ldg(zb + i);
#pragma unroll
      for (int q = 0; q < kDirTemplatesPerPass; ++q) accd[q] = dot8(zv, __ldg(prow[q] + i), accd[q]);
    }
#pragma unroll
    for (int q = 0; q < kDirTemplatesPerPass; ++q) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        accn[q] += __shfl_xor_sync(0xffffffffu, accn[q], o);
        accd[q] += __shfl_xor_sync(0xffffffffu, accd[q], o);
      }
      if (lane == 0 && a0 + q < n_inplane) {
        num[out0 + a0 + q] = accn[q];
        den[out0 + a0 + q] = accd[q];
      }
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
  cjx::k_pack_observed<<<(unsigned)n, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      static_cast<const float2*>(observed), params, py, px, (uint32_t)flags, static_cast<__half*>(y16),
      static_cast<__half*>(z16), oo, yinv, zinv);
  return cjx::check_cuda(cudaGetLastError(), "pack_observed launch");
}

int cjx_ncc_argmax(const float* num, const float* den, int64_t ld, int64_t n, int64_t T, const float* oo,
                   const float* yinv, const float* zinv, int64_t t0, float* scores, int64_t ld_scores,
                   float* best_score, int32_t* best_orientation, int accumulate_best, void* stream) {
  if (n < 0 || T < 1 || ld < T || t0 < 0 || t0 + T > 2147483647LL)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_argmax: bad sizes");
  if (n == 0) return CJX_OK;
  if (!num || !den || !oo || !yinv || !zinv || !best_score || !best_orientation)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_argmax: NULL pointer");
  cjx::k_ncc_argmax<<<(unsigned)n, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      num, den, ld, T, oo, yinv, zinv, t0, scores, ld_scores, best_score, best_orientation, accumulate_best);
  return cjx::check_cuda(cudaGetLastError(), "ncc_argmax launch");
}

int cjx_ncc_topk(const float* num, const float* den, int64_t ld, int64_t n, int64_t T, const float* oo,
                 const float* yinv, const float* zinv, int k, int32_t* indices, void* stream) {
  if (n < 0 || T < 1 || ld < T || T > 2147483647LL || k < 1 || k > cjx::kTopMMax || k > T)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_topk: need 1 <= k <= min(16, T), ld >= T");
  if (n == 0) return CJX_OK;
  if (!num || !den || !oo || !yinv || !zinv || !indices)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "ncc_topk: NULL pointer");
  cjx::k_ncc_topm<<<(unsigned)n, 256, 0, static_cast<cudaStream_t>(stream)>>>(num, den, ld, T, oo, yinv, zinv, k,
                                                                            indices);
  return cjx::check_cuda(cudaGetLastError(), "ncc_topk launch");
}


static size_t ncc_directions_workspace_bytes(int64_t n, int kd, int n_dir) {
  return sizeof(int) * ((size_t)n_dir + 1 + (size_t)n * kd);
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
  int32_t* sorted = cursor + n_dir + 1;
  const int64_t pairs = n * kd;
  if (int e = cjx::check_cuda(cudaMemsetAsync(cursor, 0, sizeof(int) * ((size_t)n_dir + 1), s), "cudaMemsetAsync"))
    return e;
  const int blocks = (int)std::min<int64_t>((pairs + 255) / 256, 1184);
  cjx::prof_begin(s);
  cjx::k_dir_count<<<blocks, 256, 0, s>>>(dirs, pairs, n_dir, cursor);
  cjx::k_dir_scan<<<1, 1024, 0, s>>>(cursor, n_dir + 1);
  cjx::k_dir_scatter<<<blocks, 256, 0, s>>>(dirs, pairs, n_dir, cursor, sorted);
  cjx::prof_end("k_dir_sort", s);
  cjx::prof_begin(s);
  cjx::k_ncc_directions<<<(unsigned)pairs, 256, 0, s>>>(
      static_cast<const uint4*>(y16), static_cast<const uint4*>(z16), static_cast<const uint4*>(s16),
      static_cast<const uint4*>(p16), kp, dirs, sorted, kd, n_dir, n_inplane, num, den);
  cjx::prof_end("k_ncc_directions", s);
  return cjx::check_cuda(cudaGetLastError(), "ncc_directions launch");
}

}  // extern "C"
