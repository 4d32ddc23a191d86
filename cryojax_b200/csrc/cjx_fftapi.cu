// cjx_fft_c2c: batched complex FFTs of contiguous rows with the library's
// warp FFTs (register/shuffle form for n = 32 R, shared-memory Stockham
// otherwise).  A utility and test hook for the transforms the resize stage
// uses; one warp per row.
#include <cuda_runtime.h>

#include "cjx_common.cuh"
#include "cjx_profile.cuh"

namespace cjx {

template <int R, int DIR>
__global__ void __launch_bounds__(256) k_fft_rows_reg(const float2* __restrict__ in, float2* __restrict__ out,
                                                      int64_t count) {
  constexpr int n = 32 * R;
  __shared__ float2 tab[32 * R];
  __shared__ float2 w32[32];
  build_reg_twiddles(tab, n);
  build_w32(w32);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + warp;
  if (row >= count) return;
  const LaneTwiddles lt = make_lane_twiddles(w32, lane);
  const float2* src = in + row * n;
  const int bl = brev5(lane);
  float2 x[R];
#pragma unroll
  for (int n1 = 0; n1 < R; ++n1) x[n1] = src[32 * n1 + bl];
  warp_fft_reg<R, DIR>(x, tab, lt, lane);
  float2* dst = out + row * n;
#pragma unroll
  for (int k1 = 0; k1 < R; ++k1) dst[k1 + R * lane] = x[k1];
}

template <int DIR>
__global__ void __launch_bounds__(256) k_fft_rows_stockham(const float2* __restrict__ in, float2* __restrict__ out,
                                                           int64_t count, FftPlan plan) {
  extern __shared__ float2 smem[];
  const int n = plan.n;
  float2* tw = smem;
  float2* bufs = smem + n;
  build_twiddles(tw, n);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row = (int64_t)blockIdx.x * (blockDim.x / 32) + warp;
  if (row >= count) return;
  float2* a = bufs + warp * 2 * n;
  for (int i = lane; i < n; i += 32) a[i] = in[row * n + i];
  __syncwarp();
  float2* r = warp_fft<DIR>(a, a + n, plan, tw, lane);
  for (int i = lane; i < n; i += 32) out[row * n + i] = r[i];
}

template <int R>
static void launch_reg(int dir, const float2* in, float2* out, int64_t count, cudaStream_t s) {
  const int blocks = (int)((count + 7) / 8);
  if (dir < 0)
    k_fft_rows_reg<R, -1><<<blocks, 256, 0, s>>>(in, out, count);
  else
    k_fft_rows_reg<R, +1><<<blocks, 256, 0, s>>>(in, out, count);
}

int launch_fft_rows(int n, int dir, const float2* in, float2* out, int64_t count, cudaStream_t s) {
  if (count <= 0) return CJX_OK;
  if (count > (int64_t)8 * 2147483647LL) return fail(CJX_ERR_UNSUPPORTED, "too many rows");
  prof_begin(s);
  switch (reg_fft_radix(n)) {
    case 1: launch_reg<1>(dir, in, out, count, s); break;
    case 2: launch_reg<2>(dir, in, out, count, s); break;
    case 3: launch_reg<3>(dir, in, out, count, s); break;
    case 4: launch_reg<4>(dir, in, out, count, s); break;
    case 5: launch_reg<5>(dir, in, out, count, s); break;
    case 6: launch_reg<6>(dir, in, out, count, s); break;
    case 8: launch_reg<8>(dir, in, out, count, s); break;
    case 10: launch_reg<10>(dir, in, out, count, s); break;
    case 12: launch_reg<12>(dir, in, out, count, s); break;
    case 16: launch_reg<16>(dir, in, out, count, s); break;
    default: {
      const size_t smem = sizeof(float2) * (size_t)(n + 8 * 2 * n);
      if (smem > 227 * 1024) return fail(CJX_ERR_UNSUPPORTED, "FFT length too large");
      cudaError_t e = cudaFuncSetAttribute(dir < 0 ? k_fft_rows_stockham<-1> : k_fft_rows_stockham<+1>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
      if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute");
      const FftPlan plan = make_fft_plan(n);
      const int blocks = (int)((count + 7) / 8);
      if (dir < 0)
        k_fft_rows_stockham<-1><<<blocks, 256, smem, s>>>(in, out, count, plan);
      else
        k_fft_rows_stockham<+1><<<blocks, 256, smem, s>>>(in, out, count, plan);
    }
  }
  prof_end("k_fft_rows", s);
  return check_cuda(cudaGetLastError(), "cjx_fft_c2c launch");
}

}  // namespace cjx

extern "C" int cjx_fft_c2c(int n, int direction, const void* in, void* out, int64_t count, void* stream) {
  using namespace cjx;
  if (n < 1 || n > CJX_MAX_SIDE) return fail(CJX_ERR_UNSUPPORTED, "FFT length must be in [1, CJX_MAX_SIDE]");
  if (direction != -1 && direction != 1) return fail(CJX_ERR_INVALID_ARGUMENT, "direction must be -1 or +1");
  if (count < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "count < 0");
  if (count == 0) return CJX_OK;
  if (!in || !out) return fail(CJX_ERR_INVALID_ARGUMENT, "in and out must be non-NULL");
  if (in == out) return fail(CJX_ERR_INVALID_ARGUMENT, "in-place transforms are not supported");
  return launch_fft_rows(n, direction, static_cast<const float2*>(in), static_cast<float2*>(out), count,
                         static_cast<cudaStream_t>(stream));
}
