// General tensor-core GEMM C = A * B^T (A: M x K, B: N x K, both K-major
// 16-bit, FP32 accumulation in TMEM) with a fused epilogue: per-column bias,
// ReLU, BF16 or FP32 store, or FP32 atomic accumulation (split-K).  Used by
// the pose-proposal network's convolution (im2col) and dense layers,
// forward and backward.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

#include "cjx_common.cuh"
#include "cjx_tc.cuh"
#include "cjx_profile.cuh"

namespace cjx {

__device__ int g_tc_status;  // first error code a tensor-core kernel recorded (0 = none)

struct GemmEpilogue {
  void* C;
  int64_t ldc;
  const float* bias;
  int flags;
  int M, N;

  __device__ void operator()(int row, int col0, float (&v)[16]) const {
    if (row >= M) return;
    const int nv = min(16, N - col0);
    if (nv <= 0) return;
    if (flags & CJX_GEMM_BIAS) {
#pragma unroll
      for (int i = 0; i < 16; ++i)
        if (i < nv) v[i] += bias[col0 + i];
    }
    if (flags & CJX_GEMM_RELU) {
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = fmaxf(v[i], 0.f);
    }
    if (flags & CJX_GEMM_OUT_BF16) {
      __nv_bfloat16* c = static_cast<__nv_bfloat16*>(C) + (size_t)row * ldc + col0;
      if (nv == 16 && (reinterpret_cast<uintptr_t>(c) & 15) == 0) {
        uint32_t w[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
          w[i] = *reinterpret_cast<uint32_t*>(&h);
        }
        reinterpret_cast<uint4*>(c)[0] = make_uint4(w[0], w[1], w[2], w[3]);
        reinterpret_cast<uint4*>(c)[1] = make_uint4(w[4], w[5], w[6], w[7]);
      } else {
        for (int i = 0; i < nv; ++i) c[i] = __float2bfloat16_rn(v[i]);
      }
    } else {
      float* c = static_cast<float*>(C) + (size_t)row * ldc + col0;
      if (flags & CJX_GEMM_ACCUMULATE) {
        for (int i = 0; i < nv; ++i) atomicAdd(c + i, v[i]);
      } else if (nv == 16 && (reinterpret_cast<uintptr_t>(c) & 15) == 0) {
#pragma unroll
        for (int i = 0; i < 4; ++i)
          reinterpret_cast<float4*>(c)[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
      } else {
        for (int i = 0; i < nv; ++i) c[i] = v[i];
      }
    }
  }
};

template <int BN, class Epi>
__global__ void __launch_bounds__(128, 1)
    k_gemm_tc(const __grid_constant__ CUtensorMap tma_a, const __grid_constant__ CUtensorMap tma_b, Epi epi, int K,
              int kb_per_split, uint32_t idesc) {
  extern __shared__ uint8_t smem_raw[];
  const int nk = (K + tc::BK - 1) / tc::BK;
  const int kb0 = blockIdx.z * kb_per_split;
  const int kb1 = min(nk, kb0 + kb_per_split);
  if (kb0 >= kb1) return;  // uniform across the CTA: this split has no k-blocks
  tc::TileMainloop<BN> ml;
  ml.carve(smem_raw);
  const int m0 = blockIdx.x * tc::BM, n0 = blockIdx.y * BN;
  const uint32_t tmem = ml.setup(&tma_a, &tma_b);
  int issued = 0;
  ml.run(&tma_a, &tma_b, m0, n0, kb0, kb1, tmem, idesc, &g_tc_status, &issued);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (ml.wait_done(&g_tc_status)) {
    const uint32_t lane_base = tmem + (static_cast<uint32_t>(warp * 32) << 16);
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      tc::tmem_ld16(lane_base + c, v);
      epi(m0 + warp * 32 + lane, n0 + c, v);
    }
  }
  ml.teardown(tmem, issued, &g_tc_status);
}

// One thread waits on an mbarrier that nothing ever arrives on: the bounded
// wait must give up after limit_ns and record kErrSelfTest in *status.
__global__ void k_selftest_bounded_wait(uint64_t limit_ns, int* status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    tc::mbar_init(tc::smem_u32(&bar), 1);
    tc::fence_barrier_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) tc::mbar_wait(tc::smem_u32(&bar), 0, nullptr, status, tc::kErrSelfTest, limit_ns);
}

// ---- host side -------------------------------------------------------------

static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 2-D K-major operand [rows][ld] of 16-bit elements, box 64 x box_rows, 128-byte swizzle.
int make_operand_map(CUtensorMap* map, const void* base, int64_t rows, int64_t k, int64_t ld, int box_rows,
                     bool f16) {
  auto enc = tensor_map_encoder();
  if (!enc) return fail(CJX_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld % 8) || ld < k || k < 1 || rows < 1)
    return fail(CJX_ERR_INVALID_ARGUMENT,
                "GEMM operands need a 16-byte aligned base, ld a multiple of 8 elements, ld >= K >= 1");
  cuuint64_t dims[2] = {static_cast<cuuint64_t>(k), static_cast<cuuint64_t>(rows)};
  cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld) * 2};
  cuuint32_t box[2] = {static_cast<cuuint32_t>(tc::BK), static_cast<cuuint32_t>(box_rows)};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, f16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                   const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(CJX_ERR_INVALID_ARGUMENT, "cuTensorMapEncodeTiled rejected the operand");
  return CJX_OK;
}

// Once per device (function attributes belong to each device's context).
template <int BN>
static cudaError_t gemm_smem_attr() {
  static PerDeviceOnce once;
  return once.run([] {
    return cudaFuncSetAttribute(k_gemm_tc<BN, GemmEpilogue>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)tc::gemm_smem_bytes(BN));
  });
}

template <int BN>
static int launch_gemm_bn(const CUtensorMap& ta, const CUtensorMap& tb, const GemmEpilogue& epi, int64_t M,
                          int64_t N, int64_t K, int split, bool f16, cudaStream_t stream) {
  if (cudaError_t e = gemm_smem_attr<BN>()) return check_cuda(e, "cudaFuncSetAttribute(gemm)");
  const int nk = (int)((K + tc::BK - 1) / tc::BK);
  const int kbps = (nk + split - 1) / split;
  const dim3 grid((unsigned)((M + tc::BM - 1) / tc::BM), (unsigned)((N + BN - 1) / BN), (unsigned)split);
  k_gemm_tc<BN, GemmEpilogue><<<grid, 128, tc::gemm_smem_bytes(BN), stream>>>(ta, tb, epi, (int)K, kbps,
                                                                            tc::f16_idesc(tc::BM, BN, f16 ? 0 : 1));
  return check_cuda(cudaGetLastError(), "gemm launch");
}

int launch_gemm(int64_t M, int64_t N, int64_t K, const void* A, int64_t lda, const void* B, int64_t ldb, void* C,
                int64_t ldc, const float* bias, int flags, int split_k, cudaStream_t stream) {
  if (M < 0 || N < 0 || K < 0) return fail(CJX_ERR_INVALID_ARGUMENT, "negative GEMM size");
  if (M == 0 || N == 0) return CJX_OK;
  if (K == 0) return fail(CJX_ERR_INVALID_ARGUMENT, "K must be >= 1");
  if (M > (int64_t)65535 * tc::BM * 1024 || N > (int64_t)65535 * 32) return fail(CJX_ERR_UNSUPPORTED, "GEMM too large");
  if (!A || !B || !C) return fail(CJX_ERR_INVALID_ARGUMENT, "A, B and C must be non-NULL");
  if ((flags & CJX_GEMM_BIAS) && !bias) return fail(CJX_ERR_INVALID_ARGUMENT, "CJX_GEMM_BIAS needs bias");
  if ((flags & CJX_GEMM_ACCUMULATE) && (flags & (CJX_GEMM_OUT_BF16 | CJX_GEMM_BIAS | CJX_GEMM_RELU)))
    return fail(CJX_ERR_INVALID_ARGUMENT, "CJX_GEMM_ACCUMULATE is FP32 only, without bias or ReLU");
  if (split_k < 1) split_k = 1;
  if (split_k > 1 && !(flags & CJX_GEMM_ACCUMULATE))
    return fail(CJX_ERR_INVALID_ARGUMENT, "split_k > 1 needs CJX_GEMM_ACCUMULATE");
  if (ldc < N) return fail(CJX_ERR_INVALID_ARGUMENT, "ldc < N");
  const int nk = (int)((K + tc::BK - 1) / tc::BK);
  split_k = std::min(split_k, nk);
  const bool f16 = (flags & CJX_GEMM_F16) != 0;
  const int bn = N > 128 ? (M >= 8 * tc::BM ? 256 : 128) : (N > 64 ? 128 : (N > 32 ? 64 : 32));
  CUtensorMap ta, tb;
  if (int e = make_operand_map(&ta, A, M, K, lda, tc::BM, f16)) return e;
  if (int e = make_operand_map(&tb, B, N, K, ldb, bn, f16)) return e;
  GemmEpilogue epi{C, ldc, bias, flags, (int)M, (int)N};
  switch (bn) {
    case 32: return launch_gemm_bn<32>(ta, tb, epi, M, N, K, split_k, f16, stream);
    case 64: return launch_gemm_bn<64>(ta, tb, epi, M, N, K, split_k, f16, stream);
    case 128: return launch_gemm_bn<128>(ta, tb, epi, M, N, K, split_k, f16, stream);
    default: return launch_gemm_bn<256>(ta, tb, epi, M, N, K, split_k, f16, stream);
  }
}

int read_tc_status(int* status, int reset, cudaStream_t stream) {
  int v = 0;
  if (cudaError_t e = cudaMemcpyFromSymbolAsync(&v, g_tc_status, sizeof(int), 0, cudaMemcpyDeviceToHost, stream))
    return check_cuda(e, "read status");
  if (cudaError_t e = cudaStreamSynchronize(stream)) return check_cuda(e, "status sync");
  if (reset) {
    const int z = 0;
    if (cudaError_t e = cudaMemcpyToSymbolAsync(g_tc_status, &z, sizeof(int), 0, cudaMemcpyHostToDevice, stream))
      return check_cuda(e, "reset status");
    if (cudaError_t e = cudaStreamSynchronize(stream)) return check_cuda(e, "status sync");
  }
  *status = v;
  return CJX_OK;
}

}  // namespace cjx

extern "C" {

int cjx_gemm(int64_t M, int64_t N, int64_t K, const void* A, int64_t lda, const void* B, int64_t ldb, void* C,
             int64_t ldc, const float* bias, int flags, int split_k, void* stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cjx::prof_begin(s);
  const int e = cjx::launch_gemm(M, N, K, A, lda, B, ldb, C, ldc, bias, flags, split_k, s);
  cjx::prof_end("gemm_tc", s);
  return e;
}

int cjx_selftest_bounded_wait(uint64_t limit_ns, int* device_status, void* stream) {
  if (!device_status) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "device_status is NULL");
  if (limit_ns < 1000 || limit_ns > cjx::tc::kWaitLimitNs)
    return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "limit_ns must be in [1 us, 2 s]");
  cjx::k_selftest_bounded_wait<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(limit_ns, device_status);
  return cjx::check_cuda(cudaGetLastError(), "selftest launch");
}

int cjx_device_status(int* status, int reset, void* stream) {
  if (!status) return cjx::fail(CJX_ERR_INVALID_ARGUMENT, "status is NULL");
  return cjx::read_tc_status(status, reset, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
