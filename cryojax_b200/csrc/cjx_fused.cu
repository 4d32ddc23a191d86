// Fused first pass of the resize path: gather + column inverse FFT + Py window.
//
// One CTA takes kCols = 8 consecutive slice columns kx of one image.  Its 256
// threads sample those columns of the rotated central plane (the gather of
// k_gather_slice, same sampler and out-of-bounds rule) into a shared-memory
// tile [column][row], each warp then runs the N-point inverse FFT of one
// column from that tile in registers (warp_fft512_t for N = 512,
// warp_fft_reg otherwise), and the CTA writes the Py rows of the real-space
// crop/pad window of its 8 columns to T1.  Against the split form (gather to
// an HBM slice buffer H, then a column kernel reading H back) this removes
// the H round trip: 2 N (N/2 + 1) complex64 values of DRAM traffic per image
// (2.1 MB at N = 512), and the FFT arithmetic of one CTA overlaps the memory
// stalls of the others on the SM.
//
// Columns kx = 0 and kx = N/2 are made Hermitian in ky before the transform
// ((S[v] + conj(S[-v])) / 2, what the reference's irfftn keeps of a
// non-Hermitian plane); the Ewald sphere's full complex surface is not.
#include "cjx_common.cuh"
#include "cjx_profile.cuh"

namespace cjx {

namespace {

constexpr int kCols = 8;  // slice columns per CTA (one per warp in the FFT phase)

// Shared-memory layout of a column: samples at pad16(row); the transform's
// output staged at stage_idx(k), which also moves the second half of the
// column by 8 entries.  With a column stride of pad16(n) + 12 (12 mod 16 at
// n = 512), the 8-byte stores of the 4 x 8 lane map, the staged outputs of the
// transpose FFT and the window reads meet no bank conflicts within a half-warp
// except the window's 2-way ones (about 830 shared-memory wavefronts per CTA
// of 8 columns, counted on the CPU, against 1860 with stride pad16(n) + 1).
__host__ __device__ constexpr int fused_stride(int n) { return pad16(n) + 12; }
__device__ __forceinline__ int stage_idx(int k) { return stage512(k); }

// Lane -> (column, row) offsets inside the CTA's 8-column x 32-row pass of the
// plane (MAP): 0: each warp 2 columns x 16 rows, 1: 4 x 8, 2: 8 x 4, 3: one
// column x 32 rows.
template <int MAP>
__device__ __forceinline__ void fused_lane_offsets(int warp, int lane, int& du, int& dv) {
  if constexpr (MAP == 0) {
    du = 2 * (warp & 3) + (lane >> 4);
    dv = 16 * (warp >> 2) + (lane & 15);
  } else if constexpr (MAP == 1) {
    du = 4 * (warp & 1) + (lane & 3);
    dv = 8 * (warp >> 1) + (lane >> 2);
  } else if constexpr (MAP == 2) {
    du = lane & 7;
    dv = 4 * warp + (lane >> 3);
  } else {
    du = warp;
    dv = lane;
  }
}

// Body for the CTA at (bx, by) (column block, image of the chunk): smem is
// the dynamic shared memory, w32 a 32-entry shared table.
template <int R, typename Layout, int S, int MAP, bool T512>
__device__ __forceinline__ void gather_colifft_body(const float2* __restrict__ grid,
                                                    const cjx_image_params* __restrict__ params,
                                                    const int32_t* __restrict__ order, float2* __restrict__ t1,
                                                    const SliceGeom& g, int64_t k0, int bx, int by, float2* smem,
                                                    float2* w32) {
  constexpr int n = 32 * R;
  constexpr int stride = fused_stride(n);
  static_assert(!T512 || R == 16, "the transpose FFT is 512-point");
  float2* tab = smem;
  float2* tile = smem + n;  // [kCols][stride], rows in the pad16 layout
  int* winy = reinterpret_cast<int*>(tile + kCols * stride);
  const Layout L(n);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j0 = bx * kCols;
  const int ncols = min(kCols, g.ncols - j0);
  const int64_t k = k0 + by;
  const int64_t img = order ? (int64_t)order[k] : k;
  const bool ewald = (g.flags & CJX_EWALD_SPHERE) != 0;

  // tables first: their (L2-resident) loads overlap the first gathers
  build_reg_twiddles(tab, n);
  build_w32(w32);
  for (int m = threadIdx.x; m < g.py; m += blockDim.x) winy[m] = win_src(m, n, g.py, g.pad_left_y);

  {
    const double* Rm = params[img].rot;
    const float r00 = (float)Rm[0], r01 = (float)Rm[1];
    const float r10 = (float)Rm[3], r11 = (float)Rm[4];
    const float r20 = (float)Rm[6], r21 = (float)Rm[7];
    const bool wrap = !(g.flags & CJX_ZERO_FILL_NEGATIVE);
    int du, dv;
    fused_lane_offsets<MAP>(warp, lane, du, dv);
    const bool col_ok = du < ncols;
    const float ux = (float)fft_index(col_ok ? j0 + du : 0, n);
    const float bx = r00 * ux, by = r10 * ux, bz = r20 * ux;
    float cw = 0.f, r02 = 0.f, r12 = 0.f, r22 = 0.f;
    if (ewald) {
      // the sphere's third coordinate w = lambda (u^2 + v^2) / (2 N pixel_size), rotated with R's third column
      cw = ewald_w(params + img, n);
      r02 = (float)Rm[2];
      r12 = (float)Rm[5];
      r22 = (float)Rm[8];
    }
    float2* col = tile + du * stride;
#pragma unroll 1
    for (int p0 = 0; p0 < R; p0 += S) {
      float ox[S], oy[S], oz[S];
      bool act[S];
      float2 val[S];
#pragma unroll
      for (int s = 0; s < S; ++s) {
        act[s] = col_ok && (p0 + s) < R;
        const float vy = (float)fft_index(act[s] ? 32 * (p0 + s) + dv : 0, n);
        ox[s] = fmaf(r01, vy, bx);
        oy[s] = fmaf(r11, vy, by);
        oz[s] = fmaf(r21, vy, bz);
        if (ewald) {
          const float w = cw * fmaf(ux, ux, vy * vy);
          ox[s] = fmaf(r02, w, ox[s]);
          oy[s] = fmaf(r12, w, oy[s]);
          oz[s] = fmaf(r22, w, oz[s]);
        }
      }
      gather_samples<S>(grid, n, L, ox, oy, oz, act, wrap, g.fill, val);
#pragma unroll
      for (int s = 0; s < S; ++s)
        if (act[s]) col[pad16(32 * (p0 + s) + dv)] = val[s];
    }
  }
  __syncthreads();

  if (warp < ncols) {
    float2* buf = tile + warp * stride;
    const int j = j0 + warp;
    const bool sym = !ewald && (j == 0 || j == n / 2);
    const int bl = T512 ? lane : brev5(lane);  // the transpose FFT takes natural lane order
    float2 x[R];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) {
      const int idx = 32 * n1 + bl;
      float2 v = buf[pad16(idx)];
      if (sym) {  // (S[v] + conj(S[-v])) / 2, as the irfftn of the reference sees it
        const float2 m = buf[pad16(idx == 0 ? 0 : n - idx)];
        v = make_float2(0.5f * (v.x + m.x), 0.5f * (v.y - m.y));
      }
      x[n1] = v;
    }
    __syncwarp();  // every lane has its column values before the buffer is reused
    if constexpr (T512) {
      warp_fft512_t<+1>(x, tab, w32, buf, lane);
#pragma unroll
      for (int q = 0; q < R; ++q) buf[stage_idx(fft512_t_out(q, lane))] = x[q];
    } else {
      const LaneTwiddles lt = make_lane_twiddles(w32, lane);
      warp_fft_reg<R, +1>(x, tab, lt, lane);
#pragma unroll
      for (int k1 = 0; k1 < R; ++k1) buf[stage_idx(k1 + R * lane)] = x[k1];
    }
  }
  __syncthreads();

  float2* dst = t1 + (size_t)by * g.py * g.ld1 + j0;
  for (int e = threadIdx.x; e < g.py * kCols; e += blockDim.x) {
    const int m = e / kCols, jj = e % kCols;
    if (jj < ncols) {
      const int src = winy[m];
      dst[(size_t)m * g.ld1 + jj] = (src >= 0) ? tile[jj * stride + stage_idx(src)] : make_float2(0.f, 0.f);
    }
  }
}

template <int R, typename Layout, int S, int MAP, bool T512>
__global__ void __launch_bounds__(kCols * 32, 4)
    k_gather_colifft_fused(const float2* __restrict__ grid, const cjx_image_params* __restrict__ params,
                           const int32_t* __restrict__ order, float2* __restrict__ t1, SliceGeom g, int64_t k0) {
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  gather_colifft_body<R, Layout, S, MAP, T512>(grid, params, order, t1, g, k0, blockIdx.x, blockIdx.y, smem, w32);
}

template <int R, typename Layout, int S, int MAP>
void launch_fused_rsm(const SliceGeom& g, const float2* grid, const cjx_image_params* params, const int32_t* order,
                      int64_t k0, int cnt, float2* t1, bool t512, cudaStream_t stream) {
  const size_t smem = sizeof(float2) * (size_t)(32 * R + kCols * fused_stride(32 * R)) + sizeof(int) * (size_t)g.py;
  const dim3 grd((g.ncols + kCols - 1) / kCols, cnt);
  if constexpr (R == 16) {
    if (t512) {
      k_gather_colifft_fused<R, Layout, S, MAP, true><<<grd, kCols * 32, smem, stream>>>(grid, params, order, t1, g,
                                                                                         k0);
      return;
    }
  }
  k_gather_colifft_fused<R, Layout, S, MAP, false><<<grd, kCols * 32, smem, stream>>>(grid, params, order, t1, g, k0);
}

// Every layout and size with the default sample count and lane map; the other
// (S, MAP) choices for the x-pair layout at N = 512, the benchmark size.  Four
// samples per lane do not fit the 64-register budget of 4 CTAs per SM (they
// spill), so an ILP of 4 runs as 2.
template <int R, typename Layout>
int launch_fused_r(const SliceGeom& g, const float2* grid, const cjx_image_params* params, const int32_t* order,
                   int64_t k0, int cnt, float2* t1, const Tuning& tn, cudaStream_t stream) {
  const bool t512 = tn.fft_mode >= 2;
  if constexpr (R == 16 && std::is_same<Layout, PairLayout>::value) {
    const int key = 10 * tn.ilp + tn.tile;
    switch (key) {
      case 10: launch_fused_rsm<R, Layout, 1, 0>(g, grid, params, order, k0, cnt, t1, t512, stream); return CJX_OK;
      case 11: launch_fused_rsm<R, Layout, 1, 1>(g, grid, params, order, k0, cnt, t1, t512, stream); return CJX_OK;
      case 12: launch_fused_rsm<R, Layout, 1, 2>(g, grid, params, order, k0, cnt, t1, t512, stream); return CJX_OK;
      case 13: launch_fused_rsm<R, Layout, 1, 3>(g, grid, params, order, k0, cnt, t1, t512, stream); return CJX_OK;
      case 20: launch_fused_rsm<R, Layout, 2, 0>(g, grid, params, order, k0, cnt, t1, t512, stream); return CJX_OK;
      case 22: launch_fused_rsm<R, Layout, 2, 2>(g, grid, params, order, k0, cnt, t1, t512, stream); return CJX_OK;
      case 23: launch_fused_rsm<R, Layout, 2, 3>(g, grid, params, order, k0, cnt, t1, t512, stream); return CJX_OK;
      default: break;
    }
  }
  launch_fused_rsm<R, Layout, 2, 1>(g, grid, params, order, k0, cnt, t1, t512, stream);
  return CJX_OK;
}

template <typename Layout>
int launch_fused_layout(const SliceGeom& g, const float2* grid, const cjx_image_params* params, const int32_t* order,
                        int64_t k0, int cnt, float2* t1, const Tuning& tn, cudaStream_t stream) {
  switch (reg_fft_radix(g.n)) {
#define CJX_FUSED_CASE(R) \
  case R: return launch_fused_r<R, Layout>(g, grid, params, order, k0, cnt, t1, tn, stream);
    CJX_FUSED_CASE(1) CJX_FUSED_CASE(2) CJX_FUSED_CASE(3) CJX_FUSED_CASE(4) CJX_FUSED_CASE(5)
    CJX_FUSED_CASE(6) CJX_FUSED_CASE(8) CJX_FUSED_CASE(10) CJX_FUSED_CASE(12) CJX_FUSED_CASE(16)
#undef CJX_FUSED_CASE
    default:
      return fail(CJX_ERR_UNSUPPORTED, "fused gather + column FFT needs N = 32 R (R in 1-6, 8, 10, 12, 16)");
  }
}

// The front pass for every group of a wave in one launch (x-pair, bricked or
// C-order grid, as the Layout), with the default sample count and lane map.
template <typename Layout>
__global__ void __launch_bounds__(kCols * 32, 4) k_front_wave(const __grid_constant__ Wave w) {
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  const int gi = wave_group(w, 0, blockIdx.x);
  const WaveGroup& q = w.grp[gi];
  const int local = blockIdx.x - q.cta0[0];
  const int cx = (q.g.ncols + kCols - 1) / kCols;
  const int bx = local % cx, by = local / cx;
  switch (reg_fft_radix(q.g.n)) {
#define CJX_FW(R)                                                                                              \
  case R:                                                                                                      \
    gather_colifft_body<R, Layout, 2, 1, false>(q.grid, q.params, q.order, q.t1, q.g, q.k0, bx, by, smem, w32); \
    break;
    CJX_FW(1) CJX_FW(2) CJX_FW(3) CJX_FW(4) CJX_FW(5) CJX_FW(6) CJX_FW(8) CJX_FW(10) CJX_FW(12)
#undef CJX_FW
    case 16:
      if (w.t512)
        gather_colifft_body<16, Layout, 2, 1, true>(q.grid, q.params, q.order, q.t1, q.g, q.k0, bx, by, smem, w32);
      else
        gather_colifft_body<16, Layout, 2, 1, false>(q.grid, q.params, q.order, q.t1, q.g, q.k0, bx, by, smem, w32);
      break;
    default:
      break;
  }
}

}  // namespace

// Dynamic shared memory of the front pass for one group.
size_t front_wave_smem(const SliceGeom& g) {
  return sizeof(float2) * (size_t)(g.n + kCols * fused_stride(g.n)) + sizeof(int) * (size_t)g.py;
}

// CTAs of the front pass per image.
int front_wave_ctas_per_image(const SliceGeom& g) { return (g.ncols + kCols - 1) / kCols; }

int launch_front_wave(const Wave& w, int ctas, size_t smem, cudaStream_t stream) {
  static PerDeviceOnce once;
  const cudaError_t ea = once.run([] {
    cudaError_t e = cudaFuncSetAttribute(k_front_wave<PairLayout>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         220 * 1024);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_front_wave<BrickLayout>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_front_wave<LinearLayout>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
    return e;
  });
  if (ea != cudaSuccess) return check_cuda(ea, "cudaFuncSetAttribute (wave front pass)");
  const uint32_t flags = w.grp[0].g.flags;
  prof_begin(stream);
  if (flags & CJX_GRID_BRICKED_PAIRS)
    k_front_wave<PairLayout><<<ctas, kCols * 32, smem, stream>>>(w);
  else if (flags & CJX_GRID_BRICKED)
    k_front_wave<BrickLayout><<<ctas, kCols * 32, smem, stream>>>(w);
  else
    k_front_wave<LinearLayout><<<ctas, kCols * 32, smem, stream>>>(w);
  prof_end("k_front_wave", stream);
  return check_cuda(cudaGetLastError(), "k_front_wave launch");
}

// True when launch_gather_colifft_fused handles this geometry: a trilinear
// voxel grid (any of the three layouts, slice or Ewald sphere) with N of the
// register-FFT form.
bool fused_gather_supported(const SliceGeom& g) {
  return !(g.flags & CJX_GRID_SPLINE) && reg_fft_radix(g.n) != 0;
}

int launch_gather_colifft_fused(const SliceGeom& g, const float2* grid, const cjx_image_params* params,
                                const int32_t* order, int64_t k0, int cnt, float2* t1, const Tuning& tn,
                                cudaStream_t stream) {
  prof_begin(stream);
  int e;
  if (g.flags & CJX_GRID_BRICKED_PAIRS)
    e = launch_fused_layout<PairLayout>(g, grid, params, order, k0, cnt, t1, tn, stream);
  else if (g.flags & CJX_GRID_BRICKED)
    e = launch_fused_layout<BrickLayout>(g, grid, params, order, k0, cnt, t1, tn, stream);
  else
    e = launch_fused_layout<LinearLayout>(g, grid, params, order, k0, cnt, t1, tn, stream);
  prof_end("k_gather_colifft_fused", stream);
  if (e) return e;
  return check_cuda(cudaGetLastError(), "k_gather_colifft_fused launch");
}

}  // namespace cjx
