// Ewald-sphere extraction (CJX_EWALD_SPHERE), sm_100a.
//
// cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:225-516
// (EwaldSphereExtraction) and cryojax/simulator/_transfer_theory/
// transfer_theory.py:100-111, 165-255 (the non-projection contrast).
//
// The gather (k_gather_slice) and the column inverse FFT + window
// (k_colifft_window*) are shared with the slice path: in Ewald mode they
// sample all N columns of the curved surface and skip the Hermitian fix.
// The two passes here finish the complex resize and the contrast:
//   B  rows: N-point inverse FFT of each complex row, Px window, Px-point
//      forward FFT (ifftn -> crop/pad -> fftn, complex throughout);
//   C  columns: Py-point forward FFT of columns x and -x together, then the
//      Ewald contrast (pairing +q with -q), envelope and translation; or,
//      without CJX_APPLY_CTF, the full spectrum times the scale.
// Without resize, k_ewald_direct samples each output pixel (and its mirror)
// and applies the same epilogue.
#include <algorithm>
#include <mutex>

#include "cjx_common.cuh"
#include "cjx_profile.cuh"

namespace cjx {

constexpr int kEwWarps = 4;  // warps per CTA in the column pass (two columns each)

// Pass B.
__global__ void __launch_bounds__(kWarps * 32)
    k_ewald_rows(const float2* __restrict__ t1, float2* __restrict__ t2, SliceGeom g) {
  extern __shared__ float2 smem[];
  const int n = g.n, px = g.px;
  const int L = max(n, px);
  float2* twn = smem;
  float2* twp = twn + n;
  float2* bufs = twp + px;
  build_twiddles(twn, n);
  build_twiddles(twp, px);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.x * kWarps + warp;
  if (r >= g.py) return;
  float2* a = bufs + warp * (2 * L + 2);
  float2* b = a + L;
  const float2* row = t1 + ((size_t)blockIdx.y * g.py + r) * g.ld1;
  for (int k = lane; k < n; k += 32) a[k] = row[k];
  __syncwarp();
  float2* z = warp_fft<+1>(a, b, g.plan_n, twn, lane);
  float2* w = (z == a) ? b : a;
  for (int m = lane; m < px; m += 32) {
    const int src = win_src(m, n, px, g.pad_left_x);
    w[m] = (src >= 0) ? z[src] : make_float2(0.f, 0.f);
  }
  __syncwarp();
  float2* W = warp_fft<-1>(w, z, g.plan_px, twp, lane);
  float2* dst = t2 + ((size_t)blockIdx.y * g.py + r) * g.ld2;
  for (int k = lane; k < px; k += 32) dst[k] = W[k];
}

// Pass C.  One warp per output column x: with the CTF, x in [0, Px/2] and
// the warp transforms columns x and (Px - x) mod Px; without it, x in
// [0, Px) and one column.
__global__ void __launch_bounds__(kEwWarps * 32)
    k_ewald_colfft(const float2* __restrict__ t2, const cjx_image_params* __restrict__ params,
                   const int32_t* __restrict__ order, float2* __restrict__ out, SliceGeom g, int64_t k0,
                   float norm) {
  extern __shared__ float2 smem[];
  const int py = g.py, px = g.px;
  const int stride = 2 * py + 2;  // one column and its Stockham ping-pong half
  float2* tw = smem;
  float2* bufs = smem + py;
  build_twiddles(tw, py);
  const int64_t k = k0 + blockIdx.y;
  const int64_t img = order ? (int64_t)order[k] : k;
  const ImageConsts c = load_image_consts(params + img, norm, py, px);
  __syncthreads();
  const bool ctf = (g.flags & CJX_APPLY_CTF) != 0;
  const int pitch = ctf ? g.pxh : px;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int x = blockIdx.x * kEwWarps + warp;
  if (x >= pitch) return;
  const int xm = (px - x) % px;
  const bool pair = ctf && xm != x;
  float2* a = bufs + warp * 2 * stride;
  float2* b = a + stride;
  const float2* src = t2 + (size_t)blockIdx.y * py * g.ld2;
  for (int i = lane; i < py; i += 32) {
    a[i] = src[(size_t)i * g.ld2 + x];
    if (pair) b[i] = src[(size_t)i * g.ld2 + xm];
  }
  __syncwarp();
  const float2* A = warp_fft<-1>(a, a + py, g.plan_py, tw, lane);
  const float2* B = pair ? warp_fft<-1>(b, b + py, g.plan_py, tw, lane) : A;
  __syncwarp();
  float2* dst = out + (size_t)img * py * pitch + x;
  for (int i = lane; i < py; i += 32) {
    float2 v;
    if (ctf) {
      v = ewald_epilogue(A[i], B[(py - i) % py], i, x, py, px, g.flags, c);
    } else {
      v = A[i];
      v.x *= c.scale;
      v.y *= c.scale;
    }
    dst[(size_t)i * pitch] = apply_filter(v, g, i, x, pitch);
  }
}

// ---------------------------------------------------------------------------
// Register-FFT forms (N, Px, Py = 32 R): the same data flow with the
// transforms in registers (cjx_fft.cuh); shared memory holds the twiddle
// tables and the transposes, so loads and stores stay coalesced.
// ---------------------------------------------------------------------------
// z holds the row in the lane's bit-reversed order, loaded by the caller
// before its table copy.
// With T512 (N = 512) the N-point transform is the 16 x 32 transpose FFT
// (z in natural lane order, output staged with stage512).
template <int RN, int RP, bool T512>
__device__ __forceinline__ void ewald_row_reg(float2 (&z)[RN], float2* __restrict__ dst, float2* buf,
                                              const float2* tabN, const float2* tabP, const LaneTwiddles& lt,
                                              int lane, const int* winx, const float2* w32) {
  constexpr int px = 32 * RP;
  const int bl = brev5(lane);
  if constexpr (T512) {
    static_assert(RN == 16, "the transpose FFT is 512-point");
    warp_fft512_t<+1>(z, tabN, w32, buf, lane);
#pragma unroll
    for (int q = 0; q < RN; ++q) buf[stage512(fft512_t_out(q, lane))] = z[q];
  } else {
    warp_fft_reg<RN, +1>(z, tabN, lt, lane);
#pragma unroll
    for (int k1 = 0; k1 < RN; ++k1) buf[pad16(k1 + RN * lane)] = z[k1];
  }
  __syncwarp();
  float2 w[RP];
#pragma unroll
  for (int n1 = 0; n1 < RP; ++n1) {
    const int src = winx[32 * n1 + bl];
    w[n1] = (src >= 0) ? buf[T512 ? stage512(src) : pad16(src)] : make_float2(0.f, 0.f);
  }
  __syncwarp();
  warp_fft_reg<RP, -1>(w, tabP, lt, lane);
#pragma unroll
  for (int k1 = 0; k1 < RP; ++k1) buf[pad16(k1 + RP * lane)] = w[k1];
  __syncwarp();
  for (int k = lane; k < px; k += 32) dst[k] = buf[pad16(k)];
}

// Per-warp buffer of the Ewald row pass: the N-point transform's staging
// (stage512 with the transpose FFT, pad16 otherwise) and the Px-point one's.
__host__ __device__ inline int ewald_rows_stride(int n, int px, bool t512) {
  const int s = (n > px ? pad16(n) : pad16(px)) + 1;
  return (t512 && kStage512Size + 1 > s) ? kStage512Size + 1 : s;
}

template <int RN, bool T512 = false>
__global__ void __launch_bounds__(kWarps * 32, 4)
    k_ewald_rows_reg(const float2* __restrict__ t1, float2* __restrict__ t2, SliceGeom g, int rp) {
  constexpr int n = 32 * RN;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  const int px = g.px;
  const int stride = ewald_rows_stride(n, px, T512);
  float2* tabN = smem;
  float2* tabP = tabN + n;
  float2* bufs = tabP + px;
  int* winx = reinterpret_cast<int*>(bufs + kWarps * stride);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.x * kWarps + warp;
  float2 z[RN];  // loaded first, so that the load latency overlaps the table copy
  if (r < g.py) {
    const float2* row = t1 + ((size_t)blockIdx.y * g.py + r) * g.ld1;
    const int bl = T512 ? lane : brev5(lane);  // the transpose FFT takes natural lane order
#pragma unroll
    for (int n1 = 0; n1 < RN; ++n1) z[n1] = row[32 * n1 + bl];
  }
  build_reg_twiddles(tabN, n);
  build_reg_twiddles(tabP, px);
  build_w32(w32);
  for (int m = threadIdx.x; m < px; m += blockDim.x) winx[m] = win_src(m, n, px, g.pad_left_x);
  __syncthreads();
  if (r >= g.py) return;
  float2* dst = t2 + ((size_t)blockIdx.y * g.py + r) * g.ld2;
  float2* buf = bufs + warp * stride;
  const LaneTwiddles lt = make_lane_twiddles(w32, lane);
  switch (rp) {
#define CJX_EROW_CASE(RPV) \
  case RPV: ewald_row_reg<RN, RPV, T512>(z, dst, buf, tabN, tabP, lt, lane, winx, w32); break;
    CJX_EROW_CASE(1) CJX_EROW_CASE(2) CJX_EROW_CASE(3) CJX_EROW_CASE(4) CJX_EROW_CASE(5)
    CJX_EROW_CASE(6) CJX_EROW_CASE(8) CJX_EROW_CASE(10) CJX_EROW_CASE(12) CJX_EROW_CASE(16)
#undef CJX_EROW_CASE
    default: break;
  }
}

// Column pass: a CTA takes kWarps consecutive output columns and (with the
// CTF) their mirror columns (Px - x) mod Px; each warp transforms its column
// and its mirror, forms the contrast in place, and the CTA stores rows of
// kWarps values.
template <int R>
__global__ void __launch_bounds__(kWarps * 32)
    k_ewald_colfft_reg(const float2* __restrict__ t2, const cjx_image_params* __restrict__ params,
                       const int32_t* __restrict__ order, float2* __restrict__ out, SliceGeom g, int64_t k0,
                       float norm) {
  constexpr int py = 32 * R;
  constexpr int stride = pad16(py) + 1;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  float2* tab = smem;
  float2* row_phase = smem + py;  // exp(-2 pi i qy(i) ty)
  float2* bufs = smem + 2 * py;   // columns [0, kWarps): own, [kWarps, 2 kWarps): mirrors
  const int px = g.px;
  const bool ctf = (g.flags & CJX_APPLY_CTF) != 0;
  const int pitch = ctf ? g.pxh : px;
  const int j0 = blockIdx.x * kWarps;
  const int ncols = min(kWarps, pitch - j0);
  const float2* src = t2 + (size_t)blockIdx.y * py * g.ld2;
  // staging: thread t moves column t % kWarps (and its mirror), rows
  // t / kWarps + 32 q; the loads are issued before the table copy
  static_assert(kWarps * 32 == 256, "the staging map assumes 256 threads");
  const int sj = threadIdx.x % kWarps, sm0 = threadIdx.x / kWarps;
  const int cj = j0 + sj, cm = (px - j0 - sj) % px;
  float2 st[R], sb[R];
  if (sj < ncols) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      st[q] = src[(size_t)(sm0 + 32 * q) * g.ld2 + cj];
      if (ctf) sb[q] = src[(size_t)(sm0 + 32 * q) * g.ld2 + cm];
    }
  }
  build_reg_twiddles(tab, py);
  build_w32(w32);
  if (sj < ncols) {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      bufs[sj * stride + pad16(sm0 + 32 * q)] = st[q];
      if (ctf) bufs[(kWarps + sj) * stride + pad16(sm0 + 32 * q)] = sb[q];
    }
  }
  const int64_t k = k0 + blockIdx.y;
  const int64_t img = order ? (int64_t)order[k] : k;
  __shared__ ImageConsts sc;  // evaluated once per CTA
  if (threadIdx.x == 0) sc = load_image_consts(params + img, norm, py, px);
  __syncthreads();
  const ImageConsts& c = sc;  // read from shared memory where used (keeps the register count down)
  if (ctf && (g.flags & CJX_APPLY_TRANSLATION)) {
    for (int i = threadIdx.x; i < py; i += blockDim.x) row_phase[i] = phase_factor((double)fft_index(i, py) * c.qy_step * c.ty);
    __syncthreads();
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < ncols) {
    const LaneTwiddles lt = make_lane_twiddles(w32, lane);
    const int bl = brev5(lane);
    float2* A = bufs + warp * stride;
    float2* B = bufs + (kWarps + warp) * stride;
    float2 x[R];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) x[n1] = A[pad16(32 * n1 + bl)];
    warp_fft_reg<R, -1>(x, tab, lt, lane);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) A[pad16(k1 + R * lane)] = x[k1];
    if (ctf) {
#pragma unroll
      for (int n1 = 0; n1 < R; ++n1) x[n1] = B[pad16(32 * n1 + bl)];
      warp_fft_reg<R, -1>(x, tab, lt, lane);
      __syncwarp();
#pragma unroll
      for (int k1 = 0; k1 < R; ++k1) B[pad16(k1 + R * lane)] = x[k1];
    }
    __syncwarp();
    const int col = j0 + warp;
    const ColumnEpilogue ce = column_epilogue(col, ctf ? g.flags : 0u, c);
    for (int i = lane; i < py; i += 32) {
      float2 v = A[pad16(i)];
      if (ctf) {
        v = ewald_column_epilogue(v, B[pad16((py - i) % py)], i, col, py, px, g.flags, c, ce, row_phase);
      } else {
        v.x *= c.scale;
        v.y *= c.scale;
      }
      A[pad16(i)] = apply_filter(v, g, i, col, pitch);
    }
  }
  __syncthreads();
  float2* dst = out + (size_t)img * py * pitch + j0;
  for (int e = threadIdx.x; e < py * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) dst[(size_t)m * pitch + jj] = bufs[jj * stride + pad16(m)];
  }
}

// Offset from the grid centre of surface entry (i, j) (pixel frequency
// indices v, u): R (u, v, cw (u^2 + v^2)).
struct SurfaceFrame {
  float r00, r01, r02, r10, r11, r12, r20, r21, r22, cw;
};

__device__ __forceinline__ SurfaceFrame surface_frame(const cjx_image_params* __restrict__ p, int n) {
  const double* R = p->rot;
  SurfaceFrame f;
  f.r00 = (float)R[0]; f.r01 = (float)R[1]; f.r02 = (float)R[2];
  f.r10 = (float)R[3]; f.r11 = (float)R[4]; f.r12 = (float)R[5];
  f.r20 = (float)R[6]; f.r21 = (float)R[7]; f.r22 = (float)R[8];
  f.cw = ewald_w(p, n);
  return f;
}

__device__ __forceinline__ void surface_offset(const SurfaceFrame& f, int i, int j, int n, float& ox, float& oy,
                                               float& oz) {
  const float ux = (float)fft_index(j, n), vy = (float)fft_index(i, n);
  // same operation order as the gather kernel's: R's first two columns, then the sphere term
  ox = fmaf(f.r01, vy, f.r00 * ux);
  oy = fmaf(f.r11, vy, f.r10 * ux);
  oz = fmaf(f.r21, vy, f.r20 * ux);
  const float w = f.cw * fmaf(ux, ux, vy * vy);
  ox = fmaf(f.r02, w, ox);
  oy = fmaf(f.r12, w, oy);
  oz = fmaf(f.r22, w, oz);
}

// No-resize path ((Py, Px) == (N, N)): one thread per output entry.
template <typename Layout>
__global__ void __launch_bounds__(256)
    k_ewald_direct(const float2* __restrict__ grid, const cjx_image_params* __restrict__ params,
                   const int32_t* __restrict__ order, float2* __restrict__ out, SliceGeom g, int64_t k0) {
  const Layout L(g.n);
  const int n = g.n;
  const int64_t k = k0 + blockIdx.y;
  const int64_t img = order ? (int64_t)order[k] : k;
  const SurfaceFrame f = surface_frame(params + img, n);
  const bool wrap = !(g.flags & CJX_ZERO_FILL_NEGATIVE);
  const bool ctf = (g.flags & CJX_APPLY_CTF) != 0;
  const ImageConsts c = load_image_consts(params + img, 1.0f, n, n);
  const int width = ctf ? g.nxh : n;
  const int total = n * width;
  float2* dst = out + (size_t)img * total;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int i = e / width, j = e - i * width;
    float ox[2], oy[2], oz[2];
    float2 v[2];
    surface_offset(f, i, j, n, ox[0], oy[0], oz[0]);
    if (ctf) {
      surface_offset(f, (n - i) % n, (n - j) % n, n, ox[1], oy[1], oz[1]);
      const bool act[2] = {true, true};
      gather_samples<2>(grid, n, L, ox, oy, oz, act, wrap, g.fill, v);
      dst[e] = apply_filter(ewald_epilogue(v[0], v[1], i, j, n, n, g.flags, c), g, i, j, width);
    } else {
      const bool act = true;
      gather_samples<1>(grid, n, L, ox, oy, oz, &act, wrap, g.fill, v);
      dst[e] = apply_filter(make_float2(v[0].x * c.scale, v[0].y * c.scale), g, i, j, width);
    }
  }
}

size_t ewald_rows_smem(const SliceGeom& g) {
  const int L = std::max(g.n, g.px);
  return sizeof(float2) * (size_t)(g.n + g.px + kWarps * (2 * L + 2));
}

size_t ewald_cols_smem(const SliceGeom& g) {
  return sizeof(float2) * (size_t)(g.py + kEwWarps * 2 * (2 * g.py + 2));
}

static int ensure_ewald_smem() {
  static PerDeviceOnce once;
  const cudaError_t err = once.run([] {
    const int kMax = 227 * 1024;
    cudaError_t e = cudaFuncSetAttribute(k_ewald_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ewald_colfft, cudaFuncAttributeMaxDynamicSharedMemorySize, kMax);
    // the register kernels also hold a static 32-entry twiddle table
    const int kMaxReg = kMax - 1024;
#define CJX_EW_ATTR(R)                                                                                        \
  if (e == cudaSuccess)                                                                                       \
    e = cudaFuncSetAttribute(k_ewald_colfft_reg<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxReg);     \
  if (e == cudaSuccess)                                                                                       \
    e = cudaFuncSetAttribute(k_ewald_rows_reg<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxReg);
    CJX_EW_ATTR(1) CJX_EW_ATTR(2) CJX_EW_ATTR(3) CJX_EW_ATTR(4) CJX_EW_ATTR(5)
    CJX_EW_ATTR(6) CJX_EW_ATTR(8) CJX_EW_ATTR(10) CJX_EW_ATTR(12) CJX_EW_ATTR(16)
#undef CJX_EW_ATTR
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_ewald_rows_reg<16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxReg);
    return e;
  });
  return err == cudaSuccess ? CJX_OK : check_cuda(err, "cudaFuncSetAttribute (Ewald kernels)");
}

int launch_ewald_rows(const SliceGeom& g, const float2* t1, float2* t2, int cnt, cudaStream_t stream,
                      const Tuning& tn) {
  if (int e = ensure_ewald_smem()) return e;
  const dim3 gd((g.py + kWarps - 1) / kWarps, cnt);
  const int rn = reg_fft_radix(g.n), rp = reg_fft_radix(g.px);
  prof_begin(stream);
  if (tn.fft_mode >= 1 && rn && rp) {
    const bool t512 = rn == 16 && tn.fft_mode >= 3;  // the 512-point transform through one transpose
    const size_t sm = sizeof(float2) * (size_t)(g.n + g.px + kWarps * ewald_rows_stride(g.n, g.px, t512)) +
                      sizeof(int) * (size_t)g.px;
    if (t512) {
      k_ewald_rows_reg<16, true><<<gd, kWarps * 32, sm, stream>>>(t1, t2, g, rp);
      prof_end("k_ewald_rows", stream);
      return check_cuda(cudaGetLastError(), "k_ewald_rows launch");
    }
    switch (rn) {
#define CJX_ER_CASE(R) \
  case R: k_ewald_rows_reg<R><<<gd, kWarps * 32, sm, stream>>>(t1, t2, g, rp); break;
      CJX_ER_CASE(1) CJX_ER_CASE(2) CJX_ER_CASE(3) CJX_ER_CASE(4) CJX_ER_CASE(5)
      CJX_ER_CASE(6) CJX_ER_CASE(8) CJX_ER_CASE(10) CJX_ER_CASE(12) CJX_ER_CASE(16)
#undef CJX_ER_CASE
    }
  } else {
    const size_t sm = ewald_rows_smem(g);
    if (sm > 227 * 1024) return fail(CJX_ERR_UNSUPPORTED, "Ewald row pass: shared memory exceeds 227 KB");
    k_ewald_rows<<<gd, kWarps * 32, sm, stream>>>(t1, t2, g);
  }
  prof_end("k_ewald_rows", stream);
  return check_cuda(cudaGetLastError(), "k_ewald_rows launch");
}

int launch_ewald_colfft(const SliceGeom& g, const float2* t2, const cjx_image_params* params, const int32_t* order,
                        float2* out, int64_t k0, int cnt, cudaStream_t stream, const Tuning& tn) {
  if (int e = ensure_ewald_smem()) return e;
  const int cols = (g.flags & CJX_APPLY_CTF) ? g.pxh : g.px;
  const float norm = (float)(1.0 / ((double)g.n * (double)g.n));
  const int ry = reg_fft_radix(g.py);
  prof_begin(stream);
  if (tn.fft_mode >= 1 && ry) {
    const dim3 gd((cols + kWarps - 1) / kWarps, cnt);
    const size_t sm = sizeof(float2) * (size_t)(2 * g.py + 2 * kWarps * (pad16(g.py) + 1));
    switch (ry) {
#define CJX_EC_CASE(R) \
  case R: k_ewald_colfft_reg<R><<<gd, kWarps * 32, sm, stream>>>(t2, params, order, out, g, k0, norm); break;
      CJX_EC_CASE(1) CJX_EC_CASE(2) CJX_EC_CASE(3) CJX_EC_CASE(4) CJX_EC_CASE(5)
      CJX_EC_CASE(6) CJX_EC_CASE(8) CJX_EC_CASE(10) CJX_EC_CASE(12) CJX_EC_CASE(16)
#undef CJX_EC_CASE
    }
  } else {
    const size_t sm = ewald_cols_smem(g);
    if (sm > 227 * 1024) return fail(CJX_ERR_UNSUPPORTED, "Ewald column pass: shared memory exceeds 227 KB");
    k_ewald_colfft<<<dim3((cols + kEwWarps - 1) / kEwWarps, cnt), kEwWarps * 32, sm, stream>>>(t2, params, order,
                                                                                                 out, g, k0, norm);
  }
  prof_end("k_ewald_colfft", stream);
  return check_cuda(cudaGetLastError(), "k_ewald_colfft launch");
}

int launch_ewald_direct(const SliceGeom& g, const float2* grid, const cjx_image_params* params, const int32_t* order,
                        int64_t n_images, float2* out, cudaStream_t stream) {
  const int width = (g.flags & CJX_APPLY_CTF) ? g.nxh : g.n;
  const int total = g.n * width;
  const int blocks = std::min((total + 255) / 256, 1024);
  const bool spline = (g.flags & CJX_GRID_SPLINE) != 0;
  for (int64_t k0 = 0; k0 < n_images; k0 += 65535) {
    const int cnt = (int)std::min<int64_t>(65535, n_images - k0);
    const dim3 gd(blocks, cnt);
    prof_begin(stream);
    if (spline && (g.flags & CJX_GRID_BRICKED_PAIRS))
      k_ewald_direct<SplinePairLayout><<<gd, 256, 0, stream>>>(grid, params, order, out, g, k0);
    else if (spline && (g.flags & CJX_GRID_BRICKED))
      k_ewald_direct<SplineBrickLayout><<<gd, 256, 0, stream>>>(grid, params, order, out, g, k0);
    else if (spline)
      k_ewald_direct<SplineLinearLayout><<<gd, 256, 0, stream>>>(grid, params, order, out, g, k0);
    else if (g.flags & CJX_GRID_BRICKED_PAIRS)
      k_ewald_direct<PairLayout><<<gd, 256, 0, stream>>>(grid, params, order, out, g, k0);
    else if (g.flags & CJX_GRID_BRICKED)
      k_ewald_direct<BrickLayout><<<gd, 256, 0, stream>>>(grid, params, order, out, g, k0);
    else
      k_ewald_direct<LinearLayout><<<gd, 256, 0, stream>>>(grid, params, order, out, g, k0);
    prof_end("k_ewald_direct", stream);
  }
  return check_cuda(cudaGetLastError(), "k_ewald_direct launch");
}

}  // namespace cjx
