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
    dst[(size_t)i * pitch] = v;
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
      dst[e] = ewald_epilogue(v[0], v[1], i, j, n, n, g.flags, c);
    } else {
      const bool act = true;
      gather_samples<1>(grid, n, L, ox, oy, oz, &act, wrap, g.fill, v);
      dst[e] = make_float2(v[0].x * c.scale, v[0].y * c.scale);
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
  static std::once_flag flags[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return check_cuda(cudaGetLastError(), "cudaGetDevice");
  int err = CJX_OK;
  std::call_once(flags[dev & 63], [&] {
    cudaError_t e = cudaFuncSetAttribute(k_ewald_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_ewald_colfft, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) err = check_cuda(e, "cudaFuncSetAttribute");
  });
  return err;
}

int launch_ewald_rows(const SliceGeom& g, const float2* t1, float2* t2, int cnt, cudaStream_t stream) {
  if (int e = ensure_ewald_smem()) return e;
  const size_t sm = ewald_rows_smem(g);
  if (sm > 227 * 1024) return fail(CJX_ERR_UNSUPPORTED, "Ewald row pass: shared memory exceeds 227 KB");
  prof_begin(stream);
  k_ewald_rows<<<dim3((g.py + kWarps - 1) / kWarps, cnt), kWarps * 32, sm, stream>>>(t1, t2, g);
  prof_end("k_ewald_rows", stream);
  return check_cuda(cudaGetLastError(), "k_ewald_rows launch");
}

int launch_ewald_colfft(const SliceGeom& g, const float2* t2, const cjx_image_params* params, const int32_t* order,
                        float2* out, int64_t k0, int cnt, cudaStream_t stream) {
  if (int e = ensure_ewald_smem()) return e;
  const size_t sm = ewald_cols_smem(g);
  if (sm > 227 * 1024) return fail(CJX_ERR_UNSUPPORTED, "Ewald column pass: shared memory exceeds 227 KB");
  const int cols = (g.flags & CJX_APPLY_CTF) ? g.pxh : g.px;
  const float norm = (float)(1.0 / ((double)g.n * (double)g.n));
  prof_begin(stream);
  k_ewald_colfft<<<dim3((cols + kEwWarps - 1) / kEwWarps, cnt), kEwWarps * 32, sm, stream>>>(t2, params, order, out,
                                                                                               g, k0, norm);
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
