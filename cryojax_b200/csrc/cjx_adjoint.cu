// Squared-residual loss and its adjoint (reverse mode) for the resize path.
//
// Loss per image: L = sum over real-space pixels of (x - obs)^2, where x is
// the simulated image (irfftn of the Fourier image F, as simulate() returns
// it with padded_shape == shape) and obs the observed image.  With O =
// rfftn(obs) and F_h = F with its kx = 0 and kx = Px/2 columns made
// Hermitian (what irfftn actually reads), Parseval gives
//   L = 1/(Py Px) sum_half w_j |F_h - O|^2,   w_j = 1 (j = 0, Px/2), else 2.
// The adjoint runs the forward passes in reverse with their transposes:
//   k_colfft_loss_adj   column FFT (forward), epilogue, loss, E = dL/dF,
//                       d/d(shift, defocus), g_X = conj(multiplier) E, then
//                       the column inverse FFT (adjoint of the forward FFT);
//   k_rows_adj          per row: adjoint of r2c_Px, of the Px window, of the
//                       unnormalised c2r_N;
//   k_colfft_adj        per column: adjoint of the Py window, forward FFT
//                       (adjoint of the unnormalised inverse), Hermitian fix
//                       of kx = 0, N/2 (self-adjoint);
//   k_scatter_slice     trilinear scatter-add of the slice gradient into the
//                       grid gradient (float2 / float4 atomics) and d/dR from the
//                       derivative of the interpolation weights.
// On the Ewald sphere (CJX_EWALD_SPHERE with CJX_APPLY_CTF) the first three
// are k_ewald_loss_adj (contrast pairing of +q with -q), k_ewald_rows_adj
// (complex rows) and k_ewald_colfft_adj (all N surface columns), and the
// scatter samples the curved surface and adds R's third column to d/dR.
// The gradient of a real loss w.r.t. a complex value z is reported as
// dL/dRe z + i dL/dIm z (jax.grad returns its complex conjugate).
#include <algorithm>
#include <cstdint>
#include <mutex>

#include "cjx_common.cuh"
#include "cjx_profile.cuh"

namespace cjx {

// Per-image gradient record (16 doubles), matches cjx_image_grads.
constexpr int kGradLoss = 0, kGradTx = 1, kGradTy = 2, kGradDf = 3, kGradRot = 4;

// Multiplier of pass C's epilogue and its defocus derivative at (i, j):
// F = mult * X, dF/d(defocus) = dmult * X (X = unnormalised column FFT).
struct EpiTerms {
  float2 mult, dmult;
  double qx, qy;
};

__device__ __forceinline__ EpiTerms epilogue_terms(int i, int j, int py, int px, uint32_t flags,
                                                   const ImageConsts& c, double wavelength) {
  EpiTerms t;
  t.qy = (double)fft_index(i, py) * c.qy_step;
  t.qx = (double)j * c.qx_step;
  const double k2 = t.qx * t.qx + t.qy * t.qy;
  float m = c.scale, dm = 0.f;
  if (flags & CJX_APPLY_CTF) {
    float c2t = 1.0f, s2t = 0.0f;
    if (k2 > 0.0) {
      const float qxf = (float)t.qx, qyf = (float)t.qy;
      const float inv = 1.0f / (float)k2;
      c2t = (qyf * qyf - qxf * qxf) * inv;
      s2t = 2.0f * qxf * qyf * inv;
    }
    const double df = c.defocus + c.half_astig * (double)(c2t * c.cos2a + s2t * c.sin2a);
    const double arg = (c.c_def * df + c.c_sph * k2) * k2 - c.phase_cycles;
    const float r = (float)(arg - rint(arg));
    float sn, cs;
    sincospif(2.0f * r, &sn, &cs);
    dm = c.scale * cs * (float)(-3.14159265358979323846 * wavelength * k2);  // d chi / d df = -pi lambda k^2
    m = c.scale * sn;
  }
  if (flags & CJX_APPLY_ENVELOPE) {
    const float e = c.env_amp * expf(-c.env_quarter_b * (float)k2);
    m *= e;
    dm *= e;
  }
  t.mult = make_float2(m, 0.f);
  t.dmult = make_float2(dm, 0.f);
  if (flags & CJX_APPLY_TRANSLATION) {
    const bool ey = (py % 2 == 0), ex = (px % 2 == 0);
    const bool self_conj = (ey && i == py / 2 && j == 0) || (ex && i == 0 && j == px / 2) ||
                           (ey && ex && i == py / 2 && j == px / 2);
    if (self_conj) {
      t.mult = make_float2(0.f, 0.f);
      t.dmult = make_float2(0.f, 0.f);
    } else {
      const double ph = t.qx * c.tx + t.qy * c.ty;
      const float r = (float)(ph - rint(ph));
      float s, co;
      sincospif(2.0f * r, &s, &co);
      const float2 p = make_float2(co, -s);
      t.mult = make_float2(m * p.x, m * p.y);
      t.dmult = make_float2(dm * p.x, dm * p.y);
    }
  }
  return t;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// Loss + column kernel (adjoint of pass C).  t2 holds T2 on entry and the
// gradient g_T2 on exit (each CTA reads and writes only its own columns).
// ---------------------------------------------------------------------------
template <int R>
__global__ void __launch_bounds__(kWarps * 32)
    k_colfft_loss_adj(float2* __restrict__ t2, const float2* __restrict__ obs, const cjx_image_params* __restrict__ params,
                      const int32_t* __restrict__ order, double* __restrict__ grads, SliceGeom g, int64_t k0,
                      float norm) {
  constexpr int py = 32 * R;
  constexpr int stride = pad16(py) + 1;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  __shared__ float red[kWarps][4];
  float2* tab = smem;
  float2* bufs = smem + py;                  // T2 columns, then F, then g_X
  float2* obuf = bufs + kWarps * stride;     // observed columns
  __shared__ ImageConsts sc;
  const int j0 = blockIdx.x * kWarps;
  const int ncols = min(kWarps, g.pxh - j0);
  const int64_t k = k0 + blockIdx.y;
  const int64_t img = order ? (int64_t)order[k] : k;
  float2* col0 = t2 + (size_t)blockIdx.y * py * g.ld2 + j0;
  const float2* ocol0 = obs + (size_t)img * py * g.pxh + j0;
  // staging: thread t moves column t % kWarps, rows t / kWarps + 32 q; the
  // loads are issued before the table copy
  static_assert(kWarps * 32 == 256, "the staging map assumes 256 threads");
  const int sj = threadIdx.x % kWarps, sm0 = threadIdx.x / kWarps;
  {
    float2 st[R], so[R];
    if (sj < ncols) {
#pragma unroll
      for (int q = 0; q < R; ++q) {
        st[q] = col0[(size_t)(sm0 + 32 * q) * g.ld2 + sj];
        so[q] = ocol0[(size_t)(sm0 + 32 * q) * g.pxh + sj];
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
  }
  if (threadIdx.x == 0) sc = load_image_consts(params + img, norm, g.py, g.px);  // once per CTA
  const double wl = params[img].wavelength;
  __syncthreads();
  const ImageConsts& c = sc;  // read from shared memory where used (keeps the register count down)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float sl = 0.f, stx = 0.f, sty = 0.f, sdf = 0.f;
  if (warp < ncols) {
    float2* buf = bufs + warp * stride;
    const float2* ob = obuf + warp * stride;
    const LaneTwiddles lt = make_lane_twiddles(w32, lane);
    const int bl = brev5(lane);
    const int j = j0 + warp;
    float2 x[R];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) x[n1] = buf[pad16(32 * n1 + bl)];
    warp_fft_reg<R, -1>(x, tab, lt, lane);  // x[k1] = X[k1 + R lane]
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) {
      const int i = k1 + R * lane;
      const EpiTerms et = epilogue_terms(i, j, py, g.px, g.flags, c, wl);
      buf[pad16(i)] = cmul(et.mult, x[k1]);
    }
    __syncwarp();
    const bool self_col = (j == 0) || ((g.px % 2 == 0) && j == g.px / 2);
    const float wj = self_col ? 1.f : 2.f;
    const float inv_pp = 1.0f / ((float)py * (float)g.px);
    float2 gx[R];
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) {
      const int i = k1 + R * lane;
      const EpiTerms et = epilogue_terms(i, j, py, g.px, g.flags, c, wl);
      const float2 f = buf[pad16(i)];
      float2 fh = f;
      if (self_col) {
        const float2 fm = buf[pad16(i == 0 ? 0 : py - i)];
        fh = make_float2(0.5f * (f.x + fm.x), 0.5f * (f.y - fm.y));
      }
      const float2 o = ob[pad16(i)];
      const float2 d = make_float2(fh.x - o.x, fh.y - o.y);
      sl += wj * inv_pp * (d.x * d.x + d.y * d.y);
      const float2 E = make_float2(2.f * wj * inv_pp * d.x, 2.f * wj * inv_pp * d.y);
      // z = conj(E) F ; dL/dt = 2 pi q Im(z)
      const float zim = E.x * f.y - E.y * f.x;
      stx += 6.283185307179586f * (float)et.qx * zim;
      sty += 6.283185307179586f * (float)et.qy * zim;
      // dL/ddf = Re(conj(E) dmult X)
      const float2 dfx = cmul(et.dmult, x[k1]);
      sdf += E.x * dfx.x + E.y * dfx.y;
      // g_X = conj(mult) E
      gx[k1] = cmul(cconj(et.mult), E);
    }
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) buf[pad16(k1 + R * lane)] = gx[k1];
    __syncwarp();
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) x[n1] = buf[pad16(32 * n1 + bl)];
    __syncwarp();
    warp_fft_reg<R, +1>(x, tab, lt, lane);  // adjoint of the forward column FFT
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) buf[pad16(k1 + R * lane)] = x[k1];
  }
  sl = warp_sum(sl);
  stx = warp_sum(stx);
  sty = warp_sum(sty);
  sdf = warp_sum(sdf);
  if (lane == 0) {
    red[warp][kGradLoss] = sl;
    red[warp][kGradTx] = stx;
    red[warp][kGradTy] = sty;
    red[warp][kGradDf] = sdf;
  }
  __syncthreads();
  if (threadIdx.x < 4) {  // loss, d/d shift_x, d/d shift_y, d/d defocus
    double acc = 0.0;
    for (int w = 0; w < kWarps; ++w) acc += (double)red[w][threadIdx.x];
    atomicAdd(&grads[img * 16 + kGradLoss + threadIdx.x], acc);
  }
  for (int e = threadIdx.x; e < py * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) col0[(size_t)m * g.ld2 + jj] = bufs[jj * stride + pad16(m)];
  }
}

// ---------------------------------------------------------------------------
// Row adjoint (transpose of pass B).  g_T2 rows -> g_T1 rows.
// ---------------------------------------------------------------------------
template <int RN, int RP>
__device__ __forceinline__ void rows_pair_adj(const float2* __restrict__ gA, const float2* __restrict__ gB, bool has_b,
                                              float2* __restrict__ outA, int ld1, float2* buf, const float2* tabN,
                                              const float2* tabP, const LaneTwiddles& lt, int lane, const int* invx) {
  constexpr int n = 32 * RN, px = 32 * RP, hp = px / 2, h = n / 2;
  const int bl = brev5(lane);
  // adjoint of r2c_Px: Z = half spectrum with interior bins halved, DC / Nyquist real
  float2 z[RP];
#pragma unroll
  for (int n1 = 0; n1 < RP; ++n1) {
    const int k = 32 * n1 + bl;
    if (k == 0 || k == hp) {
      const float2 A = gA[k];
      const float2 B = has_b ? gB[k] : make_float2(0.f, 0.f);
      z[n1] = make_float2(A.x, B.x);
    } else if (k < hp) {
      const float2 A = gA[k];
      const float2 B = has_b ? gB[k] : make_float2(0.f, 0.f);
      z[n1] = make_float2(0.5f * (A.x - B.y), 0.5f * (A.y + B.x));
    } else {
      const float2 A = gA[px - k];
      const float2 B = has_b ? gB[px - k] : make_float2(0.f, 0.f);
      z[n1] = make_float2(0.5f * (A.x + B.y), 0.5f * (B.x - A.y));
    }
  }
  warp_fft_reg<RP, +1>(z, tabP, lt, lane);  // real rows a + i b (length Px)
#pragma unroll
  for (int k1 = 0; k1 < RP; ++k1) buf[pad16(k1 + RP * lane)] = z[k1];
  __syncwarp();
  // adjoint of the Px window: place sample m at src(m), zeros elsewhere
  float2 y[RN];
#pragma unroll
  for (int n1 = 0; n1 < RN; ++n1) {
    const int m = invx[32 * n1 + bl];
    y[n1] = (m >= 0) ? buf[pad16(m)] : make_float2(0.f, 0.f);
  }
  __syncwarp();
  warp_fft_reg<RN, -1>(y, tabN, lt, lane);  // adjoint of the unnormalised inverse
#pragma unroll
  for (int k1 = 0; k1 < RN; ++k1) buf[pad16(k1 + RN * lane)] = y[k1];
  __syncwarp();
  // split A + iB and apply the c2r weights (interior x2, DC / Nyquist real)
  for (int kk = lane; kk <= h; kk += 32) {
    const float2 Wk = buf[pad16(kk)];
    const float2 Wm = buf[pad16((n - kk) % n)];
    float2 a = make_float2(0.5f * (Wk.x + Wm.x), 0.5f * (Wk.y - Wm.y));
    float2 b = make_float2(0.5f * (Wk.y + Wm.y), -0.5f * (Wk.x - Wm.x));
    if (kk == 0 || kk == h) {
      a.y = 0.f;
      b.y = 0.f;
    } else {
      a = make_float2(2.f * a.x, 2.f * a.y);
      b = make_float2(2.f * b.x, 2.f * b.y);
    }
    outA[kk] = a;
    if (has_b) outA[ld1 + kk] = b;
  }
}

template <int RN>
__global__ void __launch_bounds__(kWarps * 32)
    k_rows_adj(const float2* __restrict__ gt2, float2* __restrict__ gt1, SliceGeom g, int rp) {
  constexpr int n = 32 * RN;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  const int px = g.px;
  const int stride = pad16(max(n, px)) + 1;
  float2* tabN = smem;
  float2* tabP = tabN + n;
  float2* bufs = tabP + px;
  int* invx = reinterpret_cast<int*>(bufs + kWarps * stride);
  build_reg_twiddles(tabN, n);
  build_reg_twiddles(tabP, px);
  build_w32(w32);
  for (int q = threadIdx.x; q < n; q += blockDim.x) invx[q] = -1;
  __syncthreads();
  for (int m = threadIdx.x; m < px; m += blockDim.x) {
    const int s = win_src(m, n, px, g.pad_left_x);
    if (s >= 0) invx[s] = m;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ra = 2 * (blockIdx.x * kWarps + warp);
  if (ra >= g.py) return;
  const bool has_b = (ra + 1) < g.py;
  const float2* gA = gt2 + ((size_t)blockIdx.y * g.py + ra) * g.ld2;
  float2* outA = gt1 + ((size_t)blockIdx.y * g.py + ra) * g.ld1;
  float2* buf = bufs + warp * stride;
  const LaneTwiddles lt = make_lane_twiddles(w32, lane);
  switch (rp) {
#define CJX_RA_CASE(RPV) \
  case RPV: rows_pair_adj<RN, RPV>(gA, gA + g.ld2, has_b, outA, g.ld1, buf, tabN, tabP, lt, lane, invx); break;
    CJX_RA_CASE(1) CJX_RA_CASE(2) CJX_RA_CASE(3) CJX_RA_CASE(4) CJX_RA_CASE(5)
    CJX_RA_CASE(6) CJX_RA_CASE(8) CJX_RA_CASE(10) CJX_RA_CASE(12) CJX_RA_CASE(16)
#undef CJX_RA_CASE
    default: break;
  }
}

// ---------------------------------------------------------------------------
// Column adjoint (transpose of pass A's FFT + window).  g_T1 -> g_H.
// ---------------------------------------------------------------------------
template <int R>
__global__ void __launch_bounds__(kWarps * 32)
    k_colfft_adj(const float2* __restrict__ gt1, float2* __restrict__ gh, SliceGeom g) {
  constexpr int n = 32 * R;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  const int stride = pad16(max(n, g.py)) + 1;
  float2* tab = smem;
  float2* bufs = smem + n;
  int* invy = reinterpret_cast<int*>(bufs + kWarps * stride);
  build_reg_twiddles(tab, n);
  build_w32(w32);
  for (int q = threadIdx.x; q < n; q += blockDim.x) invy[q] = -1;
  __syncthreads();
  for (int m = threadIdx.x; m < g.py; m += blockDim.x) {
    const int s = win_src(m, n, g.py, g.pad_left_y);
    if (s >= 0) invy[s] = m;
  }
  const int j0 = blockIdx.x * kWarps;
  const int ncols = min(kWarps, g.nxh - j0);
  const float2* src = gt1 + (size_t)blockIdx.y * g.py * g.ld1 + j0;
  for (int e = threadIdx.x; e < g.py * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) bufs[jj * stride + pad16(m)] = src[(size_t)m * g.ld1 + jj];
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = j0 + warp;
  if (j < g.nxh) {
    float2* buf = bufs + warp * stride;
    const LaneTwiddles lt = make_lane_twiddles(w32, lane);
    const int bl = brev5(lane);
    float2 y[R];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) {
      const int m = invy[32 * n1 + bl];
      y[n1] = (m >= 0) ? buf[pad16(m)] : make_float2(0.f, 0.f);
    }
    __syncwarp();
    warp_fft_reg<R, -1>(y, tab, lt, lane);
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) buf[pad16(k1 + R * lane)] = y[k1];
    __syncwarp();
    float2* col = gh + ((size_t)blockIdx.y * g.nxh + j) * g.ldh;
    const bool sym = (j == 0) || (j == n / 2);
    for (int i = lane; i < n; i += 32) {
      float2 v = buf[pad16(i)];
      if (sym) {
        const float2 m = buf[pad16(i == 0 ? 0 : n - i)];
        v = make_float2(0.5f * (v.x + m.x), 0.5f * (v.y - m.y));
      }
      col[i] = v;
    }
  }
}

// ---------------------------------------------------------------------------
// Warp aggregation of atomics that hit the same address.
// ---------------------------------------------------------------------------
// Lanes holding the same key (a gradient element index, or kNoKey) form a
// group (__match_any_sync).  A binary tree over the group's ranks (lanes in
// increasing order) sums their values: at step s a lane of rank r with
// r % 2s == 0 adds the partial sum of the lane of rank r + s, the s-th group
// member above it.  The group's lowest lane ends with the total and returns
// true; it alone issues the atomic.  Called by all 32 lanes together.
constexpr unsigned kNoKey = 0xffffffffu;

__device__ __forceinline__ bool peer_sum(unsigned key, float2& v, int lane) {
  const unsigned peers = __match_any_sync(0xffffffffu, key);
  const unsigned below = peers & ((1u << lane) - 1u);
  const unsigned above = peers & ~below & ~(1u << lane);
  const int rank = __popc(below);
  const int count = __popc(peers);
  for (int s = 1; __any_sync(0xffffffffu, rank + s < count); s <<= 1) {
    unsigned m = above;
    for (int i = 1; i < s && m; ++i) m &= m - 1u;  // drop the s - 1 nearest members above
    const int src = m ? __ffs(m) - 1 : lane;
    const float tx = __shfl_sync(0xffffffffu, v.x, src);
    const float ty = __shfl_sync(0xffffffffu, v.y, src);
    if (m && (rank % (2 * s)) == 0) {
      v.x += tx;
      v.y += ty;
    }
  }
  return rank == 0 && key != kNoKey;
}

// ---------------------------------------------------------------------------
// Trilinear scatter-add of the slice gradient and d/dR.
// ---------------------------------------------------------------------------
// The 8 corner values of one sample, corner c = 4 dz + 2 dy + dx: the fill
// value where a corner lies outside the grid (and for lanes that are not
// live).  Any layout: one 8-byte load per corner.
template <typename Layout>
__device__ __forceinline__ void load_corners(const float2* __restrict__ grid, const Layout& L, const AxisNodes& ax,
                                             const AxisNodes& ay, const AxisNodes& az, bool live, float2 fill,
                                             float2* v) {
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int dz = c >> 2, dy = (c >> 1) & 1, dx = c & 1;
    const bool ok = live && (dz ? az.v1 : az.v0) && (dy ? ay.v1 : ay.v0) && (dx ? ax.v1 : ax.v0);
    const int iz = dz ? az.i1 : az.i0, iy = dy ? ay.i1 : ay.i0, ix = dx ? ax.i1 : ax.i0;
    v[c] = ok ? __ldg(&grid[L.az(iz) + L.ay(iy) + L.ax(ix)]) : fill;
  }
}

// x-pair layout: a (dz, dy) corner row whose two x-corners are adjacent and
// inside the grid is one 16-byte entry (g(x0), g(x0 + 1)); other corners
// read the low half of their own entry.
template <>
__device__ __forceinline__ void load_corners<PairLayout>(const float2* __restrict__ grid, const PairLayout& L,
                                                         const AxisNodes& ax, const AxisNodes& ay,
                                                         const AxisNodes& az, bool live, float2 fill, float2* v) {
  const float4* g4 = reinterpret_cast<const float4*>(grid);
  const bool xpair = ax.v0 && ax.v1 && ax.i1 == ax.i0 + 1;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int dz = r >> 1, dy = r & 1;
    const bool okr = live && (dz ? az.v1 : az.v0) && (dy ? ay.v1 : ay.v0);
    const size_t row = (size_t)L.az(dz ? az.i1 : az.i0) + (size_t)L.ay(dy ? ay.i1 : ay.i0);
    if (okr && xpair) {
      const float4 q = __ldg(g4 + row + L.ax(ax.i0));
      v[2 * r] = make_float2(q.x, q.y);
      v[2 * r + 1] = make_float2(q.z, q.w);
    } else {
      v[2 * r] = (okr && ax.v0) ? __ldg(&grid[2 * (row + L.ax(ax.i0))]) : fill;
      v[2 * r + 1] = (okr && ax.v1) ? __ldg(&grid[2 * (row + L.ax(ax.i1))]) : fill;
    }
  }
}

// How the grid scatter issues its atomics (CJX_TUNE_SCATTER_VEC).
constexpr int kScatterCorner = 0;  // one 8-byte float2 atomic per valid corner
constexpr int kScatterVec = 1;     // a corner row's two x-corners in one 16-byte float4 atomic where that is
                                   // 16-byte aligned in the gradient array (even x0), else two float2 atomics
constexpr int kScatterWarpAgg = 2; // lanes whose corner hits the same voxel sum first (peer_sum), float2 atomics

// The scatter of one sample's corner rows (kScatterCorner, kScatterVec):
// weight * cotangent to each valid corner of the C-order gradient array.
template <int MODE, typename GL>
__device__ __forceinline__ void scatter_rows(float2* __restrict__ gg, const GL& G, const AxisNodes& ax,
                                             const AxisNodes& ay, const AxisNodes& az, float2 gs) {
  const bool xpair = ax.v0 && ax.v1 && ax.i1 == ax.i0 + 1;
#pragma unroll
  for (int r = 0; r < 4; ++r) {  // corner rows (dz, dy); x-corners 0 and 1
    const int dz = r >> 1, dy = r & 1;
    if (!((dz ? az.v1 : az.v0) && (dy ? ay.v1 : ay.v0))) continue;
    const int iz = dz ? az.i1 : az.i0, iy = dy ? ay.i1 : ay.i0;
    const float wyz = (dz ? az.w1 : az.w0) * (dy ? ay.w1 : ay.w0);
    const size_t row = (size_t)G.az(iz) + (size_t)G.ay(iy);
    const float2 c0 = make_float2(wyz * ax.w0 * gs.x, wyz * ax.w0 * gs.y);
    const float2 c1 = make_float2(wyz * ax.w1 * gs.x, wyz * ax.w1 * gs.y);
    const size_t e0 = row + G.ax(ax.i0), e1 = row + G.ax(ax.i1);
    if (MODE == kScatterVec && xpair && (e0 & 1) == 0 && e1 == e0 + 1) {
      atomicAdd(reinterpret_cast<float4*>(gg + e0), make_float4(c0.x, c0.y, c1.x, c1.y));
    } else {
      if (ax.v0) atomicAdd(&gg[e0], c0);
      if (ax.v1) atomicAdd(&gg[e1], c1);
    }
  }
}

// grid_grad (C order [z][y][x]) += acc (the bricked accumulator of the
// scatter), two x-neighbours per thread: for even x both are one 16-byte
// entry pair in either layout.
__global__ void k_unbrick_add(float2* __restrict__ gg, const float2* __restrict__ acc, int n) {
  const BrickLayout L(n);
  const int half = n / 2;
  const int64_t total = (int64_t)n * n * half;
  float4* g4 = reinterpret_cast<float4*>(gg);
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int x = 2 * (int)(e % half);
    const int64_t t = e / half;
    const int y = (int)(t % n), z = (int)(t / n);
    const float4 a = *reinterpret_cast<const float4*>(acc + (size_t)L.az(z) + L.ay(y) + L.ax(x));
    float4 v = g4[e];
    v.x += a.x; v.y += a.y; v.z += a.z; v.w += a.w;
    g4[e] = v;
  }
}

// One thread per sample of the half plane (16 x 16 samples per CTA): the
// sample's cotangent gs = g_H, its 8 corners (read for dH/d(coordinate)),
// the scatter of w * gs to the corners (MODE above; neighbouring samples of
// a warp's 4 x 8 patch share most of their corners, about 3.3 samples per
// voxel), and the CTA's share of dL/dR.  The scatter is bound by the L1 and
// the L2's atomic units, so fewer atomic instructions and sectors is what
// shortens it.
// EW: the Ewald sphere's full surface (N columns; the third coordinate
// w = cw (u^2 + v^2) along R's third column, so dL/dR gains that column).
template <typename Layout, int MODE, typename GL, bool EW>
__global__ void __launch_bounds__(256)
    k_scatter_slice(const float2* __restrict__ grid, const float2* __restrict__ gh,
                    const cjx_image_params* __restrict__ params, const int32_t* __restrict__ order,
                    float2* __restrict__ grad_grid, double* __restrict__ grads, SliceGeom g, int64_t k0) {
  const Layout L(g.n);
  const GL G(g.n);  // the gradient array's layout: C order, or the bricked accumulator
  constexpr int NR = EW ? 9 : 6;  // dL/dR entries: columns 0 and 1 (as (row, column) pairs), then column 2
  __shared__ float red[8][NR];
  const int n = g.n;
  const int64_t k = k0 + blockIdx.z;
  const int64_t img = order ? (int64_t)order[k] : k;
  const double* Rm = params[img].rot;
  const float r00 = (float)Rm[0], r01 = (float)Rm[1];
  const float r10 = (float)Rm[3], r11 = (float)Rm[4];
  const float r20 = (float)Rm[6], r21 = (float)Rm[7];
  const bool wrap = !(g.flags & CJX_ZERO_FILL_NEGATIVE);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int du, dv;
  gather_lane_offsets<1>(warp, lane, du, dv);
  const int u = blockIdx.x * 16 + du;
  const int v = blockIdx.y * 16 + dv;
  const bool live = u < g.ncols && v < n;
  float gr[NR];
#pragma unroll
  for (int q = 0; q < NR; ++q) gr[q] = 0.f;
  // the warp-aggregated form groups all 32 lanes, so there every lane runs the sample code (inactive
  // lanes carry kNoKey)
  if (MODE == kScatterWarpAgg || live) {
    const float2 gs = live ? gh[((size_t)blockIdx.z * g.ncols + u) * g.ldh + v] : make_float2(0.f, 0.f);
    const float ux = (float)fft_index(live ? u : 0, n), vy = (float)fft_index(live ? v : 0, n);
    float o[3] = {fmaf(r01, vy, r00 * ux), fmaf(r11, vy, r10 * ux), fmaf(r21, vy, r20 * ux)};
    float ew = 0.f;  // the surface's third coordinate
    if constexpr (EW) {
      ew = ewald_w(params + img, n) * fmaf(ux, ux, vy * vy);
      o[0] = fmaf((float)Rm[2], ew, o[0]);
      o[1] = fmaf((float)Rm[5], ew, o[1]);
      o[2] = fmaf((float)Rm[8], ew, o[2]);
    }
    const AxisNodes ax = axis_nodes(o[0], n, wrap);
    const AxisNodes ay = axis_nodes(o[1], n, wrap);
    const AxisNodes az = axis_nodes(o[2], n, wrap);
    float2 val[8];
    load_corners<Layout>(grid, L, ax, ay, az, live, g.fill, val);
    float dH[3][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};  // dH/do_axis (complex)
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int dz = c >> 2, dy = (c >> 1) & 1, dx = c & 1;
      const float wx = dx ? ax.w1 : ax.w0, wy = dy ? ay.w1 : ay.w0, wz = dz ? az.w1 : az.w0;
      const float sx = dx ? 1.f : -1.f, sy = dy ? 1.f : -1.f, sz = dz ? 1.f : -1.f;
      const float gwx = sx * wy * wz, gwy = sy * wx * wz, gwz = sz * wx * wy;
      dH[0][0] += gwx * val[c].x; dH[0][1] += gwx * val[c].y;
      dH[1][0] += gwy * val[c].x; dH[1][1] += gwy * val[c].y;
      dH[2][0] += gwz * val[c].x; dH[2][1] += gwz * val[c].y;
    }
    if (grad_grid) {
      if constexpr (MODE == kScatterWarpAgg) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
          const int dz = c >> 2, dy = (c >> 1) & 1, dx = c & 1;
          const bool ok = live && (dz ? az.v1 : az.v0) && (dy ? ay.v1 : ay.v0) && (dx ? ax.v1 : ax.v0);
          const int iz = dz ? az.i1 : az.i0, iy = dy ? ay.i1 : ay.i0, ix = dx ? ax.i1 : ax.i0;
          const float w = ((dz ? az.w1 : az.w0) * (dy ? ay.w1 : ay.w0)) * (dx ? ax.w1 : ax.w0);
          const unsigned key = ok ? (unsigned)((size_t)G.az(iz) + G.ay(iy) + G.ax(ix)) : kNoKey;
          float2 c2 = make_float2(w * gs.x, w * gs.y);
          if (peer_sum(key, c2, lane)) atomicAdd(&grad_grid[key], c2);
        }
      } else {
        scatter_rows<MODE>(grad_grid, G, ax, ay, az, gs);
      }
    }
    if (live) {
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const float dLdo = gs.x * dH[a][0] + gs.y * dH[a][1];
        gr[2 * a] = dLdo * ux;
        gr[2 * a + 1] = dLdo * vy;
        if constexpr (EW) gr[6 + a] = dLdo * ew;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < NR; ++q) gr[q] = warp_sum(gr[q]);
  if (lane == 0)
    for (int q = 0; q < NR; ++q) red[warp][q] = gr[q];
  __syncthreads();
  if (threadIdx.x < NR) {
    double acc = 0.0;
    for (int w = 0; w < 8; ++w) acc += (double)red[w][threadIdx.x];
    atomicAdd(&grads[img * 16 + kGradRot + threadIdx.x], acc);
  }
}

// ---------------------------------------------------------------------------
// Cubic-spline scatter-add (FourierVoxelSplineVolume) and d/dR.
// ---------------------------------------------------------------------------
// The transpose of sample_spline_batch: every one of a sample's 64 taps
// receives weight * cotangent in the C-order (N+2)^3 coefficient gradient,
// and d(sample)/d(coordinate) uses the basis derivatives, per axis
//   -3 (1-f)^2,  -12 f + 9 f^2,  12 (1-f) - 9 (1-f)^2,  3 f^2
// (d/dc of basis(c - i + 1) for taps i = floor(c) + 0..3; floor has zero
// derivative), with fill-valued taps included as the forward reads them.
__device__ __forceinline__ void spline_dweights(float f, float* dw) {
  const float g = 1.0f - f;
  dw[0] = -3.0f * g * g;
  dw[1] = f * fmaf(9.0f, f, -12.0f);
  dw[2] = g * fmaf(-9.0f, g, 12.0f);
  dw[3] = 3.0f * f * f;
}

template <typename Layout, bool EW>
__global__ void __launch_bounds__(256)
    k_scatter_slice_spline(const float2* __restrict__ coef, const float2* __restrict__ gh,
                           const cjx_image_params* __restrict__ params, const int32_t* __restrict__ order,
                           float2* __restrict__ grad_coef, double* __restrict__ grads, SliceGeom g, int64_t k0) {
  const Layout L(g.n);
  constexpr int NR = EW ? 9 : 6;
  __shared__ float red[8][NR];
  const int n = g.n, m = n + 2;
  const int64_t k = k0 + blockIdx.z;
  const int64_t img = order ? (int64_t)order[k] : k;
  const double* Rm = params[img].rot;
  const float r00 = (float)Rm[0], r01 = (float)Rm[1];
  const float r10 = (float)Rm[3], r11 = (float)Rm[4];
  const float r20 = (float)Rm[6], r21 = (float)Rm[7];
  const bool wrap = !(g.flags & CJX_ZERO_FILL_NEGATIVE);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int du, dv;
  gather_lane_offsets<1>(warp, lane, du, dv);
  const int u = blockIdx.x * 16 + du;
  const int v = blockIdx.y * 16 + dv;
  float gr[NR];
#pragma unroll
  for (int q = 0; q < NR; ++q) gr[q] = 0.f;
  if (u < g.ncols && v < n) {
    const float2 gs = gh[((size_t)blockIdx.z * g.ncols + u) * g.ldh + v];
    const float ux = (float)fft_index(u, n), vy = (float)fft_index(v, n);
    float o[3] = {fmaf(r01, vy, r00 * ux), fmaf(r11, vy, r10 * ux), fmaf(r21, vy, r20 * ux)};
    float ew = 0.f;  // the surface's third coordinate
    if constexpr (EW) {
      ew = ewald_w(params + img, n) * fmaf(ux, ux, vy * vy);
      o[0] = fmaf((float)params[img].rot[2], ew, o[0]);
      o[1] = fmaf((float)params[img].rot[5], ew, o[1]);
      o[2] = fmaf((float)params[img].rot[8], ew, o[2]);
    }
    const SplineAxis ax = spline_axis(o[0], n, wrap);
    const SplineAxis ay = spline_axis(o[1], n, wrap);
    const SplineAxis az = spline_axis(o[2], n, wrap);
    float dwx[4], dwy[4], dwz[4];
    spline_dweights(o[0] - floorf(o[0]), dwx);
    spline_dweights(o[1] - floorf(o[1]), dwy);
    spline_dweights(o[2] - floorf(o[2]), dwz);
    float dH[3][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
    for (int dz = 0; dz < 4; ++dz) {
      for (int dy = 0; dy < 4; ++dy) {
        const bool vzy = az.v[dz] && ay.v[dy];
        const int zy = L.az(az.i[dz]) + L.ay(ay.i[dy]);
        const size_t row = ((size_t)az.i[dz] * m + ay.i[dy]) * m;
        const float wzy = az.w[dz] * ay.w[dy];
#pragma unroll
        for (int dx = 0; dx < 4; ++dx) {
          const bool ok = vzy && ax.v[dx];
          const float2 val = ok ? __ldg(coef + zy + L.ax(ax.i[dx])) : g.fill;
          const float gwx = dwx[dx] * wzy, gwy = ax.w[dx] * dwy[dy] * az.w[dz], gwz = ax.w[dx] * ay.w[dy] * dwz[dz];
          dH[0][0] += gwx * val.x; dH[0][1] += gwx * val.y;
          dH[1][0] += gwy * val.x; dH[1][1] += gwy * val.y;
          dH[2][0] += gwz * val.x; dH[2][1] += gwz * val.y;
          if (ok && grad_coef) {
            const float w = wzy * ax.w[dx];
            atomicAdd(&grad_coef[row + ax.i[dx]], make_float2(w * gs.x, w * gs.y));
          }
        }
      }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const float dLdo = gs.x * dH[a][0] + gs.y * dH[a][1];
      gr[2 * a] = dLdo * ux;
      gr[2 * a + 1] = dLdo * vy;
      if constexpr (EW) gr[6 + a] = dLdo * ew;
    }
  }
#pragma unroll
  for (int q = 0; q < NR; ++q) gr[q] = warp_sum(gr[q]);
  if (lane == 0)
    for (int q = 0; q < NR; ++q) red[warp][q] = gr[q];
  __syncthreads();
  if (threadIdx.x < NR) {
    double acc = 0.0;
    for (int w = 0; w < 8; ++w) acc += (double)red[w][threadIdx.x];
    atomicAdd(&grads[img * 16 + kGradRot + threadIdx.x], acc);
  }
}

// ---------------------------------------------------------------------------
// Ewald sphere (CJX_EWALD_SPHERE with CJX_APPLY_CTF): the transposes of
// k_ewald_colfft (column FFTs of x and -x, the contrast pairing of +q with
// -q), k_ewald_rows (complex rows: N-point inverse, Px window, Px-point
// forward) and the column inverse FFT + Py window of the full surface (no
// Hermitian fix), on the shared-memory FFTs.
// ---------------------------------------------------------------------------
constexpr int kEwAdjWarps = 4;  // warps per CTA in the Ewald loss kernel (one output column, two T2 columns each)

// Cotangents of one output entry F(i, j) = T (V(pos, neg)) of ewald_epilogue,
// given E = dL/dF: ga, gb for its inputs a = A[i] and b = B[-i] (before the
// scale), and Re(conj(E) dF/d defocus).  With P = (w2 sin - w1 cos) / 2 and
// Q = (w1 sin + w2 cos) / 2 of the aberration phase,
//   V = (P (pos + neg).re + Q (pos + neg).im,  P (pos - neg).im + Q (neg - pos).re),
// T the envelope times the translation phase; conj(T) E is dL/dV.
struct EwaldAdj {
  float2 ga, gb;
  float ddf;
};

__device__ __forceinline__ EwaldAdj ewald_epilogue_adj(float2 a, float2 b, float2 E, int i, int j, int py, int px,
                                                      uint32_t flags, const ImageConsts& c) {
  a.x *= c.scale; a.y *= c.scale;
  b.x *= c.scale; b.y *= c.scale;
  const double qy = (double)fft_index(i, py) * c.qy_step;
  const double qx = (double)j * c.qx_step;
  const double k2 = qx * qx + qy * qy;
  const double arg = aberration_cycles(qx, qy, k2, c) - c.ps_cycles;
  const float r = (float)(arg - rint(arg));
  float s, co;
  sincospif(2.0f * r, &s, &co);
  const int kNone = 0, kNyqCol = 1, kZeroColNyqRow = 2;
  int rule = kNone;
  float2 pos = a, neg = b;
  if ((px % 2 == 0) && j == px / 2) {
    rule = kNyqCol;
    pos = cconj(b);
  } else if (j == 0 && (py % 2 == 0) && i == py / 2) {
    rule = kZeroColNyqRow;
    pos = cconj(a);
    neg = a;
  }
  const float P = 0.5f * (c.w2 * s - c.w1 * co), Q = 0.5f * (c.w1 * s + c.w2 * co);
  const float Pd = 0.5f * (c.w2 * co + c.w1 * s), Qd = 0.5f * (c.w1 * co - c.w2 * s);  // d/d(2 pi arg)
  const float sr = pos.x + neg.x, si = pos.y + neg.y;
  const float dr = neg.x - pos.x, di = pos.y - neg.y;
  float2 dv = make_float2(Pd * sr + Qd * si, Pd * di + Qd * dr);
  if (rule == kZeroColNyqRow) dv.y = -dv.y;
  // T: envelope and translation (zero at the self-conjugate entries)
  float2 T = make_float2(1.f, 0.f);
  if (flags & CJX_APPLY_ENVELOPE) {
    const float e = c.env_amp * expf(-c.env_quarter_b * (float)k2);
    T = make_float2(e, 0.f);
  }
  if (flags & CJX_APPLY_TRANSLATION) {
    const bool ey = (py % 2 == 0), ex = (px % 2 == 0);
    const bool self_conj = (ey && i == py / 2 && j == 0) || (ex && i == 0 && j == px / 2) ||
                           (ey && ex && i == py / 2 && j == px / 2);
    if (self_conj) {
      T = make_float2(0.f, 0.f);
    } else {
      const double ph = qx * c.tx + qy * c.ty;
      const float rp = (float)(ph - rint(ph));
      float sp, cp;
      sincospif(2.0f * rp, &sp, &cp);
      T = cmul(T, make_float2(cp, -sp));
    }
  }
  EwaldAdj out;
  // dF/d defocus = T dV/d(2 pi arg) * 2 pi c_def k^2
  const float dth = (float)(6.283185307179586 * c.c_def * k2);
  const float2 dF = cmul(T, make_float2(dv.x * dth, dv.y * dth));
  out.ddf = E.x * dF.x + E.y * dF.y;
  float2 G = cmul(cconj(T), E);
  if (rule == kZeroColNyqRow) G.y = -G.y;
  const float2 dpos = make_float2(G.x * P - G.y * Q, G.x * Q + G.y * P);
  const float2 dneg = make_float2(G.x * P + G.y * Q, G.x * Q - G.y * P);
  float2 ga = dpos, gb = dneg;
  if (rule == kNyqCol) {
    ga = make_float2(0.f, 0.f);
    gb = make_float2(dpos.x + dneg.x, dneg.y - dpos.y);
  } else if (rule == kZeroColNyqRow) {
    ga = make_float2(dpos.x + dneg.x, dneg.y - dpos.y);
    gb = make_float2(0.f, 0.f);
  }
  out.ga = make_float2(c.scale * ga.x, c.scale * ga.y);
  out.gb = make_float2(c.scale * gb.x, c.scale * gb.y);
  return out;
}

// Loss and the adjoint of the Ewald column pass.  One warp per output column
// x in [0, Px/2]: T2 columns x and (Px - x) mod Px are transformed, the
// contrast formed, the loss taken on the Hermitian part of the x = 0 and
// Nyquist columns (what irfftn reads), and the cotangents of both T2
// columns (inverse FFT: the adjoint of the forward FFT) written back over them.
__global__ void __launch_bounds__(kEwAdjWarps * 32)
    k_ewald_loss_adj(float2* __restrict__ t2, const float2* __restrict__ obs, const cjx_image_params* __restrict__ params,
                     const int32_t* __restrict__ order, double* __restrict__ grads, SliceGeom g, int64_t k0,
                     float norm) {
  extern __shared__ float2 smem[];
  __shared__ float red[kEwAdjWarps][4];
  const int py = g.py, px = g.px;
  const int stride = 2 * py + 2;
  float2* tw = smem;
  float2* bufs = smem + py;  // per warp: A ping-pong, B ping-pong, F, gA, gB
  build_twiddles(tw, py);
  const int64_t k = k0 + blockIdx.y;
  const int64_t img = order ? (int64_t)order[k] : k;
  const ImageConsts c = load_image_consts(params + img, norm, py, px);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int x = blockIdx.x * kEwAdjWarps + warp;
  float sl = 0.f, stx = 0.f, sty = 0.f, sdf = 0.f;
  if (x < g.pxh) {
    const int xm = (px - x) % px;
    const bool pair = xm != x;
    float2* a = bufs + warp * (2 * stride + 3 * py);
    float2* b = a + stride;
    float2* F = b + stride;
    float2* gA = F + py;
    float2* gB = gA + py;
    float2* col = t2 + (size_t)blockIdx.y * py * g.ld2;
    for (int i = lane; i < py; i += 32) {
      a[i] = col[(size_t)i * g.ld2 + x];
      if (pair) b[i] = col[(size_t)i * g.ld2 + xm];
    }
    __syncwarp();
    const float2* A = warp_fft<-1>(a, a + py, g.plan_py, tw, lane);
    const float2* B = pair ? warp_fft<-1>(b, b + py, g.plan_py, tw, lane) : A;
    __syncwarp();
    for (int i = lane; i < py; i += 32) F[i] = ewald_epilogue(A[i], B[(py - i) % py], i, x, py, px, g.flags, c);
    __syncwarp();
    const bool self_col = (x == 0) || ((px % 2 == 0) && x == px / 2);
    const float wj = self_col ? 1.f : 2.f;
    const float inv_pp = 1.0f / ((float)py * (float)px);
    const float2* ocol = obs + (size_t)img * py * g.pxh + x;
    for (int i = lane; i < py; i += 32) {
      const float2 f = F[i];
      float2 fh = f;
      if (self_col) {
        const float2 fm = F[(py - i) % py];
        fh = make_float2(0.5f * (f.x + fm.x), 0.5f * (f.y - fm.y));
      }
      const float2 o = ocol[(size_t)i * g.pxh];
      const float2 d = make_float2(fh.x - o.x, fh.y - o.y);
      sl += wj * inv_pp * (d.x * d.x + d.y * d.y);
      const float2 E = make_float2(2.f * wj * inv_pp * d.x, 2.f * wj * inv_pp * d.y);
      const float zim = E.x * f.y - E.y * f.x;  // Im(conj(E) F): dL/dt = 2 pi q Im(conj(E) F)
      stx += 6.283185307179586f * (float)((double)x * c.qx_step) * zim;
      sty += 6.283185307179586f * (float)((double)fft_index(i, py) * c.qy_step) * zim;
      const EwaldAdj ad = ewald_epilogue_adj(A[i], B[(py - i) % py], E, i, x, py, px, g.flags, c);
      sdf += ad.ddf;
      gA[i] = ad.ga;
      gB[(py - i) % py] = ad.gb;
    }
    __syncwarp();
    if (!pair) {
      for (int i = lane; i < py; i += 32) gA[i] = make_float2(gA[i].x + gB[i].x, gA[i].y + gB[i].y);
      __syncwarp();
    }
    // adjoint of the forward column FFTs (unnormalised inverse), into the ping-pong buffers
    for (int i = lane; i < py; i += 32) {
      a[i] = gA[i];
      if (pair) b[i] = gB[i];
    }
    __syncwarp();
    const float2* GA = warp_fft<+1>(a, a + py, g.plan_py, tw, lane);
    const float2* GB = pair ? warp_fft<+1>(b, b + py, g.plan_py, tw, lane) : GA;
    __syncwarp();
    for (int i = lane; i < py; i += 32) {
      col[(size_t)i * g.ld2 + x] = GA[i];
      if (pair) col[(size_t)i * g.ld2 + xm] = GB[i];
    }
  }
  sl = warp_sum(sl);
  stx = warp_sum(stx);
  sty = warp_sum(sty);
  sdf = warp_sum(sdf);
  if (lane == 0) {
    red[warp][kGradLoss] = sl;
    red[warp][kGradTx] = stx;
    red[warp][kGradTy] = sty;
    red[warp][kGradDf] = sdf;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double acc = 0.0;
    for (int w = 0; w < kEwAdjWarps; ++w) acc += (double)red[w][threadIdx.x];
    atomicAdd(&grads[img * 16 + kGradLoss + threadIdx.x], acc);
  }
}

// Adjoint of k_ewald_rows, one warp per row: g_T2 row -> Px-point inverse
// (adjoint of the forward FFT) -> transpose of the Px window -> N-point
// forward FFT (adjoint of the unnormalised inverse) -> g_T1 row.
__global__ void __launch_bounds__(kWarps * 32)
    k_ewald_rows_adj(const float2* __restrict__ t2, float2* __restrict__ t1, SliceGeom g) {
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
  const float2* row = t2 + ((size_t)blockIdx.y * g.py + r) * g.ld2;
  for (int m = lane; m < px; m += 32) a[m] = row[m];
  __syncwarp();
  float2* w = warp_fft<+1>(a, b, g.plan_px, twp, lane);
  float2* z = (w == a) ? b : a;
  for (int k = lane; k < n; k += 32) z[k] = make_float2(0.f, 0.f);
  __syncwarp();
  for (int m = lane; m < px; m += 32) {
    const int src = win_src(m, n, px, g.pad_left_x);
    if (src >= 0) z[src] = w[m];
  }
  __syncwarp();
  const float2* Z = warp_fft<-1>(z, w, g.plan_n, twn, lane);
  float2* dst = t1 + ((size_t)blockIdx.y * g.py + r) * g.ld1;
  for (int k = lane; k < n; k += 32) dst[k] = Z[k];
}

// Adjoint of the column inverse FFT + Py window over the full surface, one
// warp per column j in [0, N): g_T1 column -> transpose of the window ->
// N-point forward FFT -> the surface cotangent H[j][*].
__global__ void __launch_bounds__(kWarps * 32)
    k_ewald_colfft_adj(const float2* __restrict__ t1, float2* __restrict__ hb, SliceGeom g) {
  extern __shared__ float2 smem[];
  const int n = g.n;
  float2* tw = smem;
  float2* bufs = smem + n;
  build_twiddles(tw, n);
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = blockIdx.x * kWarps + warp;
  if (j >= g.ncols) return;
  float2* a = bufs + warp * (2 * n + 2);
  float2* b = a + n;
  for (int k = lane; k < n; k += 32) a[k] = make_float2(0.f, 0.f);
  __syncwarp();
  const float2* col = t1 + (size_t)blockIdx.y * g.py * g.ld1 + j;
  for (int m = lane; m < g.py; m += 32) {
    const int src = win_src(m, n, g.py, g.pad_left_y);
    if (src >= 0) a[src] = col[(size_t)m * g.ld1];
  }
  __syncwarp();
  const float2* Z = warp_fft<-1>(a, b, g.plan_n, tw, lane);
  float2* dst = hb + ((size_t)blockIdx.y * g.ncols + j) * g.ldh;
  for (int k = lane; k < n; k += 32) dst[k] = Z[k];
}

// Register-FFT forms (N, Px = 32 R): the transforms in registers
// (cjx_fft.cuh), shared memory for the tables, the window's inverse map
// winv[k] (the m with win_src(m) = k, or -1; win_src is one-to-one) and the
// per-warp staging that keeps the row loads and stores coalesced.
template <int RN, int RP>
__device__ __forceinline__ void ewald_row_adj_reg(float2 (&w)[RP], float2* __restrict__ dst, float2* buf,
                                                  const float2* tabN, const float2* tabP, const LaneTwiddles& lt,
                                                  int lane, const int* winv) {
  constexpr int n = 32 * RN;
  const int bl = brev5(lane);
  warp_fft_reg<RP, +1>(w, tabP, lt, lane);  // adjoint of the forward Px-point FFT
#pragma unroll
  for (int k1 = 0; k1 < RP; ++k1) buf[pad16(k1 + RP * lane)] = w[k1];
  __syncwarp();
  float2 z[RN];
#pragma unroll
  for (int n1 = 0; n1 < RN; ++n1) {
    const int m = winv[32 * n1 + bl];
    z[n1] = (m >= 0) ? buf[pad16(m)] : make_float2(0.f, 0.f);
  }
  __syncwarp();
  warp_fft_reg<RN, -1>(z, tabN, lt, lane);  // adjoint of the unnormalised N-point inverse
#pragma unroll
  for (int k1 = 0; k1 < RN; ++k1) buf[pad16(k1 + RN * lane)] = z[k1];
  __syncwarp();
  for (int k = lane; k < n; k += 32) dst[k] = buf[pad16(k)];
}

template <int RN>
__global__ void __launch_bounds__(kWarps * 32)
    k_ewald_rows_adj_reg(const float2* __restrict__ t2, float2* __restrict__ t1, SliceGeom g, int rp) {
  constexpr int n = 32 * RN;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  const int px = g.px;
  const int stride = pad16(max(n, px)) + 1;
  float2* tabN = smem;
  float2* tabP = tabN + n;
  float2* bufs = tabP + px;
  int* winv = reinterpret_cast<int*>(bufs + kWarps * stride);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.x * kWarps + warp;
  const int bl = brev5(lane);
  build_reg_twiddles(tabN, n);
  build_reg_twiddles(tabP, px);
  build_w32(w32);
  for (int k = threadIdx.x; k < n; k += blockDim.x) winv[k] = -1;
  __syncthreads();
  for (int m = threadIdx.x; m < px; m += blockDim.x) {
    const int s = win_src(m, n, px, g.pad_left_x);
    if (s >= 0) winv[s] = m;
  }
  __syncthreads();
  if (r >= g.py) return;
  const float2* row = t2 + ((size_t)blockIdx.y * g.py + r) * g.ld2;
  float2* dst = t1 + ((size_t)blockIdx.y * g.py + r) * g.ld1;
  float2* buf = bufs + warp * stride;
  const LaneTwiddles lt = make_lane_twiddles(w32, lane);
  switch (rp) {
#define CJX_ERADJ_CASE(RPV)                                                  \
  case RPV: {                                                                \
    float2 v[RPV];                                                           \
    for (int q = 0; q < RPV; ++q) v[q] = row[32 * q + bl];                   \
    ewald_row_adj_reg<RN, RPV>(v, dst, buf, tabN, tabP, lt, lane, winv);     \
  } break;
    CJX_ERADJ_CASE(1) CJX_ERADJ_CASE(2) CJX_ERADJ_CASE(3) CJX_ERADJ_CASE(4) CJX_ERADJ_CASE(5)
    CJX_ERADJ_CASE(6) CJX_ERADJ_CASE(8) CJX_ERADJ_CASE(10) CJX_ERADJ_CASE(12) CJX_ERADJ_CASE(16)
#undef CJX_ERADJ_CASE
    default: break;
  }
}

// Column adjoint in registers: a CTA takes kWarps consecutive surface
// columns, stages their g_T1 entries with coalesced row loads, and each warp
// reads its column through the window transpose into the lane's
// bit-reversed inputs; the N-point FFT's output is staged so that the
// surface column is stored contiguously.
template <int RN>
__global__ void __launch_bounds__(kWarps * 32)
    k_ewald_colfft_adj_reg(const float2* __restrict__ t1, float2* __restrict__ hb, SliceGeom g) {
  constexpr int n = 32 * RN;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  const int stride = pad16(max(n, g.py)) + 1;
  float2* tab = smem;
  float2* bufs = smem + n;
  int* winv = reinterpret_cast<int*>(bufs + kWarps * stride);
  const int j0 = blockIdx.x * kWarps;
  const int ncols = min(kWarps, g.ncols - j0);
  static_assert(kWarps * 32 == 256, "the staging map assumes 256 threads");
  const int sj = threadIdx.x % kWarps, sm0 = threadIdx.x / kWarps;
  const float2* blk = t1 + (size_t)blockIdx.y * g.py * g.ld1 + j0;
  if (sj < ncols)
    for (int m = sm0; m < g.py; m += 32) bufs[sj * stride + pad16(m)] = blk[(size_t)m * g.ld1 + sj];
  build_reg_twiddles(tab, n);
  build_w32(w32);
  for (int k = threadIdx.x; k < n; k += blockDim.x) winv[k] = -1;
  __syncthreads();
  for (int m = threadIdx.x; m < g.py; m += blockDim.x) {
    const int s = win_src(m, n, g.py, g.pad_left_y);
    if (s >= 0) winv[s] = m;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp >= ncols) return;
  const int bl = brev5(lane);
  float2* buf = bufs + warp * stride;
  float2 z[RN];
#pragma unroll
  for (int n1 = 0; n1 < RN; ++n1) {
    const int m = winv[32 * n1 + bl];
    z[n1] = (m >= 0) ? buf[pad16(m)] : make_float2(0.f, 0.f);
  }
  __syncwarp();
  const LaneTwiddles lt = make_lane_twiddles(w32, lane);
  warp_fft_reg<RN, -1>(z, tab, lt, lane);
#pragma unroll
  for (int k1 = 0; k1 < RN; ++k1) buf[pad16(k1 + RN * lane)] = z[k1];
  __syncwarp();
  float2* dst = hb + ((size_t)blockIdx.y * g.ncols + j0 + warp) * g.ldh;
  for (int k = lane; k < n; k += 32) dst[k] = buf[pad16(k)];
}

// k_ewald_loss_adj with register FFTs (Py = 32 R): a CTA takes kWarps
// consecutive output columns; T2 columns x, their mirrors and the observed
// columns are staged with coalesced row loads, and the cotangents stored
// back the same way.  Shared memory per warp: the column (then its
// cotangent), the mirror (then its cotangent), the observed column, F.
template <int R>
__global__ void __launch_bounds__(kWarps * 32)
    k_ewald_loss_adj_reg(float2* __restrict__ t2, const float2* __restrict__ obs,
                         const cjx_image_params* __restrict__ params, const int32_t* __restrict__ order,
                         double* __restrict__ grads, SliceGeom g, int64_t k0, float norm) {
  constexpr int py = 32 * R;
  constexpr int stride = pad16(py) + 1;
  extern __shared__ float2 smem[];
  __shared__ float2 w32[32];
  __shared__ float red[kWarps][4];
  __shared__ ImageConsts sc;
  float2* tab = smem;
  float2* bufs = smem + py;
  const int px = g.px;
  const int j0 = blockIdx.x * kWarps;
  const int ncols = min(kWarps, g.pxh - j0);
  const int64_t k = k0 + blockIdx.y;
  const int64_t img = order ? (int64_t)order[k] : k;
  float2* src = t2 + (size_t)blockIdx.y * py * g.ld2;
  const float2* ocol0 = obs + (size_t)img * py * g.pxh + j0;
  static_assert(kWarps * 32 == 256, "the staging map assumes 256 threads");
  const int sj = threadIdx.x % kWarps, sm0 = threadIdx.x / kWarps;
  {
    const int cj = j0 + sj, cm = (px - j0 - sj) % px;
    float2 st[R], sb[R], so[R];
    if (sj < ncols) {
#pragma unroll
      for (int q = 0; q < R; ++q) {
        st[q] = src[(size_t)(sm0 + 32 * q) * g.ld2 + cj];
        sb[q] = src[(size_t)(sm0 + 32 * q) * g.ld2 + cm];
        so[q] = ocol0[(size_t)(sm0 + 32 * q) * g.pxh + sj];
      }
    }
    build_reg_twiddles(tab, py);
    build_w32(w32);
    if (sj < ncols) {
#pragma unroll
      for (int q = 0; q < R; ++q) {
        bufs[sj * stride + pad16(sm0 + 32 * q)] = st[q];
        bufs[(kWarps + sj) * stride + pad16(sm0 + 32 * q)] = sb[q];
        bufs[(2 * kWarps + sj) * stride + pad16(sm0 + 32 * q)] = so[q];
      }
    }
  }
  if (threadIdx.x == 0) sc = load_image_consts(params + img, norm, py, px);  // once per CTA
  __syncthreads();
  const ImageConsts& c = sc;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float sl = 0.f, stx = 0.f, sty = 0.f, sdf = 0.f;
  if (warp < ncols) {
    const int x = j0 + warp;
    const bool pair = (px - x) % px != x;
    float2* A = bufs + warp * stride;
    float2* B = bufs + (kWarps + warp) * stride;
    const float2* O = bufs + (2 * kWarps + warp) * stride;
    float2* F = bufs + (3 * kWarps + warp) * stride;
    const LaneTwiddles lt = make_lane_twiddles(w32, lane);
    const int bl = brev5(lane);
    float2 v[R];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) v[n1] = A[pad16(32 * n1 + bl)];
    warp_fft_reg<R, -1>(v, tab, lt, lane);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) A[pad16(k1 + R * lane)] = v[k1];
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) v[n1] = B[pad16(32 * n1 + bl)];
    warp_fft_reg<R, -1>(v, tab, lt, lane);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) B[pad16(k1 + R * lane)] = v[k1];
    __syncwarp();
    for (int i = lane; i < py; i += 32)
      F[pad16(i)] = ewald_epilogue(A[pad16(i)], B[pad16((py - i) % py)], i, x, py, px, g.flags, c);
    __syncwarp();
    const bool self_col = (x == 0) || ((px % 2 == 0) && x == px / 2);
    const float wj = self_col ? 1.f : 2.f;
    const float inv_pp = 1.0f / ((float)py * (float)px);
    // lane i alone reads A[i] and B[-i] here, so it may overwrite them with their cotangents
    for (int i = lane; i < py; i += 32) {
      const float2 f = F[pad16(i)];
      float2 fh = f;
      if (self_col) {
        const float2 fm = F[pad16((py - i) % py)];
        fh = make_float2(0.5f * (f.x + fm.x), 0.5f * (f.y - fm.y));
      }
      const float2 o = O[pad16(i)];
      const float2 d = make_float2(fh.x - o.x, fh.y - o.y);
      sl += wj * inv_pp * (d.x * d.x + d.y * d.y);
      const float2 E = make_float2(2.f * wj * inv_pp * d.x, 2.f * wj * inv_pp * d.y);
      const float zim = E.x * f.y - E.y * f.x;
      stx += 6.283185307179586f * (float)((double)x * c.qx_step) * zim;
      sty += 6.283185307179586f * (float)((double)fft_index(i, py) * c.qy_step) * zim;
      const int im = (py - i) % py;
      const EwaldAdj ad = ewald_epilogue_adj(A[pad16(i)], B[pad16(im)], E, i, x, py, px, g.flags, c);
      sdf += ad.ddf;
      A[pad16(i)] = ad.ga;
      B[pad16(im)] = ad.gb;
    }
    __syncwarp();
    if (!pair) {  // one column: its two cotangent shares add
      for (int i = lane; i < py; i += 32) {
        const float2 a = A[pad16(i)], b = B[pad16(i)];
        A[pad16(i)] = make_float2(a.x + b.x, a.y + b.y);
      }
      __syncwarp();
    }
#pragma unroll
    for (int n1 = 0; n1 < R; ++n1) v[n1] = A[pad16(32 * n1 + bl)];
    __syncwarp();
    warp_fft_reg<R, +1>(v, tab, lt, lane);  // adjoint of the forward column FFT
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) A[pad16(k1 + R * lane)] = v[k1];
    if (pair) {
#pragma unroll
      for (int n1 = 0; n1 < R; ++n1) v[n1] = B[pad16(32 * n1 + bl)];
      __syncwarp();
      warp_fft_reg<R, +1>(v, tab, lt, lane);
#pragma unroll
      for (int k1 = 0; k1 < R; ++k1) B[pad16(k1 + R * lane)] = v[k1];
    }
  }
  sl = warp_sum(sl);
  stx = warp_sum(stx);
  sty = warp_sum(sty);
  sdf = warp_sum(sdf);
  if (lane == 0) {
    red[warp][kGradLoss] = sl;
    red[warp][kGradTx] = stx;
    red[warp][kGradTy] = sty;
    red[warp][kGradDf] = sdf;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double acc = 0.0;
    for (int w = 0; w < kWarps; ++w) acc += (double)red[w][threadIdx.x];
    atomicAdd(&grads[img * 16 + kGradLoss + threadIdx.x], acc);
  }
  for (int e = threadIdx.x; e < py * kWarps; e += blockDim.x) {
    const int m = e / kWarps, jj = e % kWarps;
    if (jj < ncols) {
      const int x = j0 + jj, xm = (px - x) % px;
      src[(size_t)m * g.ld2 + x] = bufs[jj * stride + pad16(m)];
      if (xm != x) src[(size_t)m * g.ld2 + xm] = bufs[(kWarps + jj) * stride + pad16(m)];
    }
  }
}

size_t ewald_loss_adj_reg_smem(const SliceGeom& g) {
  return sizeof(float2) * (size_t)(g.py + 4 * kWarps * (pad16(g.py) + 1));
}

size_t ewald_rows_adj_reg_smem(const SliceGeom& g) {
  return sizeof(float2) * (size_t)(g.n + g.px + kWarps * (pad16(std::max(g.n, g.px)) + 1)) + sizeof(int) * g.n;
}
size_t ewald_colfft_adj_reg_smem(const SliceGeom& g) {
  return sizeof(float2) * (size_t)(g.n + kWarps * (pad16(std::max(g.n, g.py)) + 1)) + sizeof(int) * g.n;
}

size_t ewald_loss_smem(const SliceGeom& g) {
  return sizeof(float2) * (size_t)(g.py + kEwAdjWarps * (2 * (2 * g.py + 2) + 3 * g.py));
}
size_t ewald_rows_adj_smem(const SliceGeom& g) {
  return sizeof(float2) * (size_t)(g.n + g.px + kWarps * (2 * std::max(g.n, g.px) + 2));
}
size_t ewald_colfft_adj_smem(const SliceGeom& g) { return sizeof(float2) * (size_t)(g.n + kWarps * (2 * g.n + 2)); }

// ---------------------------------------------------------------------------
// Host launcher
// ---------------------------------------------------------------------------
int launch_forward_to_t2(const SliceGeom& g, const float2* grid, const cjx_image_params* params, const int32_t* order,
                         int64_t k0, int cnt, float2* t1, float2* t2, float2* hb, cudaStream_t stream,
                         const Tuning& tn);

template <typename K>
static cudaError_t allow_smem_adj(K kernel) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
}

static int ensure_adjoint_smem_attrs() {
  static PerDeviceOnce once;
  const cudaError_t err = once.run([] {
    cudaError_t e = cudaSuccess;
#define CJX_ADJ_ATTR(R)                                                    \
  if (e == cudaSuccess) e = allow_smem_adj(k_colfft_loss_adj<R>);          \
  if (e == cudaSuccess) e = allow_smem_adj(k_rows_adj<R>);                 \
  if (e == cudaSuccess) e = allow_smem_adj(k_colfft_adj<R>);
    CJX_ADJ_ATTR(1) CJX_ADJ_ATTR(2) CJX_ADJ_ATTR(3) CJX_ADJ_ATTR(4) CJX_ADJ_ATTR(5)
    CJX_ADJ_ATTR(6) CJX_ADJ_ATTR(8) CJX_ADJ_ATTR(10) CJX_ADJ_ATTR(12) CJX_ADJ_ATTR(16)
#undef CJX_ADJ_ATTR
    if (e == cudaSuccess) e = allow_smem_adj(k_ewald_loss_adj);
    if (e == cudaSuccess) e = allow_smem_adj(k_ewald_rows_adj);
    if (e == cudaSuccess) e = allow_smem_adj(k_ewald_colfft_adj);
#define CJX_EADJ_ATTR(R)                                                         \
  if (e == cudaSuccess) e = allow_smem_adj(k_ewald_rows_adj_reg<R>);             \
  if (e == cudaSuccess) e = allow_smem_adj(k_ewald_colfft_adj_reg<R>);          \
  if (e == cudaSuccess) e = allow_smem_adj(k_ewald_loss_adj_reg<R>);
    CJX_EADJ_ATTR(1) CJX_EADJ_ATTR(2) CJX_EADJ_ATTR(3) CJX_EADJ_ATTR(4) CJX_EADJ_ATTR(5)
    CJX_EADJ_ATTR(6) CJX_EADJ_ATTR(8) CJX_EADJ_ATTR(10) CJX_EADJ_ATTR(12) CJX_EADJ_ATTR(16)
#undef CJX_EADJ_ATTR
    return e;
  });
  return err == cudaSuccess ? CJX_OK : check_cuda(err, "cudaFuncSetAttribute (adjoint kernels)");
}

__global__ void k_zero_doubles(double* p, int64_t count) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = 0.0;
}

template <typename Layout, typename GL, bool EW>
static void launch_scatter(int mode, dim3 gs, cudaStream_t stream, const float2* grid, const float2* hb,
                           const cjx_image_params* params, const int32_t* order, float2* grad_grid, double* grads,
                           const SliceGeom& g, int64_t k0) {
  switch (mode) {
#define CJX_SC_CASE(M)                                                                                             \
  case M:                                                                                                          \
    k_scatter_slice<Layout, M, GL, EW><<<gs, 256, 0, stream>>>(grid, hb, params, order, grad_grid, grads, g, k0); \
    break;
    CJX_SC_CASE(kScatterCorner) CJX_SC_CASE(kScatterVec) CJX_SC_CASE(kScatterWarpAgg)
#undef CJX_SC_CASE
    default:
      break;
  }
}

// The grid scatter for one chunk: spline coefficients (C order or bricked), or voxel grids in any layout
// scattering into the bricked accumulator (use_acc) or straight into grid_grad.
template <bool EW>
static void dispatch_scatter(dim3 gs, cudaStream_t stream, const float2* grid, const float2* hb,
                             const cjx_image_params* params, const int32_t* order, float2* grad_grid, float2* target,
                             double* grads, const SliceGeom& g, int64_t k0, int mode, bool use_acc) {
  const bool pairs = (g.flags & CJX_GRID_BRICKED_PAIRS) != 0;
  const bool bricked = (g.flags & CJX_GRID_BRICKED) != 0;
  if (g.flags & CJX_GRID_SPLINE) {
    if (bricked)
      k_scatter_slice_spline<SplineBrickLayout, EW><<<gs, 256, 0, stream>>>(grid, hb, params, order, grad_grid, grads,
                                                                            g, k0);
    else
      k_scatter_slice_spline<SplineLinearLayout, EW><<<gs, 256, 0, stream>>>(grid, hb, params, order, grad_grid,
                                                                             grads, g, k0);
  } else if (use_acc) {
    if (pairs)
      launch_scatter<PairLayout, BrickLayout, EW>(mode, gs, stream, grid, hb, params, order, target, grads, g, k0);
    else if (bricked)
      launch_scatter<BrickLayout, BrickLayout, EW>(mode, gs, stream, grid, hb, params, order, target, grads, g, k0);
    else
      launch_scatter<LinearLayout, BrickLayout, EW>(mode, gs, stream, grid, hb, params, order, target, grads, g, k0);
  } else {
    if (pairs)
      launch_scatter<PairLayout, LinearLayout, EW>(mode, gs, stream, grid, hb, params, order, target, grads, g, k0);
    else if (bricked)
      launch_scatter<BrickLayout, LinearLayout, EW>(mode, gs, stream, grid, hb, params, order, target, grads, g, k0);
    else
      launch_scatter<LinearLayout, LinearLayout, EW>(mode, gs, stream, grid, hb, params, order, target, grads, g, k0);
  }
}

size_t bricked_elements(int n);

// Bytes of the bricked accumulator of the grid scatter (voxel grids), which
// follows the per-chunk scratch in the loss workspace at a 256-byte boundary.
size_t loss_accumulator_bytes(int n) { return 256 + sizeof(float2) * bricked_elements(n); }

int launch_loss_grad(const SliceGeom& g, const float2* grid, const cjx_image_params* params, const int32_t* order,
                     int64_t n_images, const float2* obs, double* grads, float2* grad_grid, float2* acc,
                     void* workspace, int64_t chunk, cudaStream_t stream, const Tuning& tn) {
  const int rn = reg_fft_radix(g.n), rpy = reg_fft_radix(g.py), rpx = reg_fft_radix(g.px);
  const bool ewald = (g.flags & CJX_EWALD_SPHERE) != 0;
  if (ewald && !(g.flags & CJX_APPLY_CTF))
    return fail(CJX_ERR_UNSUPPORTED, "loss gradient on the Ewald sphere needs the contrast transfer (CJX_APPLY_CTF)");
  // the Ewald adjoint runs on the shared-memory FFTs (any size the forward takes)
  if (!ewald && (!rn || !rpy || !rpx))
    return fail(CJX_ERR_UNSUPPORTED, "loss gradient needs N, Py, Px = 32 R with R in {1-6, 8, 10, 12, 16}");
  prof_begin(stream);
  k_zero_doubles<<<64, 256, 0, stream>>>(grads, n_images * 16);
  prof_end("k_zero_doubles", stream);
  float2* t1 = static_cast<float2*>(workspace);
  float2* t2 = t1 + (size_t)chunk * g.py * g.ld1;
  float2* hb = t2 + (size_t)chunk * g.py * g.ld2;
  const float norm = (float)(1.0 / ((double)g.n * (double)g.n));
  const size_t s_loss = sizeof(float2) * (size_t)(g.py + 2 * kWarps * (pad16(g.py) + 1));
  const size_t s_rows = sizeof(float2) * (size_t)(g.n + g.px + kWarps * (pad16(std::max(g.n, g.px)) + 1)) +
                        sizeof(int) * (size_t)g.n;
  const size_t s_cols = sizeof(float2) * (size_t)(g.n + kWarps * (pad16(std::max(g.n, g.py)) + 1)) +
                        sizeof(int) * (size_t)g.n;
  // the Ewald row and column adjoints run on register FFTs where N and Px (rows) or N (columns) are 32 R
  const bool ew_reg_rows = ewald && tn.fft_mode >= 1 && rn && rpx;
  const bool ew_reg_cols = ewald && tn.fft_mode >= 1 && rn;
  const bool ew_reg_loss = ewald && tn.fft_mode >= 1 && rpy;
  const size_t e_loss = ew_reg_loss ? ewald_loss_adj_reg_smem(g) : ewald_loss_smem(g);
  const size_t e_rows = ew_reg_rows ? ewald_rows_adj_reg_smem(g) : ewald_rows_adj_smem(g);
  const size_t e_cols = ew_reg_cols ? ewald_colfft_adj_reg_smem(g) : ewald_colfft_adj_smem(g);
  if (ewald ? (e_loss > 227 * 1024 || e_rows > 227 * 1024 || e_cols > 227 * 1024)
            : (s_loss > 227 * 1024 || s_rows > 227 * 1024 || s_cols > 227 * 1024))
    return fail(CJX_ERR_UNSUPPORTED, "loss gradient shared-memory footprint above 227 KB for these sizes");
  if (int e = ensure_adjoint_smem_attrs()) return e;
  const bool pairs = (g.flags & CJX_GRID_BRICKED_PAIRS) != 0;
  if (pairs && (g.flags & CJX_GRID_SPLINE))
    return fail(CJX_ERR_UNSUPPORTED, "the spline adjoint reads the coefficients in the linear or bricked layout");
  // the 16-byte atomics need a 16-byte aligned gradient array
  int mode = tn.scatter_vec;
  const bool aligned16 = (reinterpret_cast<uintptr_t>(grad_grid) & 15) == 0;
  if (mode == kScatterVec && !aligned16) mode = kScatterCorner;
  // voxel grids scatter into a zeroed bricked accumulator: a warp's corner rows then touch about 12 instead of
  // about 20 distinct 128-byte lines; it is added into grid_grad (C order) at the end
  const bool use_acc = grad_grid && acc && aligned16 && !(g.flags & CJX_GRID_SPLINE);
  float2* target = use_acc ? acc : grad_grid;
  if (use_acc) {
    if (int e = check_cuda(cudaMemsetAsync(acc, 0, sizeof(float2) * bricked_elements(g.n), stream),
                           "zero the gradient accumulator"))
      return e;
  }
  for (int64_t k0 = 0; k0 < n_images; k0 += chunk) {
    const int cnt = (int)std::min<int64_t>(chunk, n_images - k0);
    if (int e = launch_forward_to_t2(g, grid, params, order, k0, cnt, t1, t2, hb, stream, tn)) return e;
    if (ewald) {
      prof_begin(stream);
      if (ew_reg_loss) {
        const dim3 gl((g.pxh + kWarps - 1) / kWarps, cnt);
        switch (rpy) {
#define CJX_ELA_CASE(R) \
  case R: k_ewald_loss_adj_reg<R><<<gl, kWarps * 32, e_loss, stream>>>(t2, obs, params, order, grads, g, k0, norm); break;
          CJX_ELA_CASE(1) CJX_ELA_CASE(2) CJX_ELA_CASE(3) CJX_ELA_CASE(4) CJX_ELA_CASE(5)
          CJX_ELA_CASE(6) CJX_ELA_CASE(8) CJX_ELA_CASE(10) CJX_ELA_CASE(12) CJX_ELA_CASE(16)
#undef CJX_ELA_CASE
        }
      } else {
        k_ewald_loss_adj<<<dim3((g.pxh + kEwAdjWarps - 1) / kEwAdjWarps, cnt), kEwAdjWarps * 32, e_loss, stream>>>(
            t2, obs, params, order, grads, g, k0, norm);
      }
      prof_end("k_ewald_loss_adj", stream);
      prof_begin(stream);
      const dim3 gr((g.py + kWarps - 1) / kWarps, cnt);
      if (ew_reg_rows) {
        switch (rn) {
#define CJX_ERA_CASE(R) \
  case R: k_ewald_rows_adj_reg<R><<<gr, kWarps * 32, e_rows, stream>>>(t2, t1, g, rpx); break;
          CJX_ERA_CASE(1) CJX_ERA_CASE(2) CJX_ERA_CASE(3) CJX_ERA_CASE(4) CJX_ERA_CASE(5)
          CJX_ERA_CASE(6) CJX_ERA_CASE(8) CJX_ERA_CASE(10) CJX_ERA_CASE(12) CJX_ERA_CASE(16)
#undef CJX_ERA_CASE
        }
      } else {
        k_ewald_rows_adj<<<gr, kWarps * 32, e_rows, stream>>>(t2, t1, g);
      }
      prof_end("k_ewald_rows_adj", stream);
      prof_begin(stream);
      const dim3 gc((g.ncols + kWarps - 1) / kWarps, cnt);
      if (ew_reg_cols) {
        switch (rn) {
#define CJX_ECA_CASE(R) \
  case R: k_ewald_colfft_adj_reg<R><<<gc, kWarps * 32, e_cols, stream>>>(t1, hb, g); break;
          CJX_ECA_CASE(1) CJX_ECA_CASE(2) CJX_ECA_CASE(3) CJX_ECA_CASE(4) CJX_ECA_CASE(5)
          CJX_ECA_CASE(6) CJX_ECA_CASE(8) CJX_ECA_CASE(10) CJX_ECA_CASE(12) CJX_ECA_CASE(16)
#undef CJX_ECA_CASE
        }
      } else {
        k_ewald_colfft_adj<<<gc, kWarps * 32, e_cols, stream>>>(t1, hb, g);
      }
      prof_end("k_ewald_colfft_adj", stream);
    } else {
    prof_begin(stream);
    const dim3 gl((g.pxh + kWarps - 1) / kWarps, cnt);
    switch (rpy) {
#define CJX_L_CASE(R) \
  case R: k_colfft_loss_adj<R><<<gl, kWarps * 32, s_loss, stream>>>(t2, obs, params, order, grads, g, k0, norm); break;
      CJX_L_CASE(1) CJX_L_CASE(2) CJX_L_CASE(3) CJX_L_CASE(4) CJX_L_CASE(5)
      CJX_L_CASE(6) CJX_L_CASE(8) CJX_L_CASE(10) CJX_L_CASE(12) CJX_L_CASE(16)
#undef CJX_L_CASE
    }
    prof_end("k_colfft_loss_adj", stream);
    prof_begin(stream);
    const dim3 gr((g.py + 2 * kWarps - 1) / (2 * kWarps), cnt);
    switch (rn) {
#define CJX_RB_CASE(R) \
  case R: k_rows_adj<R><<<gr, kWarps * 32, s_rows, stream>>>(t2, t1, g, rpx); break;
      CJX_RB_CASE(1) CJX_RB_CASE(2) CJX_RB_CASE(3) CJX_RB_CASE(4) CJX_RB_CASE(5)
      CJX_RB_CASE(6) CJX_RB_CASE(8) CJX_RB_CASE(10) CJX_RB_CASE(12) CJX_RB_CASE(16)
#undef CJX_RB_CASE
    }
    prof_end("k_rows_adj", stream);
    prof_begin(stream);
    const dim3 gc((g.nxh + kWarps - 1) / kWarps, cnt);
    switch (rn) {
#define CJX_CA_CASE(R) \
  case R: k_colfft_adj<R><<<gc, kWarps * 32, s_cols, stream>>>(t1, hb, g); break;
      CJX_CA_CASE(1) CJX_CA_CASE(2) CJX_CA_CASE(3) CJX_CA_CASE(4) CJX_CA_CASE(5)
      CJX_CA_CASE(6) CJX_CA_CASE(8) CJX_CA_CASE(10) CJX_CA_CASE(12) CJX_CA_CASE(16)
#undef CJX_CA_CASE
    }
    prof_end("k_colfft_adj", stream);
    }
    prof_begin(stream);
    const dim3 gs((g.ncols + 15) / 16, (g.n + 15) / 16, cnt);
    if (ewald)
      dispatch_scatter<true>(gs, stream, grid, hb, params, order, grad_grid, target, grads, g, k0, mode, use_acc);
    else
      dispatch_scatter<false>(gs, stream, grid, hb, params, order, grad_grid, target, grads, g, k0, mode, use_acc);
    prof_end("k_scatter_slice", stream);
  }
  if (use_acc) {
    prof_begin(stream);
    k_unbrick_add<<<148 * 8, 256, 0, stream>>>(grad_grid, acc, g.n);
    prof_end("k_unbrick_add", stream);
  }
  return check_cuda(cudaGetLastError(), "loss gradient launch");
}

}  // namespace cjx
