// Shared device helpers for the cryojax_b200 kernels: geometry of one
// launch, cryoJAX's trilinear sampling rule, the CTF / envelope /
// translation epilogue, and host-side error plumbing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>
#include <string>
#include <type_traits>

#include "../../include/cryojax_b200.h"
#include "cjx_fft.cuh"

namespace cjx {

constexpr int kWarps = 8;  // warps per CTA in the column / row passes

// Geometry of one (volume side, image shape) group.
struct SliceGeom {
  int n;            // volume side N
  int py, px;       // padded image shape
  int nxh;          // N/2 + 1 (half-plane columns of the slice)
  int ncols;        // slice columns sampled: N/2 + 1, or N for the Ewald sphere's full surface
  int pxh;          // Px/2 + 1
  int ld1, ld2;     // row pitch (complex elements) of workspace T1, T2
  int ldh;          // column pitch of the slice buffer H ([kx][ky], split gather)
  int pad_left_y;   // left pad when Py > N (cryojax/ndimage/_edges.py:175-185)
  int pad_left_x;
  uint32_t flags;
  float2 fill;      // out-of-bounds fill value
  FftPlan plan_n, plan_py, plan_px;
  const float* filter;  // optional Fourier-space filter over the output grid (row pitch = output columns)
};

// Output entry (i, j) times the optional fused filter.
__device__ __forceinline__ float2 apply_filter(float2 v, const SliceGeom& g, int i, int j, int pitch) {
  if (g.filter) {
    const float f = __ldg(g.filter + (size_t)i * pitch + j);
    v.x *= f;
    v.y *= f;
  }
  return v;
}

// ---------------------------------------------------------------------------
// Index helpers
// ---------------------------------------------------------------------------

// Signed frequency index of entry i of an fftfreq-ordered axis of length n
// (numpy.fft.fftfreq(n) * n).
__device__ __forceinline__ int fft_index(int i, int n) { return (i < n - n / 2) ? i : i - n; }

// Resize window along one axis (irfftn -> fftshift -> centre crop or pad ->
// ifftshift -> rfftn, cryojax/simulator/_volume_integrator/
// fourier_voxel_extract.py:133-138 with cryojax/ndimage/_edges.py:15-62,
// 110-185): destination sample m of the unshifted length-n_dst signal comes
// from sample win_src(m) of the unshifted length-n_src signal, or is zero
// padding when win_src returns -1.
__device__ __forceinline__ int win_src(int m, int n_src, int n_dst, int pad_left) {
  const int mm = (m + n_dst / 2) % n_dst;  // position in the centred destination
  int s;
  if (n_dst <= n_src) {
    s = mm + (n_src / 2 - n_dst / 2);
  } else {
    s = mm - pad_left;
    if (s < 0 || s >= n_src) return -1;
  }
  return (s - n_src / 2 + n_src) % n_src;
}

// ---------------------------------------------------------------------------
// Trilinear sampling with cryoJAX's rule
// (cryojax/ndimage/_map_coordinates.py:85-123, 168-175): lower = floor(c),
// w_hi = c - lower, w_lo = 1 - w_hi; each of the 8 corners is read with
// `.at[idx].get(mode="fill")`: a negative index wraps once to idx + N, any
// index still outside [0, N) yields the fill value.
//
// The coordinate is passed as an offset from the grid centre N/2 (the
// logical coordinate is offset + N/2, cryojax/simulator/_volume_integrator/
// fourier_voxel_extract.py:528): floor and weights are taken on the offset,
// so the interpolation weights keep full single precision near the origin
// where the spectrum is largest.
// ---------------------------------------------------------------------------
struct AxisNodes {
  int i0, i1;      // wrapped corner indices (clamped when invalid)
  bool v0, v1;     // corner inside [0, N)
  float w0, w1;    // lower / upper weights
};

__device__ __forceinline__ AxisNodes axis_nodes(float off, int n, bool wrap_negative) {
  AxisNodes a;
  const float f = floorf(off);
  a.w1 = off - f;
  a.w0 = 1.0f - a.w1;
  int i0 = (int)f + n / 2;
  int i1 = i0 + 1;
  if (wrap_negative) {
    if (i0 < 0) i0 += n;
    if (i1 < 0) i1 += n;
  }
  a.v0 = (unsigned)i0 < (unsigned)n;
  a.v1 = (unsigned)i1 < (unsigned)n;
  a.i0 = a.v0 ? i0 : 0;
  a.i1 = a.v1 ? i1 : 0;
  return a;
}

__device__ __forceinline__ float2 sample_trilinear(const float2* __restrict__ grid, int n, float ox, float oy,
                                                   float oz, bool wrap_negative, float2 fill) {
  const AxisNodes ax = axis_nodes(ox, n, wrap_negative);
  const AxisNodes ay = axis_nodes(oy, n, wrap_negative);
  const AxisNodes az = axis_nodes(oz, n, wrap_negative);
  float2 acc = make_float2(0.f, 0.f);
#pragma unroll
  for (int dz = 0; dz < 2; ++dz) {
    const int iz = dz ? az.i1 : az.i0;
    const bool vz = dz ? az.v1 : az.v0;
    const float wz = dz ? az.w1 : az.w0;
#pragma unroll
    for (int dy = 0; dy < 2; ++dy) {
      const int iy = dy ? ay.i1 : ay.i0;
      const bool vy = dy ? ay.v1 : ay.v0;
      const float wzy = wz * (dy ? ay.w1 : ay.w0);
      const size_t row = ((size_t)iz * n + iy) * n;
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        const int ix = dx ? ax.i1 : ax.i0;
        const bool ok = vz && vy && (dx ? ax.v1 : ax.v0);
        const float w = wzy * (dx ? ax.w1 : ax.w0);
        const float2 g = ok ? __ldg(&grid[row + ix]) : fill;
        acc.x = fmaf(w, g.x, acc.x);
        acc.y = fmaf(w, g.y, acc.y);
      }
    }
  }
  return acc;
}

// S samples at once: every corner load of all S samples is issued before
// any is consumed, so one lane keeps 8*S independent loads in flight.
template <int S>
__device__ __forceinline__ void sample_trilinear_batch(const float2* __restrict__ grid, int n, const float* ox,
                                                       const float* oy, const float* oz, const bool* active,
                                                       bool wrap_negative, float2 fill, float2* out) {
  float2 v[S][8];
  float w[S][6];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const AxisNodes ax = axis_nodes(ox[s], n, wrap_negative);
    const AxisNodes ay = axis_nodes(oy[s], n, wrap_negative);
    const AxisNodes az = axis_nodes(oz[s], n, wrap_negative);
    w[s][0] = ax.w0; w[s][1] = ax.w1; w[s][2] = ay.w0; w[s][3] = ay.w1; w[s][4] = az.w0; w[s][5] = az.w1;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int dz = c >> 2, dy = (c >> 1) & 1, dx = c & 1;
      const int iz = dz ? az.i1 : az.i0, iy = dy ? ay.i1 : ay.i0, ix = dx ? ax.i1 : ax.i0;
      const bool ok = active[s] && (dz ? az.v1 : az.v0) && (dy ? ay.v1 : ay.v0) && (dx ? ax.v1 : ax.v0);
      v[s][c] = ok ? __ldg(&grid[((size_t)iz * n + iy) * n + ix]) : fill;
    }
  }
#pragma unroll
  for (int s = 0; s < S; ++s) {
    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int dz = c >> 2, dy = (c >> 1) & 1, dx = c & 1;
      const float wt = (w[s][4 + dz] * w[s][2 + dy]) * w[s][dx];
      acc.x = fmaf(wt, v[s][c].x, acc.x);
      acc.y = fmaf(wt, v[s][c].y, acc.y);
    }
    out[s] = acc;
  }
}

// ---------------------------------------------------------------------------
// Volume layouts.  The address of voxel (z, y, x) is ax(x) + ay(y) + az(z)
// in complex elements.
//  - LinearLayout: the reference's C-order [z][y][x] array.
//  - BrickLayout: 8x8x8 blocks in C order; inside a block the 512 voxels are
//    in Morton order (bit pattern z2 y2 x2 z1 y1 x1 z0 y0 x0), so every
//    2x2x2 brick is 64 contiguous bytes and every 4x4x4 brick 512 bytes.
//    A randomly oriented slice plane then touches compact clusters of
//    voxels per DRAM burst and per cache line instead of x-runs.
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int spread3(int v) { return (v & 1) | ((v & 2) << 2) | ((v & 4) << 4); }

__host__ __device__ __forceinline__ int brick_blocks(int n) { return (n + 7) / 8; }

struct LinearLayout {
  int n, nn;
  __host__ __device__ explicit LinearLayout(int n_) : n(n_), nn(n_ * n_) {}
  __device__ __forceinline__ int ax(int i) const { return i; }
  __device__ __forceinline__ int ay(int i) const { return i * n; }
  __device__ __forceinline__ int az(int i) const { return i * nn; }
};

struct BrickLayout {
  int sy, sz;  // block strides (elements) along y and z
  __host__ __device__ explicit BrickLayout(int n) : sy(brick_blocks(n) * 512), sz(brick_blocks(n) * brick_blocks(n) * 512) {}
  __device__ __forceinline__ int ax(int i) const { return ((i >> 3) << 9) + spread3(i & 7); }
  __device__ __forceinline__ int ay(int i) const { return (i >> 3) * sy + (spread3(i & 7) << 1); }
  __device__ __forceinline__ int az(int i) const { return (i >> 3) * sz + (spread3(i & 7) << 2); }
};

// Same result as sample_trilinear_batch with a fast path: when all 8 corners
// of a sample are inside [0, N)^3 (every sample away from the cube faces)
// they are read at base + {0, 1, N, N+1, N^2, ...} with 32-bit offsets and no
// per-corner checks; samples near the faces take the general rule.
template <int S, typename Layout>
__device__ __forceinline__ void sample_trilinear_batch_fast(const float2* __restrict__ grid, int n, const Layout& L,
                                                            const float* ox, const float* oy, const float* oz,
                                                            const bool* active, bool wrap_negative, float2 fill,
                                                            float2* out) {
  float2 v[S][8];
  float w[S][6];
  const int h = n / 2;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const float fx = floorf(ox[s]), fy = floorf(oy[s]), fz = floorf(oz[s]);
    w[s][1] = ox[s] - fx; w[s][0] = 1.0f - w[s][1];
    w[s][3] = oy[s] - fy; w[s][2] = 1.0f - w[s][3];
    w[s][5] = oz[s] - fz; w[s][4] = 1.0f - w[s][5];
    const int ix0 = (int)fx + h, iy0 = (int)fy + h, iz0 = (int)fz + h;
    const bool interior = (unsigned)ix0 < (unsigned)(n - 1) && (unsigned)iy0 < (unsigned)(n - 1) &&
                          (unsigned)iz0 < (unsigned)(n - 1);
    if (interior) {
      if (active[s]) {
        const int x0 = L.ax(ix0), x1 = L.ax(ix0 + 1);
        const int y0 = L.ay(iy0), y1 = L.ay(iy0 + 1);
        const int z0 = L.az(iz0), z1 = L.az(iz0 + 1);
        const int zy00 = z0 + y0, zy01 = z0 + y1, zy10 = z1 + y0, zy11 = z1 + y1;
        v[s][0] = __ldg(grid + zy00 + x0);
        v[s][1] = __ldg(grid + zy00 + x1);
        v[s][2] = __ldg(grid + zy01 + x0);
        v[s][3] = __ldg(grid + zy01 + x1);
        v[s][4] = __ldg(grid + zy10 + x0);
        v[s][5] = __ldg(grid + zy10 + x1);
        v[s][6] = __ldg(grid + zy11 + x0);
        v[s][7] = __ldg(grid + zy11 + x1);
      } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) v[s][c] = make_float2(0.f, 0.f);
      }
    } else {
      const AxisNodes ax = axis_nodes(ox[s], n, wrap_negative);
      const AxisNodes ay = axis_nodes(oy[s], n, wrap_negative);
      const AxisNodes az = axis_nodes(oz[s], n, wrap_negative);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int dz = c >> 2, dy = (c >> 1) & 1, dx = c & 1;
        const int iz = dz ? az.i1 : az.i0, iy = dy ? ay.i1 : ay.i0, ix = dx ? ax.i1 : ax.i0;
        const bool ok = active[s] && (dz ? az.v1 : az.v0) && (dy ? ay.v1 : ay.v0) && (dx ? ax.v1 : ax.v0);
        v[s][c] = ok ? __ldg(&grid[L.az(iz) + L.ay(iy) + L.ax(ix)]) : fill;
      }
    }
  }
#pragma unroll
  for (int s = 0; s < S; ++s) {
    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int dz = c >> 2, dy = (c >> 1) & 1, dx = c & 1;
      const float wt = (w[s][4 + dz] * w[s][2 + dy]) * w[s][dx];
      acc.x = fmaf(wt, v[s][c].x, acc.x);
      acc.y = fmaf(wt, v[s][c].y, acc.y);
    }
    out[s] = acc;
  }
}

// x-pair layout: the bricked (Morton-in-8^3-block) order of BrickLayout with
// 16-byte entries holding (g(x, y, z), g(x + 1, y, z)) (the second half is 0
// at x = N - 1).  An interior trilinear sample reads its 8 corners with 4
// vector loads.  The grid pointer is float4; entry e's first half is g at
// e's own coordinates, so single-corner reads use the float2 view at 2 e.
struct PairLayout : BrickLayout {
  __host__ __device__ explicit PairLayout(int n) : BrickLayout(n) {}
};

template <int S>
__device__ __forceinline__ void sample_trilinear_batch_pairs(const float4* __restrict__ grid, int n,
                                                             const PairLayout& L, const float* ox, const float* oy,
                                                             const float* oz, const bool* active, bool wrap_negative,
                                                             float2 fill, float2* out) {
  float2 v[S][8];
  float w[S][6];
  const int h = n / 2;
  const float2* g2 = reinterpret_cast<const float2*>(grid);
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const float fx = floorf(ox[s]), fy = floorf(oy[s]), fz = floorf(oz[s]);
    w[s][1] = ox[s] - fx; w[s][0] = 1.0f - w[s][1];
    w[s][3] = oy[s] - fy; w[s][2] = 1.0f - w[s][3];
    w[s][5] = oz[s] - fz; w[s][4] = 1.0f - w[s][5];
    const int ix0 = (int)fx + h, iy0 = (int)fy + h, iz0 = (int)fz + h;
    const bool interior = (unsigned)ix0 < (unsigned)(n - 1) && (unsigned)iy0 < (unsigned)(n - 1) &&
                          (unsigned)iz0 < (unsigned)(n - 1);
    if (interior) {
      if (active[s]) {
        const int x0 = L.ax(ix0);
        const int y0 = L.ay(iy0), y1 = L.ay(iy0 + 1);
        const int z0 = L.az(iz0), z1 = L.az(iz0 + 1);
        const float4 a = __ldg(grid + z0 + y0 + x0);
        const float4 b = __ldg(grid + z0 + y1 + x0);
        const float4 c = __ldg(grid + z1 + y0 + x0);
        const float4 d = __ldg(grid + z1 + y1 + x0);
        v[s][0] = make_float2(a.x, a.y); v[s][1] = make_float2(a.z, a.w);
        v[s][2] = make_float2(b.x, b.y); v[s][3] = make_float2(b.z, b.w);
        v[s][4] = make_float2(c.x, c.y); v[s][5] = make_float2(c.z, c.w);
        v[s][6] = make_float2(d.x, d.y); v[s][7] = make_float2(d.z, d.w);
      } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) v[s][c] = make_float2(0.f, 0.f);
      }
    } else {
      const AxisNodes ax = axis_nodes(ox[s], n, wrap_negative);
      const AxisNodes ay = axis_nodes(oy[s], n, wrap_negative);
      const AxisNodes az = axis_nodes(oz[s], n, wrap_negative);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int dz = c >> 2, dy = (c >> 1) & 1, dx = c & 1;
        const int iz = dz ? az.i1 : az.i0, iy = dy ? ay.i1 : ay.i0, ix = dx ? ax.i1 : ax.i0;
        const bool ok = active[s] && (dz ? az.v1 : az.v0) && (dy ? ay.v1 : ay.v0) && (dx ? ax.v1 : ax.v0);
        v[s][c] = ok ? __ldg(&g2[2 * (L.az(iz) + L.ay(iy) + L.ax(ix))]) : fill;
      }
    }
  }
#pragma unroll
  for (int s = 0; s < S; ++s) {
    float2 acc = make_float2(0.f, 0.f);
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int dz = c >> 2, dy = (c >> 1) & 1, dx = c & 1;
      const float wt = (w[s][4 + dz] * w[s][2 + dy]) * w[s][dx];
      acc.x = fmaf(wt, v[s][c].x, acc.x);
      acc.y = fmaf(wt, v[s][c].y, acc.y);
    }
    out[s] = acc;
  }
}

// ---------------------------------------------------------------------------
// Cubic-spline sampling from a FourierVoxelSplineVolume's coefficient array
// (side m = N + 2), cryojax/ndimage/_map_coordinates.py:126-142, 217-250:
// for the logical coordinate c = off + N/2 the taps are the coefficient
// indices i = floor(c) + t, t = 0..3, each weighted by basis(c - i + 1) with
// basis(u) = 4 - 6u^2 + 3|u|^3 (|u| <= 1), (2 - |u|)^3 (1 <= |u| <= 2).
// With f = c - floor(c) the four weights are (1-f)^3, 4 - 6f^2 + 3f^3,
// 4 - 6(1-f)^2 + 3(1-f)^3 and f^3.  Each tap is read with the same
// `.at[idx].get(mode="fill")` rule as the trilinear corners, on side m.
// The layouts address the coefficient array on side N + 2.
// ---------------------------------------------------------------------------
struct SplineLinearLayout : LinearLayout {
  __host__ __device__ explicit SplineLinearLayout(int n) : LinearLayout(n + 2) {}
};
struct SplineBrickLayout : BrickLayout {
  __host__ __device__ explicit SplineBrickLayout(int n) : BrickLayout(n + 2) {}
};
// x-pair entries (c(x), c(x + 1)) in the bricked order on side N + 2: a row
// of 4 x-taps is two 16-byte loads (entries x0 and x0 + 2).
struct SplinePairLayout : BrickLayout {
  __host__ __device__ explicit SplinePairLayout(int n) : BrickLayout(n + 2) {}
};
template <typename Layout>
struct is_spline_layout
    : std::integral_constant<bool, std::is_same<Layout, SplineLinearLayout>::value ||
                                       std::is_same<Layout, SplineBrickLayout>::value ||
                                       std::is_same<Layout, SplinePairLayout>::value> {};

struct SplineAxis {
  int i[4];    // wrapped tap indices (0 when invalid)
  bool v[4];   // tap inside [0, m)
  float w[4];  // basis weights
};

__device__ __forceinline__ void spline_weights(float f, float* w) {
  const float g = 1.0f - f;
  w[0] = g * g * g;
  w[1] = fmaf(fmaf(3.0f, f, -6.0f), f * f, 4.0f);
  w[2] = fmaf(fmaf(3.0f, g, -6.0f), g * g, 4.0f);
  w[3] = f * f * f;
}

__device__ __forceinline__ SplineAxis spline_axis(float off, int n, bool wrap_negative) {
  SplineAxis a;
  const float fl = floorf(off);
  spline_weights(off - fl, a.w);
  const int m = n + 2;
  const int i0 = (int)fl + n / 2;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    int i = i0 + t;
    if (wrap_negative && i < 0) i += m;
    a.v[t] = (unsigned)i < (unsigned)m;
    a.i[t] = a.v[t] ? i : 0;
  }
  return a;
}

// S cubic-spline samples.  A sample whose 64 taps all lie inside the
// coefficient array (every sample away from the faces) reads them at the
// layout's offsets with no per-tap checks; samples near the faces take the
// general rule.  The taps are summed as x rows (4 taps), each row weighted
// by its (z, y) weight.
template <int S, typename Layout>
__device__ __forceinline__ void sample_spline_batch(const float2* __restrict__ coef, int n, const Layout& L,
                                                    const float* ox, const float* oy, const float* oz,
                                                    const bool* active, bool wrap_negative, float2 fill,
                                                    float2* out) {
  const int h = n / 2;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    float2 acc = make_float2(0.f, 0.f);
    if (active[s]) {
      const float fx = floorf(ox[s]), fy = floorf(oy[s]), fz = floorf(oz[s]);
      float wx[4], wy[4], wz[4];
      spline_weights(ox[s] - fx, wx);
      spline_weights(oy[s] - fy, wy);
      spline_weights(oz[s] - fz, wz);
      const int ix0 = (int)fx + h, iy0 = (int)fy + h, iz0 = (int)fz + h;
      // taps i0..i0+3 inside [0, N + 2) on every axis
      const bool interior = (unsigned)ix0 < (unsigned)(n - 1) && (unsigned)iy0 < (unsigned)(n - 1) &&
                            (unsigned)iz0 < (unsigned)(n - 1);
      if (interior) {
        int xo[4], yo[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          xo[t] = L.ax(ix0 + t);
          yo[t] = L.ay(iy0 + t);
        }
#pragma unroll
        for (int dz = 0; dz < 4; ++dz) {
          const int zo = L.az(iz0 + dz);
#pragma unroll
          for (int dy = 0; dy < 4; ++dy) {
            float2 c0, c1, c2, c3;
            if constexpr (std::is_same<Layout, SplinePairLayout>::value) {
              const float4* row = reinterpret_cast<const float4*>(coef) + zo + yo[dy];
              const float4 p = __ldg(row + xo[0]), q = __ldg(row + xo[2]);
              c0 = make_float2(p.x, p.y); c1 = make_float2(p.z, p.w);
              c2 = make_float2(q.x, q.y); c3 = make_float2(q.z, q.w);
            } else {
              const float2* row = coef + zo + yo[dy];
              c0 = __ldg(row + xo[0]); c1 = __ldg(row + xo[1]);
              c2 = __ldg(row + xo[2]); c3 = __ldg(row + xo[3]);
            }
            float2 r;
            r.x = fmaf(wx[3], c3.x, fmaf(wx[2], c2.x, fmaf(wx[1], c1.x, wx[0] * c0.x)));
            r.y = fmaf(wx[3], c3.y, fmaf(wx[2], c2.y, fmaf(wx[1], c1.y, wx[0] * c0.y)));
            const float wzy = wz[dz] * wy[dy];
            acc.x = fmaf(wzy, r.x, acc.x);
            acc.y = fmaf(wzy, r.y, acc.y);
          }
        }
      } else {
        const SplineAxis ax = spline_axis(ox[s], n, wrap_negative);
        const SplineAxis ay = spline_axis(oy[s], n, wrap_negative);
        const SplineAxis az = spline_axis(oz[s], n, wrap_negative);
#pragma unroll
        for (int dz = 0; dz < 4; ++dz) {
#pragma unroll
          for (int dy = 0; dy < 4; ++dy) {
            const bool vzy = az.v[dz] && ay.v[dy];
            const int zy = L.az(az.i[dz]) + L.ay(ay.i[dy]);
            float2 r = make_float2(0.f, 0.f);
#pragma unroll
            for (int dx = 0; dx < 4; ++dx) {
              // a pair entry's first half is the coefficient at the entry's own coordinates
              const int e = zy + L.ax(ax.i[dx]);
              const float2 c = (vzy && ax.v[dx])
                                   ? __ldg(coef + (std::is_same<Layout, SplinePairLayout>::value ? 2 * e : e))
                                   : fill;
              r.x = fmaf(ax.w[dx], c.x, r.x);
              r.y = fmaf(ax.w[dx], c.y, r.y);
            }
            const float wzy = az.w[dz] * ay.w[dy];
            acc.x = fmaf(wzy, r.x, acc.x);
            acc.y = fmaf(wzy, r.y, acc.y);
          }
        }
      }
    }
    out[s] = acc;
  }
}

// Samples from a grid in any of the layouts: trilinear from a voxel grid,
// cubic spline from a coefficient array.
template <int S, typename Layout>
__device__ __forceinline__ void gather_samples(const float2* __restrict__ grid, int n, const Layout& L,
                                               const float* ox, const float* oy, const float* oz,
                                               const bool* active, bool wrap_negative, float2 fill, float2* out) {
  if constexpr (is_spline_layout<Layout>::value)
    sample_spline_batch<S>(grid, n, L, ox, oy, oz, active, wrap_negative, fill, out);
  else if constexpr (std::is_same<Layout, PairLayout>::value)
    sample_trilinear_batch_pairs<S>(reinterpret_cast<const float4*>(grid), n, L, ox, oy, oz, active, wrap_negative,
                                    fill, out);
  else
    sample_trilinear_batch_fast<S>(grid, n, L, ox, oy, oz, active, wrap_negative, fill, out);
}

// Lane -> sample mapping inside a CTA's 16 x 16 patch of the plane (MAP):
//   0: each warp 2 columns x 16 rows, 1: 4 x 8, 2: 8 x 4.
template <int MAP>
__device__ __forceinline__ void gather_lane_offsets(int warp, int lane, int& du, int& dv) {
  if constexpr (MAP == 0) {
    du = 2 * warp + (lane >> 4);
    dv = lane & 15;
  } else if constexpr (MAP == 1) {
    du = 4 * (warp & 3) + (lane & 3);
    dv = 8 * (warp >> 2) + (lane >> 2);
  } else {
    du = 8 * (warp & 1) + (lane & 7);
    dv = 4 * (warp >> 1) + (lane >> 3);
  }
}

// ---------------------------------------------------------------------------
// Epilogue: scale, CTF, envelope, translation
// ---------------------------------------------------------------------------
struct ImageConsts {
  double inv_px;        // 1 / pixel_size
  double qy_step;       // 1 / (py * pixel_size): qy = fftfreq index * qy_step
  double qx_step;       // 1 / (px * pixel_size)
  double defocus;
  double half_astig;    // 0.5 * astigmatism
  double c_def;         // -0.5 * wavelength                (cycles per A^2 per A)
  double c_sph;         // 0.25 * Cs * wavelength^3
  double phase_cycles;  // phase_total / (2 pi)
  double tx, ty;
  float cos2a, sin2a;   // cos / sin of 2 * astigmatism_angle
  float scale;
  float env_amp, env_quarter_b;
  double ps_cycles;     // phase_shift / (2 pi)        (Ewald contrast)
  float w1, w2;         // ac, sqrt(1 - ac^2)          (Ewald contrast)
};

__device__ __forceinline__ ImageConsts load_image_consts(const cjx_image_params* __restrict__ p, float extra_scale,
                                                         int py, int px) {
  ImageConsts c;
  c.inv_px = 1.0 / p->pixel_size;
  c.qy_step = c.inv_px / (double)py;
  c.qx_step = c.inv_px / (double)px;
  c.defocus = p->defocus;
  c.half_astig = 0.5 * p->astigmatism;
  const double wl = p->wavelength;
  c.c_def = -0.5 * wl;
  c.c_sph = 0.25 * p->spherical_aberration * wl * wl * wl;
  c.phase_cycles = p->phase_total * 0.15915494309189533577;  // 1 / (2 pi)
  c.tx = p->shift_x;
  c.ty = p->shift_y;
  double s2, c2;
  sincos(2.0 * p->astigmatism_angle, &s2, &c2);
  c.cos2a = (float)c2;
  c.sin2a = (float)s2;
  c.scale = (float)(p->scale * (double)extra_scale);
  c.env_amp = (float)p->envelope_amplitude;
  c.env_quarter_b = (float)(0.25 * p->envelope_b_factor);
  c.ps_cycles = p->phase_shift * 0.15915494309189533577;
  const double ac = p->amplitude_contrast_ratio;
  c.w1 = (float)ac;
  c.w2 = (float)sqrt(1.0 - ac * ac);
  return c;
}

// The Ewald surface's third coordinate per squared pixel frequency index:
// N q_z = N (lambda / pixel_size) |q|^2 / 2 with q = (kx, ky) / N
// (cryojax/simulator/_volume_integrator/fourier_voxel_extract.py:489-516).
__device__ __forceinline__ float ewald_w(const cjx_image_params* __restrict__ p, int n) {
  return (float)(p->wavelength / (2.0 * (double)n * p->pixel_size));
}

// Value at rfft-grid entry (i, j) of a (py, px) image.
//   qx = rfftfreq(px)[j] / pixel_size, qy = fftfreq(py)[i] / pixel_size
//   (cryojax/simulator/_image_config.py:194-201);
//   CTF = sin(chi - phase_total), chi = 2 pi (-1/2 df(theta) lambda k^2
//   + 1/4 Cs lambda^3 k^4), df(theta) = df + astig/2 cos(2 (theta - alpha)),
//   theta = atan2(qx, qy)  (cryojax/simulator/_transfer_theory/
//   common_functions.py:9-40, transfer_function.py:27-82, 130-169).
//   cos(2 theta) = (qy^2 - qx^2) / k^2 and sin(2 theta) = 2 qx qy / k^2, so
//   no per-pixel atan2 is needed; at k = 0 theta = atan2(0, 0) = 0.
//   chi is accumulated in cycles in double and reduced to [-1/2, 1/2]
//   before the single-precision sinpi, so large defocus keeps full accuracy.
//   Translation: zero the even-size Nyquist self-conjugates, then multiply
//   by exp(-2 pi i (qx tx + qy ty))  (cryojax/simulator/_pose.py:68-114).
// chi / (2 pi) without the constant phase: -1/2 df(theta) lambda k^2 + 1/4 Cs lambda^3 k^4.
__device__ __forceinline__ double aberration_cycles(double qx, double qy, double k2, const ImageConsts& c) {
  // angle terms only scale the astigmatism (|astig| / 2 <~ 1e3 A), so
  // single precision is ample for them
  float c2t = 1.0f, s2t = 0.0f;
  if (k2 > 0.0) {
    const float qxf = (float)qx, qyf = (float)qy;
    const float inv = 1.0f / (float)k2;
    c2t = (qyf * qyf - qxf * qxf) * inv;
    s2t = 2.0f * qxf * qyf * inv;
  }
  const double df = c.defocus + c.half_astig * (double)(c2t * c.cos2a + s2t * c.sin2a);
  return (c.c_def * df + c.c_sph * k2) * k2;
}

// Envelope and translation of an rfft-grid value (shared by both epilogues).
__device__ __forceinline__ float2 envelope_translate(float2 v, int i, int j, int py, int px, double qx, double qy,
                                                    double k2, uint32_t flags, const ImageConsts& c) {
  if (flags & CJX_APPLY_ENVELOPE) {
    const float e = c.env_amp * expf(-c.env_quarter_b * (float)k2);
    v.x *= e;
    v.y *= e;
  }
  if (flags & CJX_APPLY_TRANSLATION) {
    const bool ey = (py % 2 == 0), ex = (px % 2 == 0);
    const bool self_conj = (ey && i == py / 2 && j == 0) || (ex && i == 0 && j == px / 2) ||
                           (ey && ex && i == py / 2 && j == px / 2);
    if (self_conj) {
      v = make_float2(0.f, 0.f);
    } else {
      const double ph = qx * c.tx + qy * c.ty;
      const float r = (float)(ph - rint(ph));
      float s, co;
      sincospif(2.0f * r, &s, &co);
      v = make_float2(fmaf(v.x, co, v.y * s), fmaf(v.y, co, -v.x * s));
    }
  }
  return v;
}

// exp(-2 pi i ph), ph reduced to [-1/2, 1/2] in double before the float sincospi.
__device__ __forceinline__ float2 phase_factor(double ph) {
  const float r = (float)(ph - rint(ph));
  float s, co;
  sincospif(2.0f * r, &s, &co);
  return make_float2(co, -s);
}

// The epilogue of one output column j (the column pass's unit of work),
// with the per-column terms hoisted:
//   * the translation factor is separable, exp(-2 pi i qx tx) exp(-2 pi i
//     qy ty): the column factor is computed once, the row factors come from
//     a per-CTA table (row_phase[i]);
//   * chi / (2 pi) needs no angle: cos(2 theta) k^2 = qy^2 - qx^2 and
//     sin(2 theta) k^2 = 2 qx qy, so
//     chi / (2 pi) = (c_def df + c_sph k^2) k^2 + c_def (astig / 2)
//                    ((qy^2 - qx^2) cos 2 alpha + 2 qx qy sin 2 alpha),
//     the large first term in double, the astigmatic term in float.
// Same values as apply_epilogue up to rounding.
struct ColumnEpilogue {
  double qx, qx2, c_dd;
  float qxf, c_astig;
  float2 col_phase;
};

__device__ __forceinline__ ColumnEpilogue column_epilogue(int j, uint32_t flags, const ImageConsts& c) {
  ColumnEpilogue e;
  e.qx = (double)j * c.qx_step;
  e.qx2 = e.qx * e.qx;
  e.qxf = (float)e.qx;
  e.c_dd = c.c_def * c.defocus;
  e.c_astig = (float)(c.c_def * c.half_astig);
  e.col_phase = (flags & CJX_APPLY_TRANSLATION) ? phase_factor(e.qx * c.tx) : make_float2(1.f, 0.f);
  return e;
}

// chi / (2 pi) - const_cycles at (qy, k2) of column e.
__device__ __forceinline__ double column_aberration_cycles(double qy, double k2, const ImageConsts& c,
                                                           const ColumnEpilogue& e, double const_cycles) {
  const float qyf = (float)qy;
  const float astig = e.c_astig * fmaf(fmaf(qyf, qyf, -e.qxf * e.qxf), c.cos2a, 2.0f * e.qxf * qyf * c.sin2a);
  return fma(fma(c.c_sph, k2, e.c_dd), k2, (double)astig - const_cycles);
}

// Envelope and translation in column form (envelope_translate's counterpart).
__device__ __forceinline__ float2 column_envelope_translate(float2 v, int i, int j, int py, int px, double k2,
                                                            uint32_t flags, const ImageConsts& c,
                                                            const ColumnEpilogue& e,
                                                            const float2* __restrict__ row_phase) {
  if (flags & CJX_APPLY_ENVELOPE) {
    const float en = c.env_amp * expf(-c.env_quarter_b * (float)k2);
    v.x *= en;
    v.y *= en;
  }
  if (flags & CJX_APPLY_TRANSLATION) {
    const bool ey = (py % 2 == 0), ex = (px % 2 == 0);
    const bool self_conj = (ey && i == py / 2 && j == 0) || (ex && i == 0 && j == px / 2) ||
                           (ey && ex && i == py / 2 && j == px / 2);
    if (self_conj) return make_float2(0.f, 0.f);
    v = cmul(v, cmul(e.col_phase, row_phase[i]));
  }
  return v;
}

__device__ __forceinline__ float2 apply_column_epilogue(float2 v, int i, int j, int py, int px, uint32_t flags,
                                                        const ImageConsts& c, const ColumnEpilogue& e,
                                                        const float2* __restrict__ row_phase) {
  v.x *= c.scale;
  v.y *= c.scale;
  double k2 = 0.0;
  if (flags & (CJX_APPLY_CTF | CJX_APPLY_ENVELOPE)) {
    const double qy = (double)fft_index(i, py) * c.qy_step;
    k2 = fma(qy, qy, e.qx2);
    if (flags & CJX_APPLY_CTF) {
      const double arg = column_aberration_cycles(qy, k2, c, e, c.phase_cycles);
      const float r = (float)(arg - rint(arg));
      const float ctf = sinpif(2.0f * r);
      v.x *= ctf;
      v.y *= ctf;
    }
  }
  return column_envelope_translate(v, i, j, py, px, k2, flags, c, e, row_phase);
}

__device__ __forceinline__ float2 apply_epilogue(float2 v, int i, int j, int py, int px, uint32_t flags,
                                                 const ImageConsts& c) {
  v.x *= c.scale;
  v.y *= c.scale;
  if (flags & (CJX_APPLY_CTF | CJX_APPLY_ENVELOPE | CJX_APPLY_TRANSLATION)) {
    const double qy = (double)fft_index(i, py) * c.qy_step;
    const double qx = (double)j * c.qx_step;
    const double k2 = qx * qx + qy * qy;
    if (flags & CJX_APPLY_CTF) {
      const double arg = aberration_cycles(qx, qy, k2, c) - c.phase_cycles;
      const float r = (float)(arg - rint(arg));
      const float ctf = sinpif(2.0f * r);
      v.x *= ctf;
      v.y *= ctf;
    }
    v = envelope_translate(v, i, j, py, px, qx, qy, k2, flags, c);
  }
  return v;
}

// Ewald-sphere contrast at rfft-grid entry (i, j) of a (py, px) image from
// the full object spectrum's a = O[i, j] and b = O[-i, -j]
// (cryojax/simulator/_transfer_theory/transfer_theory.py:165-255):
//   K(pos, neg) = 1/2 [ (w2 (p+n)_r + w1 (p+n)_i) sin + (w2 (p+n)_i - w1 (p+n)_r) cos
//                   + i ((w2 (p-n)_i + w1 (n-p)_r) sin + (w2 (n-p)_r + w1 (n-p)_i) cos) ],
//   sin, cos of chi - deg2rad(phase_shift), w1 = ac, w2 = sqrt(1 - ac^2);
//   pos = a, neg = b, except the even-size Nyquist column (pos = conj(b)) and
//   the x = 0 column's even-size Nyquist row (conj(K(conj(a), a))).  Rows
//   y > Py/2 of the x = 0 column equal conj(K) of their mirror row, which is
//   K itself since K's imaginary part is odd in (pos, neg).
__device__ __forceinline__ float2 ewald_epilogue(float2 a, float2 b, int i, int j, int py, int px, uint32_t flags,
                                                 const ImageConsts& c) {
  a.x *= c.scale;
  a.y *= c.scale;
  b.x *= c.scale;
  b.y *= c.scale;
  const double qy = (double)fft_index(i, py) * c.qy_step;
  const double qx = (double)j * c.qx_step;
  const double k2 = qx * qx + qy * qy;
  const double arg = aberration_cycles(qx, qy, k2, c) - c.ps_cycles;
  const float r = (float)(arg - rint(arg));
  float s, co;
  sincospif(2.0f * r, &s, &co);
  float2 pos = a, neg = b;
  bool conj_out = false;
  if ((px % 2 == 0) && j == px / 2) {
    pos = make_float2(b.x, -b.y);
  } else if (j == 0 && (py % 2 == 0) && i == py / 2) {
    pos = make_float2(a.x, -a.y);
    neg = a;
    conj_out = true;
  }
  const float sr = pos.x + neg.x, si = pos.y + neg.y;
  const float dr = neg.x - pos.x, di = pos.y - neg.y;
  float2 v;
  v.x = 0.5f * ((c.w2 * sr + c.w1 * si) * s + (c.w2 * si - c.w1 * sr) * co);
  v.y = 0.5f * ((c.w2 * di + c.w1 * dr) * s + (c.w2 * dr - c.w1 * di) * co);
  if (conj_out) v.y = -v.y;
  return envelope_translate(v, i, j, py, px, qx, qy, k2, flags, c);
}

// ewald_epilogue in column form: the aberration phase without an angle or
// a division, the translation from the column factor and the per-CTA row
// table (same values up to rounding).
__device__ __forceinline__ float2 ewald_column_epilogue(float2 a, float2 b, int i, int j, int py, int px,
                                                        uint32_t flags, const ImageConsts& c,
                                                        const ColumnEpilogue& e,
                                                        const float2* __restrict__ row_phase) {
  a.x *= c.scale;
  a.y *= c.scale;
  b.x *= c.scale;
  b.y *= c.scale;
  const double qy = (double)fft_index(i, py) * c.qy_step;
  const double k2 = fma(qy, qy, e.qx2);
  const double arg = column_aberration_cycles(qy, k2, c, e, c.ps_cycles);
  const float r = (float)(arg - rint(arg));
  float s, co;
  sincospif(2.0f * r, &s, &co);
  float2 pos = a, neg = b;
  bool conj_out = false;
  if ((px % 2 == 0) && j == px / 2) {
    pos = make_float2(b.x, -b.y);
  } else if (j == 0 && (py % 2 == 0) && i == py / 2) {
    pos = make_float2(a.x, -a.y);
    neg = a;
    conj_out = true;
  }
  const float sr = pos.x + neg.x, si = pos.y + neg.y;
  const float dr = neg.x - pos.x, di = pos.y - neg.y;
  float2 v;
  v.x = 0.5f * ((c.w2 * sr + c.w1 * si) * s + (c.w2 * si - c.w1 * sr) * co);
  v.y = 0.5f * ((c.w2 * di + c.w1 * dr) * s + (c.w2 * dr - c.w1 * di) * co);
  if (conj_out) v.y = -v.y;
  return column_envelope_translate(v, i, j, py, px, k2, flags, c, e, row_phase);
}

// ---------------------------------------------------------------------------
// Per-call kernel choices (process defaults come from cjx_tuning_set)
// ---------------------------------------------------------------------------
struct Tuning {
  int ilp;          // samples per gather lane issued together (1, 2, 4)
  int tile;         // gather lane tile (0, 1, 2)
  int gather_mode;  // 1 = separate gather kernel, 0 = fused gather + column FFT
  int fft_mode;     // 1 = register FFTs where possible
  int scatter_vec;  // 1 = adjoint grid scatter merges aligned x-corner pairs into 16-byte atomics
  int spline_ilp;   // samples per lane in the cubic-spline gather (1, 2, 4)
  int multi_waves;  // 1 = mixed-size batches run in waves, one launch per pass for all groups
};
Tuning current_tuning();

// ---------------------------------------------------------------------------
// One wave of a mixed-size batch: a slice of every group's images, each pass
// of the resize path launched once for all of them (the CTAs of the groups
// follow one another in the launch: group i owns CTAs [cta0[pass], next
// group's cta0[pass]) of that pass).
// ---------------------------------------------------------------------------
constexpr int kMaxWaveGroups = 8;
struct WaveGroup {
  SliceGeom g;
  const float2* grid;
  const cjx_image_params* params;
  const int32_t* order;
  float2* t1;
  float2* t2;
  float2* out;
  int64_t k0;  // processing index of the group's first image in this wave
  int cnt;     // the group's images in this wave
  int cta0[3]; // first CTA of the group in the front, row and column passes
};
struct Wave {
  WaveGroup grp[kMaxWaveGroups];
  int n;
  int t512;       // 512-point column transforms of the front pass through the transpose FFT
  int rows_t512;  // the same for the row pass
};

// One group of a mixed-size batch, as the host hands it to launch_forward_waves.
struct WaveInput {
  SliceGeom g;
  const float2* grid;
  const cjx_image_params* params;
  const int32_t* order;
  float2* out;
  int64_t n;
};
bool wave_eligible(const SliceGeom& g, const Tuning& tn);
int64_t plan_waves(const WaveInput* in, int n_in, size_t workspace_bytes, int64_t* per_wave);
int launch_forward_waves(const WaveInput* in, int n_in, void* workspace, size_t workspace_bytes, cudaStream_t stream,
                         const Tuning& tn);

// The group that owns CTA `b` of pass `pass`.
__device__ __forceinline__ int wave_group(const Wave& w, int pass, int b) {
  int gi = 0;
  while (gi + 1 < w.n && b >= w.grp[gi + 1].cta0[pass]) ++gi;
  return gi;
}

// ---------------------------------------------------------------------------
// Host-side error plumbing
// ---------------------------------------------------------------------------
void set_last_error(const std::string& msg);
int fail(int code, const std::string& msg);
int check_cuda(cudaError_t e, const char* what);

// Per-device one-time set-up (function attributes belong to each device's
// context).  `init` runs the first time a thread reaches this with a given
// device current; its outcome is stored and returned to every later call on
// that device, so a failed set-up keeps failing instead of letting kernels
// that depend on it launch.  Device indices from kMaxDevices up are refused.
constexpr int kMaxDevices = 64;
struct PerDeviceOnce {
  std::once_flag flags[kMaxDevices];
  cudaError_t errs[kMaxDevices] = {};
  template <typename F>
  cudaError_t run(F&& init) {
    int dev = 0;
    if (cudaError_t e = cudaGetDevice(&dev)) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::call_once(flags[dev], [&] { errs[dev] = init(); });
    return errs[dev];
  }
};

}  // namespace cjx
