// Cubic-spline coefficients of a Fourier voxel grid (sm_100a).
//
// cryojax/ndimage/_map_coordinates.py:71-82, 179-215
// (compute_spline_coefficients): along each axis, last axis first, a line d
// of length L becomes L + 2 coefficients
//   c2 = d[0] / 6,  c_{L+1} = d[L-1] / 6,
//   tridiag(1, 4, 1) cs = d[1 : L-1] with d[1] -= c2 and d[L-2] -= c_{L+1},
//   c1 = 2 c2 - cs[0],  c_{L+2} = 2 c_{L+1} - cs[L-3],
// stored in the order (c1, c2, cs, c_{L+1}, c_{L+2}).  The reference solves
// the tridiagonal systems with lineax; here one thread runs the Thomas
// recurrence of one line in double precision.
//
// Three passes, one per axis: grid (N, N, N) -> out viewed as (N, N, M) ->
// workspace (N, M, M) -> out (M, M, M), M = N + 2.
#include "cjx_common.cuh"
#include "cjx_profile.cuh"

namespace cjx {

// Thomas factors of tridiag(1, 4, 1): f[0] = 1/4, f[k] = 1 / (4 - f[k-1]).
// They depend on k alone and reach their fixed point 2 - sqrt(3) (to double
// rounding) well before k = 32; f_inf holds f[31] iterated once more.
struct ThomasFactors {
  double f[32];
  double f_inf;
};

static ThomasFactors make_thomas_factors() {
  ThomasFactors t;
  double f = 0.25;
  t.f[0] = f;
  for (int k = 1; k < 32; ++k) {
    f = 1.0 / (4.0 - f);
    t.f[k] = f;
  }
  t.f_inf = 1.0 / (4.0 - f);
  return t;
}

__device__ __forceinline__ double2 ld_d2(const float2* p) {
  const float2 v = *p;
  return make_double2(v.x, v.y);
}
__device__ __forceinline__ void st_d2(float2* p, double2 v) { *p = make_float2((float)v.x, (float)v.y); }

// One axis pass.  The input is (A, L, B) in C order (the solved axis in the
// middle, B contiguous), the output (A, L + 2, B).  One thread per line
// (a, b); lines with consecutive b are adjacent in memory.
__global__ void __launch_bounds__(256)
    k_spline_axis(const float2* __restrict__ in, float2* __restrict__ out, int64_t A, int L, int64_t B,
                  const __grid_constant__ ThomasFactors tf) {
  const int64_t lines = A * B;
  const int m = L - 2;  // interior unknowns (>= 2)
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < lines; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = e / B, b = e - a * B;
    const float2* src = in + a * (int64_t)L * B + b;
    float2* dst = out + a * (int64_t)(L + 2) * B + b;
    const double2 d0 = ld_d2(src), dl = ld_d2(src + (int64_t)(L - 1) * B);
    const double2 c2 = make_double2(d0.x / 6.0, d0.y / 6.0);
    const double2 cn = make_double2(dl.x / 6.0, dl.y / 6.0);
    // forward elimination; d'_k is parked in the output slot of cs_k
    double2 dp = make_double2(0.0, 0.0);
    for (int k = 0; k < m; ++k) {
      double2 y = ld_d2(src + (int64_t)(k + 1) * B);
      if (k == 0) {
        y.x -= c2.x;
        y.y -= c2.y;
      }
      if (k == m - 1) {
        y.x -= cn.x;
        y.y -= cn.y;
      }
      const double f = k < 32 ? tf.f[k] : tf.f_inf;
      dp = make_double2((y.x - dp.x) * f, (y.y - dp.y) * f);
      st_d2(dst + (int64_t)(k + 2) * B, dp);
    }
    // back substitution: x_{m-1} = d'_{m-1}, x_k = d'_k - f_k x_{k+1}
    double2 x = dp;
    st_d2(dst + (int64_t)(m + 1) * B, x);
    const double2 x_last = x;
    for (int k = m - 2; k >= 0; --k) {
      const double2 d = ld_d2(dst + (int64_t)(k + 2) * B);
      const double f = k < 32 ? tf.f[k] : tf.f_inf;
      x = make_double2(d.x - f * x.x, d.y - f * x.y);
      st_d2(dst + (int64_t)(k + 2) * B, x);
    }
    st_d2(dst, make_double2(2.0 * c2.x - x.x, 2.0 * c2.y - x.y));
    st_d2(dst + B, c2);
    st_d2(dst + (int64_t)L * B, cn);
    st_d2(dst + (int64_t)(L + 1) * B, make_double2(2.0 * cn.x - x_last.x, 2.0 * cn.y - x_last.y));
  }
}

size_t spline_workspace_elements(int n) { return (size_t)n * (size_t)(n + 2) * (size_t)(n + 2); }

int launch_spline_coefficients(int n, const float2* grid, float2* coef, float2* work, cudaStream_t stream) {
  static const ThomasFactors tf = make_thomas_factors();
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t N = n, M = n + 2;
  auto blocks = [&](int64_t lines) { return (int)std::min<int64_t>((lines + 255) / 256, (int64_t)sms * 8); };
  prof_begin(stream);
  // x: grid (N*N, N, 1) -> coef viewed as (N*N, M, 1)
  k_spline_axis<<<blocks(N * N), 256, 0, stream>>>(grid, coef, N * N, n, 1, tf);
  // y: (N, N, M) -> work (N, M, M)
  k_spline_axis<<<blocks(N * M), 256, 0, stream>>>(coef, work, N, n, M, tf);
  // z: (1, N, M*M) -> coef (1, M, M*M)
  k_spline_axis<<<blocks(M * M), 256, 0, stream>>>(work, coef, 1, n, M * M, tf);
  prof_end("k_spline_axis", stream);
  return check_cuda(cudaGetLastError(), "k_spline_axis launch");
}

}  // namespace cjx
