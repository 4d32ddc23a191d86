// Warp-level shared-memory FFTs for the resize stage of the Fourier-slice path.
//
// One warp transforms one length-n complex sequence held in shared memory,
// out of place between two buffers (Stockham autosort, natural order in and
// out).  Radices 8, 4, 2, 3, 5 have hand-written butterflies, radix 7 uses
// the twiddle table; a length with any other prime factor falls back to a
// direct O(n^2) DFT.  Twiddles exp(-2 pi i m / n) are computed per launch in
// double precision and stored as float2 in shared memory.  The register FFTs
// (n = 32 R) copy theirs from tables the compiler evaluates.
//
// Sign convention: DIR = -1 is the forward transform (numpy.fft.fft),
// DIR = +1 the unnormalised inverse (n * numpy.fft.ifft).
#pragma once

#include <cuda_runtime.h>

#include <utility>

namespace cjx {

constexpr int kMaxStages = 16;

struct FftPlan {
  int n;
  int nstages;  // 0 => direct DFT
  int radix[kMaxStages];
};

__host__ inline FftPlan make_fft_plan(int n) {
  FftPlan p{};
  p.n = n;
  int m = n, s = 0;
  const int radices[] = {8, 4, 2, 3, 5, 7};
  for (int r : radices) {
    while (m % r == 0 && s < kMaxStages) {
      p.radix[s++] = r;
      m /= r;
    }
  }
  p.nstages = (m == 1) ? s : 0;
  return p;
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by DIR * i
template <int DIR>
__device__ __forceinline__ float2 cmul_i(float2 a) {
  return DIR > 0 ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}
// twiddle exp(DIR * 2 pi i m / n) from the forward table
template <int DIR>
__device__ __forceinline__ float2 twiddle(const float2* tw, int m) {
  float2 w = tw[m];
  return DIR > 0 ? cconj(w) : w;
}

// Fill tw[m] = exp(-2 pi i m / n), m in [0, n), cooperatively by the block.
__device__ inline void build_twiddles(float2* tw, int n) {
  for (int m = threadIdx.x; m < n; m += blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)m / (double)n, &s, &c);
    tw[m] = make_float2((float)c, (float)s);
  }
}

template <int DIR>
__device__ __forceinline__ void dft2(float2* v) {
  float2 a = v[0];
  v[0] = cadd(a, v[1]);
  v[1] = csub(a, v[1]);
}

template <int DIR>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
  float2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
  float2 s13 = cadd(a1, a3), d13 = csub(a1, a3);
  float2 t = cmul_i<DIR>(d13);
  a0 = cadd(s02, s13);
  a2 = csub(s02, s13);
  a1 = cadd(d02, t);
  a3 = csub(d02, t);
}

template <int DIR>
__device__ __forceinline__ void dft3(float2* v) {
  const float c = 0.86602540378443864676f;  // sqrt(3)/2
  float2 s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
  float2 x0 = cadd(v[0], s);
  float2 m = make_float2(fmaf(-0.5f, s.x, v[0].x), fmaf(-0.5f, s.y, v[0].y));
  float2 t = cscale(cmul_i<DIR>(d), c);
  v[0] = x0;
  v[1] = cadd(m, t);
  v[2] = csub(m, t);
}

template <int DIR>
__device__ __forceinline__ void dft5(float2* v) {
  const float c1 = 0.30901699437494742410f;   // cos(2 pi / 5)
  const float c2 = -0.80901699437494742410f;  // cos(4 pi / 5)
  const float s1 = 0.95105651629515357212f;   // sin(2 pi / 5)
  const float s2 = 0.58778525229247312917f;   // sin(4 pi / 5)
  float2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
  float2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
  float2 a0 = v[0];
  float2 m1 = make_float2(a0.x + c1 * t1.x + c2 * t2.x, a0.y + c1 * t1.y + c2 * t2.y);
  float2 m2 = make_float2(a0.x + c2 * t1.x + c1 * t2.x, a0.y + c2 * t1.y + c1 * t2.y);
  float2 n1 = cmul_i<DIR>(make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
  float2 n2 = cmul_i<DIR>(make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
  v[0] = cadd(a0, cadd(t1, t2));
  v[1] = cadd(m1, n1);
  v[4] = csub(m1, n1);
  v[2] = cadd(m2, n2);
  v[3] = csub(m2, n2);
}

template <int DIR>
__device__ __forceinline__ void dft8(float2* v) {
  const float r = 0.70710678118654752440f;
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<DIR>(e0, e1, e2, e3);
  dft4<DIR>(o0, o1, o2, o3);
  // o_k *= exp(DIR 2 pi i k / 8)
  o1 = make_float2((o1.x - DIR * o1.y) * r, (o1.y + DIR * o1.x) * r);
  o2 = cmul_i<DIR>(o2);
  o3 = make_float2((-o3.x - DIR * o3.y) * r, (-o3.y + DIR * o3.x) * r);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

// Generic radix-R DFT with twiddles exp(DIR 2 pi i r q / R) = tw[(r q n / R) mod n].
template <int R, int DIR>
__device__ __forceinline__ void dft_generic(float2* v, const float2* tw, int n) {
  float2 out[R];
  const int step = n / R;
#pragma unroll
  for (int q = 0; q < R; ++q) {
    float2 acc = v[0];
#pragma unroll
    for (int r = 1; r < R; ++r) acc = cadd(acc, cmul(v[r], twiddle<DIR>(tw, ((r * q) % R) * step)));
    out[q] = acc;
  }
#pragma unroll
  for (int q = 0; q < R; ++q) v[q] = out[q];
}

template <int R, int DIR>
__device__ __forceinline__ void stockham_stage(const float2* __restrict__ in, float2* __restrict__ out,
                                               int n, int Ns, const float2* tw, int lane) {
  const int nb = n / R;
  const int tstep = n / (Ns * R);
  for (int j = lane; j < nb; j += 32) {
    const int k = j % Ns;
    float2 v[R];
#pragma unroll
    for (int q = 0; q < R; ++q) v[q] = in[j + q * nb];
    if (Ns > 1) {
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = cmul(v[q], twiddle<DIR>(tw, (q * k * tstep) % n));
    }
    if constexpr (R == 2) dft2<DIR>(v);
    else if constexpr (R == 3) dft3<DIR>(v);
    else if constexpr (R == 4) dft4<DIR>(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 5) dft5<DIR>(v);
    else if constexpr (R == 8) dft8<DIR>(v);
    else dft_generic<R, DIR>(v, tw, n);
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int q = 0; q < R; ++q) out[base + q * Ns] = v[q];
  }
}

// Transform buffer `a` (length plan.n) with scratch `b`; returns the buffer
// holding the result (a or b).  Executed by one full warp; ends with __syncwarp.
template <int DIR>
__device__ float2* warp_fft(float2* a, float2* b, const FftPlan& plan, const float2* tw, int lane) {
  const int n = plan.n;
  if (plan.nstages == 0) {
    for (int k = lane; k < n; k += 32) {
      float2 acc = make_float2(0.f, 0.f);
      int m = 0;
      for (int j = 0; j < n; ++j) {
        acc = cadd(acc, cmul(a[j], twiddle<DIR>(tw, m)));
        m += k;
        if (m >= n) m -= n;
      }
      b[k] = acc;
    }
    __syncwarp();
    return b;
  }
  int Ns = 1;
  for (int s = 0; s < plan.nstages; ++s) {
    const int R = plan.radix[s];
    switch (R) {
      case 8: stockham_stage<8, DIR>(a, b, n, Ns, tw, lane); break;
      case 4: stockham_stage<4, DIR>(a, b, n, Ns, tw, lane); break;
      case 2: stockham_stage<2, DIR>(a, b, n, Ns, tw, lane); break;
      case 3: stockham_stage<3, DIR>(a, b, n, Ns, tw, lane); break;
      case 5: stockham_stage<5, DIR>(a, b, n, Ns, tw, lane); break;
      default: stockham_stage<7, DIR>(a, b, n, Ns, tw, lane); break;
    }
    __syncwarp();
    float2* t = a;
    a = b;
    b = t;
    Ns *= R;
  }
  return a;
}


// ===========================================================================
// Register FFT for n = 32 R (R in {1, 2, 3, 4, 5, 6, 8, 10, 12, 16}).
//
// Four-step split n = 32 n1 + n2, k = k1 + R k2 (n2, k2 across the 32 lanes;
// n1, k1 in registers):
//   X[k1 + R k2] = sum_n2 W_32^(n2 k2) W_n^(n2 k1) sum_n1 x[32 n1 + n2] W_R^(n1 k1)
// 1. lane l holds x[32 n1 + brev5(l)] for n1 = 0..R-1 (the caller loads them);
// 2. R-point DFT over n1 in registers (compile-time twiddles);
// 3. multiply by W_n^(brev5(l) k1) from a [R][32] table (conflict-free);
// 4. 32-point radix-2 decimation-in-time across lanes with warp shuffles;
//    bit-reversed lane order in, natural order out.
// Afterwards lane l holds X[k1 + R l] for k1 = 0..R-1.
// Shared-memory buffers that receive these outputs use the padded layout
// pad16(e) = e + e / 16, which keeps the stride-R stores near conflict-free.
// ===========================================================================

__host__ __device__ constexpr int pad16(int e) { return e + (e >> 4); }

__device__ __forceinline__ int brev5(int l) { return (int)(__brev((unsigned)l) >> 27); }

// Shared-memory staging of a register FFT's outputs (lane l holds k = k1 + R l)
// for reading back in natural order.  pad16 is conflict-free for the
// power-of-two R; for R = 10 (the 320-point transforms) its stride-10 stores
// meet 5-way bank conflicts within a half-warp, and k + k/16 + 14 (k/32) keeps
// both the stores and the natural-order reads conflict-free (20 + 32
// wavefronts per 320 outputs against 100 + 32, counted on the CPU).
__host__ __device__ constexpr int stage_r(int R, int k) { return R == 10 ? k + (k >> 4) + (k >> 5) * 14 : pad16(k); }
__host__ __device__ constexpr int stage_r_size(int R) { return stage_r(R, 32 * R - 1) + 1; }
// The same for warp_fft512_t's outputs (k = fft512_t_out(q, lane)): its two
// lane halves land 256 apart and, with pad16 alone, on the same banks; the
// second half moves by 8 entries.  Size 551.
__host__ __device__ constexpr int stage512(int k) { return pad16(k) + 8 * ((k >> 8) & 1); }
constexpr int kStage512Size = 551;

// Compile-time cos / sin of 2 pi m / R via Taylor series after reduction to
// |x| <= pi/4 (enough terms for double precision); used only for the small
// constant twiddles of the in-register DFTs.
namespace ct {
constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double taylor_sin(double x) {
  double term = x, sum = x;
  for (int k = 1; k < 14; ++k) {
    term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double taylor_cos(double x) {
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 14; ++k) {
    term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
    sum += term;
  }
  return sum;
}
// angle = 2 pi m / R reduced by octant symmetry
constexpr double cos2pi(int m, int R) {
  m = ((m % R) + R) % R;
  const double x = 2.0 * kPi * m / R;  // [0, 2 pi)
  if (x <= kPi / 4) return taylor_cos(x);
  if (x <= 3 * kPi / 4) return -taylor_sin(x - kPi / 2);
  if (x <= 5 * kPi / 4) return -taylor_cos(x - kPi);
  if (x <= 7 * kPi / 4) return taylor_sin(x - 3 * kPi / 2);
  return taylor_cos(x - 2 * kPi);
}
constexpr double sin2pi(int m, int R) { return cos2pi(m * 4 - R, 4 * R); }

// Register-FFT twiddle tables, evaluated by the compiler: for each n = 32 R
// with R in the register-FFT list, entries k1 * 32 + l = exp(-2 pi i brev5(l)
// k1 / n) (the layout build_reg_twiddles fills), back to back in the order
// of that list; then w32[m] = exp(-2 pi i m / 32).
__host__ __device__ constexpr int reg_table_offset(int R) {
  switch (R) {
    case 1: return 0;
    case 2: return 32;
    case 3: return 96;
    case 4: return 192;
    case 5: return 320;
    case 6: return 480;
    case 8: return 672;
    case 10: return 928;
    case 12: return 1248;
    case 16: return 1632;
    default: return -1;
  }
}
constexpr int kRegTableSize = 2144;  // 32 * (1 + 2 + 3 + 4 + 5 + 6 + 8 + 10 + 12 + 16)
constexpr int brev5c(int l) {
  int r = 0;
  for (int b = 0; b < 5; ++b) r |= ((l >> b) & 1) << (4 - b);
  return r;
}
struct TwiddleTables {
  float2 reg[kRegTableSize];
  float2 w32[32];
};
constexpr TwiddleTables make_twiddle_tables() {
  TwiddleTables t{};
  const int radices[10] = {1, 2, 3, 4, 5, 6, 8, 10, 12, 16};
  for (int q = 0; q < 10; ++q) {
    const int R = radices[q], n = 32 * R, o = reg_table_offset(R);
    for (int k1 = 0; k1 < R; ++k1)
      for (int l = 0; l < 32; ++l) {
        const int a = brev5c(l) * k1;
        t.reg[o + k1 * 32 + l] = float2{(float)cos2pi(a, n), (float)-sin2pi(a, n)};
      }
  }
  for (int m = 0; m < 32; ++m) t.w32[m] = float2{(float)cos2pi(m, 32), (float)-sin2pi(m, 32)};
  return t;
}
}  // namespace ct

// In global memory (L2-resident after the first CTAs): every CTA copies its
// table into shared memory instead of evaluating n double-precision sincospi.
// Not declared const, so that it stays an ordinary global array read through
// the L1 (lanes read different entries).
static __device__ ct::TwiddleTables kTwiddleTables = ct::make_twiddle_tables();

// exp(DIR 2 pi i m / R) as a compile-time constant
template <int DIR, int M, int R>
__device__ __forceinline__ float2 ctw() {
  constexpr float c = (float)ct::cos2pi(M, R);
  constexpr float s = (float)ct::sin2pi(M, R);
  return make_float2(c, DIR > 0 ? s : -s);
}

template <int DIR, int M, int R>
__device__ __forceinline__ float2 ctw_mul(float2 v) {
  if constexpr ((M % R) == 0) {
    return v;
  } else {
    return cmul(v, ctw<DIR, M, R>());
  }
}

template <int R, int DIR>
struct RegDft;

template <int DIR>
struct RegDft<1, DIR> {
  __device__ __forceinline__ static void run(float2*) {}
};
template <int DIR>
struct RegDft<2, DIR> {
  __device__ __forceinline__ static void run(float2* v) { dft2<DIR>(v); }
};
template <int DIR>
struct RegDft<3, DIR> {
  __device__ __forceinline__ static void run(float2* v) { dft3<DIR>(v); }
};
template <int DIR>
struct RegDft<4, DIR> {
  __device__ __forceinline__ static void run(float2* v) { dft4<DIR>(v[0], v[1], v[2], v[3]); }
};
template <int DIR>
struct RegDft<5, DIR> {
  __device__ __forceinline__ static void run(float2* v) { dft5<DIR>(v); }
};
template <int DIR>
struct RegDft<8, DIR> {
  __device__ __forceinline__ static void run(float2* v) { dft8<DIR>(v); }
};

// R = A * B: X[kA + A kB] = sum_b W_B^(b kB) W_R^(b kA) sum_a v[B a + b] W_A^(a kA)
template <int A, int B, int DIR>
struct RegDftAB {
  template <int b, int kA>
  __device__ __forceinline__ static void twiddle_one(float2 (&u)[B][A]) {
    u[b][kA] = ctw_mul<DIR, b * kA, A * B>(u[b][kA]);
  }
  template <int b, int... kA>
  __device__ __forceinline__ static void twiddle_row(float2 (&u)[B][A], std::integer_sequence<int, kA...>) {
    (twiddle_one<b, kA>(u), ...);
  }
  template <int... b>
  __device__ __forceinline__ static void twiddle_all(float2 (&u)[B][A], std::integer_sequence<int, b...>) {
    (twiddle_row<b>(u, std::make_integer_sequence<int, A>{}), ...);
  }
  __device__ __forceinline__ static void run(float2* v) {
    float2 u[B][A];
#pragma unroll
    for (int b = 0; b < B; ++b) {
#pragma unroll
      for (int a = 0; a < A; ++a) u[b][a] = v[B * a + b];
      RegDft<A, DIR>::run(u[b]);
    }
    twiddle_all(u, std::make_integer_sequence<int, B>{});
#pragma unroll
    for (int kA = 0; kA < A; ++kA) {
      float2 w[B];
#pragma unroll
      for (int b = 0; b < B; ++b) w[b] = u[b][kA];
      RegDft<B, DIR>::run(w);
#pragma unroll
      for (int kB = 0; kB < B; ++kB) v[kA + A * kB] = w[kB];
    }
  }
};

template <int DIR>
struct RegDft<6, DIR> : RegDftAB<2, 3, DIR> {};
template <int DIR>
struct RegDft<10, DIR> : RegDftAB<2, 5, DIR> {};
template <int DIR>
struct RegDft<12, DIR> : RegDftAB<4, 3, DIR> {};
template <int DIR>
struct RegDft<16, DIR> : RegDftAB<4, 4, DIR> {};

// Per-lane twiddles of the 5 cross-lane DIT stages (forward sign):
// stage s (span h = 2^s) uses exp(-2 pi i (l mod h) / (2h)) =
// W32[(l mod h) * 16 / h].  Only upper lanes (bit h set) use them.
struct LaneTwiddles {
  float2 w[5];
};

// w32[m] = exp(-2 pi i m / 32), m in [0, 32) (block-cooperative).
__device__ inline void build_w32(float2* w32) {
  if (threadIdx.x < 32) w32[threadIdx.x] = __ldg(&kTwiddleTables.w32[threadIdx.x]);
}

__device__ __forceinline__ LaneTwiddles make_lane_twiddles(const float2* w32, int lane) {
  LaneTwiddles t;
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 1 << s;
    t.w[s] = (lane & h) ? w32[(lane & (h - 1)) * (16 >> s)] : make_float2(1.f, 0.f);
  }
  return t;
}

// Fill tab[k1 * 32 + l] = exp(-2 pi i brev5(l) k1 / n), k1 in [0, R) (block-cooperative).
__device__ inline void build_reg_twiddles(float2* tab, int n) {
  const int R = n / 32;
  const int o = (n % 32 == 0) ? ct::reg_table_offset(R) : -1;
  if (o >= 0) {
    for (int e = threadIdx.x; e < n; e += blockDim.x) tab[e] = __ldg(&kTwiddleTables.reg[o + e]);
    return;
  }
  for (int e = threadIdx.x; e < R * 32; e += blockDim.x) {
    const int k1 = e >> 5, l = e & 31;
    double s, c;
    sincospi(-2.0 * (double)(brev5(l) * k1) / (double)n, &s, &c);
    tab[e] = make_float2((float)c, (float)s);
  }
}

// Steps 2-4 on the lane's R values (step 1 input already loaded).
// Cross-lane DIT butterfly: the upper lane pre-multiplies its value by the
// stage twiddle (lower lanes hold w = 1), the pair exchanges values, then
// lower = own + partner and upper = partner - own.
template <int R, int DIR>
__device__ __forceinline__ void warp_fft_reg(float2 (&x)[R], const float2* __restrict__ tab, const LaneTwiddles& lt,
                                             int lane) {
  RegDft<R, DIR>::run(x);
#pragma unroll
  for (int k1 = 1; k1 < R; ++k1) x[k1] = cmul(x[k1], twiddle<DIR>(tab, k1 * 32 + lane));
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 1 << s;
    const float sg = (lane & h) ? -1.f : 1.f;
    const float2 w = DIR > 0 ? cconj(lt.w[s]) : lt.w[s];
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) {
      float2 v = (s == 0) ? x[k1] : cmul(x[k1], w);
      float2 p;
      p.x = __shfl_xor_sync(0xffffffffu, v.x, h);
      p.y = __shfl_xor_sync(0xffffffffu, v.y, h);
      x[k1] = make_float2(fmaf(sg, v.x, p.x), fmaf(sg, v.y, p.y));
    }
  }
}

// Sizes the register FFT handles: n = 32 R with R in the list above.
__host__ __device__ inline int reg_fft_radix(int n) {
  if (n % 32 != 0) return 0;
  const int R = n / 32;
  switch (R) {
    case 1: case 2: case 3: case 4: case 5: case 6: case 8: case 10: case 12: case 16:
      return R;
    default:
      return 0;
  }
}

// 512-point warp FFT as 16 x 32 with one shared-memory transpose:
// x[n] = x[l + 32 n1] (l = lane), X[k] = X[k1 + 16 k2].
//   1. a 16-point DFT over n1 in registers, twiddle W_512^(l k1);
//   2. transpose through shared memory so that lane (k1, e) = (lane >> 1,
//      lane & 1) holds the 16 values z[2m + e] of column k1;
//   3. a 16-point DFT over m in registers (the even / odd half of the
//      32-point DFT over l), then one cross-lane radix-2 step with W_32^q:
//      X[k1 + 16 q] = Y0 + W Y1 (e = 0), X[k1 + 16 (q + 16)] = Y0 - W Y1 (e = 1).
// About 40 % fewer instructions than the five-shuffle-stage network of
// warp_fft_reg<16> (32 shuffles per lane instead of 160).
// Input: x[n1] = data[32 n1 + lane] (natural lane order, unlike
// warp_fft_reg).  Output: x[q] = X[fft512_t_out(q, lane)].  tab is the
// build_reg_twiddles(n = 512) table, w32 the build_w32 table, scr a
// per-warp shared buffer of >= 16 * 34 values (overwritten).
__device__ __forceinline__ int fft512_t_out(int q, int lane) { return (lane >> 1) + 16 * (q + 16 * (lane & 1)); }

template <int DIR>
__device__ __forceinline__ void warp_fft512_t(float2 (&x)[16], const float2* __restrict__ tab,
                                              const float2* __restrict__ w32, float2* __restrict__ scr, int lane) {
  constexpr int kStride = 34;  // row stride: conflict-free 8-byte reads within each half-warp
  RegDft<16, DIR>::run(x);
  const int bl = brev5(lane);
#pragma unroll
  for (int k1 = 1; k1 < 16; ++k1) x[k1] = cmul(x[k1], twiddle<DIR>(tab, k1 * 32 + bl));  // W_512^(lane k1)
#pragma unroll
  for (int k1 = 0; k1 < 16; ++k1) scr[k1 * kStride + lane] = x[k1];
  __syncwarp();
  const int c = lane >> 1, e = lane & 1;
#pragma unroll
  for (int m = 0; m < 16; ++m) x[m] = scr[c * kStride + 2 * m + e];
  __syncwarp();
  RegDft<16, DIR>::run(x);
  const float sg = e ? -1.f : 1.f;
#pragma unroll
  for (int q = 0; q < 16; ++q) {
    float2 w = e ? w32[q] : make_float2(1.f, 0.f);
    if (DIR > 0) w = cconj(w);
    const float2 v = cmul(x[q], w);
    float2 p;
    p.x = __shfl_xor_sync(0xffffffffu, v.x, 1);
    p.y = __shfl_xor_sync(0xffffffffu, v.y, 1);
    x[q] = make_float2(fmaf(sg, v.x, p.x), fmaf(sg, v.y, p.y));
  }
}

}  // namespace cjx
