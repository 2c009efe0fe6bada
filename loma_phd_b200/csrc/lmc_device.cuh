// lmc_device.cuh -- device building blocks of the lomacte substep kernels.
//
// y-direction operators: one warp per (kx,kz) mode.  The pencil of my
// points is split into chunks of n in {C-1, C} consecutive points, one chunk
// per active lane (LPM active lanes).  Banded matrix-vector products
// exchange a halo of H points with the neighbour lanes by shuffles.  Banded
// triangular solves run each chunk's recurrence in registers and join the
// chunks with a Kogge-Stone scan of the affine chunk maps
// state_out = M state_in + p.  For the mode-independent operators (the
// compact-derivative LUs) the scan matrices are precomputed on the host, so
// only the particular responses p travel between lanes; for the per-mode
// Poisson LUs the 2x2 maps are built in registers.
//
// x/z transforms: four-step FFTs N = N1*N2 with both factors done by one
// thread in registers, lines staged in shared memory with a skewed index
// (one pad slot per N1 entries) so that both the strided and the
// contiguous passes are free of bank conflicts.  The inverse ("nat2perm")
// leaves the samples in a permuted order and the direct transform
// ("perm2nat") is its transpose, so no permutation pass is needed.
#pragma once
#include <cuda_runtime.h>

namespace lmcd {

#define LMC_FULL 0xffffffffu

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
// (i k) * a
__device__ __forceinline__ double2 cik(double k, double2 a) { return make_double2(-k * a.y, k * a.x); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 czero() { return make_double2(0.0, 0.0); }

// The same operations on single-precision complex values (the transform
// work buffers of the mixed-precision form).
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cscale(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
__device__ __forceinline__ float2 cik(float k, float2 a) { return make_float2(-k * a.y, k * a.x); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// real type and constructors of a complex type
template <typename CT>
struct CReal;
template <>
struct CReal<double2> { using R = double; };
template <>
struct CReal<float2> { using R = float; };
template <typename CT>
__device__ __forceinline__ CT cmk(typename CReal<CT>::R a, typename CReal<CT>::R b) {
  CT c;
  c.x = a;
  c.y = b;
  return c;
}
template <typename CT>
__device__ __forceinline__ CT cz() { return cmk<CT>(0, 0); }
// FP64 value of a stored work-buffer element and back
__device__ __forceinline__ double2 to_d2(double2 a) { return a; }
__device__ __forceinline__ double2 to_d2(float2 a) { return make_double2(a.x, a.y); }
template <typename CT>
__device__ __forceinline__ CT from_d2(double2 a) { return cmk<CT>((typename CReal<CT>::R)a.x, (typename CReal<CT>::R)a.y); }

__device__ __forceinline__ double2 shfl_up2(double2 v, int d) {
  return make_double2(__shfl_up_sync(LMC_FULL, v.x, d), __shfl_up_sync(LMC_FULL, v.y, d));
}
__device__ __forceinline__ double2 shfl_down2(double2 v, int d) {
  return make_double2(__shfl_down_sync(LMC_FULL, v.x, d), __shfl_down_sync(LMC_FULL, v.y, d));
}

// ---------------------------------------------------------------------
// Chunk geometry of one lane
// ---------------------------------------------------------------------
struct Lane {
  int lane, s, n, lpm;
  bool full;  // n == C
};

template <int C>
__device__ __forceinline__ Lane make_lane(int lpm, int base, int extra) {
  Lane L;
  L.lane = threadIdx.x & 31;
  L.lpm = lpm;
  if (L.lane < lpm) {
    L.n = base + (L.lane < extra ? 1 : 0);
    L.s = L.lane * base + (L.lane < extra ? L.lane : extra);
  } else {
    L.n = 0;
    L.s = 0;
  }
  L.full = (L.n == C);
  return L;
}

// Row tables are stored chunk-major: entry (row s+t, coefficient c) of
// lane l is T[(t*W + c)*32 + l], so a warp reads 32 consecutive doubles.
__device__ __forceinline__ double tab(const double *__restrict__ T, int W, int t, int c, int lane) {
  return __ldg(T + ((size_t)t * W + c) * 32 + lane);
}

// chunk <-> pencil held in shared memory (or any pointer)
template <int C>
__device__ __forceinline__ void cld(const double2 *p, const Lane &L, double2 (&v)[C]) {
#pragma unroll
  for (int t = 0; t < C; t++) v[t] = (t < L.n) ? p[L.s + t] : czero();
}
template <int C>
__device__ __forceinline__ void cst(double2 *p, const Lane &L, const double2 (&v)[C]) {
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) p[L.s + t] = v[t];
}

// out = band(A) * v, A rows of 2H+1 coefficients (column offsets -H..H).
// The coefficient tables hold zeros for out-of-range columns and the halos
// of the first/last lanes are zero.
template <int C, int H>
__device__ __forceinline__ void matvec(const double *__restrict__ A, const Lane &L, const double2 (&v)[C],
                                       double2 (&out)[C]) {
  double2 lh[H], rh[H];
#pragma unroll
  for (int q = 0; q < H; q++) {
    const double2 tl = L.full ? v[C - H + q] : v[C - 1 - H + q];
    lh[q] = shfl_up2(tl, 1);
    rh[q] = shfl_down2(v[q], 1);
    if (L.lane == 0) lh[q] = czero();
    if (L.lane >= L.lpm - 1) rh[q] = czero();
  }
#pragma unroll
  for (int t = 0; t < C; t++) {
    double2 acc = czero();
    if (t < L.n) {
#pragma unroll
      for (int c = 0; c < 2 * H + 1; c++) {
        const int e = t - H + c;
        double2 u;
        if (e < 0) u = lh[e + H];
        else if (e < C - 1) u = v[e];
        else if (e == C - 1) u = L.full ? v[C - 1] : rh[0];
        else {
          const int i0 = (e - C < H) ? e - C : H - 1, i1 = (e - C + 1 < H) ? e - C + 1 : H - 1;
          u = L.full ? rh[i0] : rh[i1];
        }
        const double w = tab(A, 2 * H + 1, t, c, L.lane);
        acc.x = fma(w, u.x, acc.x);
        acc.y = fma(w, u.y, acc.y);
      }
    }
    out[t] = acc;
  }
}

// In-place variant: a rolling window keeps the H original values that the
// rows after them still need.
template <int C, int H>
__device__ __forceinline__ void matvec_ip(const double *__restrict__ A, const Lane &L, double2 (&v)[C]) {
  double2 lh[H], rh[H];
#pragma unroll
  for (int q = 0; q < H; q++) {
    const double2 tl = L.full ? v[C - H + q] : v[C - 1 - H + q];
    lh[q] = shfl_up2(tl, 1);
    rh[q] = shfl_down2(v[q], 1);
    if (L.lane == 0) lh[q] = czero();
    if (L.lane >= L.lpm - 1) rh[q] = czero();
  }
  double2 win[H];  // win[q] = original v[t-H+q] (left halo at first)
#pragma unroll
  for (int q = 0; q < H; q++) win[q] = lh[q];
#pragma unroll
  for (int t = 0; t < C; t++) {
    const double2 orig = v[t];
    double2 acc = czero();
    if (t < L.n) {
#pragma unroll
      for (int c = 0; c < 2 * H + 1; c++) {
        const int e = t - H + c;
        double2 u;
        if (c < H) u = win[c];
        else if (c == H) u = orig;
        else if (e < C - 1) u = v[e];
        else if (e == C - 1) u = L.full ? v[C - 1] : rh[0];
        else {
          const int i0 = (e - C < H) ? e - C : H - 1, i1 = (e - C + 1 < H) ? e - C + 1 : H - 1;
          u = L.full ? rh[i0] : rh[i1];
        }
        const double w = tab(A, 2 * H + 1, t, c, L.lane);
        acc.x = fma(w, u.x, acc.x);
        acc.y = fma(w, u.y, acc.y);
      }
    }
#pragma unroll
    for (int q = 0; q < H - 1; q++) win[q] = win[q + 1];
    win[H - 1] = orig;
    v[t] = acc;
  }
}

// ---------------------------------------------------------------------
// Band triangular solves (tables chunk-major, see tab()).
//   lower: x_j -= sum_{d=1..B} Lt[j][d-1] x_{j-d}
//   upper: x_i = (x_i - sum_{d=1..B} Ut[i][d] x_{i+d}) * Ut[i][0]
// Scan tables (constant operators): Ks[(s*32 + lane)*B*B] = the lane's
// composed chunk map at Kogge-Stone step s (row-major B x B).
// ---------------------------------------------------------------------
template <int C, int B>
__device__ __forceinline__ void lrun(double2 (&x)[C], const double *__restrict__ Lt, const Lane &L, double2 (&S)[B],
                                     bool write) {
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      double2 v = x[t];
#pragma unroll
      for (int d = 0; d < B; d++) {
        const double c = tab(Lt, B, t, d, L.lane);
        v.x = fma(-c, S[d].x, v.x);
        v.y = fma(-c, S[d].y, v.y);
      }
#pragma unroll
      for (int d = B - 1; d > 0; d--) S[d] = S[d - 1];
      S[0] = v;
      if (write) x[t] = v;
    }
}
template <int C, int B>
__device__ __forceinline__ void urun(double2 (&x)[C], const double *__restrict__ Ut, const Lane &L, double2 (&S)[B],
                                     bool write) {
#pragma unroll
  for (int t = C - 1; t >= 0; t--)
    if (t < L.n) {
      double2 v = x[t];
#pragma unroll
      for (int d = 0; d < B; d++) {
        const double c = tab(Ut, B + 1, t, 1 + d, L.lane);
        v.x = fma(-c, S[d].x, v.x);
        v.y = fma(-c, S[d].y, v.y);
      }
      const double r = tab(Ut, B + 1, t, 0, L.lane);
      v.x *= r;
      v.y *= r;
#pragma unroll
      for (int d = B - 1; d > 0; d--) S[d] = S[d - 1];
      S[0] = v;
      if (write) x[t] = v;
    }
}

// scan of the particular responses with precomputed composed maps
template <int B, bool UP>
__device__ __forceinline__ void scan_const(double2 (&S)[B], const double *__restrict__ Ks, int lane) {
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int off = 1 << s;
    double2 pp[B];
#pragma unroll
    for (int d = 0; d < B; d++) pp[d] = UP ? shfl_up2(S[d], off) : shfl_down2(S[d], off);
    const bool act = UP ? (lane >= off) : (lane + off < 32);
    if (act) {
      const double *A = Ks + (size_t)(s * 32 + lane) * B * B;
#pragma unroll
      for (int r = 0; r < B; r++) {
#pragma unroll
        for (int q = 0; q < B; q++) {
          const double a = __ldg(A + r * B + q);
          S[r].x = fma(a, pp[q].x, S[r].x);
          S[r].y = fma(a, pp[q].y, S[r].y);
        }
      }
    }
  }
}

template <int C, int B>
__device__ __forceinline__ void lsolve_c(double2 (&x)[C], const double *__restrict__ Lt, const double *__restrict__ Ks,
                                         const Lane &L) {
  double2 S[B];
#pragma unroll
  for (int d = 0; d < B; d++) S[d] = czero();
  lrun<C, B>(x, Lt, L, S, false);
  scan_const<B, true>(S, Ks, L.lane);
#pragma unroll
  for (int d = 0; d < B; d++) {
    S[d] = shfl_up2(S[d], 1);
    if (L.lane == 0) S[d] = czero();
  }
  lrun<C, B>(x, Lt, L, S, true);
}
template <int C, int B>
__device__ __forceinline__ void usolve_c(double2 (&x)[C], const double *__restrict__ Ut, const double *__restrict__ Ks,
                                         const Lane &L) {
  double2 S[B];
#pragma unroll
  for (int d = 0; d < B; d++) S[d] = czero();
  urun<C, B>(x, Ut, L, S, false);
  scan_const<B, false>(S, Ks, L.lane);
#pragma unroll
  for (int d = 0; d < B; d++) {
    S[d] = shfl_down2(S[d], 1);
    if (L.lane == 31) S[d] = czero();
  }
  urun<C, B>(x, Ut, L, S, true);
}

// General solves (per-mode factors): the chunk maps are built in registers.
template <int C, int B, bool UP>
__device__ __forceinline__ void scan_gen(double2 (&S)[B], double (&M)[B][B], int lane) {
#pragma unroll
  for (int s = 0; s < 5; s++) {
    const int off = 1 << s;
    double2 pp[B];
    double MM[B][B];
#pragma unroll
    for (int d = 0; d < B; d++) pp[d] = UP ? shfl_up2(S[d], off) : shfl_down2(S[d], off);
#pragma unroll
    for (int r = 0; r < B; r++)
#pragma unroll
      for (int q = 0; q < B; q++)
        MM[r][q] = UP ? __shfl_up_sync(LMC_FULL, M[r][q], off) : __shfl_down_sync(LMC_FULL, M[r][q], off);
    const bool act = UP ? (lane >= off) : (lane + off < 32);
    if (act) {
      double nM[B][B];
#pragma unroll
      for (int r = 0; r < B; r++) {
#pragma unroll
        for (int q = 0; q < B; q++) {
          S[r].x = fma(M[r][q], pp[q].x, S[r].x);
          S[r].y = fma(M[r][q], pp[q].y, S[r].y);
          double a = 0.0;
#pragma unroll
          for (int k = 0; k < B; k++) a = fma(M[r][k], MM[k][q], a);
          nM[r][q] = a;
        }
      }
#pragma unroll
      for (int r = 0; r < B; r++)
#pragma unroll
        for (int q = 0; q < B; q++) M[r][q] = nM[r][q];
    }
  }
}

template <int C, int B>
__device__ __forceinline__ void lsolve_g(double2 (&x)[C], const double *__restrict__ Lt, const Lane &L) {
  double2 S[B];
#pragma unroll
  for (int d = 0; d < B; d++) S[d] = czero();
  lrun<C, B>(x, Lt, L, S, false);
  double M[B][B];
#pragma unroll
  for (int q = 0; q < B; q++) {
    double2 T[B];
    double2 z[C];
#pragma unroll
    for (int t = 0; t < C; t++) z[t] = czero();
#pragma unroll
    for (int d = 0; d < B; d++) T[d] = make_double2(d == q ? 1.0 : 0.0, 0.0);
    lrun<C, B>(z, Lt, L, T, false);
#pragma unroll
    for (int r = 0; r < B; r++) M[r][q] = T[r].x;
  }
  scan_gen<C, B, true>(S, M, L.lane);
#pragma unroll
  for (int d = 0; d < B; d++) {
    S[d] = shfl_up2(S[d], 1);
    if (L.lane == 0) S[d] = czero();
  }
  lrun<C, B>(x, Lt, L, S, true);
}
template <int C, int B>
__device__ __forceinline__ void usolve_g(double2 (&x)[C], const double *__restrict__ Ut, const Lane &L) {
  double2 S[B];
#pragma unroll
  for (int d = 0; d < B; d++) S[d] = czero();
  urun<C, B>(x, Ut, L, S, false);
  double M[B][B];
#pragma unroll
  for (int q = 0; q < B; q++) {
    double2 T[B];
    double2 z[C];
#pragma unroll
    for (int t = 0; t < C; t++) z[t] = czero();
#pragma unroll
    for (int d = 0; d < B; d++) T[d] = make_double2(d == q ? 1.0 : 0.0, 0.0);
    urun<C, B>(z, Ut, L, T, false);
#pragma unroll
    for (int r = 0; r < B; r++) M[r][q] = T[r].x;
  }
  scan_gen<C, B, false>(S, M, L.lane);
#pragma unroll
  for (int d = 0; d < B; d++) {
    S[d] = shfl_down2(S[d], 1);
    if (L.lane == 31) S[d] = czero();
  }
  urun<C, B>(x, Ut, L, S, true);
}

__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    v.x += __shfl_xor_sync(LMC_FULL, v.x, off);
    v.y += __shfl_xor_sync(LMC_FULL, v.y, off);
  }
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(LMC_FULL, v, off);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v = fmax(v, __shfl_xor_sync(LMC_FULL, v, off));
  return v;
}

#ifdef LMC_FFT_TU
// ---------------------------------------------------------------------
// Register DFTs of compile-time size R (natural order in and out):
// y_k = sum_n x_n exp(SIGN 2 pi i nk/R), recursive mixed radix 4/2/3.
// Twiddles exp(-2 pi i e/R) come from a constant table (c_tw), one block
// per size, filled by the host at initialisation.
// ---------------------------------------------------------------------
constexpr int TW_SIZES[] = {4, 6, 8, 9, 12, 16, 18, 24, 32, 36, 48};
__host__ __device__ constexpr int tw_off(int R) {
  return R == 4 ? 0 : R == 6 ? 4 : R == 8 ? 10 : R == 9 ? 18 : R == 12 ? 27 : R == 16 ? 39 : R == 18 ? 55
       : R == 24 ? 73 : R == 32 ? 97 : R == 36 ? 129 : R == 48 ? 165 : -1;
}
constexpr int TW_TOTAL = 4 + 6 + 8 + 9 + 12 + 16 + 18 + 24 + 32 + 36 + 48;

static __constant__ double2 c_tw[TW_TOTAL];  // one copy per translation unit
static __constant__ float2 c_twf[TW_TOTAL];  // the same, rounded to FP32

template <int R, int SIGN, typename CT>
__device__ __forceinline__ CT ctw(int e) {
  constexpr int o = tw_off(R);
  static_assert(o >= 0, "register DFT size without twiddles");
  CT w;
  if constexpr (sizeof(CT) == sizeof(double2)) w = c_tw[o + e];
  else w = c_twf[o + e];
  return SIGN > 0 ? cconj(w) : w;
}

template <int R, int SIGN, typename CT>
__device__ __forceinline__ void bfly(CT (&x)[R]) {
  using Re = typename CReal<CT>::R;
  if constexpr (R == 2) {
    const CT a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  } else if constexpr (R == 4) {
    const CT t0 = cadd(x[0], x[2]), t1 = csub(x[0], x[2]), t2 = cadd(x[1], x[3]);
    const CT d = csub(x[1], x[3]);
    const CT t3 = (SIGN > 0) ? cmk<CT>(-d.y, d.x) : cmk<CT>(d.y, -d.x);  // d * (SIGN i)
    x[0] = cadd(t0, t2);
    x[2] = csub(t0, t2);
    x[1] = cadd(t1, t3);
    x[3] = csub(t1, t3);
  } else if constexpr (R == 3) {
    const Re s3 = (Re)0.86602540378443864676;  // sqrt(3)/2
    const CT t = cadd(x[1], x[2]);
    const CT d = csub(x[1], x[2]);
    const CT u = (SIGN > 0) ? cmk<CT>(-s3 * d.y, s3 * d.x) : cmk<CT>(s3 * d.y, -s3 * d.x);
    const CT a = cmk<CT>(x[0].x - (Re)0.5 * t.x, x[0].y - (Re)0.5 * t.y);
    x[0] = cadd(x[0], t);
    x[1] = cadd(a, u);
    x[2] = csub(a, u);
  }
}

template <int R, int SIGN, typename CT>
__device__ __forceinline__ void rdft(CT (&x)[R]) {
  if constexpr (R == 1) {
    return;
  } else if constexpr (R == 2 || R == 3 || R == 4) {
    bfly<R, SIGN>(x);
  } else {
    constexpr int p = (R % 4 == 0) ? 4 : ((R % 2 == 0) ? 2 : 3);
    constexpr int m = R / p;
    CT sub[p][m];
#pragma unroll
    for (int r = 0; r < p; r++)
#pragma unroll
      for (int j = 0; j < m; j++) sub[r][j] = x[r + p * j];
#pragma unroll
    for (int r = 0; r < p; r++) rdft<m, SIGN>(sub[r]);
#pragma unroll
    for (int k = 0; k < m; k++) {
      CT t[p];
#pragma unroll
      for (int r = 0; r < p; r++) t[r] = (r == 0 || k == 0) ? sub[r][k] : cmul(sub[r][k], ctw<R, SIGN, CT>(r * k));
      bfly<p, SIGN>(t);
#pragma unroll
      for (int q = 0; q < p; q++) x[k + m * q] = t[q];
    }
  }
}

// Four-step transform of nb lines of length N = N1*N2 in shared memory.
// Line b starts at sm + b*ld; natural index n is stored at skew(n) =
// n + n/N1.  twN[e] = exp(-2 pi i e/N).  CT is the complex type of the
// samples and of the arithmetic (double2, or float2 in the mixed form).
template <int N1, int N2, typename CT = double2>
struct Four {
  static constexpr int N = N1 * N2;
  static constexpr int LD = N2 * (N1 + 1);  // skewed line length
  __device__ static __forceinline__ int sk(int n) { return n + n / N1; }

  // natural -> permuted: X[k2 + N2 k1] lands at skew position k1 + N1 k2
  template <int SIGN, int U = 1>
  __device__ static void nat2perm(CT *sm, int nb, int ld, const CT *__restrict__ twN) {
    #pragma unroll U
    for (int idx = threadIdx.x; idx < nb * N1; idx += blockDim.x) {
      const int b = idx / N1, n1 = idx - b * N1;
      CT *p = sm + (size_t)b * ld + n1;
      CT x[N2];
#pragma unroll
      for (int j = 0; j < N2; j++) x[j] = p[j * (N1 + 1)];
      rdft<N2, SIGN>(x);
#pragma unroll
      for (int k = 0; k < N2; k++) {
        CT v = x[k];
        if (k > 0 && n1 > 0) {
          CT w = __ldg(twN + n1 * k);
          if (SIGN > 0) w = cconj(w);
          v = cmul(v, w);
        }
        p[k * (N1 + 1)] = v;
      }
    }
    __syncthreads();
    nat2perm_p2<SIGN, U>(sm, nb, ld);
  }

  // the first pass of nat2perm with sample n of line b supplied by
  // load(b, n) instead of read from shared memory (ends with a barrier)
  template <int SIGN, typename L>
  __device__ static void nat2perm_in(CT *sm, int nb, int ld, const CT *__restrict__ twN, L &&load) {
    for (int idx = threadIdx.x; idx < nb * N1; idx += blockDim.x) {
      const int b = idx / N1, n1 = idx - b * N1;
      CT *p = sm + (size_t)b * ld + n1;
      CT x[N2];
#pragma unroll
      for (int j = 0; j < N2; j++) x[j] = load(b, n1 + N1 * j);
      rdft<N2, SIGN>(x);
#pragma unroll
      for (int k = 0; k < N2; k++) {
        CT v = x[k];
        if (k > 0 && n1 > 0) {
          CT w = __ldg(twN + n1 * k);
          if (SIGN > 0) w = cconj(w);
          v = cmul(v, w);
        }
        p[k * (N1 + 1)] = v;
      }
    }
    __syncthreads();
  }

  // The first pass of nat2perm for real inputs packed two per line (A + iB)
  // under the 2/3 rule: only the N/3 lowest modes of A and B are nonzero,
  // given as rows of nkx = N/3 complex values; the transform input is A + iB
  // at n < nkx, its conjugate mirror at n > N - nkx and zero in the gap
  // (the imaginary parts of mode 0 dropped, rftsingle.f:85-88).  With
  // N2 % 3 == 0 the gap and the mirrored third are fixed ranges of the
  // sample index j of a task (n = n1 + N1 j), so no sample is tested and
  // the gap is never loaded.  rows(b, A, B) gives line b's two rows (false:
  // a padding line, all zero).  Ends with a barrier.
  template <int SIGN, typename ST, typename R>
  __device__ static void nat2perm_in3(CT *sm, int nb, int ld, const CT *__restrict__ twN, R &&rows) {
    static_assert(N2 % 3 == 0, "the 2/3-rule gap must be whole sample rows");
    constexpr int J1 = N2 / 3, J2 = 2 * N2 / 3;
    using Re = typename CReal<CT>::R;
    auto cv = [](const ST &v) { return cmk<CT>((Re)v.x, (Re)v.y); };
    for (int idx = threadIdx.x; idx < nb * N1; idx += blockDim.x) {
      const int b = idx / N1, n1 = idx - b * N1;
      CT *p = sm + (size_t)b * ld + n1;
      const ST *A = nullptr, *B = nullptr;
      const bool ok = rows(b, A, B);
      CT x[N2];
#pragma unroll
      for (int j = 0; j < N2; j++) x[j] = cz<CT>();
      if (ok) {
#pragma unroll
        for (int j = 0; j < J1; j++) {  // A + iB, n = n1 + N1 j < nkx
          const int n = n1 + N1 * j;
          const CT a = cv(A[n]), c = cv(B[n]);
          x[j] = (j == 0 && n1 == 0) ? cmk<CT>(a.x, c.x) : cmk<CT>(a.x - c.y, a.y + c.x);
        }
#pragma unroll
        for (int j = J2; j < N2; j++) {  // conj(A) + i conj(B) at k = N - n < nkx
          const int k = N - n1 - N1 * j;
          if (j > J2 || n1 > 0) {
            const CT a = cv(A[k]), c = cv(B[k]);
            x[j] = cmk<CT>(a.x + c.y, c.x - a.y);
          }
        }
      }
      rdft<N2, SIGN>(x);
#pragma unroll
      for (int k = 0; k < N2; k++) {
        CT v = x[k];
        if (k > 0 && n1 > 0) {
          CT w = __ldg(twN + n1 * k);
          if (SIGN > 0) w = cconj(w);
          v = cmul(v, w);
        }
        p[k * (N1 + 1)] = v;
      }
    }
    __syncthreads();
  }

  // The first pass of nat2perm for the 3/2-padded z lines read straight
  // from their spectral rows: sample n of line b is coefficient n (n < N/3),
  // zero (the padding N/3 .. 2N/3) or coefficient n - N/3 - 1 (the negative
  // wavenumbers, n > 2N/3); get(b, k) returns coefficient k of line b.
  // N2 % 3 == 0, so the three ranges are fixed ranges of the sample row j.
  // Ends with a barrier.
  template <int SIGN, typename G>
  __device__ static void nat2perm_zin(CT *sm, int nb, int ld, const CT *__restrict__ twN, G &&get) {
    static_assert(N2 % 3 == 0, "the padding gap must be whole sample rows");
    constexpr int J1 = N2 / 3, J2 = 2 * N2 / 3, SH = N / 3 + 1;
    for (int idx = threadIdx.x; idx < nb * N1; idx += blockDim.x) {
      const int b = idx / N1, n1 = idx - b * N1;
      CT *p = sm + (size_t)b * ld + n1;
      CT x[N2];
#pragma unroll
      for (int j = 0; j < N2; j++) {
        const int n = n1 + N1 * j;
        if (j < J1) x[j] = get(b, n);
        else if (j > J2 || (j == J2 && n1 > 0)) x[j] = get(b, n - SH);
        else x[j] = cz<CT>();
      }
      rdft<N2, SIGN>(x);
#pragma unroll
      for (int k = 0; k < N2; k++) {
        CT v = x[k];
        if (k > 0 && n1 > 0) {
          CT w = __ldg(twN + n1 * k);
          if (SIGN > 0) w = cconj(w);
          v = cmul(v, w);
        }
        p[k * (N1 + 1)] = v;
      }
    }
    __syncthreads();
  }

  // the second pass of nat2perm (ends with a barrier)
  template <int SIGN, int U = 1>
  __device__ static void nat2perm_p2(CT *sm, int nb, int ld) {
    #pragma unroll U
    for (int idx = threadIdx.x; idx < nb * N2; idx += blockDim.x) {
      const int b = idx / N2, k2 = idx - b * N2;
      CT *p = sm + (size_t)b * ld + k2 * (N1 + 1);
      CT x[N1];
#pragma unroll
      for (int j = 0; j < N1; j++) x[j] = p[j];
      rdft<N1, SIGN>(x);
#pragma unroll
      for (int j = 0; j < N1; j++) p[j] = x[j];
    }
    __syncthreads();
  }

  // permuted -> natural (transpose of nat2perm)
  template <int SIGN, int U = 1>
  __device__ static void perm2nat(CT *sm, int nb, int ld, const CT *__restrict__ twN) {
    #pragma unroll U
    for (int idx = threadIdx.x; idx < nb * N2; idx += blockDim.x) {
      const int b = idx / N2, k2 = idx - b * N2;
      CT *p = sm + (size_t)b * ld + k2 * (N1 + 1);
      CT x[N1];
#pragma unroll
      for (int j = 0; j < N1; j++) x[j] = p[j];
      rdft<N1, SIGN>(x);
#pragma unroll
      for (int j = 0; j < N1; j++) {
        CT v = x[j];
        if (j > 0 && k2 > 0) {
          CT w = __ldg(twN + j * k2);
          if (SIGN > 0) w = cconj(w);
          v = cmul(v, w);
        }
        p[j] = v;
      }
    }
    __syncthreads();
    #pragma unroll U
    for (int idx = threadIdx.x; idx < nb * N1; idx += blockDim.x) {
      const int b = idx / N1, n1 = idx - b * N1;
      CT *p = sm + (size_t)b * ld + n1;
      CT x[N2];
#pragma unroll
      for (int j = 0; j < N2; j++) x[j] = p[j * (N1 + 1)];
      rdft<N2, SIGN>(x);
#pragma unroll
      for (int j = 0; j < N2; j++) p[j * (N1 + 1)] = x[j];
    }
    __syncthreads();
  }
};

#endif  // LMC_FFT_TU

}  // namespace lmcd
