// lmc_device.cuh -- device building blocks of the lomacte substep kernels.
//
// y-direction operators: one warp per (kx,kz) mode.  The pencil of my
// points is split into chunks of n in {C-1, C} consecutive points, one chunk
// per active lane (LPM active lanes, my = sum of chunk sizes).  Banded
// matrix-vector products exchange a halo of H points with the neighbour
// lanes by shuffles.  Banded triangular solves run each chunk's recurrence
// in registers and join the chunks with a Kogge-Stone scan of the affine
// chunk maps state_out = M state_in + p (M from the homogeneous responses),
// so no pencil ever leaves registers between the forward and backward
// sweeps.
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
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 czero() { return make_double2(0.0, 0.0); }

__device__ __forceinline__ double2 shfl_up2(double2 v, int d) {
  return make_double2(__shfl_up_sync(LMC_FULL, v.x, d), __shfl_up_sync(LMC_FULL, v.y, d));
}
__device__ __forceinline__ double2 shfl_down2(double2 v, int d) {
  return make_double2(__shfl_down_sync(LMC_FULL, v.x, d), __shfl_down_sync(LMC_FULL, v.y, d));
}

// Chunk geometry of one lane.
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

template <int C>
__device__ __forceinline__ void ld(const double2 *__restrict__ p, const Lane &L, double2 (&v)[C]) {
#pragma unroll
  for (int t = 0; t < C; t++) v[t] = (t < L.n) ? __ldg(p + L.s + t) : czero();
}
template <int C>
__device__ __forceinline__ void st(double2 *__restrict__ p, const Lane &L, const double2 (&v)[C]) {
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) p[L.s + t] = v[t];
}

// out = band(A) * v, A rows of 2H+1 coefficients (column offsets -H..H).
// Rows outside 0..my-1 do not exist; the coefficient tables hold zeros for
// out-of-range columns, and the halos of the first/last lanes are zero.
template <int C, int H>
__device__ __forceinline__ void matvec(const double *__restrict__ A, const Lane &L, const double2 (&v)[C],
                                       double2 (&out)[C]) {
  double2 tl[H], hd[H], lh[H], rh[H];
#pragma unroll
  for (int q = 0; q < H; q++) {
    tl[q] = L.full ? v[C - H + q] : v[C - 1 - H + q];
    hd[q] = v[q];
  }
#pragma unroll
  for (int q = 0; q < H; q++) {
    lh[q] = shfl_up2(tl[q], 1);
    rh[q] = shfl_down2(hd[q], 1);
    if (L.lane == 0) lh[q] = czero();
    if (L.lane >= L.lpm - 1) rh[q] = czero();
  }
#pragma unroll
  for (int t = 0; t < C; t++) {
    double2 acc = czero();
    if (t < L.n) {
      const double *a = A + (size_t)(L.s + t) * (2 * H + 1);
#pragma unroll
      for (int c = 0; c < 2 * H + 1; c++) {
        const int e = t - H + c;
        double2 u;
        if (e < 0) u = lh[e + H];
        else if (e < C - 1) u = v[e];
        else if (e == C - 1) u = L.full ? v[C - 1] : rh[0];
        else {
          const int i0 = e - C, i1 = (e - C + 1 < H) ? e - C + 1 : H - 1;
          u = L.full ? rh[i0 < H ? i0 : H - 1] : rh[i1];
        }
        const double w = __ldg(a + c);
        acc.x = fma(w, u.x, acc.x);
        acc.y = fma(w, u.y, acc.y);
      }
    }
    out[t] = acc;
  }
}

// Lower unit-triangular band solve in place: x_j -= sum_{d=1..B} Lt[j][d-1] x_{j-d}.
template <int C, int B>
__device__ __forceinline__ void lsolve(double2 (&x)[C], const double *__restrict__ Lt, const Lane &L) {
  // 1) particular response with zero incoming state
  double2 S[B];
#pragma unroll
  for (int d = 0; d < B; d++) S[d] = czero();
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double *l = Lt + (size_t)(L.s + t) * B;
      double2 v = x[t];
#pragma unroll
      for (int d = 0; d < B; d++) {
        const double c = __ldg(l + d);
        v.x = fma(-c, S[d].x, v.x);
        v.y = fma(-c, S[d].y, v.y);
      }
#pragma unroll
      for (int d = B - 1; d > 0; d--) S[d] = S[d - 1];
      S[0] = v;
    }
  // 2) homogeneous responses: M[r][q] = state r after the chunk from e_q
  double M[B][B];
#pragma unroll
  for (int q = 0; q < B; q++) {
    double T[B];
#pragma unroll
    for (int d = 0; d < B; d++) T[d] = (d == q) ? 1.0 : 0.0;
#pragma unroll
    for (int t = 0; t < C; t++)
      if (t < L.n) {
        const double *l = Lt + (size_t)(L.s + t) * B;
        double v = 0.0;
#pragma unroll
        for (int d = 0; d < B; d++) v = fma(-__ldg(l + d), T[d], v);
#pragma unroll
        for (int d = B - 1; d > 0; d--) T[d] = T[d - 1];
        T[0] = v;
      }
#pragma unroll
    for (int r = 0; r < B; r++) M[r][q] = T[r];
  }
  // 3) inclusive scan over lanes (lane order = row order)
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    double2 pp[B];
    double MM[B][B];
#pragma unroll
    for (int d = 0; d < B; d++) pp[d] = shfl_up2(S[d], off);
#pragma unroll
    for (int r = 0; r < B; r++)
#pragma unroll
      for (int q = 0; q < B; q++) MM[r][q] = __shfl_up_sync(LMC_FULL, M[r][q], off);
    if (L.lane >= off) {
      double2 np[B];
      double nM[B][B];
#pragma unroll
      for (int r = 0; r < B; r++) {
        double2 a = S[r];
#pragma unroll
        for (int q = 0; q < B; q++) {
          a.x = fma(M[r][q], pp[q].x, a.x);
          a.y = fma(M[r][q], pp[q].y, a.y);
        }
        np[r] = a;
#pragma unroll
        for (int q = 0; q < B; q++) {
          double s = 0.0;
#pragma unroll
          for (int k = 0; k < B; k++) s = fma(M[r][k], MM[k][q], s);
          nM[r][q] = s;
        }
      }
#pragma unroll
      for (int r = 0; r < B; r++) {
        S[r] = np[r];
#pragma unroll
        for (int q = 0; q < B; q++) M[r][q] = nM[r][q];
      }
    }
  }
  // 4) incoming state = inclusive result of the previous lane
  double2 Sin[B];
#pragma unroll
  for (int d = 0; d < B; d++) {
    Sin[d] = shfl_up2(S[d], 1);
    if (L.lane == 0) Sin[d] = czero();
  }
  // 5) final pass
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double *l = Lt + (size_t)(L.s + t) * B;
      double2 v = x[t];
#pragma unroll
      for (int d = 0; d < B; d++) {
        const double c = __ldg(l + d);
        v.x = fma(-c, Sin[d].x, v.x);
        v.y = fma(-c, Sin[d].y, v.y);
      }
#pragma unroll
      for (int d = B - 1; d > 0; d--) Sin[d] = Sin[d - 1];
      Sin[0] = v;
      x[t] = v;
    }
}

// Upper band solve in place: x_i = (x_i - sum_{d=1..B} U[i][d] x_{i+d}) * U[i][0].
template <int C, int B>
__device__ __forceinline__ void usolve(double2 (&x)[C], const double *__restrict__ Ut, const Lane &L) {
  double2 S[B];  // S[d] = x_{i+1+d}
#pragma unroll
  for (int d = 0; d < B; d++) S[d] = czero();
#pragma unroll
  for (int t = C - 1; t >= 0; t--)
    if (t < L.n) {
      const double *u = Ut + (size_t)(L.s + t) * (B + 1);
      double2 v = x[t];
#pragma unroll
      for (int d = 0; d < B; d++) {
        const double c = __ldg(u + 1 + d);
        v.x = fma(-c, S[d].x, v.x);
        v.y = fma(-c, S[d].y, v.y);
      }
      const double r = __ldg(u);
      v.x *= r;
      v.y *= r;
#pragma unroll
      for (int d = B - 1; d > 0; d--) S[d] = S[d - 1];
      S[0] = v;
    }
  double M[B][B];
#pragma unroll
  for (int q = 0; q < B; q++) {
    double T[B];
#pragma unroll
    for (int d = 0; d < B; d++) T[d] = (d == q) ? 1.0 : 0.0;
#pragma unroll
    for (int t = C - 1; t >= 0; t--)
      if (t < L.n) {
        const double *u = Ut + (size_t)(L.s + t) * (B + 1);
        double v = 0.0;
#pragma unroll
        for (int d = 0; d < B; d++) v = fma(-__ldg(u + 1 + d), T[d], v);
        v *= __ldg(u);
#pragma unroll
        for (int d = B - 1; d > 0; d--) T[d] = T[d - 1];
        T[0] = v;
      }
#pragma unroll
    for (int r = 0; r < B; r++) M[r][q] = T[r];
  }
  // scan from the last lane downwards
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    double2 pp[B];
    double MM[B][B];
#pragma unroll
    for (int d = 0; d < B; d++) pp[d] = shfl_down2(S[d], off);
#pragma unroll
    for (int r = 0; r < B; r++)
#pragma unroll
      for (int q = 0; q < B; q++) MM[r][q] = __shfl_down_sync(LMC_FULL, M[r][q], off);
    if (L.lane + off < 32) {
      double2 np[B];
      double nM[B][B];
#pragma unroll
      for (int r = 0; r < B; r++) {
        double2 a = S[r];
#pragma unroll
        for (int q = 0; q < B; q++) {
          a.x = fma(M[r][q], pp[q].x, a.x);
          a.y = fma(M[r][q], pp[q].y, a.y);
        }
        np[r] = a;
#pragma unroll
        for (int q = 0; q < B; q++) {
          double s = 0.0;
#pragma unroll
          for (int k = 0; k < B; k++) s = fma(M[r][k], MM[k][q], s);
          nM[r][q] = s;
        }
      }
#pragma unroll
      for (int r = 0; r < B; r++) {
        S[r] = np[r];
#pragma unroll
        for (int q = 0; q < B; q++) M[r][q] = nM[r][q];
      }
    }
  }
  double2 Sin[B];
#pragma unroll
  for (int d = 0; d < B; d++) {
    Sin[d] = shfl_down2(S[d], 1);
    if (L.lane == 31) Sin[d] = czero();
  }
#pragma unroll
  for (int t = C - 1; t >= 0; t--)
    if (t < L.n) {
      const double *u = Ut + (size_t)(L.s + t) * (B + 1);
      double2 v = x[t];
#pragma unroll
      for (int d = 0; d < B; d++) {
        const double c = __ldg(u + 1 + d);
        v.x = fma(-c, Sin[d].x, v.x);
        v.y = fma(-c, Sin[d].y, v.y);
      }
      const double r = __ldg(u);
      v.x *= r;
      v.y *= r;
#pragma unroll
      for (int d = B - 1; d > 0; d--) Sin[d] = Sin[d - 1];
      Sin[0] = v;
      x[t] = v;
    }
}

// Warp sum of a complex value over all lanes.
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

// ---------------------------------------------------------------------
// Batched in-place mixed-radix FFT on shared memory.
// DIF (natural order in, digit-reversed out) and its transpose DIT
// (digit-reversed in, natural out).  The inverse transforms of the
// substep run DIF and the direct transforms DIT, so the physical-space
// samples sit in digit-reversed order and no permutation pass is needed.
// ---------------------------------------------------------------------
struct FFTPlan {
  int n, nst;
  int rad[16];
  const double2 *tw;  // tw[t] = exp(-2 pi i t/n)
};

__device__ __forceinline__ double2 twid(const FFTPlan &P, int e, int sign) {
  double2 w = __ldg(P.tw + e);
  return sign > 0 ? cconj(w) : w;
}

template <int R, int SIGN>
__device__ __forceinline__ void bfly(double2 (&x)[R]) {
  // y_q = sum_p x_p exp(SIGN 2 pi i pq/R), in place
  if (R == 2) {
    double2 a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
  } else if (R == 4) {
    double2 t0 = cadd(x[0], x[2]), t1 = csub(x[0], x[2]), t2 = cadd(x[1], x[3]);
    double2 d = csub(x[1], x[3]);
    double2 t3 = (SIGN > 0) ? make_double2(-d.y, d.x) : make_double2(d.y, -d.x);  // d * (SIGN i)
    x[0] = cadd(t0, t2);
    x[2] = csub(t0, t2);
    x[1] = cadd(t1, t3);
    x[3] = csub(t1, t3);
  } else {  // R == 3
    const double s3 = 0.86602540378443864676;  // sqrt(3)/2
    double2 t = cadd(x[1], x[2]);
    double2 d = csub(x[1], x[2]);
    double2 u = (SIGN > 0) ? make_double2(-s3 * d.y, s3 * d.x) : make_double2(s3 * d.y, -s3 * d.x);
    double2 a = make_double2(x[0].x - 0.5 * t.x, x[0].y - 0.5 * t.y);
    x[0] = cadd(x[0], t);
    x[1] = cadd(a, u);
    x[2] = csub(a, u);
  }
}

// One radix-R stage over nb transforms of length n (batch b at buf+b*ld);
// Ns is the sub-transform length of this stage.
template <int R, int SIGN, bool DIF>
__device__ __forceinline__ void fft_stage(double2 *buf, int nb, int ld, const FFTPlan &P, int Ns) {
  const int n = P.n, M = Ns / R, nbut = n / R, tot = nb * nbut, stride = n / Ns;
  for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
    const int b = idx / nbut, rem = idx - b * nbut, blk = rem / M, m = rem - blk * M;
    double2 *base = buf + (size_t)b * ld + blk * Ns + m;
    double2 x[R];
    if (DIF) {
#pragma unroll
      for (int p = 0; p < R; p++) x[p] = base[p * M];
      bfly<R, SIGN>(x);
#pragma unroll
      for (int q = 0; q < R; q++) {
        double2 v = x[q];
        if (q > 0 && m > 0) v = cmul(v, twid(P, (q * m * stride) % n, SIGN));
        base[q * M] = v;
      }
    } else {
#pragma unroll
      for (int q = 0; q < R; q++) {
        double2 v = base[q * M];
        if (q > 0 && m > 0) v = cmul(v, twid(P, (q * m * stride) % n, SIGN));
        x[q] = v;
      }
      bfly<R, SIGN>(x);
#pragma unroll
      for (int p = 0; p < R; p++) base[p * M] = x[p];
    }
  }
}

// nb transforms of length P.n, batch b at buf + b*ld.  All threads of the
// block call these; each stage ends with a __syncthreads().
template <int SIGN>
__device__ void fft_dif(double2 *buf, int nb, int ld, const FFTPlan &P) {
  int Ns = P.n;
  for (int st = 0; st < P.nst; st++) {
    const int r = P.rad[st];
    if (r == 4) fft_stage<4, SIGN, true>(buf, nb, ld, P, Ns);
    else if (r == 2) fft_stage<2, SIGN, true>(buf, nb, ld, P, Ns);
    else fft_stage<3, SIGN, true>(buf, nb, ld, P, Ns);
    __syncthreads();
    Ns /= r;
  }
}

template <int SIGN>
__device__ void fft_dit(double2 *buf, int nb, int ld, const FFTPlan &P) {
  int sizes[16];
  int Ns = P.n;
  for (int st = 0; st < P.nst; st++) {
    sizes[st] = Ns;
    Ns /= P.rad[st];
  }
  for (int st = P.nst - 1; st >= 0; st--) {
    const int r = P.rad[st];
    if (r == 4) fft_stage<4, SIGN, false>(buf, nb, ld, P, sizes[st]);
    else if (r == 2) fft_stage<2, SIGN, false>(buf, nb, ld, P, sizes[st]);
    else fft_stage<3, SIGN, false>(buf, nb, ld, P, sizes[st]);
    __syncthreads();
  }
}

}  // namespace lmcd
