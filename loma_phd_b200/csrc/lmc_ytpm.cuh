// lmc_ytpm.cuh -- mode-parallel y kernels: one thread per (kx,kz) mode.
//
// In the spectral layout [y][kx][kz] the value of mode m at row j sits at
// f[j*nmode + m], so the threads of a warp (32 consecutive modes) read and
// write every row of their pencils as one coalesced 32-value run, and the
// coefficients of a row are the same for the whole warp (one broadcast
// load).  Each banded solve A x = b with A = L U (the LU of cfdiff.f /
// laps.f in row form) runs as two sweeps along y: the forward sweep forms
// the band product of the right-hand side and applies L^-1, writing the
// intermediate pencil to an FP64 scratch field; the backward sweep reads it
// in reverse and applies U^-1.  Fields are streamed through a small queue
// of registers that is refilled K rows ahead of use, so every thread keeps
// several loads in flight.  Kernels follow the same statements of
// trunk/lomacte3/src/cross.f:307-1141 as the warp-per-mode kernels of
// lmc_ykernels.cuh (which keep serving small grids and the 00-mode tails).
#pragma once
#include <cuda_runtime.h>

#include "lmc_kernels.cuh"

namespace lmc {
namespace tpm {

using namespace lmcd;

constexpr int TB = 128;  // modes per block

template <typename CT>
__host__ __device__ constexpr bool mixed() { return sizeof(CT) == sizeof(float2); }

// Prefetching reader of one pencil, walking rows first, first+dir, ...
// Loads go through L2 (ld.global.cg), never the non-coherent read-only
// path: a kernel reads back scratch pencils and fields it wrote itself.
template <typename PT, int K>
struct Rd {
  const PT *p;
  size_t ld;
  int my, dir, nxt;
  PT q[K];
  __device__ __forceinline__ PT fetch(int r) const {
    PT z;
    z.x = 0;
    z.y = 0;
    return (r >= 0 && r < my) ? __ldcg(p + (size_t)r * ld) : z;
  }
  __device__ __forceinline__ void start(const PT *base, size_t ld_, int my_, int dir_, int first) {
    p = base;
    ld = ld_;
    my = my_;
    dir = dir_;
    nxt = first;
#pragma unroll
    for (int t = 0; t < K; t++) {
      q[t] = fetch(nxt);
      nxt += dir;
    }
  }
  __device__ __forceinline__ double2 pop() {
    const double2 v = to_d2(q[0]);
#pragma unroll
    for (int t = 0; t < K - 1; t++) q[t] = q[t + 1];
    q[K - 1] = fetch(nxt);
    nxt += dir;
    return v;
  }
};

// queue depth giving K x 16 bytes in flight for values of type PT
template <typename PT>
__host__ __device__ constexpr int kq(int K) { return K * 16 / (int)sizeof(PT); }

// the same for one real coefficient per row (per-mode tables)
template <int K>
struct RdS {
  const double *p;
  size_t ld;
  int my, dir, nxt;
  double q[K];
  __device__ __forceinline__ double fetch(int r) const {
    return (r >= 0 && r < my) ? __ldg(p + (size_t)r * ld) : 0.0;
  }
  __device__ __forceinline__ void start(const double *base, size_t ld_, int my_, int dir_, int first) {
    p = base;
    ld = ld_;
    my = my_;
    dir = dir_;
    nxt = first;
#pragma unroll
    for (int t = 0; t < K; t++) {
      q[t] = fetch(nxt);
      nxt += dir;
    }
  }
  __device__ __forceinline__ double pop() {
    const double v = q[0];
#pragma unroll
    for (int t = 0; t < K - 1; t++) q[t] = q[t + 1];
    q[K - 1] = fetch(nxt);
    nxt += dir;
    return v;
  }
};

// the per-mode LU rows of one mode, streamed: L (2 multipliers) forward,
// U (reciprocal pivot + 2) backward
template <int K>
struct LRows {
  RdS<K> l0, l1;
  __device__ __forceinline__ void start(const Dev &d, int m) {
    const size_t n = (size_t)d.nmode;
    l0.start(d.PLt + m, 2 * n, d.my, 1, 0);
    l1.start(d.PLt + n + m, 2 * n, d.my, 1, 0);
  }
};
template <int K>
struct URows {
  RdS<K> u0, u1, u2;
  __device__ __forceinline__ void start(const Dev &d, int m) {
    const size_t n = (size_t)d.nmode;
    u0.start(d.PUt + m, 3 * n, d.my, -1, d.my - 1);
    u1.start(d.PUt + n + m, 3 * n, d.my, -1, d.my - 1);
    u2.start(d.PUt + 2 * n + m, 3 * n, d.my, -1, d.my - 1);
  }
};

template <typename PT>
__device__ __forceinline__ void put(PT *base, size_t ld, int j, double2 v) {
  base[(size_t)j * ld] = from_d2<PT>(v);
}

// u_{j-3} .. u_{j+3} around the current row j
struct Win {
  double2 u[7];
  __device__ __forceinline__ void clear() {
#pragma unroll
    for (int t = 0; t < 7; t++) u[t] = czero();
  }
  __device__ __forceinline__ void push(double2 v) {
#pragma unroll
    for (int t = 0; t < 6; t++) u[t] = u[t + 1];
    u[6] = v;
  }
  __device__ __forceinline__ double2 c() const { return u[3]; }
};

// the last three results of a sweep (x_{j-+1}, x_{j-+2}, x_{j-+3})
struct Hist {
  double2 a, b, c;
  __device__ __forceinline__ void clear() { a = b = c = czero(); }
  __device__ __forceinline__ void push(double2 v) {
    c = b;
    b = a;
    a = v;
  }
};

__device__ __forceinline__ double2 fms(double2 s, double k, double2 v) {  // s - k v
  return make_double2(fma(-k, v.x, s.x), fma(-k, v.y, s.y));
}

// forward half of d/dy (deryr2, cfdiff.f:518-601): w_j = (L1^-1 dt12 u)_j
__device__ __forceinline__ double2 d1f(const Dev &d, int j, const Win &u, Hist &h) {
  const double *c = d.r_dt12 + 7 * j;
  double2 r = czero();
#pragma unroll
  for (int t = 0; t < 7; t++) {
    const double k = __ldg(c + t);
    r.x = fma(k, u.u[t].x, r.x);
    r.y = fma(k, u.u[t].y, r.y);
  }
  const double *l = d.r_p1L + 3 * j;
  r = fms(fms(fms(r, __ldg(l + 2), h.c), __ldg(l + 1), h.b), __ldg(l), h.a);
  h.push(r);
  return r;
}
// backward half of d/dy: x_j = (U1^-1 w)_j times fmap_j
__device__ __forceinline__ double2 d1b(const Dev &d, int j, double2 w, Hist &h) {
  const double *u = d.r_p1U + 4 * j;
  double2 x = fms(fms(fms(w, __ldg(u + 3), h.c), __ldg(u + 2), h.b), __ldg(u + 1), h.a);
  x = cscale(__ldg(u), x);
  h.push(x);
  return cscale(__ldg(d.r_fmap + j), x);
}
// forward half of d2/dy2 (deryyr2, cfdiff.f:735-797)
__device__ __forceinline__ double2 d2f(const Dev &d, int j, const Win &u, Hist &h) {
  const double *c = d.r_dt22 + 5 * j;
  double2 r = czero();
#pragma unroll
  for (int t = 0; t < 5; t++) {
    const double k = __ldg(c + t);
    r.x = fma(k, u.u[t + 1].x, r.x);
    r.y = fma(k, u.u[t + 1].y, r.y);
  }
  const double *l = d.r_p3L + 2 * j;
  r = fms(fms(r, __ldg(l + 1), h.b), __ldg(l), h.a);
  h.push(r);
  return r;
}
__device__ __forceinline__ double2 d2b(const Dev &d, int j, double2 w, Hist &h) {
  const double *u = d.r_p3U + 3 * j;
  double2 x = fms(fms(w, __ldg(u + 2), h.b), __ldg(u + 1), h.a);
  x = cscale(__ldg(u), x);
  h.push(x);
  return x;
}
// Dirichlet Poisson of mode m (laps.f:375-401): right-hand side dt21 f with
// zero wall rows, then the mode's LU (dt22 - k^2 dt21 with identity rows)
template <int K>
__device__ __forceinline__ double2 pf(const Dev &d, int j, const Win &u, Hist &h, LRows<K> &L) {
  double2 r = czero();
  if (j > 0 && j < d.my - 1) {
    const double *c = d.r_dt21 + 5 * j;
#pragma unroll
    for (int t = 0; t < 5; t++) {
      const double k = __ldg(c + t);
      r.x = fma(k, u.u[t + 1].x, r.x);
      r.y = fma(k, u.u[t + 1].y, r.y);
    }
  }
  const double l0 = L.l0.pop(), l1 = L.l1.pop();
  r = fms(fms(r, l1, h.b), l0, h.a);
  h.push(r);
  return r;
}
template <int K>
__device__ __forceinline__ double2 pb(double2 w, Hist &h, URows<K> &U) {
  const double u0 = U.u0.pop(), u1 = U.u1.pop(), u2 = U.u2.pop();
  double2 x = fms(fms(w, u2, h.b), u1, h.a);
  x = cscale(u0, x);
  h.push(x);
  return x;
}

struct Mode {
  int m;
  double kx, kz, k2;
};
__device__ __forceinline__ bool mode_of(const Dev &d, Mode &M) {
  M.m = blockIdx.x * TB + threadIdx.x;
  if (M.m >= d.nmode) return false;
  const int i = M.m / d.mz, k = M.m - i * d.mz;
  M.kx = __ldg(d.kx + i);
  M.kz = __ldg(d.kz + k);
  M.k2 = __ldg(d.k2 + M.m);
  return true;
}

// the exact (FP64) 00 coefficient of transform output o at row j (mixed forms)
__device__ __forceinline__ double2 mo00_row(const Dev &d, int o, int j) {
  return make_double2(d.mo_cur[(size_t)o * d.my + j] / ((double)d.mgalx * (double)d.mgalz), 0.0);
}

// ----------------------------------------------------------------------
// (1) Lapvdvhom: phi -> m_y, dm_y/dy (cross.f:329-335, 365-372)
// ----------------------------------------------------------------------
template <typename CT>
__global__ void __launch_bounds__(TB) t_lapv(Dev d) {
  Mode M;
  if (!mode_of(d, M)) return;
  const int my = d.my;
  const size_t ld = d.nmode;
  const bool zero = M.k2 == 0.0;
  double2 *s1 = d.ws[0] + M.m, *s2 = d.ws[1] + M.m;
  CT *MY = wsb<CT>(d, SB_MY) + M.m, *DMY = wsb<CT>(d, SB_DMY) + M.m;
  {  // forward Poisson half; phi with its wall values set to zero
    Rd<double2, 8> r;
    r.start(d.phi + M.m, ld, my, 1, 0);
    LRows<8> L;
    L.start(d, M.m);
    Win w;
    w.clear();
    Hist h;
    h.clear();
    for (int t = 0; t < 3; t++) {
      const double2 v = r.pop();
      w.push(t == 0 ? czero() : v);
    }
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      const double2 v = r.pop();
      w.push(j + 3 == my - 1 ? czero() : v);
      s1[(size_t)j * ld] = pf(d, j, w, h, L);
    }
  }
  {  // backward Poisson half -> m_y
    Rd<double2, 8> r;
    r.start(s1, ld, my, -1, my - 1);
    URows<8> U;
    U.start(d, M.m);
    Hist h;
    h.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) {
      double2 x = pb(r.pop(), h, U);
      if (zero) x = czero();
      put(MY, ld, j, x);
      s2[(size_t)j * ld] = x;
    }
  }
  {  // forward half of d/dy of m_y
    Rd<double2, 8> r;
    r.start(s2, ld, my, 1, 0);
    Win w;
    w.clear();
    Hist h;
    h.clear();
    for (int t = 0; t < 3; t++) w.push(r.pop());
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      w.push(r.pop());
      s1[(size_t)j * ld] = d1f(d, j, w, h);
    }
  }
  {  // backward half -> dm_y/dy
    Rd<double2, 8> r;
    r.start(s1, ld, my, -1, my - 1);
    Hist h;
    h.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) put(DMY, ld, j, d1b(d, j, r.pop(), h));
  }
}

// ----------------------------------------------------------------------
// (2)-(3) m_x, m_z, rho u_i, xi-updates of Omega_y and phi, 00 modes
// (cross.f:315-327, 395-499)
// ----------------------------------------------------------------------
// V: the 2014 variant (trunk/lomacte/src/cross.f:293-461): d(Omega_y)/dy = 0
// through two rows at each wall for m_x, m_z only, Omega_y** from the raw
// Omega_y, and T, T** and Delta T from the spectral RHS(T).
template <typename CT, bool V>
__global__ void __launch_bounds__(TB) t_assemble(Dev d, int rk) {
  Mode M;
  if (!mode_of(d, M)) return;
  const int my = d.my;
  const size_t ld = d.nmode;
  const double dtxi = d.scal_d[0] * d.xi[rk];
  const double ta = (M.k2 != 0.0) ? M.kx / M.k2 : 0.0, tb = (M.k2 != 0.0) ? M.kz / M.k2 : 0.0;
  const bool m00 = M.m == 0;
  double2 *s1 = d.ws[0] + M.m;
  {
    Rd<double2, 3> rvor, rrom, rphi, rrph;
    Rd<CT, kq<CT>(3)> rdmy;
    Rd<double2, 4> rpsi;
    rvor.start(d.vor + M.m, ld, my, 1, 0);
    rrom.start(d.Rom + M.m, ld, my, 1, 0);
    rphi.start(d.phi + M.m, ld, my, 1, 0);
    rrph.start(d.Rphi + M.m, ld, my, 1, 0);
    rdmy.start(wsb<CT>(d, SB_DMY) + M.m, ld, my, 1, 0);
    rpsi.start(d.psi + M.m, ld, my, 1, 0);
    CT *RU = wsb<CT>(d, SB_RU) + M.m, *RW = wsb<CT>(d, SB_RW) + M.m;
    const double2 vor1 = __ldg(d.vor + ld + M.m);  // wall BC of Omega_y, cross.f:315-327
    const double2 vor2 = __ldg(d.vor + 2 * ld + M.m);
    double2 vprev = czero(), vprev2 = czero();
    Rd<double2, 3> rT, rRT;
    if constexpr (V) {
      rT.start(d.scal + M.m, ld, my, 1, 0);
      rRT.start(d.RT + M.m, ld, my, 1, 0);
    }
    Win w;
    w.clear();
    Hist h;
    h.clear();
    for (int t = 0; t < 3; t++) w.push(rpsi.pop());
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      w.push(rpsi.pop());
      const double2 ps = w.c();
      const double2 vr = rvor.pop();
      double2 vo;
      if constexpr (V) {  // lomacte/cross.f:306-311
        vo = (j <= 1) ? vor2 : (j >= my - 2) ? (j == my - 2 ? vprev : vprev2) : vr;
        if (j == my - 2) vprev2 = vprev;
      } else {
        vo = (j == 0) ? vor1 : (j == my - 1) ? vprev : vr;
      }
      vprev = vr;
      const double2 a = rdmy.pop();
      double2 b = cadd(csub(cik(ta, a), cik(tb, vo)), cik(M.kx, ps));   // rho u, cross.f:402,467
      double2 c = cadd(cadd(cik(tb, a), cik(ta, vo)), cik(M.kz, ps));   // rho w, cross.f:404,469
      if (m00) {  // 00 modes injected (cross.f:486-491), then u00**, w00** (cross.f:495-498)
        b = make_double2(d.u00[j], 0.0);
        c = make_double2(d.w00[j], 0.0);
        if constexpr (mixed<CT>()) {
          d.mi[j] = b.x;
          d.mi[(size_t)2 * my + j] = c.x;
        }
        if (j >= 1 && j <= my - 2) {
          d.u00[j] += dtxi * d.rf0u[j];
          d.w00[j] += dtxi * d.rf0w[j];
        }
      }
      put(RU, ld, j, b);
      put(RW, ld, j, c);
      put(d.vor + M.m, ld, j, cadd(V ? vr : vo, cscale(dtxi, rrom.pop())));  // cross.f:420-424
      if constexpr (V) {  // T saved, T** and Delta T: lomacte/cross.f:368-396
        const double2 T = rT.pop(), inc = cscale(dtxi, rRT.pop());
        put(d.Told + M.m, ld, j, T);
        put(d.scal + M.m, ld, j, cadd(T, inc));
        put(d.dTs + M.m, ld, j, inc);
      }
      double2 ph = rphi.pop();
      if (j == 0 || j == my - 1) ph = czero();
      put(d.phi + M.m, ld, j, cadd(ph, cscale(dtxi, rrph.pop())));  // cross.f:424-425
      s1[(size_t)j * ld] = d1f(d, j, w, h);
    }
  }
  {  // rho v = m_y + d(psi)/dy (cross.f:434-437, 471)
    Rd<double2, 4> r;
    Rd<CT, kq<CT>(4)> rmy;
    r.start(s1, ld, my, -1, my - 1);
    rmy.start(wsb<CT>(d, SB_MY) + M.m, ld, my, -1, my - 1);
    CT *RV = wsb<CT>(d, SB_RV) + M.m;
    Hist h;
    h.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) {
      double2 a = cadd(d1b(d, j, r.pop(), h), rmy.pop());
      if (m00) {
        a = make_double2(d.v00[j], 0.0);
        if constexpr (mixed<CT>()) d.mi[(size_t)my + j] = a.x;
      }
      put(RV, ld, j, a);
    }
  }
}

// ----------------------------------------------------------------------
// (4) T with its wall BCs, dT/dy, lap(T) (cross.f:336-349, 521-541)
// ----------------------------------------------------------------------
// V: the 2014 variant differentiates the T saved before its update, with
// no wall values imposed (lomacte/cross.f:486-519).
template <typename CT, bool V>
__global__ void __launch_bounds__(TB) t_tder(Dev d) {
  Mode M;
  if (!mode_of(d, M)) return;
  const int my = d.my;
  const size_t ld = d.nmode;
  const bool m00 = M.m == 0;
  double2 *s1 = d.ws[2] + M.m, *s2 = d.ws[3] + M.m;  // 2, 3: runs beside lapv/assemble
  double2 *const Tsrc = V ? d.Told : d.scal;
  {
    Rd<double2, 8> r;
    r.start(Tsrc + M.m, ld, my, 1, 0);
    const double2 v0 = r.pop();
    const double2 wb = V ? v0 : (m00 ? make_double2(1.0 / d.scal_d[3], 0.0) : czero());
    const double2 wt_bc = m00 ? make_double2(1.0 / d.scal_d[4], 0.0) : czero();
    Win w;
    w.clear();
    Hist h1, h2;
    h1.clear();
    h2.clear();
    w.push(wb);
    for (int t = 1; t < 3; t++) w.push(r.pop());
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      const double2 v = r.pop();
      w.push((!V && j + 3 == my - 1) ? wt_bc : v);
      const double2 T = w.c();
      if constexpr (!V) put(d.scal + M.m, ld, j, T);
      if constexpr (mixed<CT>()) {
        put(wsb<CT>(d, SB_T32) + M.m, ld, j, T);
        if (m00) d.mi[(size_t)5 * my + j] = T.x;
      }
      s1[(size_t)j * ld] = d1f(d, j, w, h1);
      s2[(size_t)j * ld] = d2f(d, j, w, h2);
    }
  }
  {
    Rd<double2, 4> r1, r2, rT;
    r1.start(s1, ld, my, -1, my - 1);
    r2.start(s2, ld, my, -1, my - 1);
    rT.start(Tsrc + M.m, ld, my, -1, my - 1);
    CT *DY = wsb<CT>(d, SB_DTDY) + M.m, *LT = wsb<CT>(d, SB_LAPT) + M.m;
    Hist h1, h2;
    h1.clear();
    h2.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) {
      const double2 dT = d1b(d, j, r1.pop(), h1);
      const double2 lT = csub(d2b(d, j, r2.pop(), h2), cscale(M.k2, rT.pop()));
      if constexpr (mixed<CT>())
        if (m00) {
          d.mi[(size_t)4 * my + j] = dT.x;
          d.mi[(size_t)3 * my + j] = lT.x;
        }
      put(DY, ld, j, dT);
      put(LT, ld, j, lT);
    }
  }
}

// ----------------------------------------------------------------------
// Passive scalar Z, treated as t_tder treats T: zero at the walls except
// the 00 mode (held at scal_d[5], scal_d[6]), dZ/dy and lap Z for the
// transforms, an FP32 copy of Z in the mixed forms (the z transforms form
// dZ/dx, dZ/dz from it) and its 00 profiles (mi rows 6, 7).  Runs after
// t_tder on the second stream and shares its scratch fields.
// ----------------------------------------------------------------------
template <typename CT>
__global__ void __launch_bounds__(TB) t_zder(Dev d) {
  Mode M;
  if (!mode_of(d, M)) return;
  const int my = d.my;
  const size_t ld = d.nmode;
  const bool m00 = M.m == 0;
  double2 *s1 = d.ws[2] + M.m, *s2 = d.ws[3] + M.m;
  {
    Rd<double2, 8> r;
    r.start(d.zsc + M.m, ld, my, 1, 0);
    r.pop();
    const double2 wb = m00 ? make_double2(d.scal_d[5], 0.0) : czero();
    const double2 wt_bc = m00 ? make_double2(d.scal_d[6], 0.0) : czero();
    Win w;
    w.clear();
    Hist h1, h2;
    h1.clear();
    h2.clear();
    w.push(wb);
    for (int t = 1; t < 3; t++) w.push(r.pop());
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      const double2 v = r.pop();
      w.push(j + 3 == my - 1 ? wt_bc : v);
      const double2 Z = w.c();
      put(d.zsc + M.m, ld, j, Z);
      if constexpr (mixed<CT>()) put(wsb<CT>(d, SB_Z32) + M.m, ld, j, Z);
      s1[(size_t)j * ld] = d1f(d, j, w, h1);
      s2[(size_t)j * ld] = d2f(d, j, w, h2);
    }
  }
  {
    Rd<double2, 4> r1, r2, rZ;
    r1.start(s1, ld, my, -1, my - 1);
    r2.start(s2, ld, my, -1, my - 1);
    rZ.start(d.zsc + M.m, ld, my, -1, my - 1);
    CT *DY = wsb<CT>(d, SB_DZDY) + M.m, *LZ = wsb<CT>(d, SB_LAPZ) + M.m;
    Hist h1, h2;
    h1.clear();
    h2.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) {
      const double2 dZ = d1b(d, j, r1.pop(), h1);
      const double2 lZ = csub(d2b(d, j, r2.pop(), h2), cscale(M.k2, rZ.pop()));
      if constexpr (mixed<CT>())
        if (m00) {
          d.mi[(size_t)7 * my + j] = dZ.x;
          d.mi[(size_t)6 * my + j] = lZ.x;
        }
      put(DY, ld, j, dZ);
      put(LZ, ld, j, lZ);
    }
  }
}

// Z += Delta Z (the scalar's counterpart of cross.f:619-627); the mixed
// forms take the exact FP64 00 mode of Delta Z from the plane sums
template <typename CT>
__global__ void __launch_bounds__(TB) t_zupd(Dev d) {
  Mode M;
  if (!mode_of(d, M)) return;
  const int my = d.my;
  const size_t ld = d.nmode;
  Rd<double2, 4> rz;
  Rd<CT, kq<CT>(4)> rd;
  rz.start(d.zsc + M.m, ld, my, 1, 0);
  rd.start(wsb<CT>(d, ODZ) + M.m, ld, my, 1, 0);
  #pragma unroll 4
  for (int j = 0; j < my; j++) {
    double2 dz = rd.pop();
    if constexpr (mixed<CT>())
      if (M.m == 0) dz = mo00_row(d, ODZ, j);
    put(d.zsc + M.m, ld, j, cadd(rz.pop(), dz));
  }
}

// ----------------------------------------------------------------------
// Variable viscosity: the spectral inputs of the strain rates.  In
// physical space d(u_i)/dx_j = T d(rho u_i)/dx_j + rho u_i dT/dx_j, and the
// stress needs d(rho u_i)/dx_j only in the symmetric sums; this kernel
// writes d(rho v)/dy and the three off-diagonal sums (d(rho u)/dx and
// d(rho w)/dz are formed by the inverse z transforms from rho u and rho w).
// The y derivatives are deryr2's (cfdiff.f:518-601), as every first y
// derivative of the substep.  Runs after t_assemble on the same stream;
// scratch fields 0, 1 and 4 hold the forward halves (2 and 3 belong to
// t_tder / t_zder on the second stream, 4 is free until the psi solve).
// The mixed forms also form the 00 profiles of the results exactly, from
// the FP64 profiles of rho u_i (mi rows 0..2) into mi rows 8..10.
// ----------------------------------------------------------------------
// an FP64 profile read as a pencil (imaginary parts zero)
struct RdM {
  RdS<4> s;
  __device__ __forceinline__ void start(const double *p, int my, int dir, int first) { s.start(p, 1, my, dir, first); }
  __device__ __forceinline__ double2 pop() { return make_double2(s.pop(), 0.0); }
};

// d/dy of the three pencils (forward halves into s0, s1, s2, then the
// backward halves), sink(j, du, dv, dw, u, v, w) per row, j descending;
// start(reader, field 0..2, direction, first row) opens the readers
template <typename RT, typename Start, typename Sink>
__device__ __forceinline__ void sgrad_pass(const Dev &d, size_t ld, double2 *s0, double2 *s1, double2 *s2,
                                           Start start, Sink sink) {
  const int my = d.my;
  {
    RT ru, rv, rw;
    start(ru, 0, 1, 0);
    start(rv, 1, 1, 0);
    start(rw, 2, 1, 0);
    Win wu, wv, ww;
    wu.clear();
    wv.clear();
    ww.clear();
    Hist hu, hv, hw;
    hu.clear();
    hv.clear();
    hw.clear();
    for (int t = 0; t < 3; t++) {
      wu.push(ru.pop());
      wv.push(rv.pop());
      ww.push(rw.pop());
    }
    #pragma unroll 2
    for (int j = 0; j < my; j++) {
      wu.push(ru.pop());
      wv.push(rv.pop());
      ww.push(rw.pop());
      s0[(size_t)j * ld] = d1f(d, j, wu, hu);
      s1[(size_t)j * ld] = d1f(d, j, wv, hv);
      s2[(size_t)j * ld] = d1f(d, j, ww, hw);
    }
  }
  Rd<double2, 3> r0, r1, r2;
  r0.start(s0, ld, my, -1, my - 1);
  r1.start(s1, ld, my, -1, my - 1);
  r2.start(s2, ld, my, -1, my - 1);
  RT ru, rv, rw;
  start(ru, 0, -1, my - 1);
  start(rv, 1, -1, my - 1);
  start(rw, 2, -1, my - 1);
  Hist hu, hv, hw;
  hu.clear();
  hv.clear();
  hw.clear();
  #pragma unroll 2
  for (int j = my - 1; j >= 0; j--) {
    const double2 du = d1b(d, j, r0.pop(), hu), dv = d1b(d, j, r1.pop(), hv), dw = d1b(d, j, r2.pop(), hw);
    sink(j, du, dv, dw, ru.pop(), rv.pop(), rw.pop());
  }
}

// The mixed forms launch one block more than the pencils need: its first
// thread runs the exact 00 profiles (mi rows 0..2 into rows 8..10, scratch
// vscr) beside the pencils; the FP32 buffers' 00 coefficients are not read
// (the transforms drop them).
template <typename CT>
__global__ void __launch_bounds__(TB) t_sgrad(Dev d) {
  const int my = d.my;
  if constexpr (mixed<CT>()) {
    if (blockIdx.x == gridDim.x - 1) {
      if (threadIdx.x != 0) return;
      sgrad_pass<RdM>(
          d, 1, d.vscr, d.vscr + my, d.vscr + 2 * my,
          [&](auto &r, int f, int dir, int first) { r.start(d.mi + (size_t)f * my, my, dir, first); },
          [&](int j, double2 du, double2 dv, double2 dw, double2, double2, double2) {
            d.mi[(size_t)8 * my + j] = dv.x;
            d.mi[(size_t)9 * my + j] = du.x;
            d.mi[(size_t)10 * my + j] = dw.x;
          });
      return;
    }
  }
  Mode M;
  if (!mode_of(d, M)) return;
  const size_t ld = d.nmode;
  double2 *s0 = d.ws[0] + M.m, *s1 = d.ws[1] + M.m, *s2 = d.ws[4] + M.m;
  const CT *src[3] = {wsb<CT>(d, SB_RU) + M.m, wsb<CT>(d, SB_RV) + M.m, wsb<CT>(d, SB_RW) + M.m};
  CT *GYY = wsb<CT>(d, SB_GYY) + M.m, *G12 = wsb<CT>(d, SB_G12) + M.m;
  CT *G13 = wsb<CT>(d, SB_G13) + M.m, *G23 = wsb<CT>(d, SB_G23) + M.m;
  sgrad_pass<Rd<CT, kq<CT>(3)>>(
      d, ld, s0, s1, s2, [&](auto &r, int f, int dir, int first) { r.start(src[f], ld, my, dir, first); },
      [&](int j, double2 du, double2 dv, double2 dw, double2 u, double2 v, double2 w) {
        put(GYY, ld, j, dv);
        put(G12, ld, j, cadd(du, cik(M.kx, v)));
        put(G13, ld, j, cadd(cik(M.kz, u), cik(M.kx, w)));
        put(G23, ld, j, cadd(cik(M.kz, v), dw));
      });
}

// ----------------------------------------------------------------------
// Physical-field export (lmc_physical_f64), FP64: the transform inputs of
// tofis_loma's escrphys quantities from the state, without writing it:
// rho u_i assembled as the substep does (the wall conditions of Omega_y and
// phi, cross.f:315-335, then cross.f:395-499 with xi = 0), T and Z as
// stored (as tofis_loma reads them), grad T, and C = curl(rho u).  Reads
// m_y, dm_y/dy from SB_MY, SB_DMY (launch_lapv before); writes the export
// slots xslot(0..10) (lmc_kernels.cuh); scratch ws[0..3].
// ----------------------------------------------------------------------
__global__ void __launch_bounds__(TB) t_xprep(Dev d) {
  Mode M;
  if (!mode_of(d, M)) return;
  const int my = d.my;
  const size_t ld = d.nmode;
  const bool m00 = M.m == 0;
  const double ta = (M.k2 != 0.0) ? M.kx / M.k2 : 0.0, tb = (M.k2 != 0.0) ? M.kz / M.k2 : 0.0;
  double2 *s0 = d.ws[0] + M.m, *s1 = d.ws[1] + M.m, *s2 = d.ws[2] + M.m, *s3 = d.ws[3] + M.m;
  double2 *F[11];
  for (int q = 0; q < 11; q++) F[q] = d.sb[xslot(q)] + M.m;
  const double2 vor1 = d.vor[ld + M.m], vorn = d.vor[(size_t)(my - 2) * ld + M.m];  // cross.f:315-327
  {
    Rd<double2, 3> rpsi, rT, rvor, rdmy;
    rpsi.start(d.psi + M.m, ld, my, 1, 0);
    rT.start(d.scal + M.m, ld, my, 1, 0);
    rvor.start(d.vor + M.m, ld, my, 1, 0);
    rdmy.start(d.sb[SB_DMY] + M.m, ld, my, 1, 0);
    Win wp, wt, wu, ww;
    wp.clear();
    wt.clear();
    wu.clear();
    ww.clear();
    Hist hp, ht, hu, hw;
    hp.clear();
    ht.clear();
    hu.clear();
    hw.clear();
    // row r of rho u, rho w (the psi value of row r is the newest in wp)
    auto ru_rw = [&](int r, double2 ps, double2 &ru, double2 &rw) {
      const double2 a = rdmy.pop(), vr = rvor.pop();
      const double2 vo = r == 0 ? vor1 : r == my - 1 ? vorn : vr;
      ru = cadd(csub(cik(ta, a), cik(tb, vo)), cik(M.kx, ps));
      rw = cadd(cadd(cik(tb, a), cik(ta, vo)), cik(M.kz, ps));
      if (m00) {
        const bool in = r >= 0 && r < my;
        ru = make_double2(in ? d.u00[r] : 0.0, 0.0);
        rw = make_double2(in ? d.w00[r] : 0.0, 0.0);
      }
      if (r >= my) ru = rw = czero();
    };
    for (int r = 0; r < 3; r++) {
      const double2 ps = rpsi.pop();
      wp.push(ps);
      wt.push(rT.pop());
      double2 ru, rw;
      ru_rw(r, ps, ru, rw);
      wu.push(ru);
      ww.push(rw);
    }
    #pragma unroll 1
    for (int j = 0; j < my; j++) {
      const int r = j + 3;
      const double2 ps = rpsi.pop();
      wp.push(ps);
      wt.push(rT.pop());
      double2 ru, rw;
      ru_rw(r, ps, ru, rw);
      wu.push(ru);
      ww.push(rw);
      const double2 T = wt.c();
      put(F[0], ld, j, wu.c());
      put(F[2], ld, j, ww.c());
      put(F[3], ld, j, T);
      put(F[4], ld, j, cik(M.kx, T));
      put(F[6], ld, j, cik(M.kz, T));
      s0[(size_t)j * ld] = d1f(d, j, wp, hp);
      s1[(size_t)j * ld] = d1f(d, j, wt, ht);
      s2[(size_t)j * ld] = d1f(d, j, wu, hu);
      s3[(size_t)j * ld] = d1f(d, j, ww, hw);
    }
  }
  Rd<double2, 3> r0, r1, r2, r3, rmy, ru, rw;
  r0.start(s0, ld, my, -1, my - 1);
  r1.start(s1, ld, my, -1, my - 1);
  r2.start(s2, ld, my, -1, my - 1);
  r3.start(s3, ld, my, -1, my - 1);
  rmy.start(d.sb[SB_MY] + M.m, ld, my, -1, my - 1);
  ru.start(F[0], ld, my, -1, my - 1);
  rw.start(F[2], ld, my, -1, my - 1);
  Hist hp, ht, hu, hw;
  hp.clear();
  ht.clear();
  hu.clear();
  hw.clear();
  #pragma unroll 1
  for (int j = my - 1; j >= 0; j--) {
    double2 rv = cadd(d1b(d, j, r0.pop(), hp), rmy.pop());  // cross.f:434-437, 471
    if (m00) rv = make_double2(d.v00[j], 0.0);
    const double2 Ty = d1b(d, j, r1.pop(), ht), dudy = d1b(d, j, r2.pop(), hu), dwdy = d1b(d, j, r3.pop(), hw);
    const double2 u = ru.pop(), w = rw.pop();
    put(F[1], ld, j, rv);
    put(F[5], ld, j, Ty);
    put(F[7], ld, j, csub(dwdy, cik(M.kz, rv)));
    put(F[8], ld, j, csub(cik(M.kz, u), cik(M.kx, w)));
    put(F[9], ld, j, csub(cik(M.kx, rv), dudy));
    if (d.scalar) put(F[10], ld, j, d.zsc[(size_t)j * ld + M.m]);
  }
}

// ----------------------------------------------------------------------
// (6a)-(6b) T update and N_i (cross.f:619-682); rf0u / rf0w get the 00
// pencils of d(rho uv)/dy and d(rho vw)/dy for the 00 tail.
// ----------------------------------------------------------------------
// V: the 2014 variant advances the spectral T with this substep's RHS(T)
// (in the d(rho)/dt slot) and accumulates Delta T (lomacte/cross.f:563-570).
template <typename CT, bool V>
__global__ void __launch_bounds__(TB) t_post1(Dev d, int rk) {
  Mode M;
  if (!mode_of(d, M)) return;
  const int my = d.my;
  const size_t ld = d.nmode;
  const bool m00 = M.m == 0;
  const double dtg = d.scal_d[0] * d.gama[rk];
  double2 *s1 = d.ws[0] + M.m, *s2 = d.ws[1] + M.m, *s3 = d.ws[2] + M.m;
  {
    Rd<double2, 2> rT;
    Rd<CT, kq<CT>(2)> rDT;
    Rd<CT, kq<CT>(3)> rvv, ruv, rvw;
    rT.start(d.scal + M.m, ld, my, 1, 0);
    rDT.start(wsb<CT>(d, V ? ODRHO : ODT) + M.m, ld, my, 1, 0);
    Rd<double2, 2> rdT;
    if constexpr (V) rdT.start(d.dTs + M.m, ld, my, 1, 0);
    rvv.start(wsb<CT>(d, ORVV) + M.m, ld, my, 1, 0);
    ruv.start(wsb<CT>(d, ORUV) + M.m, ld, my, 1, 0);
    rvw.start(wsb<CT>(d, ORVW) + M.m, ld, my, 1, 0);
    Win wvv, wuv, wvw;
    wvv.clear();
    wuv.clear();
    wvw.clear();
    Hist h1, h2, h3;
    h1.clear();
    h2.clear();
    h3.clear();
    auto feed = [&](int r) {  // row r of the three derivative inputs
      double2 a = rvv.pop(), b = ruv.pop(), c = rvw.pop();
      if constexpr (mixed<CT>())
        if (m00 && r < my) {
          b = mo00_row(d, ORUV, r);
          c = mo00_row(d, ORVW, r);
        }
      wvv.push(a);
      wuv.push(b);
      wvw.push(c);
    };
    for (int t = 0; t < 3; t++) feed(t);
    #pragma unroll 2
    for (int j = 0; j < my; j++) {
      feed(j + 3);
      double2 dT = rDT.pop();
      if constexpr (mixed<CT>())
        if (m00) dT = mo00_row(d, ODT, j);
      if constexpr (V) {
        put(d.RT + M.m, ld, j, dT);
        put(d.dTs + M.m, ld, j, cadd(rdT.pop(), cscale(dtg, dT)));
        dT = cscale(dtg, dT);
      }
      put(d.scal + M.m, ld, j, cadd(rT.pop(), dT));  // cross.f:619-627
      s1[(size_t)j * ld] = d1f(d, j, wvv, h1);
      s2[(size_t)j * ld] = d1f(d, j, wuv, h2);
      s3[(size_t)j * ld] = d1f(d, j, wvw, h3);
    }
  }
  {
    Rd<double2, 2> r1, r2, r3;
    Rd<CT, kq<CT>(2)> ruv, rvw, ruu, ruw, rww;
    r1.start(s1, ld, my, -1, my - 1);
    r2.start(s2, ld, my, -1, my - 1);
    r3.start(s3, ld, my, -1, my - 1);
    CT *VV = wsb<CT>(d, ORVV) + M.m, *UU = wsb<CT>(d, ORUU) + M.m, *WW = wsb<CT>(d, ORWW) + M.m;
    ruv.start(wsb<CT>(d, ORUV) + M.m, ld, my, -1, my - 1);
    rvw.start(wsb<CT>(d, ORVW) + M.m, ld, my, -1, my - 1);
    ruu.start(UU, ld, my, -1, my - 1);
    ruw.start(wsb<CT>(d, ORUW) + M.m, ld, my, -1, my - 1);
    rww.start(WW, ld, my, -1, my - 1);
    Hist h1, h2, h3;
    h1.clear();
    h2.clear();
    h3.clear();
    #pragma unroll 2
    for (int j = my - 1; j >= 0; j--) {
      const double2 dvv = d1b(d, j, r1.pop(), h1), duv = d1b(d, j, r2.pop(), h2), dvw = d1b(d, j, r3.pop(), h3);
      const double2 uv = ruv.pop(), vw = rvw.pop(), uu = ruu.pop(), uw = ruw.pop(), ww = rww.pop();
      if (m00) {
        d.rf0u[j] = duv.x;
        d.rf0w[j] = dvw.x;
      }
      put(VV, ld, j, csub(czero(), cadd(cadd(dvv, cik(M.kx, uv)), cik(M.kz, vw))));  // N_y
      put(UU, ld, j, csub(czero(), cadd(cadd(duv, cik(M.kx, uu)), cik(M.kz, uw))));  // N_x
      put(WW, ld, j, csub(czero(), cadd(cadd(dvw, cik(M.kx, uw)), cik(M.kz, ww))));  // N_z
    }
  }
}

// ----------------------------------------------------------------------
// (6c)-(9) vorticity, the two Laplacians, RHS(Omega_y), RHS(phi) and the
// RK3 update (cross.f:748-981)
// ----------------------------------------------------------------------
template <typename CT>
__global__ void __launch_bounds__(TB) t_post2(Dev d, int rk) {
  Mode M;
  if (!mode_of(d, M)) return;
  const int my = d.my;
  const size_t ld = d.nmode;
  const double kx = M.kx, kz = M.kz, k2 = M.k2;
  const double dtg = d.scal_d[0] * d.gama[rk];
  double2 *s1 = d.ws[0] + M.m, *s2 = d.ws[1] + M.m, *s3 = d.ws[2] + M.m, *s4 = d.ws[3] + M.m;
  {  // forward halves of dw/dy, du/dy and d2(omega_y)/dy2
    Rd<CT, kq<CT>(4)> ru, rw;
    ru.start(wsb<CT>(d, OU) + M.m, ld, my, 1, 0);
    rw.start(wsb<CT>(d, OW) + M.m, ld, my, 1, 0);
    Win wu, ww, wy;
    wu.clear();
    ww.clear();
    wy.clear();
    Hist h1, h2, h3;
    h1.clear();
    h2.clear();
    h3.clear();
    auto feed = [&]() {
      const double2 u = ru.pop(), w = rw.pop();
      wu.push(u);
      ww.push(w);
      wy.push(csub(cik(kz, u), cik(kx, w)));  // omega_y, cross.f:760
    };
    for (int t = 0; t < 3; t++) feed();
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      feed();
      s1[(size_t)j * ld] = d1f(d, j, ww, h1);
      s2[(size_t)j * ld] = d1f(d, j, wu, h2);
      s3[(size_t)j * ld] = d2f(d, j, wy, h3);
    }
  }
  {  // forward half of d/dy of i kx N_x + i kz N_z (cross.f:900-907)
    Rd<CT, kq<CT>(4)> rx, rz;
    rx.start(wsb<CT>(d, ORUU) + M.m, ld, my, 1, 0);
    rz.start(wsb<CT>(d, ORWW) + M.m, ld, my, 1, 0);
    Win wc;
    wc.clear();
    Hist h;
    h.clear();
    for (int t = 0; t < 3; t++) wc.push(cadd(cik(kx, rx.pop()), cik(kz, rz.pop())));
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      wc.push(cadd(cik(kx, rx.pop()), cik(kz, rz.pop())));
      s4[(size_t)j * ld] = d1f(d, j, wc, h);
    }
  }
  {  // omega_x, omega_z, (curl omega)_y -> s1
    Rd<double2, 4> r1, r2;
    Rd<CT, kq<CT>(4)> rv;
    r1.start(s1, ld, my, -1, my - 1);
    r2.start(s2, ld, my, -1, my - 1);
    rv.start(wsb<CT>(d, OV) + M.m, ld, my, -1, my - 1);
    Hist h1, h2;
    h1.clear();
    h2.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) {
      const double2 dw = d1b(d, j, r1.pop(), h1), du = d1b(d, j, r2.pop(), h2), v = rv.pop();
      const double2 ox = csub(dw, cik(kz, v));                 // cross.f:757
      const double2 oz = csub(cik(kx, v), du);                 // cross.f:763
      s1[(size_t)j * ld] = csub(cik(kz, ox), cik(kx, oz));     // cross.f:839
    }
  }
  {  // RHS(Omega_y), Omega_y update; d/dy part of RHS(phi) (cross.f:885-917, 966-981)
    Rd<double2, 2> r3, r4, rvo;
    Rd<CT, kq<CT>(2)> ru, rw, rx, rz, ry;
    r3.start(s3, ld, my, -1, my - 1);
    r4.start(s4, ld, my, -1, my - 1);
    rvo.start(d.vor + M.m, ld, my, -1, my - 1);
    ru.start(wsb<CT>(d, OU) + M.m, ld, my, -1, my - 1);
    rw.start(wsb<CT>(d, OW) + M.m, ld, my, -1, my - 1);
    rx.start(wsb<CT>(d, ORUU) + M.m, ld, my, -1, my - 1);
    rz.start(wsb<CT>(d, ORWW) + M.m, ld, my, -1, my - 1);
    ry.start(wsb<CT>(d, ORVV) + M.m, ld, my, -1, my - 1);
    Hist h3, h4;
    h3.clear();
    h4.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) {
      const double2 u = ru.pop(), w = rw.pop(), nx = rx.pop(), nz = rz.pop(), ny = ry.pop();
      const double2 oy = csub(cik(kz, u), cik(kx, w));
      const double2 lw = csub(d2b(d, j, r3.pop(), h3), cscale(k2, oy));                   // cross.f:822-832
      const double2 rom = cadd(csub(cik(kz, nx), cik(kx, nz)), cscale(d.ire, lw));        // cross.f:889
      put(d.Rom + M.m, ld, j, rom);
      put(d.vor + M.m, ld, j, cadd(rvo.pop(), cscale(dtg, rom)));                         // cross.f:969
      const double2 dc = d1b(d, j, r4.pop(), h4);
      put(d.Rphi + M.m, ld, j, csub(cscale(-k2, ny), dc));
    }
  }
  {  // forward half of d2/dy2 of (curl omega)_y
    Rd<double2, 8> r;
    r.start(s1, ld, my, 1, 0);
    Win w;
    w.clear();
    Hist h;
    h.clear();
    for (int t = 0; t < 3; t++) w.push(r.pop());
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      w.push(r.pop());
      s2[(size_t)j * ld] = d2f(d, j, w, h);
    }
  }
  {  // lap(curl omega)_y, RHS(phi), phi update (cross.f:847-857, 917, 978)
    Rd<double2, 3> r2, rc, rrp, rph;
    r2.start(s2, ld, my, -1, my - 1);
    rc.start(s1, ld, my, -1, my - 1);
    rrp.start(d.Rphi + M.m, ld, my, -1, my - 1);
    rph.start(d.phi + M.m, ld, my, -1, my - 1);
    Hist h;
    h.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) {
      const double2 lc = csub(d2b(d, j, r2.pop(), h), cscale(k2, rc.pop()));
      const double2 rp = csub(rrp.pop(), cscale(d.ire, lc));
      put(d.Rphi + M.m, ld, j, rp);
      put(d.phi + M.m, ld, j, cadd(rph.pop(), cscale(dtg, rp)));
    }
  }
}

// ----------------------------------------------------------------------
// (8) psi^{n+1} by solvepsi (cross.f:1092-1104, laps.f:580-730)
// ----------------------------------------------------------------------
// V: the 2014 variant solves the Dirichlet problem for
// psi = -d(rho) / (Deltat (gamma + xi)) (lomacte/cross.f:970-983).
template <typename CT, bool V>
__global__ void __launch_bounds__(TB) t_psi(Dev d, int rk) {
  Mode M;
  if (!mode_of(d, M)) return;
  const int my = d.my;
  const size_t ld = d.nmode;
  double2 *s1 = d.ws[4] + M.m;  // its own scratch: runs beside post1 and post2
  const double sc = V ? -1.0 / (d.scal_d[0] * (d.gama[rk] + d.xi[rk])) : 1.0;
  {
    Rd<CT, kq<CT>(8)> r;
    r.start(wsb<CT>(d, ODRHO) + M.m, ld, my, 1, 0);
    LRows<8> L;
    L.start(d, M.m);
    Win w;
    w.clear();
    Hist h;
    h.clear();
    for (int t = 0; t < 3; t++) w.push(cscale(sc, r.pop()));
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      w.push(cscale(sc, r.pop()));
      s1[(size_t)j * ld] = pf(d, j, w, h, L);
    }
  }
  if constexpr (V) {
    const bool zero = M.k2 == 0.0;
    Rd<double2, 8> r;
    r.start(s1, ld, my, -1, my - 1);
    URows<8> U;
    U.start(d, M.m);
    Hist h;
    h.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) {
      const double2 x = pb(r.pop(), h, U);
      put(d.psi + M.m, ld, j, zero ? czero() : x);
    }
    return;
  }
  double2 db = czero(), dt = czero();
  {
    Rd<double2, 8> r;
    r.start(s1, ld, my, -1, my - 1);
    URows<8> U;
    U.start(d, M.m);
    Hist h;
    h.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) {
      const double2 x = pb(r.pop(), h, U);
      const double eb = __ldg(d.r_ebot + j), et = __ldg(d.r_etop + j);
      db.x = fma(eb, x.x, db.x);
      db.y = fma(eb, x.y, db.y);
      dt.x = fma(et, x.x, dt.x);
      dt.y = fma(et, x.y, dt.y);
      s1[(size_t)j * ld] = x;
    }
  }
  {  // Neumann walls through the homogeneous solutions (laps.f:700-730)
    const double *ai = d.AAinv + (size_t)M.m * 4;
    const double a0 = __ldg(ai), a1 = __ldg(ai + 1), a2 = __ldg(ai + 2), a3 = __ldg(ai + 3);
    const double2 c1 = make_double2(-(a0 * db.x + a1 * dt.x), -(a0 * db.y + a1 * dt.y));
    const double2 c2 = make_double2(-(a2 * db.x + a3 * dt.x), -(a2 * db.y + a3 * dt.y));
    const bool zero = M.k2 == 0.0;
    Rd<double2, 8> r;
    r.start(s1, ld, my, 1, 0);
    const size_t n = (size_t)d.nmode;
    RdS<8> rv1, rv2;
    rv1.start(d.V12t + M.m, 2 * n, my, 1, 0);
    rv2.start(d.V12t + n + M.m, 2 * n, my, 1, 0);
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      double2 x = r.pop();
      const double v1 = rv1.pop(), v2 = rv2.pop();
      x.x += c1.x * v1 + c2.x * v2;
      x.y += c1.y * v1 + c2.y * v2;
      put(d.psi + M.m, ld, j, zero ? czero() : x);
    }
  }
}

// single y operator on FP64 device-layout fields (tests): 1 d/dy, 2 d2/dy2,
// 3 Lapvdvhom (out = v, out2 = dv/dy), 4 solvepsi
__global__ void __launch_bounds__(TB) t_op_y(Dev d, int op, const double2 *in, double2 *out, double2 *out2) {
  Mode M;
  if (!mode_of(d, M)) return;
  const int my = d.my;
  const size_t ld = d.nmode;
  const bool zero = M.k2 == 0.0;
  double2 *s1 = d.ws[0] + M.m, *s2 = d.ws[1] + M.m;
  in += M.m;
  out += M.m;
  {
    Rd<double2, 8> r;
    r.start(in, ld, my, 1, 0);
    Win w;
    w.clear();
    Hist h;
    h.clear();
    LRows<4> L;
    if (op >= 3) L.start(d, M.m);
    for (int t = 0; t < 3; t++) w.push(r.pop());
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      w.push(r.pop());
      s1[(size_t)j * ld] = op == 1 ? d1f(d, j, w, h) : op == 2 ? d2f(d, j, w, h) : pf(d, j, w, h, L);
    }
  }
  double2 db = czero(), dt = czero();
  {
    Rd<double2, 8> r;
    r.start(s1, ld, my, -1, my - 1);
    URows<4> U;
    if (op >= 3) U.start(d, M.m);
    Hist h;
    h.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) {
      const double2 w = r.pop();
      double2 x = op == 1 ? d1b(d, j, w, h) : op == 2 ? d2b(d, j, w, h) : pb(w, h, U);
      if (op == 4) {
        const double eb = __ldg(d.r_ebot + j), et = __ldg(d.r_etop + j);
        db.x = fma(eb, x.x, db.x);
        db.y = fma(eb, x.y, db.y);
        dt.x = fma(et, x.x, dt.x);
        dt.y = fma(et, x.y, dt.y);
      }
      if (op == 3 && zero) x = czero();
      out[(size_t)j * ld] = x;
      s2[(size_t)j * ld] = x;
    }
  }
  if (op == 3) {
    out2 += M.m;
    {
      Rd<double2, 8> r;
      r.start(s2, ld, my, 1, 0);
      Win w;
      w.clear();
      Hist h;
      h.clear();
      for (int t = 0; t < 3; t++) w.push(r.pop());
      #pragma unroll 4
      for (int j = 0; j < my; j++) {
        w.push(r.pop());
        s1[(size_t)j * ld] = d1f(d, j, w, h);
      }
    }
    Rd<double2, 8> r;
    r.start(s1, ld, my, -1, my - 1);
    Hist h;
    h.clear();
    #pragma unroll 4
    for (int j = my - 1; j >= 0; j--) out2[(size_t)j * ld] = d1b(d, j, r.pop(), h);
  } else if (op == 4) {
    const double *ai = d.AAinv + (size_t)M.m * 4;
    const double a0 = __ldg(ai), a1 = __ldg(ai + 1), a2 = __ldg(ai + 2), a3 = __ldg(ai + 3);
    const double2 c1 = make_double2(-(a0 * db.x + a1 * dt.x), -(a0 * db.y + a1 * dt.y));
    const double2 c2 = make_double2(-(a2 * db.x + a3 * dt.x), -(a2 * db.y + a3 * dt.y));
    const size_t n = (size_t)d.nmode;
    #pragma unroll 4
    for (int j = 0; j < my; j++) {
      double2 x = out[(size_t)j * ld];
      const double v1 = __ldg(d.V12t + (size_t)j * 2 * n + M.m), v2 = __ldg(d.V12t + (size_t)j * 2 * n + n + M.m);
      x.x += c1.x * v1 + c2.x * v2;
      x.y += c1.y * v1 + c2.y * v2;
      out[(size_t)j * ld] = zero ? czero() : x;
    }
  }
}

// 2014 variant: Deltat of the first substep of a CFL step, from the
// velocity maxima of the x stage (lomacte/cross.f:1547-1574); the new
// Deltat applies from this substep on.
__global__ void k_cfl14(Dev d, int do_cfl) {
  if (!do_cfl || threadIdx.x != 0 || blockIdx.x != 0) return;
  double hmin = d.hy[0];
  for (int j = 1; j < d.my; j++) hmin = fmin(hmin, d.hy[j]);
  const double hyy = 2.0 * d.ire * pow(fmax(1.0 / hmin, fmax(0.5 * d.hxalp, 0.5 * d.hzbet)), 2.0);
  const double cx = __longlong_as_double((long long)d.cflmax[0]) * d.hxalp;
  const double cy = __longlong_as_double((long long)d.cflmax[1]);
  const double cz = __longlong_as_double((long long)d.cflmax[2]) * d.hzbet;
  const double reig = fmax(fmax(cx, fmax(cy, cz)), hyy);
  d.scal_d[0] = (double)(float)(d.cfl / reig);  // Deltat is real*4
}

// 2014 variant, 00 modes after the substep (lomacte/cross.f:931-1002):
// rho u00 / rho w00 RK3 update, masses, rho v00 = -(cumulative trapezoid of
// d(rho)00 / (Deltat (gamma + xi)) - rho_bot trapz / (rho_top + rho_bot)),
// end-of-step time.  One thread: the sums run in the reference's order.
__global__ void k_psi00_14(Dev d, int rk) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int my = d.my;
  const double dt = d.scal_d[0], dtg = dt * d.gama[rk], den = dt * (d.gama[rk] + d.xi[rk]);
  double mu = 0.0, mv = 0.0, mw = 0.0;
  #pragma unroll 4
  for (int j = 0; j < my; j++) {
    if (j >= 1 && j <= my - 2) {
      d.u00[j] += dtg * d.rf0u[j];
      d.w00[j] += dtg * d.rf0w[j];
    }
    mu += d.u00[j] * d.hy[j];
    mv += d.v00[j] * d.hy[j];
    mw += d.w00[j] * d.hy[j];
  }
  const double2 *dr = d.sb[ODRHO];
  const size_t ld = d.nmode;
  double f = 0.0, prev = dr[0].x / den;
  d.rf0v[0] = 0.0;
  for (int j = 0; j < my - 1; j++) {
    const double nxt = dr[(size_t)(j + 1) * ld].x / den;
    f += 0.5 * (d.y[j + 1] - d.y[j]) * (nxt + prev);
    d.rf0v[j + 1] = f;
    prev = nxt;
  }
  const double trapz = f;
  const double sh = d.scal_d[3] * trapz / (d.scal_d[4] + d.scal_d[3]);
  #pragma unroll 4
  for (int j = 0; j < my; j++) {
    d.rf0v[j] -= sh;
    d.v00[j] = -d.rf0v[j];
  }
  d.diag[5] = trapz;
  d.diag[7] = mu; d.diag[8] = mv; d.diag[9] = mw;
  if (rk == 2) {
    d.diag[0] = d.scal_d[2];
    d.diag[1] = dt;
    d.scal_d[2] += dt;
    d.diag[12] = dt;
  }
}

}  // namespace tpm
}  // namespace lmc
