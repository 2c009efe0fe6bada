// lmc_ykernels.cuh -- y-direction kernels of one lomacte RK3 substep.
//
// Each block owns a tile of TM modes that share the kx plane and have
// consecutive kz (one warp per mode).  Fields are staged through shared
// memory: the block reads the tile [y][kz0..kz0+TM) of the device layout
// [y][kx][kz] with coalesced TM-wide runs and each warp then takes the
// chunks of its own pencil.  The y-operators run in registers (see
// lmc_device.cuh).  Kernels follow trunk/lomacte3/src/cross.f:307-1141.
//
// All arithmetic is FP64.  The kernels are templated on the complex type CT
// of the spectral work buffers: double2 in the FP64 form, float2 in the
// mixed form (values are widened on load and rounded on store; the state
// fields, the RK3 accumulators and the 00 modes stay FP64 in both).
// The lmc_y_*.cu translation units instantiate YL<C, CT> for their chunk
// sizes; lmc_ykernels.cu dispatches.
#pragma once
#include <cuda_runtime.h>

#include "lmc_ylaunch.h"

using namespace lmcd;

namespace lmc {

namespace {

constexpr int TM = 8;  // modes (warps) per block

struct Tile {
  int i, k0, nt, w, k, m;
  bool act;
};

__device__ __forceinline__ Tile make_tile(const Dev &d) {
  Tile T;
  T.i = blockIdx.y;
  T.k0 = blockIdx.x * TM;
  T.nt = min(TM, d.mz - T.k0);
  T.w = threadIdx.x >> 5;
  T.act = T.w < T.nt;
  T.k = T.act ? T.k0 + T.w : d.mz - 1;  // idle warps compute on a valid mode and store nothing
  T.m = T.i * d.mz + T.k;
  return T;
}

// block-cooperative staged load of one spectral field, then the warp's chunk
template <int C, typename PT>
__device__ __forceinline__ void tload(const Dev &d, const Tile &T, const PT *__restrict__ f, double2 *S,
                                      const Lane &L, double2 (&v)[C]) {
  __syncthreads();
  const int tot = d.my * TM;
  const size_t rs = (size_t)d.nkx * d.mz;
  const PT *base = f + (size_t)T.i * d.mz + T.k0;
  for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
    const int y = idx / TM, m = idx - y * TM;
    if (m < T.nt) S[m * d.ldy + y] = to_d2(__ldg(base + y * rs + m));
  }
  __syncthreads();
  cld<C>(S + T.w * d.ldy, L, v);
}

// block-cooperative staging of one field into S without taking a chunk;
// the warp then reads its elements on the fly with sv()
template <typename PT>
__device__ __forceinline__ void tstage(const Dev &d, const Tile &T, const PT *__restrict__ f, double2 *S) {
  __syncthreads();
  const int tot = d.my * TM;
  const size_t rs = (size_t)d.nkx * d.mz;
  const PT *base = f + (size_t)T.i * d.mz + T.k0;
  for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
    const int y = idx / TM, m = idx - y * TM;
    if (m < T.nt) S[m * d.ldy + y] = to_d2(__ldg(base + y * rs + m));
  }
  __syncthreads();
}
__device__ __forceinline__ double2 sv(const Dev &d, const Tile &T, const double2 *S, const Lane &L, int t) {
  return (t < L.n) ? S[T.w * d.ldy + L.s + t] : czero();
}

template <int C, typename PT>
__device__ __forceinline__ void tstore(const Dev &d, const Tile &T, PT *f, double2 *S, const Lane &L,
                                       const double2 (&v)[C]) {
  __syncthreads();
  if (T.act) cst<C>(S + T.w * d.ldy, L, v);
  __syncthreads();
  const int tot = d.my * TM;
  const size_t rs = (size_t)d.nkx * d.mz;
  PT *base = f + (size_t)T.i * d.mz + T.k0;
  for (int idx = threadIdx.x; idx < tot; idx += blockDim.x) {
    const int y = idx / TM, m = idx - y * TM;
    if (m < T.nt) base[y * rs + m] = from_d2<PT>(S[m * d.ldy + y]);
  }
}

template <int C>
__device__ __forceinline__ void set_row(double2 (&v)[C], const Lane &L, int row, double2 val) {
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n && L.s + t == row) v[t] = val;
}
template <int C>
__device__ __forceinline__ double2 get_row(const double2 (&v)[C], const Lane &L, int row) {
  double2 r = czero();
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n && L.s + t == row) r = v[t];
  return r;
}
template <int C>
__device__ __forceinline__ double2 bcast_row(const double2 (&v)[C], const Lane &L, int row) {
  double2 r = get_row(v, L, row);
  r.x = warp_sum(r.x);
  r.y = warp_sum(r.y);
  return r;
}

// Mixed form: the FP64 00 profiles (see Dev::mi / Dev::mo_cur)
template <typename CT>
__host__ __device__ constexpr bool is_mixed() { return sizeof(CT) == sizeof(float2); }
template <int C>
__device__ __forceinline__ void put_mi(const Dev &d, int q, const Lane &L, const double2 (&v)[C]) {
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) d.mi[(size_t)q * d.my + L.s + t] = v[t].x;
}
// exact 00 coefficient of transform output o at row s+t (plane mean)
__device__ __forceinline__ double2 mo00(const Dev &d, int o, const Lane &L, int t) {
  if (t >= L.n) return czero();
  return make_double2(d.mo_cur[(size_t)o * d.my + L.s + t] / ((double)d.mgalx * (double)d.mgalz), 0.0);
}
template <int C>
__device__ __forceinline__ void load_mo00(const Dev &d, int o, const Lane &L, double2 (&v)[C]) {
#pragma unroll
  for (int t = 0; t < C; t++) v[t] = mo00(d, o, L, t);
}

// compact first derivative in place (deryr2, cfdiff.f:518-601)
template <int C>
__device__ __forceinline__ void d1(const Dev &d, const Lane &L, double2 (&u)[C]) {
  matvec_ip<C, 3>(d.dt12, L, u);
  lsolve_c<C, 3>(u, d.p1L, d.k1L, L);
  usolve_c<C, 3>(u, d.p1U, d.k1U, L);
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) u[t] = cscale(tab(d.fmap, 1, t, 0, L.lane), u[t]);
}
// compact second derivative in place (deryyr2, cfdiff.f:735-797)
template <int C>
__device__ __forceinline__ void d2(const Dev &d, const Lane &L, double2 (&u)[C]) {
  matvec_ip<C, 2>(d.dt22, L, u);
  lsolve_c<C, 2>(u, d.p3L, d.k3L, L);
  usolve_c<C, 2>(u, d.p3U, d.k3U, L);
}
// Dirichlet Poisson solve of mode m: rhs = dt21 f with zero wall rows
// (laps.f:375-401, calcrhslap laps.f:17-47), then the per-mode LU.
template <int C>
__device__ __forceinline__ void poisson(const Dev &d, const Lane &L, int m, double2 (&v)[C]) {
  matvec_ip<C, 2>(d.dt21, L, v);
  set_row(v, L, 0, czero());
  set_row(v, L, d.my - 1, czero());
  lsolve_g<C, 2>(v, d.PL + (size_t)m * C * 2 * 32, L);
  usolve_g<C, 2>(v, d.PU + (size_t)m * C * 3 * 32, L);
}
// solvepsi (laps.f:580-730): Neumann walls through the precomputed
// homogeneous solutions v1, v2 and the inverse of their 2x2 wall matrix.
template <int C>
__device__ __forceinline__ void neumann(const Dev &d, const Lane &L, int m, double2 (&psi)[C]) {
  poisson<C>(d, L, m, psi);
  double2 db = czero(), dt = czero();
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double eb = tab(d.ebot, 1, t, 0, L.lane), et = tab(d.etop, 1, t, 0, L.lane);
      db.x = fma(eb, psi[t].x, db.x); db.y = fma(eb, psi[t].y, db.y);
      dt.x = fma(et, psi[t].x, dt.x); dt.y = fma(et, psi[t].y, dt.y);
    }
  db = warp_sum2(db);
  dt = warp_sum2(dt);
  const double *ai = d.AAinv + (size_t)m * 4;
  const double a0 = __ldg(ai), a1 = __ldg(ai + 1), a2 = __ldg(ai + 2), a3 = __ldg(ai + 3);
  const double2 c1 = make_double2(-(a0 * db.x + a1 * dt.x), -(a0 * db.y + a1 * dt.y));
  const double2 c2 = make_double2(-(a2 * db.x + a3 * dt.x), -(a2 * db.y + a3 * dt.y));
  const double *vv = d.V12 + (size_t)m * C * 2 * 32;
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double v1 = tab(vv, 2, t, 0, L.lane), v2 = tab(vv, 2, t, 1, L.lane);
      psi[t].x += c1.x * v1 + c2.x * v2;
      psi[t].y += c1.y * v1 + c2.y * v2;
    }
}

#define YKERNEL_PROLOGUE                                  \
  extern __shared__ double2 S[];                          \
  const Tile T = make_tile(d);                            \
  const Lane L = make_lane<C>(d.lpm, d.base, d.extra);

// ----------------------------------------------------------------------
// (1) Lapvdvhom phi -> m_y, dm_y/dy: BC on phi (cross.f:329-335) and
// cross.f:365-372.
// ----------------------------------------------------------------------
template <int C, typename CT>
__global__ void __launch_bounds__(TM * 32, 2) k_lapv(Dev d) {
  YKERNEL_PROLOGUE
  double2 a[C];
  tload<C>(d, T, d.phi, S, L, a);
  set_row(a, L, 0, czero());
  set_row(a, L, d.my - 1, czero());
  const bool zero = (__ldg(d.k2 + T.m) == 0.0);
  poisson<C>(d, L, T.m, a);
  if (zero) {
#pragma unroll
    for (int t = 0; t < C; t++) a[t] = czero();
  }
  tstore<C>(d, T, wsb<CT>(d, SB_MY), S, L, a);
  d1<C>(d, L, a);
  tstore<C>(d, T, wsb<CT>(d, SB_DMY), S, L, a);
}

// ----------------------------------------------------------------------
// (2)-(3) m_x, m_z, rho u_i, xi-updates of Omega_y and phi, 00 modes:
// cross.f:315-327 (BC on Omega_y), 395-499.
// ----------------------------------------------------------------------
template <int C, typename CT>
__global__ void __launch_bounds__(TM * 32, 2) k_assemble(Dev d, int rk) {
  YKERNEL_PROLOGUE
  const double kx = __ldg(d.kx + T.i), kz = __ldg(d.kz + T.k), k2 = __ldg(d.k2 + T.m);
  const double dtxi = d.scal_d[0] * d.xi[rk];
  const double ta = (k2 != 0.0) ? kx / k2 : 0.0, tb = (k2 != 0.0) ? kz / k2 : 0.0;
  const bool m00 = T.act && T.m == 0;
  double2 vo[C], a[C], b[C];
  tload<C>(d, T, d.vor, S, L, vo);
  set_row(vo, L, 0, get_row(vo, L, 1));
  set_row(vo, L, d.my - 1, get_row(vo, L, d.my - 2));
  tload<C>(d, T, wsb<CT>(d, SB_DMY), S, L, a);
  tstage(d, T, d.psi, S);
#pragma unroll
  for (int t = 0; t < C; t++) {
    const double2 ps = sv(d, T, S, L, t);
    b[t] = cadd(csub(cik(ta, a[t]), cik(tb, vo[t])), cik(kx, ps));  // rho u, cross.f:402,467
    a[t] = cadd(cadd(cik(tb, a[t]), cik(ta, vo[t])), cik(kz, ps));  // rho w, cross.f:404,469
  }
  if (m00) {  // 00 modes injected: cross.f:486-491
#pragma unroll
    for (int t = 0; t < C; t++)
      if (t < L.n) {
        b[t] = make_double2(d.u00[L.s + t], 0.0);
        a[t] = make_double2(d.w00[L.s + t], 0.0);
      }
    if constexpr (is_mixed<CT>()) {
      put_mi<C>(d, 0, L, b);
      put_mi<C>(d, 2, L, a);
    }
  }
  tstore<C>(d, T, wsb<CT>(d, SB_RU), S, L, b);
  tstore<C>(d, T, wsb<CT>(d, SB_RW), S, L, a);
  // xi-update of Omega_y (cross.f:420-424), written with this substep's BC
  tstage(d, T, d.Rom, S);
#pragma unroll
  for (int t = 0; t < C; t++) vo[t] = cadd(vo[t], cscale(dtxi, sv(d, T, S, L, t)));
  tstore<C>(d, T, d.vor, S, L, vo);
  // rho v = m_y + d(psi)/dy (cross.f:434-437, 471)
  tload<C>(d, T, d.psi, S, L, a);
  d1<C>(d, L, a);
  tstage(d, T, wsb<CT>(d, SB_MY), S);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = cadd(a[t], sv(d, T, S, L, t));
  if (m00) {
#pragma unroll
    for (int t = 0; t < C; t++)
      if (t < L.n) a[t] = make_double2(d.v00[L.s + t], 0.0);
    if constexpr (is_mixed<CT>()) put_mi<C>(d, 1, L, a);
  }
  tstore<C>(d, T, wsb<CT>(d, SB_RV), S, L, a);
  // xi-update of phi (cross.f:424-425), with its wall BC
  tload<C>(d, T, d.phi, S, L, b);
  set_row(b, L, 0, czero());
  set_row(b, L, d.my - 1, czero());
  tstage(d, T, d.Rphi, S);
#pragma unroll
  for (int t = 0; t < C; t++) b[t] = cadd(b[t], cscale(dtxi, sv(d, T, S, L, t)));
  tstore<C>(d, T, d.phi, S, L, b);
  if (m00) {  // u00**, w00** (cross.f:495-498)
#pragma unroll
    for (int t = 0; t < C; t++)
      if (t < L.n) {
        const int j = L.s + t;
        if (j >= 1 && j <= d.my - 2) {
          d.u00[j] += dtxi * d.rf0u[j];
          d.w00[j] += dtxi * d.rf0w[j];
        }
      }
  }
}

// ----------------------------------------------------------------------
// (4) T with its wall BCs, dT/dy, lap(T): cross.f:336-349, 521-541.
// ----------------------------------------------------------------------
template <int C, typename CT>
__global__ void __launch_bounds__(TM * 32, 2) k_tder(Dev d) {
  YKERNEL_PROLOGUE
  const double k2 = __ldg(d.k2 + T.m);
  double2 Tv[C], a[C];
  tload<C>(d, T, d.scal, S, L, Tv);
  if (T.m == 0) {
    set_row(Tv, L, 0, make_double2(1.0 / d.scal_d[3], 0.0));
    set_row(Tv, L, d.my - 1, make_double2(1.0 / d.scal_d[4], 0.0));
  } else {
    set_row(Tv, L, 0, czero());
    set_row(Tv, L, d.my - 1, czero());
  }
  tstore<C>(d, T, d.scal, S, L, Tv);
  const bool m00 = T.act && T.m == 0;
  if constexpr (is_mixed<CT>()) {
    tstore<C>(d, T, wsb<CT>(d, SB_T32), S, L, Tv);
    if (m00) put_mi<C>(d, 5, L, Tv);
  }
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = Tv[t];
  d1<C>(d, L, a);
  if constexpr (is_mixed<CT>())
    if (m00) put_mi<C>(d, 4, L, a);
  tstore<C>(d, T, wsb<CT>(d, SB_DTDY), S, L, a);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = Tv[t];
  d2<C>(d, L, a);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(a[t], cscale(k2, Tv[t]));
  if constexpr (is_mixed<CT>())
    if (m00) put_mi<C>(d, 3, L, a);
  tstore<C>(d, T, wsb<CT>(d, SB_LAPT), S, L, a);
}

// ----------------------------------------------------------------------
// (6a)-(6b) T update and N_i: cross.f:619-682; 00-mode RHS, dw, H00, dm,
// masst and the CFL Deltat: cross.f:686-722, 1416-1429, 1778-1826.
// The 00 pencils of d(rho uv)/dy and d(rho vw)/dy are parked in rf0u and
// rf0w until the 00 RHS replaces them at the end of the kernel.
// ----------------------------------------------------------------------
// 00 mode of post1 (block (0,0); warp 0 computes): dw, dm, masst, the
// viscous 00 RHS of rho u00 / rho w00 (its d(rho uv)/dy, d(rho vw)/dy parts
// parked in rf0u / rf0w), H00 and the CFL Deltat: cross.f:686-722,
// 1416-1429, 1778-1826.  All threads of the block take part in the staging.
template <int C, typename CT>
__device__ __forceinline__ void post1_00(const Dev &d, const Tile &T, const Lane &L, double2 *S, int rk, int do_cfl,
                                         int do_diag) {
  double2 a[C], b[C];
  tload<C>(d, T, wsb<CT>(d, OU), S, L, a);
  if (T.w != 0) return;
  if constexpr (is_mixed<CT>()) {  // the u pencil (and its staged copy) in FP64
    load_mo00<C>(d, OU, L, a);
    const double inn = 1.0 / ((double)d.mgalx * (double)d.mgalz);
    for (int j = L.lane; j < d.my; j += 32) S[j] = make_double2(d.mo_cur[(size_t)OU * d.my + j] * inn, 0.0);
    __syncwarp();
  }
#pragma unroll
  for (int t = 0; t < C; t++) a[t].y = 0.0;
  if (rk == 2 && do_diag) {  // vorticity thickness, cross.f:692-699
#pragma unroll
    for (int t = 0; t < C; t++) b[t] = a[t];
    d1<C>(d, L, b);
    double mx = 0.0;
#pragma unroll
    for (int t = 0; t < C; t++)
      if (t < L.n) mx = fmax(mx, fabs(b[t].x));
    mx = warp_max(mx);
    if (L.lane == 0) { d.diag[3] = 1.0 / mx; d.diag[4] = d.diag[3] / d.ire; }
  }
  if (rk == 0 && do_diag) {  // momentum thickness, cross.f:1416-1429
    const double2 *U = S;  // the 00 pencil is staged in S[0..my)
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < C; t++)
      if (t < L.n) {
        const int j = L.s + t;
        double a1, a2;
        if (j == 0) { a1 = U[1].x; a2 = U[0].x; }
        else if (j == d.my - 1) { a1 = U[d.my - 1].x; a2 = U[d.my - 2].x; }
        else { a1 = U[j + 1].x; a2 = U[j - 1].x; }
        s += d.trp[j] * (a1 * a1 + a2 * a2);
      }
    s = warp_sum(s);
    double ms = 0.0;  // masst, escru.f:372-376 (one accumulation)
    for (int j = L.lane; j < d.my; j += 32) ms += d.rhom[j] * d.hy[j];
    ms = warp_sum(ms);
    if (L.lane == 0) {
      const double du0 = U[d.my - 1].x - U[0].x;
      d.diag[2] = 0.25 * (d.y[d.my - 1] - d.y[0]) - s / (du0 * du0);
      d.diag[6] = ms / ((double)d.mgalx * (double)d.mgalz);
    }
  }
  d2<C>(d, L, a);
  double hu = 0.0, hw = 0.0;
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double r = -d.rf0u[L.s + t] + d.ire * a[t].x;  // cross.f:705
      d.rf0u[L.s + t] = r;
      hu += r * d.hy[L.s + t];
    }
  {  // w00 pencil read directly (the block has left)
    const size_t rs = (size_t)d.nkx * d.mz;
#pragma unroll
    for (int t = 0; t < C; t++) a[t] = (t < L.n) ? make_double2(wsb<CT>(d, OW)[(size_t)(L.s + t) * rs].x, 0.0) : czero();
    if constexpr (is_mixed<CT>()) load_mo00<C>(d, OW, L, a);
  }
  d2<C>(d, L, a);
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double r = -d.rf0w[L.s + t] + d.ire * a[t].x;  // cross.f:706
      d.rf0w[L.s + t] = r;
      hw += r * d.hy[L.s + t];
    }
  hu = warp_sum(hu);
  hw = warp_sum(hw);
  if (L.lane == 0) {
    if (rk == 2 && do_diag) { d.diag[10] = 0.25 * hu; d.diag[11] = 0.25 * hw; }
    if (rk == 0 && do_cfl) {  // cross.f:1781-1817, one compute rank
      const double cx = __longlong_as_double((long long)d.cflmax[0]) * d.hxalp * 0.5;
      const double cy = __longlong_as_double((long long)d.cflmax[1]);
      const double cz = __longlong_as_double((long long)d.cflmax[2]) * d.hzbet * 0.5;
      const double ct = __longlong_as_double((long long)d.cflmax[3]);
      d.scal_d[1] = (double)(float)(d.cfl / (cx + cy + cz + ct));  // dtr is real*4
    }
  }
}

template <int C, typename CT>
__global__ void __launch_bounds__(TM * 32, 2) k_post1(Dev d, int rk, int do_cfl, int do_diag) {
  YKERNEL_PROLOGUE
  const double kx = __ldg(d.kx + T.i), kz = __ldg(d.kz + T.k);
  const bool m00 = T.act && T.m == 0;
  double2 a[C], b[C];
  tload<C>(d, T, d.scal, S, L, a);
  tstage(d, T, wsb<CT>(d, ODT), S);
#pragma unroll
  for (int t = 0; t < C; t++) {
    double2 dT = sv(d, T, S, L, t);
    if constexpr (is_mixed<CT>())
      if (m00) dT = mo00(d, ODT, L, t);
    a[t] = cadd(a[t], dT);  // cross.f:619-627
  }
  tstore<C>(d, T, d.scal, S, L, a);
  // N_y = -ikx rho uv - d(rho vv)/dy - ikz rho vw
  tload<C>(d, T, wsb<CT>(d, ORVV), S, L, a);
  d1<C>(d, L, a);
  tstage(d, T, wsb<CT>(d, ORUV), S);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(czero(), cadd(a[t], cik(kx, sv(d, T, S, L, t))));
  tstage(d, T, wsb<CT>(d, ORVW), S);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(a[t], cik(kz, sv(d, T, S, L, t)));
  tstore<C>(d, T, wsb<CT>(d, ORVV), S, L, a);
  // N_x = -ikx rho uu - d(rho uv)/dy - ikz rho uw
  tload<C>(d, T, wsb<CT>(d, ORUV), S, L, a);
  if constexpr (is_mixed<CT>())
    if (m00) load_mo00<C>(d, ORUV, L, a);
  d1<C>(d, L, a);
  if (m00) {
#pragma unroll
    for (int t = 0; t < C; t++)
      if (t < L.n) d.rf0u[L.s + t] = a[t].x;
  }
  tstage(d, T, wsb<CT>(d, ORUU), S);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(czero(), cadd(a[t], cik(kx, sv(d, T, S, L, t))));
  tload<C>(d, T, wsb<CT>(d, ORUW), S, L, b);  // kept for N_z
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(a[t], cik(kz, b[t]));
  tstore<C>(d, T, wsb<CT>(d, ORUU), S, L, a);
  // N_z = -ikx rho uw - d(rho vw)/dy - ikz rho ww
  tload<C>(d, T, wsb<CT>(d, ORVW), S, L, a);
  if constexpr (is_mixed<CT>())
    if (m00) load_mo00<C>(d, ORVW, L, a);
  d1<C>(d, L, a);
  if (m00) {
#pragma unroll
    for (int t = 0; t < C; t++)
      if (t < L.n) d.rf0w[L.s + t] = a[t].x;
  }
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(czero(), cadd(a[t], cik(kx, b[t])));
  tstage(d, T, wsb<CT>(d, ORWW), S);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(a[t], cik(kz, sv(d, T, S, L, t)));
  tstore<C>(d, T, wsb<CT>(d, ORWW), S, L, a);
  if (!(blockIdx.x == 0 && blockIdx.y == 0)) return;
  post1_00<C, CT>(d, T, L, S, rk, do_cfl, do_diag);
}

// ----------------------------------------------------------------------
// (6c)-(6d) vorticity and the two Laplacians: cross.f:748-857.
// lap(curl omega)_y goes to the DT buffer (consumed by post1) and
// lap(omega_y) to the v buffer (consumed here).
// ----------------------------------------------------------------------
template <int C, typename CT>
__global__ void __launch_bounds__(TM * 32, 2) k_post2a(Dev d) {
  YKERNEL_PROLOGUE
  const double kx = __ldg(d.kx + T.i), kz = __ldg(d.kz + T.k), k2 = __ldg(d.k2 + T.m);
  double2 a[C], b[C], c[C];
  tload<C>(d, T, wsb<CT>(d, OW), S, L, a);
  d1<C>(d, L, a);                                                  // dw/dy
  tstage(d, T, wsb<CT>(d, OV), S);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(a[t], cik(kz, sv(d, T, S, L, t)));  // omega_x, cross.f:757
  tload<C>(d, T, wsb<CT>(d, OU), S, L, c);
  d1<C>(d, L, c);                                                  // du/dy
  tstage(d, T, wsb<CT>(d, OV), S);
#pragma unroll
  for (int t = 0; t < C; t++) {
    c[t] = csub(cik(kx, sv(d, T, S, L, t)), c[t]);  // omega_z, cross.f:763
    b[t] = csub(cik(kz, a[t]), cik(kx, c[t]));      // (curl omega)_y, cross.f:839
    a[t] = b[t];
  }
  d2<C>(d, L, a);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(a[t], cscale(k2, b[t]));  // cross.f:847-857
  tstore<C>(d, T, wsb<CT>(d, ODT), S, L, a);
  tload<C>(d, T, wsb<CT>(d, OU), S, L, a);
  tstage(d, T, wsb<CT>(d, OW), S);
#pragma unroll
  for (int t = 0; t < C; t++) {
    b[t] = csub(cik(kz, a[t]), cik(kx, sv(d, T, S, L, t)));  // omega_y, cross.f:760
    a[t] = b[t];
  }
  d2<C>(d, L, a);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(a[t], cscale(k2, b[t]));  // cross.f:822-832
  tstore<C>(d, T, wsb<CT>(d, OV), S, L, a);
}

// ----------------------------------------------------------------------
// (9) RHS(Omega_y), RHS(phi) and the RK3 update: cross.f:885-981.
// ----------------------------------------------------------------------
template <int C, typename CT>
__global__ void __launch_bounds__(TM * 32, 2) k_post2b(Dev d, int rk) {
  YKERNEL_PROLOGUE
  const double kx = __ldg(d.kx + T.i), kz = __ldg(d.kz + T.k), k2 = __ldg(d.k2 + T.m);
  const double dtg = d.scal_d[0] * d.gama[rk];
  double2 a[C], b[C], c[C];
  tload<C>(d, T, wsb<CT>(d, ORUU), S, L, a);  // N_x
  tload<C>(d, T, wsb<CT>(d, ORWW), S, L, b);  // N_z
#pragma unroll
  for (int t = 0; t < C; t++) {
    c[t] = cadd(cik(kx, a[t]), cik(kz, b[t]));  // cross.f:900
    a[t] = csub(cik(kz, a[t]), cik(kx, b[t]));
  }
  tstage(d, T, wsb<CT>(d, OV), S);  // lap omega_y
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = cadd(a[t], cscale(d.ire, sv(d, T, S, L, t)));  // RHS(Omega_y), cross.f:889
  tstore<C>(d, T, d.Rom, S, L, a);
  tstage(d, T, d.vor, S);
#pragma unroll
  for (int t = 0; t < C; t++) b[t] = cadd(sv(d, T, S, L, t), cscale(dtg, a[t]));  // cross.f:969
  tstore<C>(d, T, d.vor, S, L, b);
  d1<C>(d, L, c);  // cross.f:907
  tstage(d, T, wsb<CT>(d, ORVV), S);  // N_y
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(cscale(-k2, sv(d, T, S, L, t)), c[t]);
  tstage(d, T, wsb<CT>(d, ODT), S);  // lap (curl omega)_y
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(a[t], cscale(d.ire, sv(d, T, S, L, t)));  // RHS(phi), cross.f:917
  tstore<C>(d, T, d.Rphi, S, L, a);
  tstage(d, T, d.phi, S);
#pragma unroll
  for (int t = 0; t < C; t++) b[t] = cadd(sv(d, T, S, L, t), cscale(dtg, a[t]));  // cross.f:978
  tstore<C>(d, T, d.phi, S, L, b);
}

// ----------------------------------------------------------------------
// (8) psi^{n+1} by solvepsi (cross.f:1092-1104); block (0,0) / warp 0
// then advances the 00 modes and integrates d(rho)/dt for rho v00
// (cross.f:1006-1074).
// ----------------------------------------------------------------------
// 00 mode of the psi stage (block (0,0); warp 0 computes): rho u00 / rho
// w00 RK3 update, masses, inty8 of d(rho)/dt00 for rho v00 with the
// acoustic wall correction, end-of-step time and Deltat: cross.f:1006-1074,
// 1196-1204.  All threads of the block take part in the staging.
template <int C, typename CT>
__device__ __forceinline__ void psi_00(const Dev &d, const Tile &T, const Lane &L, double2 *S, int rk, int cfl_step) {
  double2 a[C];
  tload<C>(d, T, wsb<CT>(d, ODRHO), S, L, a);
  if (T.w != 0) return;
  if constexpr (is_mixed<CT>()) load_mo00<C>(d, ODRHO, L, a);
  const double dt = d.scal_d[0], dtg = dt * d.gama[rk];
  double mu = 0.0, mv = 0.0, mw = 0.0;
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const int j = L.s + t;
      if (j >= 1 && j <= d.my - 2) {  // cross.f:1008-1011
        d.u00[j] += dtg * d.rf0u[j];
        d.w00[j] += dtg * d.rf0w[j];
      }
      const double h = d.hy[j];  // cross.f:1016-1020
      mu += d.u00[j] * h;
      mv += d.v00[j] * h;
      mw += d.w00[j] * h;
    }
  mu = warp_sum(mu); mv = warp_sum(mv); mw = warp_sum(mw);
  // inty8 (laps.f:484-575): rf0v(y) = int d(rho)/dt00 dy with rf0v(1) = 0
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = make_double2((t < L.n) ? a[t].x / tab(d.fmap, 1, t, 0, L.lane) : 0.0, 0.0);
  matvec_ip<C, 3>(d.dt11, L, a);
  lsolve_c<C, 3>(a, d.i8L, d.k8L, L);
  usolve_c<C, 3>(a, d.i8U, d.k8U, L);
  const double v0 = bcast_row(a, L, 0).x, vn = bcast_row(a, L, d.my - 1).x;
  const double trapz = -(vn - v0);                                       // cross.f:1046
  const double corr = trapz / (1.0 + sqrt(d.scal_d[4] / d.scal_d[3]));  // cross.f:1064-1065
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double r = a[t].x - v0;
      d.rf0v[L.s + t] = r;
      d.v00[L.s + t] = r + corr;
    }
  if (L.lane == 0) {
    d.diag[5] = trapz;
    d.diag[7] = mu; d.diag[8] = mv; d.diag[9] = mw;
    if (rk == 2) {  // end of the time step: cross.f:1196-1204
      d.diag[0] = d.scal_d[2];
      d.diag[1] = dt;
      d.scal_d[2] += dt;
      if (cfl_step) d.scal_d[0] = d.scal_d[1];
      d.diag[12] = d.scal_d[0];
    }
  }
}

template <int C, typename CT>
__global__ void __launch_bounds__(TM * 32, 2) k_psi(Dev d, int rk, int cfl_step, int do_diag) {
  YKERNEL_PROLOGUE
  double2 a[C];
  tload<C>(d, T, wsb<CT>(d, ODRHO), S, L, a);
  const bool zero = (__ldg(d.k2 + T.m) == 0.0);
  neumann<C>(d, L, T.m, a);
  if (zero) {
#pragma unroll
    for (int t = 0; t < C; t++) a[t] = czero();
  }
  tstore<C>(d, T, d.psi, S, L, a);
  if (!(blockIdx.x == 0 && blockIdx.y == 0)) return;
  psi_00<C, CT>(d, T, L, S, rk, cfl_step);
}

// the 00-mode tails alone (one block), after the mode-parallel kernels of
// lmc_ytpm.cuh
template <int C, typename CT>
__global__ void __launch_bounds__(TM * 32, 1) k_post1_00(Dev d, int rk, int do_cfl, int do_diag) {
  YKERNEL_PROLOGUE
  post1_00<C, CT>(d, T, L, S, rk, do_cfl, do_diag);
}
template <int C, typename CT>
__global__ void __launch_bounds__(TM * 32, 1) k_psi_00(Dev d, int rk, int cfl_step) {
  YKERNEL_PROLOGUE
  psi_00<C, CT>(d, T, L, S, rk, cfl_step);
}

// single-operator kernel (tests), device layout
template <int C>
__global__ void __launch_bounds__(TM * 32, 2) k_op_y(Dev d, int op, const double2 *in, double2 *out, double2 *out2) {
  YKERNEL_PROLOGUE
  double2 a[C];
  tload<C>(d, T, in, S, L, a);
  const bool zero = (__ldg(d.k2 + T.m) == 0.0);
  if (op == 1) {
    d1<C>(d, L, a);
  } else if (op == 2) {
    d2<C>(d, L, a);
  } else if (op == 3) {
    poisson<C>(d, L, T.m, a);
    if (zero) {
#pragma unroll
      for (int t = 0; t < C; t++) a[t] = czero();
    }
    tstore<C>(d, T, out, S, L, a);
    d1<C>(d, L, a);
    tstore<C>(d, T, out2, S, L, a);
    return;
  } else {
    neumann<C>(d, L, T.m, a);
    if (zero) {
#pragma unroll
      for (int t = 0; t < C; t++) a[t] = czero();
    }
  }
  tstore<C>(d, T, out, S, L, a);
}

inline dim3 ygrid(const Dev &d) { return dim3((unsigned)((d.mz + TM - 1) / TM), (unsigned)d.nkx); }
inline size_t ysmem(const Dev &d) { return (size_t)TM * d.ldy * sizeof(double2); }

inline cudaError_t yoptin(const void *fn, int limit) {
  cudaError_t e;
  cudaFuncAttributes fa;
  if ((e = cudaFuncGetAttributes(&fa, fn)) != cudaSuccess) return e;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, limit - (int)fa.sharedSizeBytes);
}

}  // namespace

#define LMC_YL(K, ...) K<<<ygrid(d), TM * 32, ysmem(d), s>>>(__VA_ARGS__)
template <int C, typename CT>
void YL<C, CT>::lapv(const Dev &d, cudaStream_t s) { LMC_YL((k_lapv<C, CT>), d); }
template <int C, typename CT>
void YL<C, CT>::assemble(const Dev &d, int rk, cudaStream_t s) { LMC_YL((k_assemble<C, CT>), d, rk); }
template <int C, typename CT>
void YL<C, CT>::tder(const Dev &d, cudaStream_t s) { LMC_YL((k_tder<C, CT>), d); }
template <int C, typename CT>
void YL<C, CT>::post1(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s) {
  LMC_YL((k_post1<C, CT>), d, rk, do_cfl, do_diag);
}
template <int C, typename CT>
void YL<C, CT>::post2(const Dev &d, int rk, cudaStream_t s) {
  LMC_YL((k_post2a<C, CT>), d);
  LMC_YL((k_post2b<C, CT>), d, rk);
}
template <int C, typename CT>
void YL<C, CT>::psi(const Dev &d, int rk, int cfl_step, int do_diag, cudaStream_t s) {
  LMC_YL((k_psi<C, CT>), d, rk, cfl_step, do_diag);
}
template <int C, typename CT>
void YL<C, CT>::post1_00(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s) {
  k_post1_00<C, CT><<<dim3(1, 1), TM * 32, ysmem(d), s>>>(d, rk, do_cfl, do_diag);
}
template <int C, typename CT>
void YL<C, CT>::psi_00(const Dev &d, int rk, int cfl_step, cudaStream_t s) {
  k_psi_00<C, CT><<<dim3(1, 1), TM * 32, ysmem(d), s>>>(d, rk, cfl_step);
}
template <int C, typename CT>
void YL<C, CT>::op_y(const Dev &d, int op, const double2 *in, double2 *out, double2 *out2, cudaStream_t s) {
  LMC_YL(k_op_y<C>, d, op, in, out, out2);
}
template <int C, typename CT>
cudaError_t YL<C, CT>::optin(int limit) {
  const void *fns[] = {(const void *)k_lapv<C, CT>, (const void *)k_assemble<C, CT>, (const void *)k_tder<C, CT>,
                       (const void *)k_post1<C, CT>, (const void *)k_post2a<C, CT>, (const void *)k_post2b<C, CT>,
                       (const void *)k_psi<C, CT>, (const void *)k_op_y<C>, (const void *)k_post1_00<C, CT>,
                       (const void *)k_psi_00<C, CT>};
  for (const void *fn : fns) {
    const cudaError_t e = yoptin(fn, limit);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}
#undef LMC_YL

}  // namespace lmc
