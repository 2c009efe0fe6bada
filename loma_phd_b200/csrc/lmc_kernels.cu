// lmc_kernels.cu -- sm_100a kernels of one lomacte RK3 substep (FP64 path).
//
// Substep = lapv -> assemble -> tder -> zinv -> xphys -> zfwd -> post1 ->
// post2 -> psi, following trunk/lomacte3/src/cross.f:307-1141.  The y
// kernels run one (kx,kz) mode per warp (see lmc_device.cuh); the
// transform kernels run batched mixed-radix FFTs in shared memory.
#include <cuda_runtime.h>

#include "lmc_kernels.cuh"

using namespace lmcd;

namespace lmc {

namespace {

constexpr int YWARPS = 4;  // warps (modes) per block of the y kernels

__device__ __forceinline__ int mode_of_warp() { return (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); }

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
// value of global row `row` held by whichever lane owns it, broadcast to the warp
template <int C>
__device__ __forceinline__ double2 bcast_row(const double2 (&v)[C], const Lane &L, int row) {
  double2 r = get_row(v, L, row);
  r.x = warp_sum(r.x);
  r.y = warp_sum(r.y);
  return r;
}

// compact first derivative (deryr2, cfdiff.f:518-601)
template <int C>
__device__ __forceinline__ void d1(const Dev &d, const Lane &L, const double2 (&u)[C], double2 (&du)[C]) {
  matvec<C, 3>(d.dt12, L, u, du);
  lsolve<C, 3>(du, d.p1L, L);
  usolve<C, 3>(du, d.p1U, L);
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) du[t] = cscale(__ldg(d.fmap + L.s + t), du[t]);
}
// compact second derivative (deryyr2, cfdiff.f:735-797)
template <int C>
__device__ __forceinline__ void d2(const Dev &d, const Lane &L, const double2 (&u)[C], double2 (&du)[C]) {
  matvec<C, 2>(d.dt22, L, u, du);
  lsolve<C, 2>(du, d.p3L, L);
  usolve<C, 2>(du, d.p3U, L);
}
// Dirichlet Poisson solve of mode m: rhs = dt21 f with zero wall rows
// (laps.f:375-401 / calcrhslap laps.f:17-47), then the per-mode LU.
template <int C>
__device__ __forceinline__ void poisson(const Dev &d, const Lane &L, int m, const double2 (&f)[C], double2 (&v)[C]) {
  matvec<C, 2>(d.dt21, L, f, v);
  set_row(v, L, 0, czero());
  set_row(v, L, d.my - 1, czero());
  lsolve<C, 2>(v, d.PL + (size_t)m * d.my * 2, L);
  usolve<C, 2>(v, d.PU + (size_t)m * d.my * 3, L);
}
// solvepsi (laps.f:580-730): Neumann walls via the precomputed homogeneous
// solutions v1, v2 and the inverse 2x2 matrix of their wall derivatives.
template <int C>
__device__ __forceinline__ void neumann(const Dev &d, const Lane &L, int m, const double2 (&f)[C], double2 (&psi)[C]) {
  poisson<C>(d, L, m, f, psi);
  double2 db = czero(), dt = czero();
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double eb = __ldg(d.ebot + L.s + t), et = __ldg(d.etop + L.s + t);
      db.x = fma(eb, psi[t].x, db.x); db.y = fma(eb, psi[t].y, db.y);
      dt.x = fma(et, psi[t].x, dt.x); dt.y = fma(et, psi[t].y, dt.y);
    }
  db = warp_sum2(db);
  dt = warp_sum2(dt);
  const double *ai = d.AAinv + (size_t)m * 4;
  const double a0 = __ldg(ai), a1 = __ldg(ai + 1), a2 = __ldg(ai + 2), a3 = __ldg(ai + 3);
  const double2 c1 = make_double2(-(a0 * db.x + a1 * dt.x), -(a0 * db.y + a1 * dt.y));
  const double2 c2 = make_double2(-(a2 * db.x + a3 * dt.x), -(a2 * db.y + a3 * dt.y));
  const double *vv = d.V12 + (size_t)m * d.my * 2;
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double v1 = __ldg(vv + 2 * (L.s + t)), v2 = __ldg(vv + 2 * (L.s + t) + 1);
      psi[t].x += c1.x * v1 + c2.x * v2;
      psi[t].y += c1.y * v1 + c2.y * v2;
    }
}

template <int C>
__device__ __forceinline__ void ld_real(const double *p, const Lane &L, double2 (&v)[C]) {
#pragma unroll
  for (int t = 0; t < C; t++) v[t] = make_double2((t < L.n) ? p[L.s + t] : 0.0, 0.0);
}

// ----------------------------------------------------------------------
// (1) Lapvdvhom phi -> m_y, dm_y/dy: cross.f:315-349 (BC on phi) and
// cross.f:365-372.
// ----------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(YWARPS * 32) k_lapv(Dev d) {
  const int m = mode_of_warp();
  if (m >= d.nmode) return;
  const Lane L = make_lane<C>(d.lpm, d.base, d.extra);
  const size_t off = (size_t)m * d.my;
  double2 a[C], b[C];
  if (__ldg(d.k2 + m) == 0.0) {
#pragma unroll
    for (int t = 0; t < C; t++) a[t] = czero();
    st(d.sb[SB_MY] + off, L, a);
    st(d.sb[SB_DMY] + off, L, a);
    return;
  }
  ld(d.phi + off, L, a);
  set_row(a, L, 0, czero());
  set_row(a, L, d.my - 1, czero());
  poisson<C>(d, L, m, a, b);
  st(d.sb[SB_MY] + off, L, b);
  d1<C>(d, L, b, a);
  st(d.sb[SB_DMY] + off, L, a);
}

// ----------------------------------------------------------------------
// (2)-(3) m_x, m_z, rho u_i, xi-update of Omega_y and phi, 00 modes:
// cross.f:395-499.
// ----------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(YWARPS * 32) k_assemble(Dev d, int rk) {
  const int m = mode_of_warp();
  if (m >= d.nmode) return;
  const Lane L = make_lane<C>(d.lpm, d.base, d.extra);
  const size_t off = (size_t)m * d.my;
  const int i = m / d.mz, k = m - i * d.mz;
  const double kx = __ldg(d.kx + i), kz = __ldg(d.kz + k), k2 = __ldg(d.k2 + m);
  const double dtxi = d.scal_d[0] * d.xi[rk];
  const double ta = (k2 != 0.0) ? kx / k2 : 0.0, tb = (k2 != 0.0) ? kz / k2 : 0.0;
  double2 vo[C], dm[C], mx[C], mz[C], ps[C], w[C];
  // Omega_y with its wall BC d(Omega_y)/dy = 0 by copy (cross.f:315-327)
  ld(d.vor + off, L, vo);
  set_row(vo, L, 0, get_row(vo, L, 1) );
  set_row(vo, L, d.my - 1, get_row(vo, L, d.my - 2));
  ld(d.sb[SB_DMY] + off, L, dm);
#pragma unroll
  for (int t = 0; t < C; t++) {
    mx[t] = csub(cik(ta, dm[t]), cik(tb, vo[t]));  // cross.f:402
    mz[t] = cadd(cik(tb, dm[t]), cik(ta, vo[t]));  // cross.f:404
  }
  ld(d.psi + off, L, ps);
#pragma unroll
  for (int t = 0; t < C; t++) {
    mx[t] = cadd(mx[t], cik(kx, ps[t]));  // cross.f:467
    mz[t] = cadd(mz[t], cik(kz, ps[t]));  // cross.f:469
  }
  d1<C>(d, L, ps, w);  // d(psi)/dy, cross.f:434-437
  ld(d.sb[SB_MY] + off, L, dm);
#pragma unroll
  for (int t = 0; t < C; t++) dm[t] = cadd(dm[t], w[t]);  // cross.f:471
  if (m == 0) {  // 00 modes injected: cross.f:486-491
#pragma unroll
    for (int t = 0; t < C; t++)
      if (t < L.n) {
        mx[t] = make_double2(d.u00[L.s + t], 0.0);
        dm[t] = make_double2(d.v00[L.s + t], 0.0);
        mz[t] = make_double2(d.w00[L.s + t], 0.0);
      }
  }
  st(d.sb[SB_RU] + off, L, mx);
  st(d.sb[SB_RV] + off, L, dm);
  st(d.sb[SB_RW] + off, L, mz);
  // xi-updates (cross.f:420-430), written with the wall BCs of this substep
  ld(d.Rom + off, L, w);
#pragma unroll
  for (int t = 0; t < C; t++) vo[t] = cadd(vo[t], cscale(dtxi, w[t]));
  st(d.vor + off, L, vo);
  ld(d.phi + off, L, vo);
  set_row(vo, L, 0, czero());
  set_row(vo, L, d.my - 1, czero());
  ld(d.Rphi + off, L, w);
#pragma unroll
  for (int t = 0; t < C; t++) vo[t] = cadd(vo[t], cscale(dtxi, w[t]));
  st(d.phi + off, L, vo);
  if (m == 0) {  // u00**, w00** (cross.f:495-498)
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
template <int C>
__global__ void __launch_bounds__(YWARPS * 32) k_tder(Dev d) {
  const int m = mode_of_warp();
  if (m >= d.nmode) return;
  const Lane L = make_lane<C>(d.lpm, d.base, d.extra);
  const size_t off = (size_t)m * d.my;
  const double k2 = __ldg(d.k2 + m);
  double2 T[C], a[C];
  ld(d.scal + off, L, T);
  if (m == 0) {
    set_row(T, L, 0, make_double2(1.0 / d.scal_d[3], 0.0));
    set_row(T, L, d.my - 1, make_double2(1.0 / d.scal_d[4], 0.0));
  } else {
    set_row(T, L, 0, czero());
    set_row(T, L, d.my - 1, czero());
  }
  st(d.scal + off, L, T);
  d1<C>(d, L, T, a);
  st(d.sb[SB_DTDY] + off, L, a);
  d2<C>(d, L, T, a);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(a[t], cscale(k2, T[t]));
  st(d.sb[SB_LAPT] + off, L, a);
}

// ----------------------------------------------------------------------
// z transforms (fourz + localyz2zy / localzy2yz, fou3D.f:80-189)
// ----------------------------------------------------------------------
constexpr int ZYB = 8;  // y lines per block of the z kernels

__device__ __forceinline__ int kz_pad(const Dev &d, int k) { return k <= d.nz1 ? k : k + (d.mgalz - d.mz); }

__global__ void __launch_bounds__(256) k_zinv(Dev d) {
  extern __shared__ double2 sm[];
  const int f = blockIdx.z, i = blockIdx.x, y0 = blockIdx.y * ZYB;
  const int nyb = min(ZYB, d.my - y0), ldz = d.mgalz + 1;
  const double2 *src;
  int mult = 0;  // 0: as is, 1: * i kx, 2: * i kz
  switch (f) {
    case 0: src = d.sb[SB_RU]; break;
    case 1: src = d.sb[SB_RV]; break;
    case 2: src = d.sb[SB_RW]; break;
    case 3: src = d.sb[SB_LAPT]; break;
    case 4: src = d.scal; mult = 1; break;
    case 5: src = d.sb[SB_DTDY]; break;
    case 6: src = d.scal; mult = 2; break;
    default: src = d.scal; break;
  }
  for (int idx = threadIdx.x; idx < ZYB * ldz; idx += blockDim.x) sm[idx] = czero();
  __syncthreads();
  const double kx = d.kx[i];
  for (int idx = threadIdx.x; idx < d.mz * ZYB; idx += blockDim.x) {
    const int k = idx / ZYB, yl = idx - k * ZYB;
    if (yl < nyb) {
      double2 v = __ldg(src + ((size_t)i * d.mz + k) * d.my + y0 + yl);
      if (mult == 1) v = cik(kx, v);
      else if (mult == 2) v = cik(__ldg(d.kz + k), v);
      sm[yl * ldz + kz_pad(d, k)] = v;
    }
  }
  __syncthreads();
  fft_dif<+1>(sm, nyb, ldz, d.fz);
  double2 *dst = d.zb[f];
  for (int idx = threadIdx.x; idx < nyb * d.mgalz; idx += blockDim.x) {
    const int yl = idx / d.mgalz, z = idx - yl * d.mgalz;
    dst[((size_t)i * d.my + y0 + yl) * d.mgalz + z] = sm[yl * ldz + z];
  }
}

__global__ void __launch_bounds__(256) k_zfwd(Dev d) {
  extern __shared__ double2 sm[];
  const int f = blockIdx.z, i = blockIdx.x, y0 = blockIdx.y * ZYB;
  const int nyb = min(ZYB, d.my - y0), ldz = d.mgalz + 1;
  const double2 *src = d.zb[f];
  for (int idx = threadIdx.x; idx < nyb * d.mgalz; idx += blockDim.x) {
    const int yl = idx / d.mgalz, z = idx - yl * d.mgalz;
    sm[yl * ldz + z] = __ldg(src + ((size_t)i * d.my + y0 + yl) * d.mgalz + z);
  }
  __syncthreads();
  fft_dit<-1>(sm, nyb, ldz, d.fz);
  const double dn = 1.0 / (double)d.mgalz;
  double2 *dst = d.sb[f];
  for (int idx = threadIdx.x; idx < d.mz * nyb; idx += blockDim.x) {
    const int k = idx / nyb, yl = idx - k * nyb;
    dst[((size_t)i * d.mz + k) * d.my + y0 + yl] = cscale(dn, sm[yl * ldz + kz_pad(d, k)]);
  }
}

// ----------------------------------------------------------------------
// x transforms + physical-space products: phys2, cross.f:1440-1828.
// Inputs (pairs packed as one complex line each, A + iB):
//   (rho u, rho v) (rho w, lap T) (dT/dx, dT/dy) (dT/dz, T)
// Outputs: (u, v) (w, rho uu) (rho vv, rho ww) (rho uv, rho uw)
//          (rho vw, drho) (DT, 0)
// ----------------------------------------------------------------------
__device__ __forceinline__ void atomic_max_pos(unsigned long long *a, double v) {
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

__global__ void __launch_bounds__(256) k_xphys(Dev d, int ZB, int rk, int do_cfl, int do_diag) {
  extern __shared__ double2 sm[];
  __shared__ unsigned long long s_tmax[32];
  __shared__ double s_red[4][8];
  const int y = blockIdx.y, z0 = blockIdx.x * ZB;
  const int nzb = min(ZB, d.mgalz - z0), N = d.mgalx, ldx = N + 1, nkx = d.nkx;
  for (int idx = threadIdx.x; idx < 4 * ZB * ldx; idx += blockDim.x) sm[idx] = czero();
  if (threadIdx.x < 32) s_tmax[threadIdx.x] = 0ull;
  __syncthreads();
  for (int p = 0; p < 4; p++) {
    const double2 *A = d.zb[2 * p], *B = d.zb[2 * p + 1];
    double2 *cb = sm + (size_t)p * ZB * ldx;
    for (int idx = threadIdx.x; idx < nkx * nzb; idx += blockDim.x) {
      const int k = idx / nzb, l = idx - k * nzb;
      const size_t g = ((size_t)k * d.my + y) * d.mgalz + z0 + l;
      const double2 a = __ldg(A + g), b = __ldg(B + g);
      if (k == 0) {
        cb[l * ldx] = make_double2(a.x, b.x);  // Im of mode 0 dropped (rftsingle.f:85-88)
      } else {
        cb[l * ldx + k] = make_double2(a.x - b.y, a.y + b.x);
        cb[l * ldx + N - k] = make_double2(a.x + b.y, b.x - a.y);
      }
    }
  }
  __syncthreads();
  fft_dif<+1>(sm, 4 * ZB, ldx, d.fx);

  const double dt = d.scal_d[0];
  const double dtxi = dt * d.xi[rk], dtg = dt * d.gama[rk], dtb = dt * d.beta[rk];
  const double ab = d.alpha[rk] / d.beta[rk], ipe = 1.0 / d.peclet;
  double mu = 0.0, mv = 0.0, mw = 0.0, rs = 0.0;
  for (int idx = threadIdx.x; idx < nzb * N; idx += blockDim.x) {
    const int l = idx / N, x = idx - l * N;
    double2 *c0 = sm + (size_t)(0 * ZB + l) * ldx + x;
    double2 *c1 = c0 + (size_t)ZB * ldx, *c2 = c1 + (size_t)ZB * ldx, *c3 = c2 + (size_t)ZB * ldx;
    double2 *c4 = c3 + (size_t)ZB * ldx, *c5 = c4 + (size_t)ZB * ldx;
    const double2 p0 = *c0, p1 = *c1, p2 = *c2, p3 = *c3;
    const double ru = p0.x, rv = p0.y, rw = p1.x, lapT = p1.y, tx = p2.x, ty = p2.y, tz = p3.x, T = p3.y;
    double *rh = d.rhst + ((size_t)y * d.mgalz + z0 + l) * N + x;
    const double rhp = *rh;
    const double u = ru * T, v = rv * T, w = rw * T;            // cross.f:1613-1622
    double tn = T + dtxi * rhp;                                  // cross.f:1626
    double d8 = dtxi * rhp;                                      // cross.f:1627
    const double rhs = -u * tx - v * ty - w * tz + T * lapT * ipe;  // cross.f:1632-1634
    *rh = rhs;
    tn = tn + dtg * rhs;                                         // cross.f:1641
    d8 = d8 + dtg * rhs;                                         // cross.f:1642
    const double drho = (d8 / (T * tn)) / dtb - ab * rhs / (T * T);  // cross.f:1670-1671
    *c0 = make_double2(u, v);
    *c1 = make_double2(w, ru * u);
    *c2 = make_double2(rv * v, rw * w);
    *c3 = make_double2(ru * v, ru * w);
    *c4 = make_double2(rv * w, drho);
    *c5 = make_double2(d8, 0.0);
    if (do_cfl) {
      mu = fmax(mu, fabs(u));
      mv = fmax(mv, fabs(v));
      mw = fmax(mw, fabs(w));
      atomicMax(&s_tmax[l], (unsigned long long)__double_as_longlong(fmax(T, 0.0)));
    }
    if (do_diag) rs += 1.0 / T;
  }
  __syncthreads();
  fft_dit<-1>(sm, 6 * ZB, ldx, d.fx);
  const double dn = 1.0 / (double)N, hdn = 0.5 * dn;
  for (int p = 0; p < 6; p++) {
    const double2 *cb = sm + (size_t)p * ZB * ldx;
    double2 *A = d.zb[2 * p];
    double2 *B = (2 * p + 1 < 11) ? d.zb[2 * p + 1] : nullptr;
    for (int idx = threadIdx.x; idx < nkx * nzb; idx += blockDim.x) {
      const int k = idx / nzb, l = idx - k * nzb;
      const size_t g = ((size_t)k * d.my + y) * d.mgalz + z0 + l;
      const double2 c = cb[l * ldx + k];
      double2 a, b;
      if (k == 0) {
        a = make_double2(c.x * dn, 0.0);
        b = make_double2(c.y * dn, 0.0);
      } else {
        const double2 q = cb[l * ldx + N - k];
        a = make_double2((c.x + q.x) * hdn, (c.y - q.y) * hdn);
        b = make_double2((c.y + q.y) * hdn, (q.x - c.x) * hdn);
      }
      A[g] = a;
      if (B) B[g] = b;
    }
  }
  if (do_cfl || do_diag) {
    mu = warp_max(mu); mv = warp_max(mv); mw = warp_max(mw); rs = warp_sum(rs);
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { s_red[0][wid] = mu; s_red[1][wid] = mv; s_red[2][wid] = mw; s_red[3][wid] = rs; }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int nw = blockDim.x >> 5;
      double a = 0, b = 0, c = 0, r = 0;
      for (int q = 0; q < nw; q++) {
        a = fmax(a, s_red[0][q]); b = fmax(b, s_red[1][q]); c = fmax(c, s_red[2][q]); r += s_red[3][q];
      }
      if (do_cfl) {
        const double hy = d.hy[y];
        double ct = 0.0;
        for (int l = 0; l < nzb; l++) {
          const double DD = ipe * __longlong_as_double((long long)s_tmax[l]);  // cross.f:1704
          ct = fmax(ct, 2.0 * DD * ((d.hxalp / 2) * (d.hxalp / 2) + (d.hzbet / 2) * (d.hzbet / 2) + (1.0 / hy) * (1.0 / hy)));
        }
        atomic_max_pos(d.cflmax + 0, a);
        atomic_max_pos(d.cflmax + 1, b / hy);
        atomic_max_pos(d.cflmax + 2, c);
        atomic_max_pos(d.cflmax + 3, ct);
      }
      if (do_diag) atomicAdd(d.rhom + y, r);
    }
  }
}

// ----------------------------------------------------------------------
// (6a)-(6b) T update and N_i: cross.f:619-682; 00-mode RHS, dw, H00,
// dm, masst and the CFL Deltat: cross.f:686-722, 1416-1429, 1778-1826.
// ----------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(YWARPS * 32) k_post1(Dev d, int rk, int do_cfl, int do_diag) {
  const int m = mode_of_warp();
  if (m >= d.nmode) return;
  const Lane L = make_lane<C>(d.lpm, d.base, d.extra);
  const size_t off = (size_t)m * d.my;
  const int i = m / d.mz, k = m - i * d.mz;
  const double kx = __ldg(d.kx + i), kz = __ldg(d.kz + k);
  double2 a[C], b[C], e[C], g[C];
  ld(d.scal + off, L, a);
  ld(d.sb[ODT] + off, L, b);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = cadd(a[t], b[t]);
  st(d.scal + off, L, a);
  // N_y = -ikx rho uv - d(rho vv)/dy - ikz rho vw
  ld(d.sb[ORVV] + off, L, a);
  d1<C>(d, L, a, b);
  ld(d.sb[ORUV] + off, L, a);
  ld(d.sb[ORVW] + off, L, e);
#pragma unroll
  for (int t = 0; t < C; t++) b[t] = csub(csub(czero(), cik(kx, a[t])), cadd(b[t], cik(kz, e[t])));
  st(d.sb[ORVV] + off, L, b);
  // N_x = -ikx rho uu - d(rho uv)/dy - ikz rho uw
  d1<C>(d, L, a, b);  // b = d(rho uv)/dy
  ld(d.sb[ORUU] + off, L, g);
  ld(d.sb[ORUW] + off, L, a);
#pragma unroll
  for (int t = 0; t < C; t++) g[t] = csub(csub(czero(), cik(kx, g[t])), cadd(b[t], cik(kz, a[t])));
  st(d.sb[ORUU] + off, L, g);
  // N_z = -ikx rho uw - d(rho vw)/dy - ikz rho ww
  d1<C>(d, L, e, g);  // g = d(rho vw)/dy
  ld(d.sb[ORWW] + off, L, e);
#pragma unroll
  for (int t = 0; t < C; t++) e[t] = csub(csub(czero(), cik(kx, a[t])), cadd(g[t], cik(kz, e[t])));
  st(d.sb[ORWW] + off, L, e);
  if (m != 0) return;
  // ---- 00 mode (warp 0): b = d(rho uv)00/dy, g = d(rho vw)00/dy ----
  double2 u[C], du[C];
  ld(d.sb[OU] + off, L, u);
#pragma unroll
  for (int t = 0; t < C; t++) u[t].y = 0.0;
  if (rk == 2 && do_diag) {  // vorticity thickness, cross.f:692-699
    d1<C>(d, L, u, du);
    double mx = 0.0;
#pragma unroll
    for (int t = 0; t < C; t++)
      if (t < L.n) mx = fmax(mx, fabs(du[t].x));
    mx = warp_max(mx);
    if (L.lane == 0) { d.diag[3] = 1.0 / mx; d.diag[4] = d.diag[3] / d.ire; }
  }
  if (rk == 0 && do_diag) {  // momentum thickness, cross.f:1416-1429
    const double2 *U = d.sb[OU];
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
  d2<C>(d, L, u, du);
  double hu = 0.0, hw = 0.0;
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double r = -b[t].x + d.ire * du[t].x;  // cross.f:705
      d.rf0u[L.s + t] = r;
      hu += r * d.hy[L.s + t];
    }
  ld(d.sb[OW] + off, L, u);
#pragma unroll
  for (int t = 0; t < C; t++) u[t].y = 0.0;
  d2<C>(d, L, u, du);
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double r = -g[t].x + d.ire * du[t].x;  // cross.f:706
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

// ----------------------------------------------------------------------
// (6c)-(9) vorticity, Laplacians, RHS(Omega_y), RHS(phi), RK3 update:
// cross.f:748-981.
// ----------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(YWARPS * 32) k_post2(Dev d, int rk) {
  const int m = mode_of_warp();
  if (m >= d.nmode) return;
  const Lane L = make_lane<C>(d.lpm, d.base, d.extra);
  const size_t off = (size_t)m * d.my;
  const int i = m / d.mz, k = m - i * d.mz;
  const double kx = __ldg(d.kx + i), kz = __ldg(d.kz + k), k2 = __ldg(d.k2 + m);
  const double dtg = d.scal_d[0] * d.gama[rk];
  double2 a[C], b[C], oz[C], lc[C];
  ld(d.sb[OU] + off, L, a);
  d1<C>(d, L, a, b);  // du/dy
  ld(d.sb[OV] + off, L, a);
#pragma unroll
  for (int t = 0; t < C; t++) oz[t] = csub(cik(kx, a[t]), b[t]);  // omega_z, cross.f:763
  ld(d.sb[OW] + off, L, b);
  d1<C>(d, L, b, lc);  // dw/dy
#pragma unroll
  for (int t = 0; t < C; t++) {
    const double2 ox = csub(lc[t], cik(kz, a[t]));  // omega_x, cross.f:757
    b[t] = csub(cik(kz, ox), cik(kx, oz[t]));       // (curl omega)_y, cross.f:839
  }
  d2<C>(d, L, b, lc);
#pragma unroll
  for (int t = 0; t < C; t++) lc[t] = csub(lc[t], cscale(k2, b[t]));  // lap (curl omega)_y, cross.f:854
  ld(d.sb[OU] + off, L, a);
  ld(d.sb[OW] + off, L, b);
#pragma unroll
  for (int t = 0; t < C; t++) oz[t] = csub(cik(kz, a[t]), cik(kx, b[t]));  // omega_y, cross.f:760
  d2<C>(d, L, oz, a);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(a[t], cscale(k2, oz[t]));  // lap omega_y, cross.f:829
  ld(d.sb[ORUU] + off, L, b);   // N_x
  ld(d.sb[ORWW] + off, L, oz);  // N_z
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = cadd(csub(cik(kz, b[t]), cik(kx, oz[t])), cscale(d.ire, a[t]));  // cross.f:889
  st(d.Rom + off, L, a);
  {
    double2 v[C];
    ld(d.vor + off, L, v);
#pragma unroll
    for (int t = 0; t < C; t++) v[t] = cadd(v[t], cscale(dtg, a[t]));  // cross.f:969
    st(d.vor + off, L, v);
  }
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = cadd(cik(kx, b[t]), cik(kz, oz[t]));  // cross.f:900
  d1<C>(d, L, a, b);
  ld(d.sb[ORVV] + off, L, a);  // N_y
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = csub(csub(cscale(-k2, a[t]), b[t]), cscale(d.ire, lc[t]));  // cross.f:917
  st(d.Rphi + off, L, a);
  ld(d.phi + off, L, b);
#pragma unroll
  for (int t = 0; t < C; t++) b[t] = cadd(b[t], cscale(dtg, a[t]));  // cross.f:978
  st(d.phi + off, L, b);
}

// ----------------------------------------------------------------------
// (8) psi^{n+1} by solvepsi (cross.f:1092-1104); warp 0 advances the 00
// modes and integrates d(rho)/dt for rho v00 (cross.f:1006-1074).
// ----------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(YWARPS * 32) k_psi(Dev d, int rk, int cfl_step, int do_diag) {
  const int m = mode_of_warp();
  if (m >= d.nmode) return;
  const Lane L = make_lane<C>(d.lpm, d.base, d.extra);
  const size_t off = (size_t)m * d.my;
  double2 a[C], b[C];
  if (m != 0) {
    ld(d.sb[ODRHO] + off, L, a);
    neumann<C>(d, L, m, a, b);
    st(d.psi + off, L, b);
    return;
  }
  // psi00 = 0 (solvepsi with rK = 0)
#pragma unroll
  for (int t = 0; t < C; t++) b[t] = czero();
  st(d.psi + off, L, b);
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
  ld(d.sb[ODRHO] + off, L, a);
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = make_double2((t < L.n) ? a[t].x / d.fmap[L.s + t] : 0.0, 0.0);
  matvec<C, 3>(d.dt11, L, a, b);
  lsolve<C, 3>(b, d.i8L, L);
  usolve<C, 3>(b, d.i8U, L);
  const double v0 = bcast_row(b, L, 0).x, vn = bcast_row(b, L, d.my - 1).x;
  const double trapz = -(vn - v0);  // cross.f:1046
  const double corr = trapz / (1.0 + sqrt(d.scal_d[4] / d.scal_d[3]));  // cross.f:1064-1065
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) {
      const double r = b[t].x - v0;
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

// ----------------------------------------------------------------------
// single-operator kernels (tests)
// ----------------------------------------------------------------------
template <int C>
__global__ void __launch_bounds__(YWARPS * 32) k_op_y(Dev d, int op, const double2 *in, double2 *out, double2 *out2) {
  const int m = mode_of_warp();
  if (m >= d.nmode) return;
  const Lane L = make_lane<C>(d.lpm, d.base, d.extra);
  const size_t off = (size_t)m * d.my;
  double2 a[C], b[C];
  ld(in + off, L, a);
  const double k2 = __ldg(d.k2 + m);
  if (op == 1) {
    d1<C>(d, L, a, b);
    st(out + off, L, b);
  } else if (op == 2) {
    d2<C>(d, L, a, b);
    st(out + off, L, b);
  } else if (op == 3) {
    if (k2 == 0.0) {
#pragma unroll
      for (int t = 0; t < C; t++) b[t] = czero();
      st(out + off, L, b);
      st(out2 + off, L, b);
      return;
    }
    poisson<C>(d, L, m, a, b);
    st(out + off, L, b);
    d1<C>(d, L, b, a);
    st(out2 + off, L, a);
  } else {
    if (k2 == 0.0) {
#pragma unroll
      for (int t = 0; t < C; t++) b[t] = czero();
    } else {
      neumann<C>(d, L, m, a, b);
    }
    st(out + off, L, b);
  }
}

inline dim3 ygrid(const Dev &d) { return dim3((unsigned)((d.nmode + YWARPS - 1) / YWARPS)); }

#define LMC_DISPATCH_C(KERNEL, ...)                                                     \
  do {                                                                                  \
    switch (d.C) {                                                                      \
      case 4: KERNEL<4><<<ygrid(d), YWARPS * 32, 0, s>>>(__VA_ARGS__); break;           \
      case 5: KERNEL<5><<<ygrid(d), YWARPS * 32, 0, s>>>(__VA_ARGS__); break;           \
      case 7: KERNEL<7><<<ygrid(d), YWARPS * 32, 0, s>>>(__VA_ARGS__); break;           \
      case 9: KERNEL<9><<<ygrid(d), YWARPS * 32, 0, s>>>(__VA_ARGS__); break;           \
      case 13: KERNEL<13><<<ygrid(d), YWARPS * 32, 0, s>>>(__VA_ARGS__); break;         \
      default: KERNEL<17><<<ygrid(d), YWARPS * 32, 0, s>>>(__VA_ARGS__); break;         \
    }                                                                                   \
  } while (0)

}  // namespace

void launch_lapv(const Dev &d, cudaStream_t s) { LMC_DISPATCH_C(k_lapv, d); }
void launch_assemble(const Dev &d, int rk, cudaStream_t s) { LMC_DISPATCH_C(k_assemble, d, rk); }
void launch_tder(const Dev &d, cudaStream_t s) { LMC_DISPATCH_C(k_tder, d); }
void launch_post1(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s) {
  LMC_DISPATCH_C(k_post1, d, rk, do_cfl, do_diag);
}
void launch_post2(const Dev &d, int rk, cudaStream_t s) { LMC_DISPATCH_C(k_post2, d, rk); }
void launch_psi(const Dev &d, int rk, int cfl_step, int do_diag, cudaStream_t s) {
  LMC_DISPATCH_C(k_psi, d, rk, cfl_step, do_diag);
}
void launch_op_y(const Dev &d, int op, const double2 *in, double2 *out, double2 *out2, cudaStream_t s) {
  LMC_DISPATCH_C(k_op_y, d, op, in, out, out2);
}

static size_t zsmem(const Dev &d) { return (size_t)ZYB * (d.mgalz + 1) * sizeof(double2); }

void launch_zinv(const Dev &d, cudaStream_t s) {
  dim3 g(d.nkx, (d.my + ZYB - 1) / ZYB, 8);
  k_zinv<<<g, 256, zsmem(d), s>>>(d);
}
void launch_zfwd(const Dev &d, cudaStream_t s) {
  dim3 g(d.nkx, (d.my + ZYB - 1) / ZYB, 11);
  k_zfwd<<<g, 256, zsmem(d), s>>>(d);
}

int xphys_zb(const Dev &d) {
  const size_t per = (size_t)6 * (d.mgalx + 1) * sizeof(double2);
  int zb = (int)((110 * 1024) / per);
  if (zb < 1) zb = 1;
  if (zb > 16) zb = 16;
  return zb;
}
size_t xphys_smem(const Dev &d) { return (size_t)6 * xphys_zb(d) * (d.mgalx + 1) * sizeof(double2); }

void launch_xphys(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s) {
  const int zb = xphys_zb(d);
  dim3 g((d.mgalz + zb - 1) / zb, d.my);
  k_xphys<<<g, 256, xphys_smem(d), s>>>(d, zb, rk, do_cfl, do_diag);
}

// Opt-in to the largest dynamic shared memory each transform kernel can
// use on this device (the opt-in limit minus the kernel's static shared
// memory), so that handles of any grid size can launch them.
static cudaError_t optin(const void *fn, int limit) {
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, fn);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, limit - (int)fa.sharedSizeBytes);
}

cudaError_t kernels_init(const Dev &d) {
  int dev = 0, limit = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if ((size_t)limit < xphys_smem(d) + 1024 || (size_t)limit < zsmem(d) + 1024) return cudaErrorInvalidValue;
  if ((e = optin((const void *)k_xphys, limit)) != cudaSuccess) return e;
  if ((e = optin((const void *)k_zinv, limit)) != cudaSuccess) return e;
  return optin((const void *)k_zfwd, limit);
}

}  // namespace lmc
