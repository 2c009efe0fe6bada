// lmc_stats.cuh -- statistics and spectra of an accumulating step on the
// device: addstats1 (cross.f:1981-2064) and addstats2 (cross.f:2070-2290)
// of trunk/lomacte3.  The physical-space sums of phys2 (cross.f:1583-1607)
// are k_xstats in lmc_fft_impl.cuh.
//
// Row kernels (one block per y row, threads over the row's modes) form the
// per-row sums over all modes; every sum is added in a fixed order (each
// thread its modes in order, then a shuffle tree, then the warps in order),
// so a run is reproducible bit for bit.  Weights follow the reference: the
// kx = 0 plane once, every other plane twice (its conjugate half of the x
// spectrum).  In the mixed forms the FP32 work buffers carry the 00 mode
// only rounded (rho u_i) or not at all (u, v, w: the transforms carry
// fluctuations), so the 00 values come from the FP64 profiles.
#pragma once
#include "lmc_ytpm.cuh"

namespace lmc {
namespace stats {

using namespace lmcd;
using tpm::mixed;

constexpr int SRT = 256;  // threads of a row kernel

// NV sums over the block, valid in thread 0; sh holds (SRT/32)*NV doubles
template <int NV>
__device__ __forceinline__ void block_sums(double (&v)[NV], double *sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; q++) v[q] = warp_sum(v[q]);
  if (lane == 0)
#pragma unroll
    for (int q = 0; q < NV; q++) sh[wid * NV + q] = v[q];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NV; q++) {
      double s = 0.0;
      for (int w = 0; w < SRT / 32; w++) s += sh[w * NV + q];
      v[q] = s;
    }
  __syncthreads();
}

// rho u_i (f = 0, 1, 2) at row j, mode m, before the transforms
template <typename CT>
__device__ __forceinline__ double2 ru_val(const Dev &d, int f, size_t row, int j, int m) {
  if constexpr (mixed<CT>())
    if (m == 0) return make_double2(d.mi[(size_t)f * d.my + j], 0.0);
  return to_d2(wsb<CT>(d, SB_RU + f)[row + m]);
}
// u, v, w (q = 0, 1, 2) at row j, mode m, after the transforms
template <typename CT>
__device__ __forceinline__ double2 uvw_val(const Dev &d, int q, size_t row, int j, int m) {
  if constexpr (mixed<CT>())
    if (m == 0) return tpm::mo00_row(d, OU + q, j);
  return to_d2(wsb<CT>(d, OU + q)[row + m]);
}

__device__ __forceinline__ double abs2(double2 a) { return a.x * a.x + a.y * a.y; }

// vorticity of one mode from u, v, w and du/dy, dw/dy (cross.f:755-766):
// o1 = dw/dy - i kz v, o2 = i kz u - i kx w, o3 = i kx v - du/dy
struct Vort {
  double2 o1, o2, o3;
  __device__ __forceinline__ Vort(double a, double b, double2 u, double2 v, double2 w, double2 du, double2 dw) {
    o1 = make_double2(dw.x + b * v.y, dw.y - b * v.x);
    o2 = make_double2(-b * u.y + a * w.y, b * u.x - a * w.x);
    o3 = make_double2(-a * v.y - du.x, a * v.x - du.y);
  }
};

// spectra slot of (kx plane i, field var, spectra plane iy, |kz| k)
__device__ __forceinline__ double *spec_at(const Dev &d, const Stats &st, int i, int var, int iy, int k) {
  return st.spec + (((size_t)i * 12 + var) * st.nsp + iy) * (d.nz1 + 1) + k;
}

// ----------------------------------------------------------------------
// addstats1 (cross.f:1981-2064): spectra of rho u, rho v, rho w, T at the
// spectra planes, Tp, and the 00 means rum, rvm, rwm, Tm.  T is the state
// at the start of the substep with its wall values set (k_tder wrote them).
// ----------------------------------------------------------------------
template <typename CT>
__global__ void __launch_bounds__(SRT) k_srow1(Dev d, Stats st) {
  __shared__ double sh[SRT / 32];
  const int j = blockIdx.x, my = d.my, nm = d.nmode, mz = d.mz, nk = d.nz1 + 1;
  const size_t row = (size_t)j * nm;
  const double2 *T = d.scal + row;
  double v[1] = {0.0};
  for (int m = threadIdx.x; m < nm; m += SRT) v[0] += (m < mz ? 1.0 : 2.0) * abs2(T[m]);  // cross.f:2034-2046
  block_sums<1>(v, sh);
  if (threadIdx.x == 0) {  // cross.f:2050-2058
    st.prof[(size_t)ST_TP * my + j] += v[0];
    st.prof[(size_t)ST_RUM * my + j] += ru_val<CT>(d, 0, row, j, 0).x;
    st.prof[(size_t)ST_RVM * my + j] += ru_val<CT>(d, 1, row, j, 0).x;
    st.prof[(size_t)ST_RWM * my + j] += ru_val<CT>(d, 2, row, j, 0).x;
    st.prof[(size_t)ST_TM * my + j] += T[0].x;
  }
  for (int iy = 0; iy < st.nsp; iy++) {  // cross.f:2005-2031
    if (st.jsp[iy] != j) continue;
    for (int p = threadIdx.x; p < d.nkx * nk; p += SRT) {
      const int i = p / nk, k = p - i * nk;
      const double f = i ? 2.0 : 1.0;
      const int m1 = i * mz + k, m2 = i * mz + (mz - k);
#pragma unroll
      for (int q = 0; q < 4; q++) {
        double *sp = spec_at(d, st, i, 8 + q, iy, k);
        double s = *sp + f * abs2(q < 3 ? ru_val<CT>(d, q, row, j, m1) : T[m1]);
        if (k > 0) s += f * abs2(q < 3 ? ru_val<CT>(d, q, row, j, m2) : T[m2]);
        *sp = s;
      }
    }
  }
}

// ----------------------------------------------------------------------
// du/dy, dv/dy, dw/dy of the transform outputs u, v, w into st.dy: one
// thread per mode, the forward half of deryr2 written to st.dy and the
// backward half applied in place (cross.f:749-750, 2152)
// ----------------------------------------------------------------------
template <typename CT>
__global__ void __launch_bounds__(tpm::TB) t_sdy(Dev d, Stats st) {
  using namespace tpm;
  Mode M;
  if (!mode_of(d, M)) return;
  const int my = d.my;
  const size_t ld = d.nmode;
  const bool m00 = M.m == 0;
  double2 *o0 = st.dy[0] + M.m, *o1 = st.dy[1] + M.m, *o2 = st.dy[2] + M.m;
  {
    Rd<CT, kq<CT>(3)> ru, rv, rw;
    ru.start(wsb<CT>(d, OU) + M.m, ld, my, 1, 0);
    rv.start(wsb<CT>(d, OV) + M.m, ld, my, 1, 0);
    rw.start(wsb<CT>(d, OW) + M.m, ld, my, 1, 0);
    Win wu, wv, ww;
    wu.clear();
    wv.clear();
    ww.clear();
    Hist h0, h1, h2;
    h0.clear();
    h1.clear();
    h2.clear();
    auto feed = [&](int r) {
      double2 a = ru.pop(), b = rv.pop(), c = rw.pop();
      if constexpr (mixed<CT>())
        if (m00 && r < my) {
          a = mo00_row(d, OU, r);
          b = mo00_row(d, OV, r);
          c = mo00_row(d, OW, r);
        }
      wu.push(a);
      wv.push(b);
      ww.push(c);
    };
    for (int t = 0; t < 3; t++) feed(t);
    #pragma unroll 2
    for (int j = 0; j < my; j++) {
      feed(j + 3);
      o0[(size_t)j * ld] = d1f(d, j, wu, h0);
      o1[(size_t)j * ld] = d1f(d, j, wv, h1);
      o2[(size_t)j * ld] = d1f(d, j, ww, h2);
    }
  }
  {
    // each row is read (queued) before the same thread overwrites it
    Rd<double2, 4> r0, r1, r2;
    r0.start(o0, ld, my, -1, my - 1);
    r1.start(o1, ld, my, -1, my - 1);
    r2.start(o2, ld, my, -1, my - 1);
    Hist h0, h1, h2;
    h0.clear();
    h1.clear();
    h2.clear();
    #pragma unroll 2
    for (int j = my - 1; j >= 0; j--) {
      const double2 a = d1b(d, j, r0.pop(), h0), b = d1b(d, j, r1.pop(), h1), c = d1b(d, j, r2.pop(), h2);
      o0[(size_t)j * ld] = a;
      o1[(size_t)j * ld] = b;
      o2[(size_t)j * ld] = c;
    }
  }
}

// ----------------------------------------------------------------------
// addstats2 (cross.f:2070-2290): intensities, Reynolds stresses and
// vorticity intensities (nine energies), the dilatation terms thep and
// theup, the dissipation ep, the 00 means, and the spectra of u, v, w,
// uv (re, im) and the vorticities at the spectra planes
// ----------------------------------------------------------------------
template <typename CT>
__global__ void __launch_bounds__(SRT) k_srow2(Dev d, Stats st) {
  __shared__ double sh[(SRT / 32) * 12];
  const int j = blockIdx.x, my = d.my, nm = d.nmode, mz = d.mz, nk = d.nz1 + 1;
  const size_t row = (size_t)j * nm;
  const double2 *DU = st.dy[0] + row, *DV = st.dy[1] + row, *DW = st.dy[2] + row;
  double e[12];  // nine energies (cross.f:2153-2182), thep, theup, ep
#pragma unroll
  for (int q = 0; q < 12; q++) e[q] = 0.0;
  for (int m = threadIdx.x; m < nm; m += SRT) {
    const int i = m / mz, kk = m - i * mz;
    const double a = __ldg(d.kx + i), b = __ldg(d.kz + kk), f = i ? 2.0 : 1.0;
    const double2 u = uvw_val<CT>(d, 0, row, j, m), v = uvw_val<CT>(d, 1, row, j, m),
                  w = uvw_val<CT>(d, 2, row, j, m);
    const double2 du = DU[m], dv = DV[m], dw = DW[m];
    const Vort o(a, b, u, v, w, du, dw);
    const double uu = abs2(u), vv = abs2(v), ww = abs2(w);
    e[0] += f * uu;
    e[1] += f * vv;
    e[2] += f * ww;
    e[3] += f * (u.x * v.x + u.y * v.y);
    e[4] += f * (u.x * w.x + u.y * w.y);
    e[5] += f * (w.x * v.x + w.y * v.y);
    e[6] += f * abs2(o.o1);
    e[7] += f * abs2(o.o2);
    e[8] += f * abs2(o.o3);
    // dilatation i kx u + dv/dy + i kz w (cross.f:2184-2188)
    const double2 cc = make_double2(-a * u.y + dv.x - b * w.y, a * u.x + dv.y + b * w.x);
    e[9] += f * abs2(cc);
    e[10] += f * (cc.x * v.x + cc.y * v.y);
    // dissipation (cross.f:2190-2203)
    const double2 c1 = make_double2(o.o1.x - b * v.y, o.o1.y + b * v.x);
    const double2 c3 = make_double2(o.o3.x + a * v.y, o.o3.y - a * v.x);
    e[11] += f * ((a * a + b * b) * (uu + vv + ww) + abs2(dv) + abs2(c1) + abs2(c3));
  }
  block_sums<12>(e, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < 9; q++) {
      st.prof[(size_t)(ST_UP + q) * my + j] += e[q];
      st.erow[(size_t)q * my + j] = e[q];
    }
    st.prof[(size_t)ST_THEP * my + j] += e[9];
    st.prof[(size_t)ST_THEUP * my + j] += e[10];
    st.prof[(size_t)ST_EP * my + j] += e[11];
    // 00 means (cross.f:2279-2289)
    const double2 u = uvw_val<CT>(d, 0, row, j, 0), v = uvw_val<CT>(d, 1, row, j, 0),
                  w = uvw_val<CT>(d, 2, row, j, 0);
    const Vort o(0.0, 0.0, u, v, w, DU[0], DW[0]);
    st.prof[(size_t)ST_UM * my + j] += u.x;
    st.prof[(size_t)ST_VM * my + j] += v.x;
    st.prof[(size_t)ST_WM * my + j] += w.x;
    st.prof[(size_t)ST_W1M * my + j] += o.o1.x;
    st.prof[(size_t)ST_W2M * my + j] += o.o2.x;
    st.prof[(size_t)ST_W3M * my + j] += o.o3.x;
    st.prof[(size_t)ST_THEM * my + j] += DV[0].x;
  }
  for (int iy = 0; iy < st.nsp; iy++) {  // cross.f:2100-2147
    if (st.jsp[iy] != j) continue;
    for (int p = threadIdx.x; p < d.nkx * nk; p += SRT) {
      const int i = p / nk, k = p - i * nk;
      const double f = i ? 2.0 : 1.0, a = __ldg(d.kx + i);
      double s[8];
#pragma unroll
      for (int q = 0; q < 8; q++) s[q] = *spec_at(d, st, i, q, iy, k);
      for (int h = 0; h < (k > 0 ? 2 : 1); h++) {
        const int kk = h ? mz - k : k, m = i * mz + kk;
        const double b = __ldg(d.kz + kk);
        const double2 u = uvw_val<CT>(d, 0, row, j, m), v = uvw_val<CT>(d, 1, row, j, m),
                      w = uvw_val<CT>(d, 2, row, j, m);
        const Vort o(a, b, u, v, w, DU[m], DW[m]);
        s[0] += f * abs2(u);
        s[1] += f * abs2(v);
        s[2] += f * abs2(w);
        s[3] += f * (u.x * v.x + u.y * v.y);
        s[4] += f * (u.y * v.x - u.x * v.y);
        s[5] += f * abs2(o.o1);
        s[6] += f * abs2(o.o2);
        s[7] += f * abs2(o.o3);
      }
#pragma unroll
      for (int q = 0; q < 8; q++) *spec_at(d, st, i, q, iy, k) = s[q];
    }
  }
}

// uner_q = sum_j hy_j erow_q(j), j in order (cross.f:2207-2210)
__global__ void k_suner(Dev d, Stats st) {
  const int q = threadIdx.x;
  if (q >= 9) return;
  double s = 0.0;
  for (int j = 0; j < d.my; j++) s += st.erow[(size_t)q * d.my + j] * d.hy[j];
  st.uner[q] = s;
}

}  // namespace stats
}  // namespace lmc
