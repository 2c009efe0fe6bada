// lmc_fft_impl.cuh -- transform kernels of one lomacte RK3 substep,
// templated on the four-step factorisation N = N1*N2 of the transform
// length, on the complex type CT of the butterflies (and of the lines in
// shared memory) and on the complex type ST of the work buffers in HBM:
//   <double2, double2>  FP64 plain form
//   <float2,  float2>   mixed form (FP32 transforms)
//   <double2, float2>   mixed form with FP64 transform arithmetic
// The pointwise products, the T update and the d(rho)/dt source are FP64
// in every form.  Included by the lmc_fft_*.cu translation units, each of which
// instantiates a group of lengths (they compile in parallel).
//
//   zinv : localyz2zy + fourz(+1) (fou3D.f:80-145): spectral [y][kx][kz]
//          -> zero-padded kz -> inverse c2c along z -> z-physical [y][z][kx]
//   xphys: phys2 (cross.f:1440-1828): per (y,z) line, inverse real x
//          transforms of 8 fields (two per complex transform), FP64
//          products, T update, d(rho)/dt source, CFL maxima, direct x
//          transforms of 11 fields truncated to kx < mx/2
//   zfwd : fourz(-1) + localzy2yz (fou3D.f:149-189): direct c2c along z,
//          truncation to the mz retained kz, back to [y][kx][kz]
#pragma once
#define LMC_FFT_TU
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "lmc_async.cuh"
#include "lmc_kernels.cuh"

using namespace lmcd;

namespace lmc {
namespace LMC_FFT_NS {

// Small blocks (about 64 threads, one task of the first FFT pass per
// thread) so that several blocks share an SM and overlap their
// barrier-separated phases.
constexpr int round32(int v) { return ((v + 31) / 32) * 32; }
template <int N1, int N2>
struct Geo {
  static constexpr int N = N1 * N2;
  static constexpr int LD = Four<N1, N2>::LD | 1;           // odd line stride
  static constexpr int KB = (64 / N1) > 0 ? (64 / N1) : 1;  // kx lines per z-transform block (FP64)
  static constexpr int ZT = round32(KB * N1);               // threads of a z-transform block (FP64)
  static constexpr int ZB = (16 / N1) > 0 ? (16 / N1) : 1;  // z lines per x-transform block
  static constexpr int XT = round32(4 * ZB * N1);           // threads of an x-transform block
  static constexpr int PT = (ZB * N + XT - 1) / XT;         // physical points per thread
};

// Threads of an x-stage block.  With the passive scalar or the variable
// viscosity the x stage stages 12 to 18 inputs and transforms 6 to 9 lines
// per z line, so shared memory admits fewer blocks per SM: those blocks
// get twice the threads (four warps), and for lines of 1152 points and
// more (N1 >= 32), of which only one or two blocks fit an SM, eight warps
// (FP64 butterflies) or nine (FP32: one task per thread in the first pass
// of the nine inverse lines, 9 x 32, and four physical points per thread
// at 1152, kept at two blocks per SM).  At most XW_MAX warps.
template <int N1, int N2, bool WIDE, bool F32>
struct XGeo {
  static constexpr int XT = !WIDE ? Geo<N1, N2>::XT
                            : N1 >= 32 ? (F32 ? 288 : 256)
                                       : (2 * Geo<N1, N2>::XT < 128 ? 2 * Geo<N1, N2>::XT : 128);
  static constexpr int PT = (Geo<N1, N2>::ZB * Geo<N1, N2>::N + XT - 1) / XT;
  // blocks per SM the register budget is sized for (FP32 butterflies; one
  // block of lines longer than 1152 fits an SM's shared memory)
  static constexpr int MINB = !F32 ? 1 : (WIDE && N1 >= 32) ? (N1 * N2 <= 1152 ? 2 : 1) : 512 / XT;
};

// z-transform blocks by butterfly type: twice as many kx lines for FP32
// butterflies (and FP32 storage), so that every strided z row moves the same
// number of bytes; FP64 butterflies keep the FP64 block, whose shared-memory
// lines are twice as wide
template <int N1, int N2, typename CT>
struct ZGeo {
  static constexpr int W = sizeof(CT) == sizeof(float2) ? 2 : 1;
  static constexpr int KB = (64 * W / N1) > 0 ? (64 * W / N1) : 1;
  static constexpr int ZT = round32(KB * N1);
};

__host__ __device__ constexpr size_t round16(size_t b) { return (b + 15) / 16 * 16; }
template <typename TO, typename FROM>
__device__ __forceinline__ TO ccvt(FROM a) {
  return cmk<TO>((typename CReal<TO>::R)a.x, (typename CReal<TO>::R)a.y);
}

__device__ __forceinline__ int kz_pad(const Dev &d, int k) { return k <= d.nz1 ? k : k + (d.mgalz - d.mz); }

// Persistent: each block walks tiles (field, y, kx block) with stride
// gridDim.x; the next tile's kz rows (one contiguous run of nb*mz complex
// values in the [y][kx][kz] layout) arrive by a TMA bulk copy while the
// current tile is transformed.  A bulk copy moves whole 16-byte units, so
// for FP32 values the run is widened to an even start and length and the
// tile is read from offset `lead` in the staging buffer.
// mode 0: the transform inputs of the substep (vbase); mode 1 (2014
// variant, FP64): T before the substep and Delta T, for d(rho)
// (lomacte/cross.f:1760-1770); mode 2 (physical-field export, FP64): the
// export inputs, written in natural z order
template <int N1, int N2, typename CT, typename ST>
__global__ void __launch_bounds__(ZGeo<N1, N2, CT>::ZT) k_zinv(Dev d, int ntiles, int mode, int f0) {
  using F = Four<N1, N2, CT>;
  using G = Geo<N1, N2>;
  using Re = typename CReal<CT>::R;
  constexpr int KB = ZGeo<N1, N2, CT>::KB, LD = G::LD;
  constexpr int E = 16 / (int)sizeof(ST);  // stored values per 16-byte unit
  extern __shared__ __align__(16) unsigned char smraw[];
  CT *W = (CT *)smraw;
  ST *St = (ST *)(smraw + round16(sizeof(CT) * KB * LD));
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_ok;
  // the kx planes zp0 .. zp0+zkn-1 (a slab block; all planes by default),
  // written into z-physical rows of zkn values
  const int nkb = (d.zkn + KB - 1) / KB, per_f = d.my * nkb, vb = vbase(d);
  auto src_of = [&](int f) -> const ST * {
    if constexpr (sizeof(ST) == sizeof(double2)) {
      if (mode == 1) return f == 0 ? d.Told : d.dTs;
      if (mode == 2) return wsb<ST>(d, xslot(f));
    }
    if (f >= vb) {  // variable viscosity: rho u (for d/dx), the sums, rho w (for d/dz)
      switch (f - vb) {
        case 0: return wsb<ST>(d, SB_RU);
        case 1: return wsb<ST>(d, SB_GYY);
        case 2: return wsb<ST>(d, SB_RW);
        case 3: return wsb<ST>(d, SB_G12);
        case 4: return wsb<ST>(d, SB_G13);
        default: return wsb<ST>(d, SB_G23);
      }
    }
    switch (f) {
      case 0: return wsb<ST>(d, SB_RU);
      case 1: return wsb<ST>(d, SB_RV);
      case 2: return wsb<ST>(d, SB_RW);
      case 3: return wsb<ST>(d, SB_LAPT);
      case 5: return wsb<ST>(d, SB_DTDY);
      case 8: return wsb<ST>(d, SB_LAPZ);   // passive scalar: lap Z,
      case 10: return wsb<ST>(d, SB_DZDY);  // dZ/dy,
      case 9:
      case 11:                              // and Z for dZ/dx, dZ/dz
        if constexpr (sizeof(ST) == sizeof(double2)) return d.zsc;
        else return wsb<ST>(d, SB_Z32);
      default:
        if constexpr (sizeof(ST) == sizeof(double2)) return d.tsrc;
        else return wsb<ST>(d, SB_T32);
    }
  };
  auto lead_of = [&](int t) {
    const int r = t % per_f, y = r / nkb, kb = r - y * nkb;
    return (int)((((size_t)y * d.nkx + d.zp0 + kb * KB) * d.mz) % E);
  };
  auto issue = [&](int t) {
    const int fr = t / per_f, f = f0 + fr, r = t - fr * per_f, y = r / nkb, kb = r - y * nkb;
    const int nb = min(KB, d.zkn - kb * KB);
    const size_t start = ((size_t)y * d.nkx + d.zp0 + kb * KB) * d.mz;
    const int lead = (int)(start % E);
    const uint32_t cnt = (uint32_t)(((nb * d.mz + lead + E - 1) / E) * E);
    const uint32_t bytes = cnt * (uint32_t)sizeof(ST);
    mbar_expect_tx(&bar, bytes);
    bulk_g2s(St, src_of(f) + (start - lead), bytes, &bar);
  };
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  int t = blockIdx.x;
  if (threadIdx.x == 0 && t < ntiles) issue(t);
  uint32_t ph = 0;
  const int gap = d.mgalz - d.mz;  // zero-padded kz positions nz1+1 .. nz1+gap
  for (; t < ntiles; t += gridDim.x) {
    if (threadIdx.x == 0) s_ok = mbar_wait(&bar, ph, d.status);
    __syncthreads();
    if (!s_ok) return;
    ph ^= 1;
    const int fr = t / per_f, f = f0 + fr, r = t - fr * per_f, y = r / nkb, kb = r - y * nkb;
    const int i0 = d.zp0 + kb * KB, nb = min(KB, d.zp0 + d.zkn - i0);
    const int lead = lead_of(t);
    // i kx, i kz: of T, Z, and with the variable viscosity of rho u, rho w
    const int mult = mode ? 0 : f >= vb ? (f == vb ? 1 : f == vb + 2 ? 2 : 0)
                                        : (f == 4 || f == 9) ? 1 : (f == 6 || f == 11) ? 2 : 0;
    if constexpr (N2 % 3 == 0) {
      // the first pass reads the staged rows: coefficient k of line il
      auto get = [&](int il, int k) -> CT {
        CT v = ccvt<CT>(St[lead + il * d.mz + k]);
        if (mult == 1) v = cik((Re)__ldg(d.kx + i0 + il), v);
        else if (mult == 2) v = cik((Re)__ldg(d.kz + k), v);
        if constexpr (sizeof(ST) == sizeof(float2))
          if (i0 + il == 0 && k == 0) v = cz<CT>();  // 00 mode: added back in FP64 by xphys
        return v;
      };
      F::template nat2perm_zin<+1>(W, nb, LD, wtwz<CT>(d), get);
      if (threadIdx.x == 0 && t + (int)gridDim.x < ntiles) {  // the staged rows are consumed
        fence_proxy_async();
        issue(t + gridDim.x);
      }
      F::template nat2perm_p2<+1>(W, nb, LD);
    } else {
      for (int idx = threadIdx.x; idx < nb * gap; idx += blockDim.x) {
        const int il = idx / gap, g = idx - il * gap;
        W[il * LD + F::sk(d.nz1 + 1 + g)] = cz<CT>();
      }
      for (int il = 0; il < nb; il++) {
        const Re kx = (Re)__ldg(d.kx + i0 + il);
        const ST *row = St + lead + il * d.mz;
        for (int k = threadIdx.x; k < d.mz; k += blockDim.x) {
          CT v = ccvt<CT>(row[k]);
          if (mult == 1) v = cik(kx, v);
          else if (mult == 2) v = cik((Re)__ldg(d.kz + k), v);
          if constexpr (sizeof(ST) == sizeof(float2))
            if (i0 + il == 0 && k == 0) v = cz<CT>();  // 00 mode: added back in FP64 by xphys
          W[il * LD + F::sk(kz_pad(d, k))] = v;
        }
      }
      __syncthreads();
      if (threadIdx.x == 0 && t + (int)gridDim.x < ntiles) {
        fence_proxy_async();
        issue(t + gridDim.x);
      }
      F::template nat2perm<+1>(W, nb, LD, wtwz<CT>(d));
    }
    ST *dst = wzb<ST>(d, f) + (size_t)y * F::N * d.zkn + (i0 - d.zp0);
    for (int idx = threadIdx.x; idx < F::N * KB; idx += blockDim.x) {
      const int z = idx / KB, il = idx - z * KB;
      // the samples stay in the transform's order (z = k1 + N1 k2 holds the
      // natural sample k2 + N2 k1), except for the export
      const int zr = mode == 2 ? z / N1 + N2 * (z % N1) : z;
      if (il < nb) dst[(size_t)zr * d.zkn + il] = ccvt<ST>(W[il * LD + F::sk(z)]);
    }
    __syncthreads();
  }
}

// mode 0: the substep's outputs (field blockIdx.z in place); mode 1 (2014
// variant): d(rho) from z-physical buffer 0 into the d(rho) spectral slot
template <int N1, int N2, typename CT, typename ST>
__global__ void __launch_bounds__(ZGeo<N1, N2, CT>::ZT) k_zfwd(Dev d, int mode) {
  using F = Four<N1, N2, CT>;
  using G = Geo<N1, N2>;
  using Re = typename CReal<CT>::R;
  extern __shared__ __align__(16) unsigned char smraw[];
  CT *sm = (CT *)smraw;
  constexpr int KB = ZGeo<N1, N2, CT>::KB;
  // the kx planes zp0 .. zp0+zkn-1, from z-physical rows of zkn values
  const int f = mode ? ODRHO : (int)blockIdx.z, y = blockIdx.y, i0 = d.zp0 + blockIdx.x * KB;
  const int nb = min(KB, d.zp0 + d.zkn - i0);
  const ST *src = wzb<ST>(d, mode ? 0 : f) + (size_t)y * N1 * N2 * d.zkn + (i0 - d.zp0);
  // each z row of the tile is a short run (KB values) at stride zkn: every
  // thread issues a batch of BT of these loads before storing any
  constexpr int ZT = ZGeo<N1, N2, CT>::ZT;
  if constexpr (ZT == KB * N1) {  // thread (z0, il) reads rows z0, z0 + N1, ... of line il
    constexpr int BT = N2 % 12 == 0 ? 12 : 8;
    const int il = threadIdx.x % KB, z0 = threadIdx.x / KB;
    if (il < nb) {
      const ST *p = src + (size_t)z0 * d.zkn + il;
      const size_t st = (size_t)N1 * d.zkn;
      CT *q = sm + il * G::LD;
      for (int i = 0; i < N2; i += BT) {
        ST v[BT];
#pragma unroll
        for (int u = 0; u < BT; u++)
          if (i + u < N2) v[u] = __ldg(p + (size_t)(i + u) * st);
#pragma unroll
        for (int u = 0; u < BT; u++)
          if (i + u < N2) q[F::sk(z0 + (i + u) * N1)] = ccvt<CT>(v[u]);
      }
    }
  } else {
    for (int idx = threadIdx.x; idx < F::N * KB; idx += blockDim.x) {
      const int z = idx / KB, il = idx - z * KB;
      if (il < nb) sm[il * G::LD + F::sk(z)] = ccvt<CT>(__ldg(src + (size_t)z * d.zkn + il));
    }
  }
  __syncthreads();
  F::template perm2nat<-1, 2>(sm, nb, G::LD, wtwz<CT>(d));
  const Re dn = (Re)(1.0 / (double)F::N);
  for (int il = 0; il < nb; il++) {
    ST *row = wsb<ST>(d, f) + ((size_t)y * d.nkx + i0 + il) * d.mz;
    for (int k = threadIdx.x; k < d.mz; k += blockDim.x)
      row[k] = ccvt<ST>(cscale(dn, sm[il * G::LD + F::sk(kz_pad(d, k))]));
  }
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long *a, double v) {
  atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

// Input pairs (A + iB per complex transform):
//   (rho u, rho v) (rho w, lap T) (dT/dx, dT/dy) (dT/dz, T)
// Output pairs, first round: (u, v) (w, rho uu) (rho vv, rho ww) (rho uv, rho uw)
// second round (kept in registers meanwhile): (rho vw, drho) (DT, 0)
template <int N1, int N2, typename CT, typename ST>
__device__ __forceinline__ void x_extract(const Dev &d, const CT *sm, int p, int fa, int fb, int y, int z0,
                                          int nzb) {
  using F = Four<N1, N2, CT>;
  using G = Geo<N1, N2>;
  using Re = typename CReal<CT>::R;
  constexpr int N = F::N;
  const Re dn = (Re)(1.0 / (double)N), hdn = (Re)(0.5 / (double)N);
  ST *A = wzb<ST>(d, fa);
  ST *B = fb >= 0 ? wzb<ST>(d, fb) : nullptr;
  for (int l = 0; l < nzb; l++) {
    const size_t g0 = ((size_t)y * d.mgalz + z0 + l - d.xl0) * d.nkx;
    const CT *line = sm + (size_t)(p * G::ZB + l) * G::LD;
    for (int k = threadIdx.x; k < d.nkx; k += blockDim.x) {
      const CT c = line[F::sk(k)];
      CT a, b;
      if (k == 0) {
        a = cmk<CT>(c.x * dn, 0);
        b = cmk<CT>(c.y * dn, 0);
      } else {
        const CT q = line[F::sk(N - k)];
        a = cmk<CT>((c.x + q.x) * hdn, (c.y - q.y) * hdn);
        b = cmk<CT>((c.y + q.y) * hdn, (q.x - c.x) * hdn);
      }
      A[g0 + k] = ccvt<ST>(a);
      if (B) B[g0 + k] = ccvt<ST>(b);
    }
  }
}

// Persistent: each block walks tiles (y, z block of ZB lines).  The next
// tile's eight input rows (each ZB*nkx contiguous complex values in the
// [y][z][kx] layout) and its RHS(T) row arrive by TMA bulk copies while the
// current tile is transformed.  stg = 0 (lengths whose staged rows do not
// fit in shared memory beside the transform lines): only the RHS rows are
// staged and the first transform pass reads the input rows from global
// memory; every row of a tile is read in that pass, before any output row
// of the tile is written (in place, after the direct transforms).  ZS: the passive scalar's four more input
// rows (lap Z, dZ/dx, dZ/dy, dZ/dz), its RHS(Z) row and Delta Z as a
// twelfth output, packed beside Delta T.  VS: the variable viscosity's six
// more input rows (vbase), with T^sigma in the diffusion of T and Z and
// the variable part of the stress taken off the products rho u_i u_j.
// FP32 butterflies: the registers of XGeo::MINB blocks per SM
template <int N1, int N2, typename CT, typename ST, bool ZS, bool VS>
__global__ void __launch_bounds__(XGeo<N1, N2, ZS || VS, sizeof(CT) == sizeof(float2)>::XT,
                                  XGeo<N1, N2, ZS || VS, sizeof(CT) == sizeof(float2)>::MINB)
    k_xphys(Dev d, int rk, int do_cfl, int do_diag, int ntiles, int stg) {
  using F = Four<N1, N2, CT>;
  using G = Geo<N1, N2>;
  using Re = typename CReal<CT>::R;
  constexpr int N = F::N, ZB = G::ZB, LD = G::LD, PT = XGeo<N1, N2, ZS || VS, sizeof(CT) == sizeof(float2)>::PT,
                XT = XGeo<N1, N2, ZS || VS, sizeof(CT) == sizeof(float2)>::XT;
  constexpr int VB = ZS ? 12 : 8;  // first viscosity input
  constexpr int NI = VB + (VS ? 6 : 0), NL = NI / 2, NO = ZS ? 12 : 11, NM = VS ? NMI : ZS ? 8 : 6;
  static_assert(XT / 32 <= XW_MAX, "partial-sum slots assume at most XW_MAX warps per x tile");
  // with six or more transform lines the eleven (twelve) outputs fit in
  // place and go through the direct transforms in one round
  constexpr bool ONE = NL >= 6;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int nkx = d.nkx;  // a multiple of 8 for every supported length
  CT *W = (CT *)smraw;                                        // NL buffers x ZB lines x LD
  ST *St = (ST *)(smraw + round16(sizeof(CT) * NL * ZB * LD));  // NI rows of ZB*nkx inputs (stg)
  double *Sr = (double *)(St + (stg ? NI * ZB * nkx : 0));  // ZB*N RHS(T)
  double *Srz = Sr + ZB * N;                    // ZB*N RHS(Z) (ZS)
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_ok;
  __shared__ unsigned long long s_tmax[ZB], s_vmax;
  __shared__ double s_red[3][XW_MAX];
  __shared__ double s_min[NM], s_est[NO];  // mixed form, per tile
  const int nzk = (d.mgalz + ZB - 1) / ZB;
  // tile t of this launch is tile xt0 + t of the substep (the x stage of a
  // slab block of lines, or all of them); its z-physical rows are local to
  // the block, which starts at line xl0
  auto issue = [&](int t) {
    t += d.xt0;
    const int y = t / nzk, z0 = (t - y * nzk) * ZB, nzb = min(ZB, d.mgalz - z0);
    const uint32_t rb = (uint32_t)nzb * nkx * sizeof(ST), hb = d.variant ? 0u : (uint32_t)nzb * N * sizeof(double);
    mbar_expect_tx(&bar, (stg ? NI * rb : 0u) + (ZS ? 2 : 1) * hb);
    const size_t g0 = ((size_t)y * d.mgalz + z0 - d.xl0) * nkx;
    if (stg)
      for (int f = 0; f < NI; f++) bulk_g2s(St + f * ZB * nkx, wzb<ST>(d, f) + g0, rb, &bar);
    if (hb) bulk_g2s(Sr, d.rhst + ((size_t)y * d.mgalz + z0) * N, hb, &bar);
    if (ZS && hb) bulk_g2s(Srz, d.rhsz + ((size_t)y * d.mgalz + z0) * N, hb, &bar);
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    s_vmax = 0ull;
  }
  for (int l = threadIdx.x; l < ZB; l += blockDim.x) s_tmax[l] = 0ull;
  __syncthreads();
  int t = blockIdx.x;
  if (threadIdx.x == 0 && t < ntiles) issue(t);
  uint32_t ph = 0;
  const double ipe = 1.0 / d.peclet;
  const double dt = d.scal_d[0];
  const double dtxi = dt * d.xi[rk], dtg = dt * d.gama[rk], dtb = dt * d.beta[rk];
  const double ab = d.alpha[rk] / d.beta[rk];
  double mu = 0.0, mw = 0.0, cfy = 0.0, cft = 0.0;  // running maxima (cfy, cft: thread 0)
  for (; t < ntiles; t += gridDim.x) {
    if (threadIdx.x == 0) s_ok = mbar_wait(&bar, ph, d.status);
    __syncthreads();
    if (!s_ok) return;
    ph ^= 1;
    const int tg = d.xt0 + t, y = tg / nzk, z0 = (tg - y * nzk) * ZB, nzb = min(ZB, d.mgalz - z0);
    if constexpr (sizeof(ST) == sizeof(float2)) {  // mixed form: see s_min / s_est below
      const int q = threadIdx.x;
      if (q < NM) s_min[q] = d.mi[(size_t)q * d.my + y];
      if (q < NO) {
        double e;
        if (d.mean_ok) {
          e = d.mo_prev[(size_t)q * d.my + y] / ((double)d.mgalx * (double)d.mgalz);
        } else {  // products of the input means
          const double ru = d.mi[y], rv = d.mi[(size_t)d.my + y], rw = d.mi[(size_t)2 * d.my + y];
          const double T = d.mi[(size_t)5 * d.my + y];
          const double u = ru * T, v = rv * T, w = rw * T;
          switch (q) {
            case OU: e = u; break;
            case OV: e = v; break;
            case OW: e = w; break;
            case ORUU: e = ru * u; break;
            case ORVV: e = rv * v; break;
            case ORWW: e = rw * w; break;
            case ORUV: e = ru * v; break;
            case ORUW: e = ru * w; break;
            case ORVW: e = rv * w; break;
            default: e = 0.0; break;
          }
        }
        s_est[q] = e;
      }
    }
    double rh[PT], rz[ZS ? PT : 1];
#pragma unroll
    for (int j = 0; j < PT; j++) {
      const int q = threadIdx.x + j * blockDim.x;
      rh[j] = (q < nzb * N && !d.variant) ? Sr[q] : 0.0;
      if constexpr (ZS) rz[j] = (q < nzb * N) ? Srz[q] : 0.0;
    }
    // the first transform pass reads the staged input rows directly: line
    // p*ZB + l packs fields 2p, 2p+1 of z line l as A + iB of the complex
    // spectrum, kx = nkx .. N-nkx (the dealiased gap) are zero, and the
    // imaginary part of mode 0 is dropped (rftsingle.f:85-88)
    const size_t gt = ((size_t)y * d.mgalz + z0 - d.xl0) * nkx;  // the tile's rows in global memory
    auto load = [&](int b, int n) -> CT {
      const int p = b / ZB, l = b - p * ZB;
      if (l >= nzb) return cz<CT>();
      const ST *A = stg ? St + (2 * p) * ZB * nkx + l * nkx : wzb<ST>(d, 2 * p) + gt + l * nkx;
      const ST *B = stg ? A + ZB * nkx : wzb<ST>(d, 2 * p + 1) + gt + l * nkx;
      if (n < nkx) {
        const CT a = ccvt<CT>(A[n]), c = ccvt<CT>(B[n]);
        return n == 0 ? cmk<CT>(a.x, c.x) : cmk<CT>(a.x - c.y, a.y + c.x);
      }
      const int k = N - n;
      if (k < nkx) {
        const CT a = ccvt<CT>(A[k]), c = ccvt<CT>(B[k]);
        return cmk<CT>(a.x + c.y, c.x - a.y);
      }
      return cz<CT>();
    };
    if constexpr (N2 % 3 == 0) {  // the gap and the mirrored third by sample row
      auto rows = [&](int b, const ST *&A, const ST *&B) -> bool {
        const int p = b / ZB, l = b - p * ZB;
        if (l >= nzb) return false;
        A = stg ? St + (2 * p) * ZB * nkx + l * nkx : wzb<ST>(d, 2 * p) + gt + l * nkx;
        B = stg ? A + ZB * nkx : wzb<ST>(d, 2 * p + 1) + gt + l * nkx;
        return true;
      };
      F::template nat2perm_in3<+1, ST>(W, NL * ZB, LD, wtwx<CT>(d), rows);
    } else {
      F::template nat2perm_in<+1>(W, NL * ZB, LD, wtwx<CT>(d), load);
    }
    // the staged rows are consumed: stage the next tile meanwhile
    if (threadIdx.x == 0 && t + (int)gridDim.x < ntiles) {
      fence_proxy_async();
      issue(t + gridDim.x);
    }
    F::template nat2perm_p2<+1>(W, NL * ZB, LD);

    // mixed form: s_min / s_est (filled before the transform above) hold the
    // FP64 00 profiles of the inputs at this y and the values subtracted from
    // the outputs before they are rounded to FP32
    constexpr bool MX = sizeof(ST) == sizeof(float2);
    double acc[NO];
    if constexpr (MX) {
#pragma unroll
      for (int o = 0; o < NO; o++) acc[o] = 0.0;
    }

    Re r0[ONE ? 1 : PT], r1[ONE ? 1 : PT], r2[ONE ? 1 : PT], r3[ZS && !ONE ? PT : 1];
    double rs = 0.0, mv = 0.0;
#pragma unroll
    for (int j = 0; j < PT; j++) {
      const int q = threadIdx.x + j * blockDim.x;
      if constexpr (!ONE) {
        r0[j] = r1[j] = r2[j] = 0.0;
        if constexpr (ZS) r3[j] = 0.0;
      }
      if (q < nzb * N) {
        const int l = q / N, pos = q - l * N;
        CT *c0 = W + (size_t)l * LD + F::sk(pos);
        CT *c1 = c0 + (size_t)ZB * LD, *c2 = c1 + (size_t)ZB * LD, *c3 = c2 + (size_t)ZB * LD;
        double2 p0 = to_d2(*c0), p1 = to_d2(*c1), p2 = to_d2(*c2), p3 = to_d2(*c3);
        if constexpr (MX) {
          p0.x += s_min[0]; p0.y += s_min[1]; p1.x += s_min[2]; p1.y += s_min[3]; p2.y += s_min[4];
          p3.y += s_min[5];
        }
        const double ru = p0.x, rv = p0.y, rw = p1.x, lapT = p1.y, tx = p2.x, ty = p2.y, tz = p3.x, T = p3.y;
        const double rhp = rh[j];
        const double u = ru * T, v = rv * T, w = rw * T;                // cross.f:1613-1622
        double tn = T + dtxi * rhp;                                      // cross.f:1626
        double d8 = dtxi * rhp;                                          // cross.f:1627
        double tsg = 1.0;                                                // mu = k = rho D = T^sigma
        double rhs;
        if constexpr (VS) {  // branches/loma/src/cross.f:1591-1596
          tsg = exp(d.sigma * log(T));  // T > 0
          rhs = -u * tx - v * ty - w * tz + tsg * (T * lapT + d.sigma * (tx * tx + ty * ty + tz * tz)) * ipe;
        } else {
          rhs = -u * tx - v * ty - w * tz + T * lapT * ipe;              // cross.f:1632-1634
        }
        if (!d.variant) {  // the 2014 variant keeps RHS(T) spectral (lomacte/cross.f:1452-1456)
          d.rhst[((size_t)y * d.mgalz + z0 + l) * N + pos] = rhs;
          tn = tn + dtg * rhs;                                           // cross.f:1641
          d8 = d8 + dtg * rhs;                                           // cross.f:1642
        }
        double o[NO];
        if constexpr (ZS) {  // the passive scalar, advanced as T is
          CT *c4 = c3 + (size_t)ZB * LD, *c5 = c4 + (size_t)ZB * LD;
          double2 p4 = to_d2(*c4), p5 = to_d2(*c5);
          if constexpr (MX) {
            p4.x += s_min[6];
            p5.x += s_min[7];
          }
          const double lapZ = p4.x, zx = p4.y, zy = p5.x, zz = p5.y;
          double rzs;
          if constexpr (VS) rzs = -u * zx - v * zy - w * zz + tsg * (T * lapZ + d.sigma * (tx * zx + ty * zy + tz * zz)) / d.pez;
          else rzs = -u * zx - v * zy - w * zz + T * lapZ / d.pez;
          d.rhsz[((size_t)y * d.mgalz + z0 + l) * N + pos] = rzs;
          o[ODZ] = dtxi * rz[j] + dtg * rzs;
        }
        o[OU] = u; o[OV] = v; o[OW] = w;
        o[ORUU] = ru * u; o[ORVV] = rv * v; o[ORWW] = rw * w;              // cross.f:1655-1666
        o[ORUV] = ru * v; o[ORUW] = ru * w; o[ORVW] = rv * w;
        if constexpr (VS) {  // minus the variable part of the stress, 2 (T^sigma - 1) S_ij / Re
          const CT *cv = c0 + (size_t)(VB / 2) * ZB * LD;
          double2 g0 = to_d2(cv[0]), g1 = to_d2(cv[(size_t)ZB * LD]), g2 = to_d2(cv[(size_t)2 * ZB * LD]);
          if constexpr (MX) {
            g0.y += s_min[8];
            g1.y += s_min[9];
            g2.y += s_min[10];
          }
          const double c = d.ire * (tsg - 1.0);
          o[ORUU] -= 2.0 * c * (T * g0.x + ru * tx);
          o[ORVV] -= 2.0 * c * (T * g0.y + rv * ty);
          o[ORWW] -= 2.0 * c * (T * g1.x + rw * tz);
          o[ORUV] -= c * (T * g1.y + ru * ty + rv * tx);
          o[ORUW] -= c * (T * g2.x + ru * tz + rw * tx);
          o[ORVW] -= c * (T * g2.y + rv * tz + rw * ty);
        }
        o[ODRHO] = d.variant ? rhs : (d8 / (T * tn)) / dtb - ab * rhs / (T * T);  // cross.f:1670-1671
        o[ODT] = d8;                                                     // cross.f:1645-1647
        if constexpr (MX) {
#pragma unroll
          for (int q = 0; q < NO; q++) {
            acc[q] += o[q];
            o[q] -= s_est[q];
          }
        }
        *c0 = from_d2<CT>(make_double2(o[OU], o[OV]));
        *c1 = from_d2<CT>(make_double2(o[OW], o[ORUU]));
        *c2 = from_d2<CT>(make_double2(o[ORVV], o[ORWW]));
        *c3 = from_d2<CT>(make_double2(o[ORUV], o[ORUW]));
        if constexpr (ONE) {  // lines 4 and 5 of this point are read above
          CT *c4 = c3 + (size_t)ZB * LD, *c5 = c4 + (size_t)ZB * LD;
          *c4 = from_d2<CT>(make_double2(o[ORVW], o[ODRHO]));
          if constexpr (ZS) *c5 = from_d2<CT>(make_double2(o[ODT], o[ODZ]));  // (Delta T, Delta Z)
          else *c5 = from_d2<CT>(make_double2(o[ODT], 0.0));
        } else {
          r0[j] = (Re)o[ORVW];
          r1[j] = (Re)o[ODRHO];
          r2[j] = (Re)o[ODT];
          if constexpr (ZS) r3[j] = (Re)o[ODZ];
        }
        if (do_cfl) {
          mu = fmax(mu, fabs(u));
          mv = fmax(mv, fabs(v));
          mw = fmax(mw, fabs(w));
          if (!d.variant) atomic_max_pos(&s_tmax[l], fmax(T, 0.0));
        }
        if (do_diag) rs += 1.0 / T;
      }
    }
    if (do_diag) {
      rs = warp_sum(rs);
      if ((threadIdx.x & 31) == 0) atomicAdd(d.rhom + y, rs);
    }
    if constexpr (MX) {  // FP64 partial plane sums, one slot per (tile, warp)
      const int slot = (z0 / ZB) * (XT / 32) + (threadIdx.x >> 5);
#pragma unroll
      for (int q = 0; q < NO; q++) {
        const double v = warp_sum(acc[q]);
        if ((threadIdx.x & 31) == 0) d.mpart[((size_t)q * d.my + y) * d.mpart_ld + slot] = v;
      }
    }
    if (do_cfl) {
      mv = warp_max(mv);
      if ((threadIdx.x & 31) == 0) atomic_max_pos(&s_vmax, mv);
    }
    __syncthreads();
    if (do_cfl && threadIdx.x == 0) {  // cross.f:1690-1708 for the lines of this tile
      const double hy = d.hy[y];
      cfy = fmax(cfy, __longlong_as_double((long long)s_vmax) / hy);
      for (int l = 0; l < nzb; l++) {
        // cross.f:1704; with the scalar the larger of the two diffusivities
        const double tm = __longlong_as_double((long long)s_tmax[l]);
        const double DD = (ZS ? fmax(ipe, 1.0 / d.pez) : ipe) * (VS ? pow(tm, 1.0 + d.sigma) : tm);
        cft = fmax(cft, 2.0 * DD * ((d.hxalp / 2) * (d.hxalp / 2) + (d.hzbet / 2) * (d.hzbet / 2) + (1.0 / hy) * (1.0 / hy)));
        s_tmax[l] = 0ull;
      }
      s_vmax = 0ull;
    }
    if constexpr (ONE) {
      F::template perm2nat<-1>(W, 6 * ZB, LD, wtwx<CT>(d));
      x_extract<N1, N2, CT, ST>(d, W, 0, OU, OV, y, z0, nzb);
      x_extract<N1, N2, CT, ST>(d, W, 1, OW, ORUU, y, z0, nzb);
      x_extract<N1, N2, CT, ST>(d, W, 2, ORVV, ORWW, y, z0, nzb);
      x_extract<N1, N2, CT, ST>(d, W, 3, ORUV, ORUW, y, z0, nzb);
      x_extract<N1, N2, CT, ST>(d, W, 4, ORVW, ODRHO, y, z0, nzb);
      if (!d.variant) x_extract<N1, N2, CT, ST>(d, W, 5, ODT, ZS ? ODZ : -1, y, z0, nzb);
      __syncthreads();
      continue;
    }
    F::template perm2nat<-1>(W, 4 * ZB, LD, wtwx<CT>(d));
    x_extract<N1, N2, CT, ST>(d, W, 0, OU, OV, y, z0, nzb);
    x_extract<N1, N2, CT, ST>(d, W, 1, OW, ORUU, y, z0, nzb);
    x_extract<N1, N2, CT, ST>(d, W, 2, ORVV, ORWW, y, z0, nzb);
    x_extract<N1, N2, CT, ST>(d, W, 3, ORUV, ORUW, y, z0, nzb);
    __syncthreads();
#pragma unroll
    for (int j = 0; j < PT; j++) {
      const int q = threadIdx.x + j * blockDim.x;
      if (q < ZB * N) {
        const int l = q / N, pos = q - l * N;
        CT *c0 = W + (size_t)l * LD + F::sk(pos);
        c0[0] = cmk<CT>(r0[j], r1[j]);
        if constexpr (ZS) c0[(size_t)ZB * LD] = cmk<CT>(r2[j], r3[j]);  // (Delta T, Delta Z)
        else c0[(size_t)ZB * LD] = cmk<CT>(r2[j], 0);
      }
    }
    __syncthreads();
    F::template perm2nat<-1>(W, 2 * ZB, LD, wtwx<CT>(d));
    x_extract<N1, N2, CT, ST>(d, W, 0, ORVW, ODRHO, y, z0, nzb);
    if (!d.variant) x_extract<N1, N2, CT, ST>(d, W, 1, ODT, ZS ? ODZ : -1, y, z0, nzb);
    __syncthreads();
  }
  if (do_cfl) {
    mu = warp_max(mu);
    mw = warp_max(mw);
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { s_red[0][wid] = mu; s_red[1][wid] = mw; }
    __syncthreads();
    if (threadIdx.x == 0) {
      double a = 0, c = 0;
      for (int q = 0; q < (int)(blockDim.x >> 5); q++) { a = fmax(a, s_red[0][q]); c = fmax(c, s_red[1][q]); }
      atomic_max_pos(d.cflmax + 0, a);
      atomic_max_pos(d.cflmax + 1, cfy);
      atomic_max_pos(d.cflmax + 2, c);
      atomic_max_pos(d.cflmax + 3, cft);
    }
  }
}

// Physical-field export (FP64): one block per (plane, z tile); the inverse
// x transforms of the export inputs (rows in natural z order, zinv mode 2),
// then per point u = T rho u, v, w, T, omega = T curl(rho u) + grad T x
// rho u (the quantities of tofis_loma's escrphys, trunk/tofis_loma/src/
// escru.f:101-314) and Z, written in natural x order to out[p][q][z][x]
template <int N1, int N2>
__global__ void __launch_bounds__(Geo<N1, N2>::XT) k_xexport(Dev d, const int *jrow, int nplanes, int nf,
                                                             double *out) {
  using F = Four<N1, N2, double2>;
  using G = Geo<N1, N2>;
  constexpr int N = F::N, ZB = G::ZB, LD = G::LD;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2 *W = (double2 *)smraw;
  const int nkx = d.nkx, nzk = (d.mgalz + ZB - 1) / ZB, NL = (nf + 1) / 2, nq = d.scalar ? 8 : 7;
  const int p = blockIdx.x / nzk, z0 = (blockIdx.x - p * nzk) * ZB, nzb = min(ZB, d.mgalz - z0);
  if (p >= nplanes) return;
  const int y = jrow[p];
  auto load = [&](int b, int n) -> double2 {
    const int pr = b / ZB, l = b - pr * ZB;
    if (l >= nzb) return czero();
    const size_t g = ((size_t)y * d.mgalz + z0 + l) * nkx;
    const double2 *A = d.zb[2 * pr] + g;
    const double2 *B = 2 * pr + 1 < nf ? d.zb[2 * pr + 1] + g : nullptr;
    int k = n;
    bool up = false;
    if (n >= nkx) {
      k = N - n;
      up = true;
      if (k >= nkx) return czero();
    }
    const double2 a = A[k], c = B ? B[k] : czero();
    if (!up) return k == 0 ? make_double2(a.x, c.x) : make_double2(a.x - c.y, a.y + c.x);
    return make_double2(a.x + c.y, c.x - a.y);
  };
  F::template nat2perm_in<+1>(W, NL * ZB, LD, d.twx, load);
  F::template nat2perm_p2<+1>(W, NL * ZB, LD);
  for (int q = threadIdx.x; q < nzb * N; q += blockDim.x) {
    const int l = q / N, pos = q - l * N;
    const int x = pos / N1 + N2 * (pos % N1);  // natural x of the sample at pos
    const double2 *c = W + (size_t)l * LD + F::sk(pos);
    const double2 p0 = c[0], p1 = c[(size_t)ZB * LD], p2 = c[(size_t)2 * ZB * LD], p3 = c[(size_t)3 * ZB * LD];
    const double2 p4 = c[(size_t)4 * ZB * LD];
    const double ru = p0.x, rv = p0.y, rw = p1.x, T = p1.y, tx = p2.x, ty = p2.y, tz = p3.x;
    const double v[8] = {ru * T, rv * T, rw * T, T, T * p3.y + ty * rw - tz * rv, T * p4.x + tz * ru - tx * rw,
                         T * p4.y + tx * rv - ty * ru, nf > 10 ? c[(size_t)5 * ZB * LD].x : 0.0};
    double *o = out + (((size_t)p * nq) * d.mgalz + z0 + l) * d.mgalx + x;
    for (int k = 0; k < nq; k++) o[(size_t)k * d.mgalz * d.mgalx] = v[k];
  }
}

// 2014 variant: d(rho) = -Delta T / (T (T + Delta T)) at every physical
// point (tensor2, lomacte/cross.f:1819-1908): T and Delta T arrive as one
// complex line per (y, z), the result leaves in z-physical buffer 0.
template <int N1, int N2>
__global__ void __launch_bounds__(Geo<N1, N2>::XT) k_xdrho(Dev d) {
  using F = Four<N1, N2, double2>;
  using G = Geo<N1, N2>;
  constexpr int N = F::N, ZB = G::ZB, LD = G::LD;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2 *W = (double2 *)smraw;
  const int y = blockIdx.y, z0 = blockIdx.x * ZB, nzb = min(ZB, d.mgalz - z0), nkx = d.nkx;
  const int gap = N - 2 * nkx + 1;
  for (int idx = threadIdx.x; idx < ZB * gap; idx += blockDim.x) {
    const int ln = idx / gap, g = idx - ln * gap;
    W[ln * LD + F::sk(nkx + g)] = czero();
  }
  for (int l = 0; l < ZB; l++) {
    double2 *line = W + l * LD;
    const size_t g0 = ((size_t)y * d.mgalz + z0 + l) * nkx;
    for (int k = threadIdx.x; k < nkx; k += blockDim.x) {
      double2 a = czero(), b = czero();
      if (l < nzb) {
        a = d.zb[0][g0 + k];
        b = d.zb[1][g0 + k];
      }
      if (k == 0) {
        line[F::sk(0)] = make_double2(a.x, b.x);
      } else {
        line[F::sk(k)] = make_double2(a.x - b.y, a.y + b.x);
        line[F::sk(N - k)] = make_double2(a.x + b.y, b.x - a.y);
      }
    }
  }
  __syncthreads();
  F::template nat2perm<+1>(W, ZB, LD, d.twx);
  for (int q = threadIdx.x; q < ZB * N; q += blockDim.x) {
    const int l = q / N, pos = q - l * N;
    double2 *c = W + (size_t)l * LD + F::sk(pos);
    const double T = c->x, dT = c->y;
    *c = make_double2(-dT / (T * (T + dT)), 0.0);  // lomacte/cross.f:1881
  }
  __syncthreads();
  F::template perm2nat<-1>(W, ZB, LD, d.twx);
  x_extract<N1, N2, double2, double2>(d, W, 0, 0, -1, y, z0, nzb);
}

// Statistics of the physical fields on an accumulating substep (phys2,
// cross.f:1583-1607): per y row the plane sums of u rho u, u rho v,
// u rho w, v rho v, v rho w, w rho w (u_i = rho u_i T), 1/T, T^sigma and
// T^(sigma+1).  Block (g, y) inverts rho u, rho v, rho w and T (three
// complex x transforms per z line, the same packing as k_xphys) on the z
// tiles g, g + ngrp, ... of row y before k_xphys overwrites its inputs and
// writes its partial sums to st.xpart; k_xsum adds the ngrp partials of a
// row in order, so the sums are reproducible.
template <int N1, int N2, typename CT, typename ST>
__global__ void __launch_bounds__(Geo<N1, N2>::XT) k_xstats(Dev d, Stats st, int ngrp) {
  using F = Four<N1, N2, CT>;
  using G = Geo<N1, N2>;
  constexpr int N = F::N, ZB = G::ZB, LD = G::LD, NW = G::XT / 32;
  extern __shared__ __align__(16) unsigned char smraw[];
  CT *W = (CT *)smraw;  // 3 groups x ZB lines x LD
  __shared__ double sh[NW * 9];
  const int y = blockIdx.y, grp = blockIdx.x, nkx = d.nkx, my = d.my;
  double m0 = 0.0, m1 = 0.0, m2 = 0.0, m5 = 0.0;  // mixed form: FP64 00 profiles
  if constexpr (sizeof(ST) == sizeof(float2)) {
    m0 = d.mi[y];
    m1 = d.mi[(size_t)my + y];
    m2 = d.mi[(size_t)2 * my + y];
    m5 = d.mi[(size_t)5 * my + y];
  }
  const double sg = st.sigma, sg1 = st.sigma + 1.0;
  double a[9];
#pragma unroll
  for (int q = 0; q < 9; q++) a[q] = 0.0;
  const int gap = N - 2 * nkx + 1;
  for (int z0 = grp * ZB; z0 < d.mgalz; z0 += ngrp * ZB) {
    const int nzb = min(ZB, d.mgalz - z0);
    for (int idx = threadIdx.x; idx < 3 * ZB * gap; idx += blockDim.x) {
      const int ln = idx / gap, g = idx - ln * gap;
      W[ln * LD + F::sk(nkx + g)] = cz<CT>();
    }
    for (int gp = 0; gp < 3; gp++) {
      const int p = gp < 2 ? gp : 3;  // line pairs (rho u, rho v), (rho w, -), (-, T)
      for (int l = 0; l < ZB; l++) {
        CT *line = W + (gp * ZB + l) * LD;
        const size_t g0 = ((size_t)y * d.mgalz + z0 + l) * nkx;
        const ST *A = wzb<ST>(d, 2 * p) + g0, *B = wzb<ST>(d, 2 * p + 1) + g0;
        for (int k = threadIdx.x; k < nkx; k += blockDim.x) {
          CT ca = cz<CT>(), cb = cz<CT>();
          if (l < nzb) { ca = ccvt<CT>(A[k]); cb = ccvt<CT>(B[k]); }
          if (k == 0) {
            line[F::sk(0)] = cmk<CT>(ca.x, cb.x);
          } else {
            line[F::sk(k)] = cmk<CT>(ca.x - cb.y, ca.y + cb.x);
            line[F::sk(N - k)] = cmk<CT>(ca.x + cb.y, cb.x - ca.y);
          }
        }
      }
    }
    __syncthreads();
    F::template nat2perm<+1>(W, 3 * ZB, LD, wtwx<CT>(d));
    for (int q = threadIdx.x; q < nzb * N; q += blockDim.x) {
      const int l = q / N, pos = q - l * N;
      const CT *c0 = W + (size_t)l * LD + F::sk(pos);
      const double2 p0 = to_d2(c0[0]), p1 = to_d2(c0[(size_t)ZB * LD]), p3 = to_d2(c0[(size_t)2 * ZB * LD]);
      const double ru = p0.x + m0, rv = p0.y + m1, rw = p1.x + m2, T = p3.y + m5;
      const double u = ru * T, v = rv * T, w = rw * T;
      a[0] += u * ru;
      a[1] += u * rv;
      a[2] += u * rw;
      a[3] += v * rv;
      a[4] += v * rw;
      a[5] += w * rw;
      a[6] += 1.0 / T;
      a[7] += pow(T, sg);
      a[8] += pow(T, sg1);
    }
    __syncthreads();
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 9; q++) {
    const double v = warp_sum(a[q]);
    if (lane == 0) sh[wid * 9 + q] = v;
  }
  __syncthreads();
  if (threadIdx.x < 9) {
    const int q = threadIdx.x;
    double s = 0.0;
    for (int w = 0; w < NW; w++) s += sh[w * 9 + q];
    st.xpart[((size_t)q * my + y) * ngrp + grp] = s;
  }
}

// the partial sums of k_xstats, group by group, into the profiles
template <int N1, int N2>
__global__ void k_xsum(Dev d, Stats st, int ngrp) {
  const int y = blockIdx.x, q = threadIdx.x;
  if (q >= 9) return;
  const double *src = st.xpart + ((size_t)q * d.my + y) * ngrp;
  double s = 0.0;
  for (int g = 0; g < ngrp; g++) s += src[g];
  const int dst = q < 7 ? ST_RUU + q : ST_MUM + (q - 7);  // ruu..rww, rhom, mum, num
  st.prof[(size_t)dst * d.my + y] += s;
}

// Plane sums of the mixed form's outputs from the partial sums of k_xphys,
// added in a fixed order so that a run is reproducible bit for bit.
template <int N1, int N2>
__global__ void __launch_bounds__(128) k_msum(Dev d, int nslot) {
  __shared__ double red[128];
  const int y = blockIdx.x, q = blockIdx.y;
  const double *src = d.mpart + ((size_t)q * d.my + y) * d.mpart_ld;
  double s = 0.0;
  for (int i = threadIdx.x; i < nslot; i += blockDim.x) s += src[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int h = 64; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) d.mo_cur[(size_t)q * d.my + y] = red[0];
}

template <int N1, int N2, typename CT, typename ST>
struct Launch {
  using G = Geo<N1, N2>;
  static constexpr int E = 16 / (int)sizeof(ST);
  using ZG = ZGeo<N1, N2, CT>;
  static size_t zsm() { return (size_t)ZG::KB * G::LD * sizeof(CT); }
  static size_t zinv_sm(int mz) {
    return round16(sizeof(CT) * ZG::KB * G::LD) + ((size_t)ZG::KB * mz + 2 * E) * sizeof(ST);
  }
  static constexpr int nin(bool zs, bool vs) { return (zs ? 12 : 8) + (vs ? 6 : 0); }
  static size_t xsm(bool zs, bool vs) { return round16(sizeof(CT) * (nin(zs, vs) / 2) * G::ZB * G::LD); }
  // stg: with the input rows staged in shared memory
  static size_t xphys_sm(int nkx, bool zs = false, bool vs = false, bool stg = true) {
    return xsm(zs, vs) + (stg ? (size_t)nin(zs, vs) * G::ZB * nkx * sizeof(ST) : 0) +
           (size_t)(zs ? 2 : 1) * G::ZB * G::N * sizeof(double);
  }
  // the staged form where it fits in a block's shared memory
  static bool xphys_stg(int nkx, bool zs, bool vs, int limit) {
    return xphys_sm(nkx, zs, vs, true) + 1024 <= (size_t)limit;
  }
  // resident blocks per SM x SMs, for the persistent kernels
  static int grid_for(const void *fn, int threads, size_t smem, int ntiles) {
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem);
    if (per < 1) per = 1;
    const int g = sms * per;
    return g < ntiles ? g : ntiles;
  }
  // fields f0 .. f0+nf-1 of the eight inputs (nf <= 0: all of them)
  static void zinv(const Dev &d, int mode, int f0, int nf, cudaStream_t s) {
    if (nf <= 0) {
      f0 = 0;
      nf = mode ? 2 : 8;
    }
    const int ntiles = nf * d.my * ((d.zkn + ZG::KB - 1) / ZG::KB);
    const size_t sm = zinv_sm(d.mz);
    const int g = grid_for((const void *)k_zinv<N1, N2, CT, ST>, ZG::ZT, sm, ntiles);
    k_zinv<N1, N2, CT, ST><<<g, ZG::ZT, sm, s>>>(d, ntiles, mode, f0);
  }
  static void zfwd(const Dev &d, int mode, cudaStream_t s) {
    dim3 g((d.zkn + ZG::KB - 1) / ZG::KB, d.my, mode ? 1 : (d.variant ? 10 : n_out(d)));
    k_zfwd<N1, N2, CT, ST><<<g, ZG::ZT, zsm(), s>>>(d, mode);
  }
  static size_t xexport_sm() { return (size_t)6 * G::ZB * G::LD * sizeof(double2); }
  static void xexport(const Dev &d, const int *jrow, int nplanes, int nf, double *out, cudaStream_t s) {
    if constexpr (sizeof(CT) == sizeof(double2) && sizeof(ST) == sizeof(double2)) {
      const int nzk = (d.mgalz + G::ZB - 1) / G::ZB;
      k_xexport<N1, N2><<<nplanes * nzk, G::XT, xexport_sm(), s>>>(d, jrow, nplanes, nf, out);
    }
  }
  static void xdrho(const Dev &d, cudaStream_t s) {
    if constexpr (sizeof(CT) == sizeof(double2) && sizeof(ST) == sizeof(double2)) {
      dim3 g((d.mgalz + G::ZB - 1) / G::ZB, d.my);
      k_xdrho<N1, N2><<<g, G::XT, (size_t)G::ZB * G::LD * sizeof(double2), s>>>(d);
    }
  }
  template <bool ZS, bool VS>
  static void xphys_zs(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s) {
    const int ntiles = d.xnt > 0 ? d.xnt : d.my * ((d.mgalz + G::ZB - 1) / G::ZB);
    constexpr int XT = XGeo<N1, N2, ZS || VS, sizeof(CT) == sizeof(float2)>::XT;
    const void *fn = (const void *)k_xphys<N1, N2, CT, ST, ZS, VS>;
    // stage the input rows (TMA, one tile ahead) where that keeps as many
    // blocks per SM as reading them in the first transform pass would
    bool stg = d.xstg && xphys_stg(d.nkx, ZS, VS, d.smem_limit);
    if (stg) {
      int a = 0, b = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, fn, XT, xphys_sm(d.nkx, ZS, VS, true));
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, XT, xphys_sm(d.nkx, ZS, VS, false));
      stg = a >= b;
    }
    const size_t sm = xphys_sm(d.nkx, ZS, VS, stg);
    const int g = grid_for(fn, XT, sm, ntiles);
    k_xphys<N1, N2, CT, ST, ZS, VS><<<g, XT, sm, s>>>(d, rk, do_cfl, do_diag, ntiles, (int)stg);
    if (sizeof(ST) == sizeof(float2) && d.msum) {
      const int nslot = ((d.mgalz + G::ZB - 1) / G::ZB) * (XT / 32);
      k_msum<N1, N2><<<dim3(d.my, n_out(d)), 128, 0, s>>>(d, nslot);
    }
  }
  static void xphys(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s) {
    if (d.visc) {
      if (d.scalar) xphys_zs<true, true>(d, rk, do_cfl, do_diag, s);
      else xphys_zs<false, true>(d, rk, do_cfl, do_diag, s);
    } else {
      if (d.scalar) xphys_zs<true, false>(d, rk, do_cfl, do_diag, s);
      else xphys_zs<false, false>(d, rk, do_cfl, do_diag, s);
    }
  }
  static size_t xstats_sm() { return (size_t)3 * G::ZB * G::LD * sizeof(CT); }
  static void xstats(const Dev &d, const Stats &st, cudaStream_t s) {
    const int ntile = (d.mgalz + G::ZB - 1) / G::ZB, ngrp = ntile < XGRP ? ntile : XGRP;
    k_xstats<N1, N2, CT, ST><<<dim3(ngrp, d.my), G::XT, xstats_sm(), s>>>(d, st, ngrp);
    k_xsum<N1, N2><<<d.my, 32, 0, s>>>(d, st, ngrp);
  }
  static cudaError_t optin1(const void *fn, int limit) {
    cudaError_t e;
    cudaFuncAttributes fa;
    if ((e = cudaFuncGetAttributes(&fa, fn)) != cudaSuccess) return e;
    return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, limit - (int)fa.sharedSizeBytes);
  }
  static cudaError_t optin(int limit) {
    cudaError_t e;
    if ((e = optin1((const void *)k_zinv<N1, N2, CT, ST>, limit)) != cudaSuccess) return e;
    if ((e = optin1((const void *)k_zfwd<N1, N2, CT, ST>, limit)) != cudaSuccess) return e;
    if ((e = optin1((const void *)k_xstats<N1, N2, CT, ST>, limit)) != cudaSuccess) return e;
    if constexpr (sizeof(CT) == sizeof(double2) && sizeof(ST) == sizeof(double2))
      if ((e = optin1((const void *)k_xexport<N1, N2>, limit)) != cudaSuccess) return e;
    if ((e = optin1((const void *)k_xphys<N1, N2, CT, ST, true, true>, limit)) != cudaSuccess) return e;
    if ((e = optin1((const void *)k_xphys<N1, N2, CT, ST, false, true>, limit)) != cudaSuccess) return e;
    if ((e = optin1((const void *)k_xphys<N1, N2, CT, ST, true, false>, limit)) != cudaSuccess) return e;
    return optin1((const void *)k_xphys<N1, N2, CT, ST, false, false>, limit);
  }
};

// register-DFT twiddles exp(-2 pi i e / R) of every block size
inline cudaError_t upload_twiddles() {
  std::vector<double2> t;
  std::vector<float2> tf;
  for (int R : TW_SIZES)
    for (int e = 0; e < R; e++) {
      const long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)e / (long double)R;
      t.push_back(make_double2((double)cosl(a), (double)(-sinl(a))));
      tf.push_back(make_float2((float)cosl(a), (float)(-sinl(a))));
    }
  cudaError_t e = cudaMemcpyToSymbol(c_tw, t.data(), t.size() * sizeof(double2));
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_twf, tf.data(), tf.size() * sizeof(float2));
}

}  // namespace LMC_FFT_NS
}  // namespace lmc

// Each translation unit defines LMC_FFT_SIZES(X) as X(N, N1, N2) entries and
// then expands LMC_FFT_TU_BODY(suffix) to get its dispatch functions.
#define LMC_FFT_FORMS(N1, N2, CALL)                                   \
  switch (d.prec) {                                                   \
    case 1: Launch<N1, N2, float2, float2>::CALL; break;              \
    case 2: Launch<N1, N2, double2, float2>::CALL; break;             \
    default: Launch<N1, N2, double2, double2>::CALL; break;           \
  }
// precision 1 with bit BIT of d.fft64 set: FP64 butterflies for this stage
#define LMC_FFT_FORMS_M(N1, N2, BIT, CALL)                                \
  switch (d.prec) {                                                       \
    case 1:                                                               \
      if (d.fft64 & (BIT)) Launch<N1, N2, double2, float2>::CALL;         \
      else Launch<N1, N2, float2, float2>::CALL;                          \
      break;                                                              \
    case 2: Launch<N1, N2, double2, float2>::CALL; break;                 \
    default: Launch<N1, N2, double2, double2>::CALL; break;               \
  }
#define LMC_FFT_CASE_Z(N, N1, N2, WHAT) \
  case N: LMC_FFT_FORMS_M(N1, N2, 4, WHAT(d, mode, s)) return true;
#define LMC_FFT_CASE_XD(N, N1, N2) \
  case N: Launch<N1, N2, double2, double2>::xdrho(d, s); return true;
#define LMC_FFT_CASE_X(N, N1, N2) \
  case N: LMC_FFT_FORMS_M(N1, N2, 2, xphys(d, rk, do_cfl, do_diag, s)) return true;
#define LMC_FFT_CASE_XE(N, N1, N2) \
  case N: Launch<N1, N2, double2, double2>::xexport(d, jrow, nplanes, nf, out, s); return true;
#define LMC_FFT_CASE_XST(N, N1, N2) \
  case N: LMC_FFT_FORMS(N1, N2, xstats(d, st, s)) return true;
#define LMC_FFT_CASE_ZI(N, N1, N2) \
  case N: LMC_FFT_FORMS_M(N1, N2, 1, zinv(d, mode, f0, nf, s)) return true;
#define LMC_FFT_CASE_ZF(N, N1, N2) LMC_FFT_CASE_Z(N, N1, N2, zfwd)
#define LMC_FFT_CASE_ZS(N, N1, N2) case N: return Launch<N1, N2, double2, double2>::zinv_sm(2 * (N / 3));
#define LMC_FFT_CASE_XS(N, N1, N2) case N: return Launch<N1, N2, double2, double2>::xphys_sm(N / 3, zs, vs, false);
#define LMC_FFT_CASE_OPT(N, N1, N2)                                                         \
  if ((e = Launch<N1, N2, double2, double2>::optin(limit)) != cudaSuccess) return e;        \
  if ((e = Launch<N1, N2, float2, float2>::optin(limit)) != cudaSuccess) return e;          \
  if ((e = Launch<N1, N2, double2, float2>::optin(limit)) != cudaSuccess) return e;
#define LMC_FFT_CASE_HAS(N, N1, N2) case N: return true;

#define LMC_FFT_TU_BODY(SUF)                                                                      \
  namespace lmc {                                                                                 \
  using namespace LMC_FFT_NS;                                                                     \
  bool fft_has_##SUF(int n) {                                                                     \
    switch (n) { LMC_FFT_SIZES(LMC_FFT_CASE_HAS) default: return false; }                         \
  }                                                                                               \
  bool fft_zinv_##SUF(const Dev &d, int mode, int f0, int nf, cudaStream_t s) {                   \
    switch (d.mgalz) { LMC_FFT_SIZES(LMC_FFT_CASE_ZI) default: return false; }                     \
  }                                                                                               \
  bool fft_zfwd_##SUF(const Dev &d, int mode, cudaStream_t s) {                                   \
    switch (d.mgalz) { LMC_FFT_SIZES(LMC_FFT_CASE_ZF) default: return false; }                     \
  }                                                                                               \
  bool fft_xdrho_##SUF(const Dev &d, cudaStream_t s) {                                            \
    switch (d.mgalx) { LMC_FFT_SIZES(LMC_FFT_CASE_XD) default: return false; }                     \
  }                                                                                               \
  bool fft_xphys_##SUF(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s) {           \
    switch (d.mgalx) { LMC_FFT_SIZES(LMC_FFT_CASE_X) default: return false; }                      \
  }                                                                                               \
  bool fft_xexport_##SUF(const Dev &d, const int *jrow, int nplanes, int nf, double *out, cudaStream_t s) { \
    switch (d.mgalx) { LMC_FFT_SIZES(LMC_FFT_CASE_XE) default: return false; }                     \
  }                                                                                               \
  bool fft_xstats_##SUF(const Dev &d, const Stats &st, cudaStream_t s) {                          \
    switch (d.mgalx) { LMC_FFT_SIZES(LMC_FFT_CASE_XST) default: return false; }                    \
  }                                                                                               \
  size_t fft_zsm_##SUF(int n) {                                                                   \
    switch (n) { LMC_FFT_SIZES(LMC_FFT_CASE_ZS) default: return 0; }                             \
  }                                                                                               \
  size_t fft_xsm_##SUF(int n, bool zs, bool vs) {                                                \
    switch (n) { LMC_FFT_SIZES(LMC_FFT_CASE_XS) default: return 0; }                              \
  }                                                                                               \
  cudaError_t fft_init_##SUF(int limit) {                                                         \
    cudaError_t e = upload_twiddles();                                                            \
    if (e != cudaSuccess) return e;                                                               \
    LMC_FFT_SIZES(LMC_FFT_CASE_OPT)                                                               \
    return cudaSuccess;                                                                           \
  }                                                                                               \
  }
