// lmc_kernels.cuh -- kernel parameter blocks and launch entry points.
#pragma once
#include <cuda_runtime.h>

#include "lmc_device.cuh"

namespace lmc {

constexpr int NWB = 18;  // work-buffer slots: 12 + 6 transform inputs at most

// Device-side view of one case.
//   spectral fields   complex [y][kx][kz]            (kz fastest)
//   z-physical fields complex [y][z][kx]             (kx fastest, z permuted)
//   RHS(T) physical   real    [y][z][x]              (x permuted)
// The reference layout [kx][kz][y] is used only at the C ABI and converted
// by the transpose kernels.
struct Dev {
  int prec;  // 0: FP64; 1: mixed (FP32 work buffers and transforms);
             // 2: mixed with FP64 transform arithmetic (FP32 work buffers)
  int fft64;  // precision 1: FP64 butterflies for the stages set here
              // (1 inverse z, 2 x stage, 4 direct z)
  int my, mgalx, mgalz, nkx, mz, nz1, nmode;
  int lpm, base, extra, C;  // y-chunking of a pencil over the lanes of a warp
  int ldy;                  // staging stride of a pencil (odd, >= my)
  int zb_x, kb_z;           // lines per block of the x / z transform kernels
  int smem_limit;           // opt-in shared memory per block of the device (bytes)
  int xstg;                 // 1: the x stage stages its input rows where they fit (LMC_XSTG=0: never)
  // Slab blocks (lmc_step_split; the whole domain otherwise): the z
  // transforms cover kx planes zp0 .. zp0+zkn-1 with z-physical rows of zkn
  // values; the x stage covers its tiles xt0 .. xt0+xnt-1 (xnt 0: all), whose
  // z-physical rows start at line xl0; msum 0 skips the mixed form's plane
  // sums after the x stage (all blocks but the last)
  int zp0, zkn, xt0, xnt, xl0, msum;
  double ire, peclet, cfl, hxalp, hzbet;
  double gama[3], xi[3], alpha[3], beta[3];
  // y operators: band rows and precomputed scan tables
  const double *dt12, *dt11, *dt22, *dt21, *p1L, *p1U, *p3L, *p3U, *i8L, *i8U;
  const double *k1L, *k1U, *k3L, *k3U, *k8L, *k8U;
  const double *fmap, *hy, *trp, *y, *ebot, *etop;
  // per-mode Poisson data
  const double *PL, *PU, *V12, *AAinv, *k2;
  // Mode-parallel y kernels (tpm = 1, lmc_ytpm.cuh): the same operators in
  // row form ([my][band], one row read by all threads of a warp), per-mode
  // Poisson tables mode-fastest ([my][band][nmode]), and five FP64
  // spectral scratch fields for the forward halves of the banded solves
  // (the fifth is the psi solve's, which runs beside post1 and post2).
  int tpm;
  // 2014 variant (trunk/lomacte): spectral T before this substep's update,
  // its increment Delta T, and the previous substep's spectral RHS(T);
  // tsrc is the T the transforms read (scal, or Told in the variant)
  int variant;
  double2 *Told, *dTs, *RT;
  const double2 *tsrc;
  const double *r_dt12, *r_dt11, *r_dt22, *r_dt21, *r_p1L, *r_p1U, *r_p3L, *r_p3U, *r_fmap, *r_ebot, *r_etop;
  const double *PLt, *PUt, *V12t;
  double2 *ws[5];
  const double *kx, *kz;  // wavenumber per kx plane / kz index
  const double2 *twx, *twz;  // exp(-2 pi i e / N) for the x / z transform lengths
  const float2 *twxf, *twzf;  // the same in FP32 (mixed form)
  // state
  double2 *vor, *phi, *psi, *scal, *Rom, *Rphi;
  double *u00, *v00, *w00, *rf0u, *rf0w, *rf0v;
  double2 *sb[NWB];  // spectral work buffers (FP64 form; [7..9] also staging)
  double2 *zb[NWB];  // z-physical work buffers (FP64 form)
  float2 *sbf[NWB];  // spectral work buffers (mixed form)
  float2 *zbf[NWB];  // z-physical work buffers (mixed form)
  // buffers beyond the 11th exist only with the passive scalar or the
  // variable viscosity
  // Passive scalar Z (scalar = 1): the spectral state, the physical RHS(Z)
  // of the previous substep, and Re*Sc; its wall values live in scal_d[5],
  // scal_d[6].  Z is advanced as T is: derivatives, transforms, physical
  // RK3 accumulator, increment transformed back.
  int scalar;
  double pez;
  double2 *zsc;
  double *rhsz;
  // Variable viscosity (visc = 1): mu = k = rho D = T^sigma.  The products
  // rho u_i u_j lose the variable part of the stress 2 (T^sigma - 1) S_ij /
  // Re, formed per point from six more transform inputs (the symmetric sums
  // of d(rho u_i)/dx_j, see vbase); T's and Z's diffusion take T^sigma.
  int visc;
  double sigma;
  double2 *vscr;  // [3][my] scratch of the mixed forms' exact 00 strain-rate inputs
  double *rhst;
  // device scalars: [0] Deltat, [1] dtr, [2] time, [3] rhobot, [4] rhotop
  double *scal_d;
  unsigned long long *cflmax;  // [4] max|u|, max|v|/hy, max|w|, max cflT (ordered bits)
  double *rhom;                // [my] plane sums of 1/T
  // Mixed form: the kx = kz = 0 (00) modes bypass the FP32 transforms.
  //   mi     [11][my] 00 profiles of the transform inputs rho u, rho v,
  //                   rho w, lap T, dT/dy, T, with the scalar lap Z,
  //                   dZ/dy, and with the variable viscosity d(rho v)/dy,
  //                   d(rho u)/dy, d(rho w)/dy (FP64); zinv drops the 00
  //                   coefficient and xphys adds the profile back per point
  //   mo_cur [12][my] FP64 plane sums of the 11 (12) transform outputs (their
  //                   exact 00 modes times mgalx*mgalz), read by post1/psi
  //   mo_prev[11][my] the sums of the previous substep: xphys subtracts
  //                   prev/(mgalx*mgalz) before rounding an output to FP32,
  //                   so the FP32 transforms carry fluctuations only
  //   mean_ok         0 until mo_prev holds a substep's sums
  //   mpart  [11][my][mpart_ld] per-(tile, warp) partial sums of xphys,
  //          added in a fixed order into mo_cur by k_msum
  double *mi, *mo_cur, *mo_prev, *mpart;
  int mean_ok, mpart_ld;
  double *diag;                // [16]
  int *status;
};

// Statistics accumulators of one case (lmc_stats_reset allocates them):
// what addstats1 / addstats2 (cross.f:1981-2290) and the physical sums of
// phys2 (cross.f:1583-1607) accumulate while istati = 1.
//   prof [NSTAT][my]  raw profiles in the order of the .sta record
//                     (escru.f:381-402), without its 1/(mgalx*mgalz)
//   spec [nkx][12][nsp][nz1+1] spectra (the .spe plane records,
//                     escru.f:445-448), FP64 here, real*4 in the reference
//   erow [9][my]      this step's per-row sums of the nine energies
//   uner [9]          sum_j hy_j erow_j (cross.f:2207-2210)
//   dy   [3]          du/dy, dv/dy, dw/dy of the step ([y][kx][kz])
//   jsp  [nsp]        0-based rows of the spectra planes
//   xpart[9][my][XGRP] partial physical-space sums (z-tile groups)
struct Stats {
  double *prof, *spec, *erow, *uner, *xpart;
  double2 *dy[3];
  const int *jsp;
  int nsp;
  double sigma;  // mu/mu0 = T^sigma (main.f:570)
};
constexpr int NSTAT = 33;
constexpr int XGRP = 32;  // z-tile groups of the physical-space sums
// warps of an x-stage block at most: the mixed form's partial-sum slots
// (Dev::mpart) hold one value per (z tile, warp)
constexpr int XW_MAX = 9;
enum {
  ST_UM = 0, ST_VM, ST_WM, ST_RUM, ST_RVM, ST_RWM, ST_TM, ST_W1M, ST_W2M, ST_W3M, ST_THEM,
  ST_UP, ST_VP, ST_WP, ST_UVR, ST_UWR, ST_VWR, ST_W1P, ST_W2P, ST_W3P, ST_TP, ST_EP,
  ST_RUU, ST_RUV, ST_RUW, ST_RVV, ST_RVW, ST_RWW, ST_RHOM, ST_THEP, ST_THEUP, ST_MUM, ST_NUM
};

// Spectral work-buffer roles before / after the transforms.
// SB_T32 holds an FP32 copy of T for the z transforms of the mixed form;
// SB_LAPZ, SB_DZDY and SB_Z32 (the same for Z) are used with the scalar;
// SB_GYY .. SB_G23 with the variable viscosity: d(rho v)/dy and the sums
// d(rho u)/dy + d(rho v)/dx, d(rho u)/dz + d(rho w)/dx, d(rho v)/dz +
// d(rho w)/dy (written by t_sgrad, read by the inverse z transforms).
enum { SB_RU = 0, SB_RV, SB_RW, SB_LAPT, SB_DTDY, SB_MY, SB_DMY, SB_T32, SB_LAPZ, SB_DZDY, SB_Z32,
       SB_GYY, SB_G12, SB_G13, SB_G23 };
enum { OU = 0, OV, OW, ORUU, ORVV, ORWW, ORUV, ORUW, ORVW, ODRHO, ODT, ODZ };
// Transform inputs: 8 (rho u, rho v, rho w, lap T, dT/dx, dT/dy, dT/dz,
// T), 4 more with the scalar (lap Z, dZ/dx, dZ/dy, dZ/dz), and from vbase
// 6 more with the variable viscosity (d(rho u)/dx, d(rho v)/dy,
// d(rho w)/dz, and the SB_G12, SB_G13, SB_G23 sums); outputs 11, 12 with
// the scalar.
__host__ __device__ inline int vbase(const Dev &d) { return d.scalar ? 12 : 8; }
__host__ __device__ inline int n_in(const Dev &d) { return vbase(d) + (d.visc ? 6 : 0); }
__host__ __device__ inline int n_out(const Dev &d) { return d.scalar ? 12 : 11; }
// spectral and z-physical work buffers a case allocates
__host__ __device__ inline int n_sbuf(const Dev &d) { return d.visc ? SB_G23 + 1 : n_out(d); }
__host__ __device__ inline int n_zbuf(const Dev &d) { return n_in(d) > n_out(d) ? n_in(d) : n_out(d); }
// 00 profiles held for the mixed form's transform inputs
constexpr int NMI = 11;
// Physical-field export (FP64 work buffers of its own): spectral slot of
// export input q = 0..10 (rho u, rho v, rho w, T, dT/dx, dT/dy, dT/dz,
// curl(rho u) x, y, z, Z), past SB_MY and SB_DMY, which Lapvdvhom fills
__host__ __device__ inline int xslot(int q) { return q < 5 ? q : q + 2; }

// work-buffer views of the two precisions
template <typename CT>
__device__ __forceinline__ CT *wsb(const Dev &d, int i) {
  if constexpr (sizeof(CT) == sizeof(double2)) return d.sb[i];
  else return d.sbf[i];
}
template <typename CT>
__device__ __forceinline__ CT *wzb(const Dev &d, int i) {
  if constexpr (sizeof(CT) == sizeof(double2)) return d.zb[i];
  else return d.zbf[i];
}
template <typename CT>
__device__ __forceinline__ const CT *wtwx(const Dev &d) {
  if constexpr (sizeof(CT) == sizeof(double2)) return d.twx;
  else return d.twxf;
}
template <typename CT>
__device__ __forceinline__ const CT *wtwz(const Dev &d) {
  if constexpr (sizeof(CT) == sizeof(double2)) return d.twz;
  else return d.twzf;
}

bool fft_supported(int n);
void launch_lapv(const Dev &d, cudaStream_t s);
void launch_assemble(const Dev &d, int rk, cudaStream_t s);
void launch_tder(const Dev &d, cudaStream_t s);
// passive scalar: Z wall values, dZ/dy, lap Z; and Z += Delta Z
void launch_zder(const Dev &d, cudaStream_t s);
void launch_zupd(const Dev &d, cudaStream_t s);
// variable viscosity: the SB_GYY .. SB_G23 inputs from rho u_i (after
// launch_assemble)
void launch_sgrad(const Dev &d, cudaStream_t s);
// physical-field export (FP64 Dev of the export's own buffers): the
// spectral inputs (after launch_lapv), then, after launch_zinv mode 2, the
// planes jrow[0..nplanes-1] (0-based) of the nq quantities into
// out[p][q][z][x]
void launch_xprep(const Dev &d, cudaStream_t s);
void launch_xexport(const Dev &d, const int *jrow, int nplanes, int nf, double *out, cudaStream_t s);
// mode 1 (2014 variant): the d(rho) round trip of T and Delta T; mode 2
// (export, FP64): the inputs in slots xslot(f), rows in natural z order;
// f0, nf: only inputs f0 .. f0+nf-1 (nf <= 0: all)
void launch_zinv(const Dev &d, cudaStream_t s, int mode = 0, int f0 = 0, int nf = 0);
void launch_xdrho(const Dev &d, cudaStream_t s);
void launch_xphys(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s);
void launch_zfwd(const Dev &d, cudaStream_t s, int mode = 0);
void launch_cfl14(const Dev &d, int do_cfl, cudaStream_t s);
void launch_post1(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s);
void launch_post2(const Dev &d, int rk, cudaStream_t s);
void launch_psi(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s);
void launch_psi_main(const Dev &d, int rk, cudaStream_t s);
void launch_psi_tail(const Dev &d, int rk, int cfl_step, cudaStream_t s);
// reference layout [kx][kz][y] <-> device layout [y][kx][kz]
void launch_ref2dev(const Dev &d, const double2 *in, double2 *out, cudaStream_t s);
void launch_dev2ref(const Dev &d, const double2 *in, double2 *out, cudaStream_t s);
// operator-level entry point (tests), device layout
void launch_op_y(const Dev &d, int op, const double2 *in, double2 *out, double2 *out2, cudaStream_t s);
// statistics of an accumulating substep: addstats1 after the assembly of
// rho u_i (before the transforms), the physical sums between the inverse z
// transforms and k_xphys, addstats2 after the direct z transforms
void launch_stats1(const Dev &d, const Stats &st, cudaStream_t s);
void launch_xstats(const Dev &d, const Stats &st, cudaStream_t s);
void launch_stats2(const Dev &d, const Stats &st, cudaStream_t s);
size_t xphys_smem(const Dev &d);
size_t z_smem(const Dev &d);
cudaError_t kernels_init(const Dev &d);

}  // namespace lmc
