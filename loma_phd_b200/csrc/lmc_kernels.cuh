// lmc_kernels.cuh -- kernel parameter blocks and launch entry points.
#pragma once
#include <cuda_runtime.h>

#include "lmc_device.cuh"

namespace lmc {

// Device-side view of one case.  Spectral fields are complex double in the
// reference layout [kx][kz][y]; z-physical intermediates are [kx][y][z]
// (z in digit-reversed order); the physical RHS(T) accumulator is
// [y][z][x] (x in digit-reversed order).
struct Dev {
  int my, mgalx, mgalz, nkx, mz, nz1, nmode;
  int lpm, base, extra, C;  // y-chunking of a pencil over the lanes of a warp
  double ire, peclet, cfl, hxalp, hzbet;
  double gama[3], xi[3], alpha[3], beta[3];
  // y operators
  const double *dt12, *dt11, *dt22, *dt21, *p1L, *p1U, *p3L, *p3U, *i8L, *i8U;
  const double *fmap, *hy, *trp, *y, *ebot, *etop;
  // per-mode Poisson data
  const double *PL, *PU, *V12, *AAinv, *k2;
  const double *kx, *kz;  // wavenumber per kx plane / kz index
  lmcd::FFTPlan fx, fz;
  // state
  double2 *vor, *phi, *psi, *scal, *Rom, *Rphi;
  double *u00, *v00, *w00, *rf0u, *rf0w, *rf0v;
  // spectral work buffers (11) and z-physical buffers (11)
  double2 *sb[11];
  double2 *zb[11];
  double *rhst;
  // device scalars: [0] Deltat, [1] dtr, [2] time, [3] rhobot, [4] rhotop
  double *scal_d;
  unsigned long long *cflmax;  // [4] max|u|, max|v|/hy, max|w|, max cflT (as ordered bits)
  double *rhom;                // [my] plane sums of 1/T
  double *diag;                // [16]
  int *status;
};

// Spectral work-buffer roles.
enum { SB_RU = 0, SB_RV, SB_RW, SB_LAPT, SB_DTDY, SB_MY, SB_DMY };
enum { OU = 0, OV, OW, ORUU, ORVV, ORWW, ORUV, ORUW, ORVW, ODRHO, ODT };

// Launchers (lmc_kernels.cu).
void launch_lapv(const Dev &d, cudaStream_t s);
void launch_assemble(const Dev &d, int rk, cudaStream_t s);
void launch_tder(const Dev &d, cudaStream_t s);
void launch_zinv(const Dev &d, cudaStream_t s);
void launch_xphys(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s);
void launch_zfwd(const Dev &d, cudaStream_t s);
void launch_post1(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s);
void launch_post2(const Dev &d, int rk, cudaStream_t s);
void launch_psi(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s);
int xphys_zb(const Dev &d);
size_t xphys_smem(const Dev &d);
cudaError_t kernels_init(const Dev &d);
// operator-level entry points (tests)
void launch_op_y(const Dev &d, int op, const double2 *in, double2 *out, double2 *out2, cudaStream_t s);

}  // namespace lmc
