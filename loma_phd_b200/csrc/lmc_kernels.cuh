// lmc_kernels.cuh -- kernel parameter blocks and launch entry points.
#pragma once
#include <cuda_runtime.h>

#include "lmc_device.cuh"

namespace lmc {

// Device-side view of one case.
//   spectral fields   complex [y][kx][kz]            (kz fastest)
//   z-physical fields complex [y][z][kx]             (kx fastest, z permuted)
//   RHS(T) physical   real    [y][z][x]              (x permuted)
// The reference layout [kx][kz][y] is used only at the C ABI and converted
// by the transpose kernels.
struct Dev {
  int my, mgalx, mgalz, nkx, mz, nz1, nmode;
  int lpm, base, extra, C;  // y-chunking of a pencil over the lanes of a warp
  int ldy;                  // staging stride of a pencil (odd, >= my)
  int zb_x, kb_z;           // lines per block of the x / z transform kernels
  double ire, peclet, cfl, hxalp, hzbet;
  double gama[3], xi[3], alpha[3], beta[3];
  // y operators: band rows and precomputed scan tables
  const double *dt12, *dt11, *dt22, *dt21, *p1L, *p1U, *p3L, *p3U, *i8L, *i8U;
  const double *k1L, *k1U, *k3L, *k3U, *k8L, *k8U;
  const double *fmap, *hy, *trp, *y, *ebot, *etop;
  // per-mode Poisson data
  const double *PL, *PU, *V12, *AAinv, *k2;
  const double *kx, *kz;  // wavenumber per kx plane / kz index
  const double2 *twx, *twz;  // exp(-2 pi i e / N) for the x / z transform lengths
  // state
  double2 *vor, *phi, *psi, *scal, *Rom, *Rphi;
  double *u00, *v00, *w00, *rf0u, *rf0w, *rf0v;
  double2 *sb[11];  // spectral work buffers
  double2 *zb[11];  // z-physical work buffers
  double *rhst;
  // device scalars: [0] Deltat, [1] dtr, [2] time, [3] rhobot, [4] rhotop
  double *scal_d;
  unsigned long long *cflmax;  // [4] max|u|, max|v|/hy, max|w|, max cflT (ordered bits)
  double *rhom;                // [my] plane sums of 1/T
  double *diag;                // [16]
  int *status;
};

// Spectral work-buffer roles before / after the transforms.
enum { SB_RU = 0, SB_RV, SB_RW, SB_LAPT, SB_DTDY, SB_MY, SB_DMY };
enum { OU = 0, OV, OW, ORUU, ORVV, ORWW, ORUV, ORUW, ORVW, ODRHO, ODT };

bool fft_supported(int n);
void launch_lapv(const Dev &d, cudaStream_t s);
void launch_assemble(const Dev &d, int rk, cudaStream_t s);
void launch_tder(const Dev &d, cudaStream_t s);
void launch_zinv(const Dev &d, cudaStream_t s);
void launch_xphys(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s);
void launch_zfwd(const Dev &d, cudaStream_t s);
void launch_post1(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s);
void launch_post2(const Dev &d, int rk, cudaStream_t s);
void launch_psi(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s);
// reference layout [kx][kz][y] <-> device layout [y][kx][kz]
void launch_ref2dev(const Dev &d, const double2 *in, double2 *out, cudaStream_t s);
void launch_dev2ref(const Dev &d, const double2 *in, double2 *out, cudaStream_t s);
// operator-level entry point (tests), device layout
void launch_op_y(const Dev &d, int op, const double2 *in, double2 *out, double2 *out2, cudaStream_t s);
size_t xphys_smem(const Dev &d);
size_t z_smem(const Dev &d);
cudaError_t kernels_init(const Dev &d);

}  // namespace lmc
