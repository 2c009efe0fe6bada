// lmc_ykernels.cu -- dispatch of the y-direction kernels to the chunk size
// and work-buffer precision of a case, their one-time set-up, and the
// layout transposes of the C ABI.
#include <cuda_runtime.h>

#include "lmc_ylaunch.h"

namespace lmc {

namespace {

// ----------------------------------------------------------------------
// layout transposes: reference [kx][kz][y] <-> device [y][kx][kz]
// ----------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_ref2dev(int my, int nkx, int mz, const double2 *__restrict__ in,
                                                 double2 *__restrict__ out) {
  __shared__ double2 t[32][33];
  const int i = blockIdx.z, y0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int k = k0 + r, y = y0 + threadIdx.x;
    if (k < mz && y < my) t[r][threadIdx.x] = in[((size_t)i * mz + k) * my + y];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int y = y0 + r, k = k0 + threadIdx.x;
    if (k < mz && y < my) out[((size_t)y * nkx + i) * mz + k] = t[threadIdx.x][r];
  }
}
__global__ void __launch_bounds__(256) k_dev2ref(int my, int nkx, int mz, const double2 *__restrict__ in,
                                                 double2 *__restrict__ out) {
  __shared__ double2 t[32][33];
  const int i = blockIdx.z, y0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int y = y0 + r, k = k0 + threadIdx.x;
    if (k < mz && y < my) t[r][threadIdx.x] = in[((size_t)y * nkx + i) * mz + k];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int k = k0 + r, y = y0 + threadIdx.x;
    if (k < mz && y < my) out[((size_t)i * mz + k) * my + y] = t[threadIdx.x][r];
  }
}

}  // namespace

#define LMC_YCASE(C, CALL)                                       \
  case C:                                                        \
    if (d.prec) YL<C, float2>::CALL;                             \
    else YL<C, double2>::CALL;                                   \
    break;
#define LMC_YDISPATCH(CALL)                                                                   \
  switch (d.C) {                                                                              \
    LMC_YCASE(4, CALL) LMC_YCASE(5, CALL) LMC_YCASE(7, CALL) LMC_YCASE(9, CALL)              \
    LMC_YCASE(13, CALL) default : LMC_YCASE(17, CALL)                                         \
  }

// d.tpm selects the mode-parallel kernels (lmc_ytpm.cu) over the
// warp-per-mode ones; the 00-mode tails always run the warp code.
void launch_lapv(const Dev &d, cudaStream_t s) {
  if (d.tpm) tpm_lapv(d, s);
  else LMC_YDISPATCH(lapv(d, s))
}
void launch_assemble(const Dev &d, int rk, cudaStream_t s) {
  if (d.tpm) tpm_assemble(d, rk, s);
  else LMC_YDISPATCH(assemble(d, rk, s))
}
void launch_tder(const Dev &d, cudaStream_t s) {
  if (d.tpm) tpm_tder(d, s);
  else LMC_YDISPATCH(tder(d, s))
}
void launch_post1(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s) {
  if (d.tpm) {
    tpm_post1(d, rk, s);
    LMC_YDISPATCH(post1_00(d, rk, d.variant ? 0 : do_cfl, do_diag, s))
  } else {
    LMC_YDISPATCH(post1(d, rk, do_cfl, do_diag, s))
  }
}
void launch_cfl14(const Dev &d, int do_cfl, cudaStream_t s) { tpm_cfl14(d, do_cfl, s); }
void launch_post2(const Dev &d, int rk, cudaStream_t s) {
  if (d.tpm) tpm_post2(d, rk, s);
  else LMC_YDISPATCH(post2(d, rk, s))
}
// mode-parallel family, non-variant: the psi solve and its 00 tail apart,
// so that the solve can run beside post1 on a second stream
void launch_psi_main(const Dev &d, int rk, cudaStream_t s) { tpm_psi(d, rk, s); }
void launch_psi_tail(const Dev &d, int rk, int cfl_step, cudaStream_t s) {
  LMC_YDISPATCH(psi_00(d, rk, cfl_step, s))
}
void launch_psi(const Dev &d, int rk, int cfl_step, int do_diag, cudaStream_t s) {
  if (d.tpm) {
    tpm_psi(d, rk, s);
    if (d.variant) tpm_psi00_14(d, rk, s);
    else LMC_YDISPATCH(psi_00(d, rk, cfl_step, s))
  } else {
    LMC_YDISPATCH(psi(d, rk, cfl_step, do_diag, s))
  }
}
void launch_op_y(const Dev &d, int op, const double2 *in, double2 *out, double2 *out2, cudaStream_t s) {
  if (d.tpm) {
    tpm_op_y(d, op, in, out, out2, s);
    return;
  }
  switch (d.C) {
    case 4: YL<4, double2>::op_y(d, op, in, out, out2, s); break;
    case 5: YL<5, double2>::op_y(d, op, in, out, out2, s); break;
    case 7: YL<7, double2>::op_y(d, op, in, out, out2, s); break;
    case 9: YL<9, double2>::op_y(d, op, in, out, out2, s); break;
    case 13: YL<13, double2>::op_y(d, op, in, out, out2, s); break;
    default: YL<17, double2>::op_y(d, op, in, out, out2, s); break;
  }
}

// Opt the y kernels in to the device's largest dynamic shared memory.
cudaError_t ykernels_init(int limit) {
  cudaError_t e = cudaSuccess;
#define LMC_YOPT(C)                                                          \
  if ((e = YL<C, double2>::optin(limit)) != cudaSuccess) return e;           \
  if ((e = YL<C, float2>::optin(limit)) != cudaSuccess) return e;
  LMC_Y_CHUNKS(LMC_YOPT)
#undef LMC_YOPT
  return cudaSuccess;
}

void launch_ref2dev(const Dev &d, const double2 *in, double2 *out, cudaStream_t s) {
  dim3 g((d.my + 31) / 32, (d.mz + 31) / 32, d.nkx);
  k_ref2dev<<<g, dim3(32, 8), 0, s>>>(d.my, d.nkx, d.mz, in, out);
}
void launch_dev2ref(const Dev &d, const double2 *in, double2 *out, cudaStream_t s) {
  dim3 g((d.my + 31) / 32, (d.mz + 31) / 32, d.nkx);
  k_dev2ref<<<g, dim3(32, 8), 0, s>>>(d.my, d.nkx, d.mz, in, out);
}

}  // namespace lmc
