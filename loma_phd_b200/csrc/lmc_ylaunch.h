// lmc_ylaunch.h -- launchers of the y-direction kernels for one chunk size
// C and one work-buffer type CT (double2: FP64 form, float2: mixed form).
// The definitions are in lmc_ykernels.cuh; each lmc_y_*.cu translation unit
// instantiates its chunk sizes so that they compile in parallel.
#pragma once
#include <cuda_runtime.h>

#include "lmc_kernels.cuh"

namespace lmc {

template <int C, typename CT>
struct YL {
  static void lapv(const Dev &d, cudaStream_t s);
  static void assemble(const Dev &d, int rk, cudaStream_t s);
  static void tder(const Dev &d, cudaStream_t s);
  static void post1(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s);
  static void post2(const Dev &d, int rk, cudaStream_t s);
  static void psi(const Dev &d, int rk, int cfl_step, int do_diag, cudaStream_t s);
  static void post1_00(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s);
  static void psi_00(const Dev &d, int rk, int cfl_step, cudaStream_t s);
  static void op_y(const Dev &d, int op, const double2 *in, double2 *out, double2 *out2, cudaStream_t s);
  static cudaError_t optin(int limit);
};

// mode-parallel kernels (lmc_ytpm.cu); the 00 tails of post1 and psi run
// as YL<C, CT>::post1_00 / psi_00 after them
void tpm_lapv(const Dev &d, cudaStream_t s);
void tpm_assemble(const Dev &d, int rk, cudaStream_t s);
void tpm_tder(const Dev &d, cudaStream_t s);
void tpm_post1(const Dev &d, int rk, cudaStream_t s);
void tpm_post2(const Dev &d, int rk, cudaStream_t s);
void tpm_psi(const Dev &d, int rk, cudaStream_t s);
void tpm_cfl14(const Dev &d, int do_cfl, cudaStream_t s);
void tpm_psi00_14(const Dev &d, int rk, cudaStream_t s);
void tpm_op_y(const Dev &d, int op, const double2 *in, double2 *out, double2 *out2, cudaStream_t s);

#define LMC_Y_CHUNKS(X) X(4) X(5) X(7) X(9) X(13) X(17)
#define LMC_Y_EXTERN(C)                   \
  extern template struct YL<C, double2>; \
  extern template struct YL<C, float2>;
LMC_Y_CHUNKS(LMC_Y_EXTERN)
#undef LMC_Y_EXTERN

}  // namespace lmc
