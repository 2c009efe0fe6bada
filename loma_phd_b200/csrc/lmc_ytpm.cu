// lmc_ytpm.cu -- launchers of the mode-parallel y kernels (lmc_ytpm.cuh)
// for both work-buffer types and, in FP64, the 2014 variant.
#include "lmc_ylaunch.h"
#include "lmc_stats.cuh"
#include "lmc_ytpm.cuh"

namespace lmc {

namespace {
inline unsigned tgrid(const Dev &d) { return (unsigned)((d.nmode + tpm::TB - 1) / tpm::TB); }
}  // namespace

// kernels without a variant form
#define LMC_TPM(K, ...)                                                       \
  do {                                                                        \
    if (d.prec) tpm::K<float2><<<tgrid(d), tpm::TB, 0, s>>>(__VA_ARGS__);    \
    else tpm::K<double2><<<tgrid(d), tpm::TB, 0, s>>>(__VA_ARGS__);          \
  } while (0)
// kernels with a 2014-variant form (FP64 only)
#define LMC_TPMV(K, ...)                                                             \
  do {                                                                               \
    if (d.prec) tpm::K<float2, false><<<tgrid(d), tpm::TB, 0, s>>>(__VA_ARGS__);    \
    else if (d.variant) tpm::K<double2, true><<<tgrid(d), tpm::TB, 0, s>>>(__VA_ARGS__); \
    else tpm::K<double2, false><<<tgrid(d), tpm::TB, 0, s>>>(__VA_ARGS__);          \
  } while (0)

void tpm_lapv(const Dev &d, cudaStream_t s) { LMC_TPM(t_lapv, d); }
void tpm_assemble(const Dev &d, int rk, cudaStream_t s) { LMC_TPMV(t_assemble, d, rk); }
void tpm_tder(const Dev &d, cudaStream_t s) { LMC_TPMV(t_tder, d); }
void tpm_post1(const Dev &d, int rk, cudaStream_t s) { LMC_TPMV(t_post1, d, rk); }
void tpm_post2(const Dev &d, int rk, cudaStream_t s) { LMC_TPM(t_post2, d, rk); }
void tpm_psi(const Dev &d, int rk, cudaStream_t s) { LMC_TPMV(t_psi, d, rk); }
void tpm_op_y(const Dev &d, int op, const double2 *in, double2 *out, double2 *out2, cudaStream_t s) {
  tpm::t_op_y<<<tgrid(d), tpm::TB, 0, s>>>(d, op, in, out, out2);
}
void launch_zder(const Dev &d, cudaStream_t s) { LMC_TPM(t_zder, d); }
void launch_zupd(const Dev &d, cudaStream_t s) { LMC_TPM(t_zupd, d); }
void launch_xprep(const Dev &d, cudaStream_t s) { tpm::t_xprep<<<tgrid(d), tpm::TB, 0, s>>>(d); }
void launch_sgrad(const Dev &d, cudaStream_t s) {  // mixed: one more block for the exact 00 profiles
  if (d.prec) tpm::t_sgrad<float2><<<tgrid(d) + 1, tpm::TB, 0, s>>>(d);
  else tpm::t_sgrad<double2><<<tgrid(d), tpm::TB, 0, s>>>(d);
}
void tpm_cfl14(const Dev &d, int do_cfl, cudaStream_t s) { tpm::k_cfl14<<<1, 32, 0, s>>>(d, do_cfl); }
void tpm_psi00_14(const Dev &d, int rk, cudaStream_t s) { tpm::k_psi00_14<<<1, 32, 0, s>>>(d, rk); }

// statistics (lmc_stats.cuh); every grid, either y family
void launch_stats1(const Dev &d, const Stats &st, cudaStream_t s) {
  if (d.prec) stats::k_srow1<float2><<<d.my, stats::SRT, 0, s>>>(d, st);
  else stats::k_srow1<double2><<<d.my, stats::SRT, 0, s>>>(d, st);
}
void launch_stats2(const Dev &d, const Stats &st, cudaStream_t s) {
  if (d.prec) {
    stats::t_sdy<float2><<<tgrid(d), tpm::TB, 0, s>>>(d, st);
    stats::k_srow2<float2><<<d.my, stats::SRT, 0, s>>>(d, st);
  } else {
    stats::t_sdy<double2><<<tgrid(d), tpm::TB, 0, s>>>(d, st);
    stats::k_srow2<double2><<<d.my, stats::SRT, 0, s>>>(d, st);
  }
  stats::k_suner<<<1, 32, 0, s>>>(d, st);
}

}  // namespace lmc
