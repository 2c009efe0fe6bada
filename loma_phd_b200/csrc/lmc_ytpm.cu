// lmc_ytpm.cu -- launchers of the mode-parallel y kernels (lmc_ytpm.cuh)
// for both work-buffer types.
#include "lmc_ylaunch.h"
#include "lmc_ytpm.cuh"

namespace lmc {

namespace {
inline unsigned tgrid(const Dev &d) { return (unsigned)((d.nmode + tpm::TB - 1) / tpm::TB); }
}  // namespace

#define LMC_TPM(K, ...)                                                       \
  do {                                                                        \
    if (d.prec) tpm::K<float2><<<tgrid(d), tpm::TB, 0, s>>>(__VA_ARGS__);    \
    else tpm::K<double2><<<tgrid(d), tpm::TB, 0, s>>>(__VA_ARGS__);          \
  } while (0)

void tpm_lapv(const Dev &d, cudaStream_t s) { LMC_TPM(t_lapv, d); }
void tpm_assemble(const Dev &d, int rk, cudaStream_t s) { LMC_TPM(t_assemble, d, rk); }
void tpm_tder(const Dev &d, cudaStream_t s) { LMC_TPM(t_tder, d); }
void tpm_post1(const Dev &d, cudaStream_t s) { LMC_TPM(t_post1, d); }
void tpm_post2(const Dev &d, int rk, cudaStream_t s) { LMC_TPM(t_post2, d, rk); }
void tpm_psi(const Dev &d, cudaStream_t s) { LMC_TPM(t_psi, d); }
void tpm_op_y(const Dev &d, int op, const double2 *in, double2 *out, double2 *out2, cudaStream_t s) {
  tpm::t_op_y<<<tgrid(d), tpm::TB, 0, s>>>(d, op, in, out, out2);
}

}  // namespace lmc
