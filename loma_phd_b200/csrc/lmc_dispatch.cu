// lmc_dispatch.cu -- routes the transform launches to the translation unit
// that instantiates the grid's transform lengths, and performs the one-time
// per-device set-up of all kernels.
#include <cuda_runtime.h>

#include <mutex>

#include "lmc_kernels.cuh"

namespace lmc {

#define LMC_FFT_DECL(SUF)                                                              \
  bool fft_has_##SUF(int n);                                                           \
  bool fft_zinv_##SUF(const Dev &d, int mode, int f0, int nf, cudaStream_t s);         \
  bool fft_zfwd_##SUF(const Dev &d, int mode, cudaStream_t s);                         \
  bool fft_xdrho_##SUF(const Dev &d, cudaStream_t s);                                  \
  bool fft_xphys_##SUF(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s); \
  bool fft_xstats_##SUF(const Dev &d, const Stats &st, cudaStream_t s);                \
  bool fft_xexport_##SUF(const Dev &d, const int *jrow, int nplanes, int nf, double *out, cudaStream_t s); \
  size_t fft_zsm_##SUF(int n);                                                         \
  size_t fft_xsm_##SUF(int n, bool zs, bool vs);                                       \
  cudaError_t fft_init_##SUF(int limit);
LMC_FFT_DECL(a)
LMC_FFT_DECL(b)
LMC_FFT_DECL(c)
cudaError_t ykernels_init(int limit);

bool fft_supported(int n) { return fft_has_a(n) || fft_has_b(n) || fft_has_c(n); }

void launch_zinv(const Dev &d, cudaStream_t s, int mode, int f0, int nf) {
  if (!fft_zinv_a(d, mode, f0, nf, s) && !fft_zinv_b(d, mode, f0, nf, s)) fft_zinv_c(d, mode, f0, nf, s);
}
void launch_zfwd(const Dev &d, cudaStream_t s, int mode) {
  if (!fft_zfwd_a(d, mode, s) && !fft_zfwd_b(d, mode, s)) fft_zfwd_c(d, mode, s);
}
void launch_xdrho(const Dev &d, cudaStream_t s) {
  if (!fft_xdrho_a(d, s) && !fft_xdrho_b(d, s)) fft_xdrho_c(d, s);
}
void launch_xphys(const Dev &d, int rk, int do_cfl, int do_diag, cudaStream_t s) {
  if (!fft_xphys_a(d, rk, do_cfl, do_diag, s) && !fft_xphys_b(d, rk, do_cfl, do_diag, s))
    fft_xphys_c(d, rk, do_cfl, do_diag, s);
}
void launch_xexport(const Dev &d, const int *jrow, int nplanes, int nf, double *out, cudaStream_t s) {
  if (!fft_xexport_a(d, jrow, nplanes, nf, out, s) && !fft_xexport_b(d, jrow, nplanes, nf, out, s))
    fft_xexport_c(d, jrow, nplanes, nf, out, s);
}
void launch_xstats(const Dev &d, const Stats &st, cudaStream_t s) {
  if (!fft_xstats_a(d, st, s) && !fft_xstats_b(d, st, s)) fft_xstats_c(d, st, s);
}
size_t xphys_smem(const Dev &d) {
  const bool zs = d.scalar != 0, vs = d.visc != 0;
  size_t v = fft_xsm_a(d.mgalx, zs, vs);
  if (!v) v = fft_xsm_b(d.mgalx, zs, vs);
  if (!v) v = fft_xsm_c(d.mgalx, zs, vs);
  return v;
}
size_t z_smem(const Dev &d) {
  size_t v = fft_zsm_a(d.mgalz);
  if (!v) v = fft_zsm_b(d.mgalz);
  if (!v) v = fft_zsm_c(d.mgalz);
  return v;
}

// Checks the grid's shared-memory needs against the device, and once per
// device (not on every case: the constant-memory twiddles would be
// rewritten under running kernels) uploads the twiddles and opts the
// kernels in to the large shared-memory carve-out.
cudaError_t kernels_init(const Dev &d) {
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0, limit = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
  const size_t need_y = (size_t)8 * d.ldy * sizeof(double2);
  if ((size_t)limit < xphys_smem(d) + 1024 || (size_t)limit < z_smem(d) + 1024 || (size_t)limit < need_y + 1024)
    return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return cudaSuccess;
  if ((e = fft_init_a(limit)) != cudaSuccess) return e;
  if ((e = fft_init_b(limit)) != cudaSuccess) return e;
  if ((e = fft_init_c(limit)) != cudaSuccess) return e;
  if ((e = ykernels_init(limit)) != cudaSuccess) return e;
  if (dev >= 0 && dev < 64) done[dev] = true;
  return cudaSuccess;
}

}  // namespace lmc
