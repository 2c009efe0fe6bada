// Transform kernels for lengths 24..96 (see lmc_fft_impl.cuh).
#define LMC_FFT_NS fft_a
#include "lmc_fft_impl.cuh"
#define LMC_FFT_SIZES(X) X(24, 4, 6) X(36, 6, 6) X(48, 6, 8) X(72, 8, 9) X(96, 8, 12)
LMC_FFT_TU_BODY(a)
