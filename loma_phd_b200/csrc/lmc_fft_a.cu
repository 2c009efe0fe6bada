// Transform kernels for lengths 3 (the z length of 2-D runs) and 24..96 (see lmc_fft_impl.cuh).
#define LMC_FFT_NS fft_a
#include "lmc_fft_impl.cuh"
#define LMC_FFT_SIZES(X) X(3, 1, 3) X(24, 4, 6) X(36, 6, 6) X(48, 6, 8) X(72, 8, 9) X(96, 8, 12)
LMC_FFT_TU_BODY(a)
