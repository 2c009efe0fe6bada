// Transform kernels for lengths 144..384 (see lmc_fft_impl.cuh).
#define LMC_FFT_NS fft_b
#include "lmc_fft_impl.cuh"
#define LMC_FFT_SIZES(X) X(144, 12, 12) X(192, 12, 16) X(288, 16, 18) X(384, 16, 24)
LMC_FFT_TU_BODY(b)
