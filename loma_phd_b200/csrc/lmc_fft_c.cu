// Transform kernels for lengths 576..1536 (see lmc_fft_impl.cuh).
#define LMC_FFT_NS fft_c
#include "lmc_fft_impl.cuh"
#define LMC_FFT_SIZES(X) X(576, 24, 24) X(768, 24, 32) X(1152, 32, 36) X(1536, 32, 48)
LMC_FFT_TU_BODY(c)
