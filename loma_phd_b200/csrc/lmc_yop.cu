// lmc_yop.cu -- the compact y operators as dense my x my matrices applied to
// every mode at once as one GEMM on the tensor cores (cuBLAS), and the
// autotuner that times them against the banded solves of the substep.
//
// d/dy (deryr2, cfdiff.f:518-601) and d2/dy2 (deryyr2, cfdiff.f:735-797)
// do not depend on the mode, so each is one dense matrix D (column j = the
// operator applied to the unit vector e_j).  In the device layout a field is
// a row-major my x (2 nmode) real matrix F (row y, columns the real and
// imaginary parts of every mode), and the operator is D F:
//   method 1  FP64 GEMM (DGEMM, FP64 tensor cores)
//   method 2  3xTF32: F = Fh + Fl and D = Dh + Dl with Fh, Dh rounded to TF32
//             (10-bit mantissa) and Fl, Dl the FP32 remainders;
//             D F ~ Dh Fh + Dh Fl + Dl Fh in three TF32 GEMMs accumulated in
//             FP32 (the split-precision scheme of the error-free
//             transformation literature: Markidis et al. 2018, "NVIDIA
//             tensor core programmability, performance & precision")
// The banded solve costs O(my) per point and streams its operands once;
// the dense product costs O(my) multiply-adds per point on the tensor
// cores.  The autotuner measures both on the device and reports which is
// faster within the precision form's error budget.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "lmc_internal.h"
#include "lmc_kernels.cuh"

namespace lmc {

struct DenseY {
  int my = 0;
  size_t ncol = 0;  // 2 * nmode real columns
  cublasHandle_t cb = nullptr;
  double *D[2] = {nullptr, nullptr};                   // d/dy, d2/dy2 (row-major my x my)
  float *Dh[2] = {nullptr, nullptr}, *Dl[2] = {nullptr, nullptr};
  float *Fh = nullptr, *Fl = nullptr, *C = nullptr;    // 3xTF32 operands (my x ncol)
};

namespace {

// round to nearest TF32 (FP32 with the 13 low mantissa bits cleared), ties
// to even; finite inputs
__device__ __forceinline__ float tf32_round(float x) {
  unsigned u = __float_as_uint(x);
  u += 0xFFFu + ((u >> 13) & 1u);
  return __uint_as_float(u & 0xFFFFE000u);
}

__global__ void k_split_tf32(const double *__restrict__ a, float *__restrict__ hi, float *__restrict__ lo, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const double v = a[i];
    const float h = tf32_round((float)v);
    hi[i] = h;
    lo[i] = (float)(v - (double)h);
  }
}

__global__ void k_widen(const float *__restrict__ c, double *__restrict__ out, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = (double)c[i];
}

int grid_1d(size_t n) {
  const size_t b = (n + 255) / 256;
  return (int)(b < 148 * 16 ? b : 148 * 16);
}

// dense matrix of a banded operator: D[i][j] = (op e_j)[i], host FP64
std::vector<double> dense_of(const YOps &o, int op) {
  const int my = o.my;
  std::vector<double> D((size_t)my * my), e(my), t(my);
  for (int j = 0; j < my; j++) {
    std::fill(e.begin(), e.end(), 0.0);
    e[j] = 1.0;
    if (op == 1) {  // deryr2: fmap * prem1^-1 (dt12 u)
      band_matvec(my, 3, o.dt12.data(), e.data(), t.data());
      band_solve(my, 3, 3, o.p1L.data(), o.p1U.data(), t.data());
      for (int i = 0; i < my; i++) t[i] *= o.fmap[i];
    } else {  // deryyr2: prem3^-1 (dt22 u)
      band_matvec(my, 2, o.dt22.data(), e.data(), t.data());
      band_solve(my, 2, 2, o.p3L.data(), o.p3U.data(), t.data());
    }
    for (int i = 0; i < my; i++) D[(size_t)i * my + j] = t[i];
  }
  return D;
}

}  // namespace

void dense_destroy(DenseY *z) {
  if (!z) return;
  if (z->cb) cublasDestroy(z->cb);
  for (int q = 0; q < 2; q++) {
    cudaFree(z->D[q]);
    cudaFree(z->Dh[q]);
    cudaFree(z->Dl[q]);
  }
  cudaFree(z->Fh);
  cudaFree(z->Fl);
  cudaFree(z->C);
  delete z;
}

// The dense operators of a grid and the GEMM workspace (set up on first use
// by lmc_op_y_dense / lmc_yop_tune; freed with the handle).
DenseY *dense_create(const YOps &ops, size_t ncol, cudaStream_t s, int *rc) {
  DenseY *z = new DenseY();
  z->my = ops.my;
  z->ncol = ncol;
  *rc = LMC_ECUDA;
  const size_t mm = (size_t)ops.my * ops.my, nf = (size_t)ops.my * ncol;
  if (cublasCreate(&z->cb) != CUBLAS_STATUS_SUCCESS || cublasSetStream(z->cb, s) != CUBLAS_STATUS_SUCCESS) {
    dense_destroy(z);
    return nullptr;
  }
  for (int q = 0; q < 2; q++) {
    const std::vector<double> D = dense_of(ops, q + 1);
    if (cudaMalloc(&z->D[q], mm * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&z->Dh[q], mm * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&z->Dl[q], mm * sizeof(float)) != cudaSuccess ||
        cudaMemcpyAsync(z->D[q], D.data(), mm * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess) {
      *rc = LMC_ENOMEM;
      dense_destroy(z);
      return nullptr;
    }
    k_split_tf32<<<grid_1d(mm), 256, 0, s>>>(z->D[q], z->Dh[q], z->Dl[q], mm);
  }
  if (cudaMalloc(&z->Fh, nf * sizeof(float)) != cudaSuccess || cudaMalloc(&z->Fl, nf * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&z->C, nf * sizeof(float)) != cudaSuccess) {
    *rc = LMC_ENOMEM;
    dense_destroy(z);
    return nullptr;
  }
  if (cudaStreamSynchronize(s) != cudaSuccess) {  // the host matrices go out of scope
    dense_destroy(z);
    return nullptr;
  }
  *rc = LMC_OK;
  return z;
}

// out = D_op in on the device layout (row-major my x ncol, FP64).  In
// cuBLAS's column-major terms out^T = in^T D^T, with D stored row-major
// (= D^T column-major, leading dimension my).
int dense_apply(DenseY *z, int op, int method, const double *in, double *out, cudaStream_t s) {
  if (!z || op < 1 || op > 2 || method < 1 || method > 2) return LMC_EINVAL;
  const int q = op - 1, my = z->my, n = (int)z->ncol;
  if (cublasSetStream(z->cb, s) != CUBLAS_STATUS_SUCCESS) return LMC_ECUDA;
  if (method == 1) {
    const double one = 1.0, zero = 0.0;
    if (cublasDgemm(z->cb, CUBLAS_OP_N, CUBLAS_OP_N, n, my, my, &one, in, n, z->D[q], my, &zero, out, n) !=
        CUBLAS_STATUS_SUCCESS)
      return LMC_ECUDA;
    return LMC_OK;
  }
  const size_t nf = (size_t)my * z->ncol;
  k_split_tf32<<<grid_1d(nf), 256, 0, s>>>(in, z->Fh, z->Fl, nf);
  const float one = 1.0f, zero = 0.0f;
  const float *A[3] = {z->Fh, z->Fl, z->Fh};
  const float *B[3] = {z->Dh[q], z->Dh[q], z->Dl[q]};
  for (int k = 0; k < 3; k++)
    if (cublasGemmEx(z->cb, CUBLAS_OP_N, CUBLAS_OP_N, n, my, my, &one, A[k], CUDA_R_32F, n, B[k], CUDA_R_32F, my,
                     k ? &one : &zero, z->C, CUDA_R_32F, n, CUBLAS_COMPUTE_32F_FAST_TF32,
                     CUBLAS_GEMM_DEFAULT) != CUBLAS_STATUS_SUCCESS)
      return LMC_ECUDA;
  k_widen<<<grid_1d(nf), 256, 0, s>>>(z->C, out, nf);
  return cudaGetLastError() == cudaSuccess ? LMC_OK : LMC_ECUDA;
}

}  // namespace lmc
