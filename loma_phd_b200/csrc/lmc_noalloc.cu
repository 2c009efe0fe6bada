// lmc_noalloc.cu -- lmc_deryr2_noalloc: the compact first y-derivative
// (deryr2) on caller-owned device pencils, with its operator workspace in a
// fixed file-scope device array instead of memory from cudaMalloc.
//
// Who needs it: callers that may not allocate device memory at run time.
// A Fortran or C driver that hands the library a fixed device-memory
// budget (its own pools, or HBM already reserved for other cases) cannot
// let the library grab more, and a time loop that must not stall cannot
// afford cudaFree, which synchronises the whole device.  This entry point
// takes only the caller's input and output buffers; everything else it
// needs lives in g_noalloc_scratch below.
//
// Contract:
//   * The scratch array is LMC_NOALLOC_SCRATCH_BYTES (256 KiB) per device;
//     a grid whose tables do not fit (my > 544, the largest pencil one warp
//     handles) is rejected with LMC_EINVAL before anything is launched.
//   * in_dev and out_dev must be 16-byte aligned (the kernel moves whole
//     complex values) and must not overlap; otherwise LMC_EINVAL, with
//     nothing launched.
//   * The array is shared by every call on a device and keeps the contents
//     of the last call.  Each call rewrites the whole table region it reads
//     (zero entries included), so nothing depends on earlier contents.
//     Calls that overlap on the GPU (different streams, or another host
//     thread) race on the array: serialise them.
//   * The first call in a CUDA context (with that device current) looks up
//     the array's device address with cudaGetSymbolAddress and caches it
//     for that context; make that first call before any stream capture
//     starts.
//   * The tables are built in host memory and copied with cudaMemcpyAsync
//     from a buffer that is released when the call returns, so the call
//     returns LMC_EINVAL while `stream` is being captured (a captured copy
//     would read the released buffer when the graph is replayed).
//   * No cudaMalloc, cudaFree or other device allocation is made.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "lmc_internal.h"
#include "lmc_kernels.cuh"

using namespace lmcd;

namespace {

constexpr size_t LMC_NOALLOC_SCRATCH_BYTES = 256 * 1024;
constexpr int LMC_NOALLOC_MAX_DEVICES = 64;

// Operator tables of the last call: chunk-major dt12 (7), LU of prem1
// (3 + 4), fmap (1), then the Kogge-Stone scan tables of both LU factors.
static __device__ __align__(256) unsigned char g_noalloc_scratch[LMC_NOALLOC_SCRATCH_BYTES];

std::mutex g_mu;
// device address of the array per (device, CUDA context): a context made
// after cudaDeviceReset, or a non-primary one, gets its own look-up
std::map<std::pair<int, void *>, void *> g_scratch_ptr;

// the calling thread's current CUDA context (driver entry point reached
// through the runtime, so the library does not link libcuda itself)
void *current_context() {
  using GetCtx = int (*)(void **);
  static GetCtx fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (GetCtx)f;
  });
  void *ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

struct View {
  const double *dt12, *p1L, *p1U, *fmap, *k1L, *k1U;
  int lpm, base, extra;
};

// one warp per pencil; the pencil (my complex values, y fastest) is read and
// written in place of the caller's buffers, chunk by chunk
template <int C>
__global__ void __launch_bounds__(256) k_deryr2_noalloc(View v, int my, int npencil, const double2 *__restrict__ in,
                                                        double2 *__restrict__ out) {
  const int p = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (p >= npencil) return;  // whole warps leave together
  const Lane L = make_lane<C>(v.lpm, v.base, v.extra);
  double2 a[C];
  const double2 *src = in + (size_t)p * my;
#pragma unroll
  for (int t = 0; t < C; t++) a[t] = (t < L.n) ? __ldg(src + L.s + t) : czero();
  matvec_ip<C, 3>(v.dt12, L, a);
  lsolve_c<C, 3>(a, v.p1L, v.k1L, L);
  usolve_c<C, 3>(a, v.p1U, v.k1U, L);
  double2 *dst = out + (size_t)p * my;
#pragma unroll
  for (int t = 0; t < C; t++)
    if (t < L.n) dst[L.s + t] = cscale(tab(v.fmap, 1, t, 0, L.lane), a[t]);
}

int chunks(int my, int &C, int &lpm, int &base, int &extra) {
  static const int Cs[] = {4, 5, 7, 9, 13, 17};
  const int need = (my + 31) / 32;
  C = 0;
  for (int c : Cs)
    if (c >= need) { C = c; break; }
  if (!C) return LMC_EINVAL;
  lpm = (my + C - 1) / C;
  base = my / lpm;
  extra = my % lpm;
  if (lpm > 32 || base < 3) return LMC_EINVAL;
  if (!(base == C - 1 || (base == C && extra == 0))) return LMC_EINVAL;
  return LMC_OK;
}

// device address of the scratch array in the current context (set-up once
// per device and context)
int scratch_ptr(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= LMC_NOALLOC_MAX_DEVICES) return LMC_ECUDA;
  const std::pair<int, void *> key(dev, current_context());
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_scratch_ptr.find(key);
  if (it == g_scratch_ptr.end()) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      std::fprintf(stderr, "lomacte_b200: scratch symbol address: %s\n", cudaGetErrorString(e));
      return LMC_ECUDA;
    }
    it = g_scratch_ptr.emplace(key, p).first;
  }
  *out = it->second;
  return LMC_OK;
}

}  // namespace

extern "C" int lmc_deryr2_noalloc(int my, const double *y, int npencil, const double *in_dev, double *out_dev,
                                  void *stream) {
  if (!y || !in_dev || !out_dev || npencil < 0 || my < 12) return LMC_EINVAL;
  int C, lpm, base, extra;
  if (chunks(my, C, lpm, base, extra) != LMC_OK) {
    std::fprintf(stderr, "lomacte_b200: lmc_deryr2_noalloc: my=%d exceeds the largest supported pencil (544)\n", my);
    return LMC_EINVAL;
  }
  if (npencil == 0) return LMC_OK;
  const uintptr_t ia = (uintptr_t)in_dev, oa = (uintptr_t)out_dev;
  if ((ia | oa) & 15) {
    std::fprintf(stderr, "lomacte_b200: lmc_deryr2_noalloc: in_dev and out_dev must be 16-byte aligned\n");
    return LMC_EINVAL;
  }
  const uintptr_t nb = (uintptr_t)npencil * (uintptr_t)my * sizeof(double2);
  if (ia < oa + nb && oa < ia + nb) {
    std::fprintf(stderr, "lomacte_b200: lmc_deryr2_noalloc: in_dev and out_dev overlap\n");
    return LMC_EINVAL;
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) return LMC_ECUDA;
  if (cs != cudaStreamCaptureStatusNone) {
    std::fprintf(stderr, "lomacte_b200: lmc_deryr2_noalloc: the stream is being captured\n");
    return LMC_EINVAL;
  }
  // operator tables in host memory (the host code of lmc_create)
  std::vector<double> pack;
  size_t off[6];
  try {
    lmc::YOps o;
    lmc::build_yops(my, y, o);
    lmc::build_scans(o, lpm, base, extra);
    const std::vector<double> parts[6] = {
        lmc::chunk_major(o.dt12, my, 7, C, lpm, base, extra), lmc::chunk_major(o.p1L, my, 3, C, lpm, base, extra),
        lmc::chunk_major(o.p1U, my, 4, C, lpm, base, extra), lmc::chunk_major(o.fmap, my, 1, C, lpm, base, extra),
        o.k1L, o.k1U};
    for (int i = 0; i < 6; i++) {
      off[i] = pack.size();
      pack.insert(pack.end(), parts[i].begin(), parts[i].end());
      while (pack.size() % 32) pack.push_back(0.0);  // 256-byte aligned parts
    }
  } catch (...) {
    return LMC_EINVAL;
  }
  if (pack.size() * sizeof(double) > LMC_NOALLOC_SCRATCH_BYTES) {
    std::fprintf(stderr, "lomacte_b200: lmc_deryr2_noalloc: tables need %zu bytes, scratch holds %zu\n",
                 pack.size() * sizeof(double), LMC_NOALLOC_SCRATCH_BYTES);
    return LMC_EINVAL;
  }
  void *scr = nullptr;
  int rc = scratch_ptr(&scr);
  if (rc) return rc;
  if (cudaMemcpyAsync(scr, pack.data(), pack.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return LMC_ECUDA;
  const double *base_ptr = (const double *)scr;
  View v{base_ptr + off[0], base_ptr + off[1], base_ptr + off[2], base_ptr + off[3], base_ptr + off[4],
         base_ptr + off[5], lpm, base, extra};
  const dim3 grid((unsigned)((npencil + 7) / 8)), block(256);
  const double2 *in = (const double2 *)in_dev;
  double2 *out = (double2 *)out_dev;
  switch (C) {
    case 4: k_deryr2_noalloc<4><<<grid, block, 0, s>>>(v, my, npencil, in, out); break;
    case 5: k_deryr2_noalloc<5><<<grid, block, 0, s>>>(v, my, npencil, in, out); break;
    case 7: k_deryr2_noalloc<7><<<grid, block, 0, s>>>(v, my, npencil, in, out); break;
    case 9: k_deryr2_noalloc<9><<<grid, block, 0, s>>>(v, my, npencil, in, out); break;
    case 13: k_deryr2_noalloc<13><<<grid, block, 0, s>>>(v, my, npencil, in, out); break;
    default: k_deryr2_noalloc<17><<<grid, block, 0, s>>>(v, my, npencil, in, out); break;
  }
  return cudaGetLastError() == cudaSuccess ? LMC_OK : LMC_ECUDA;
}
