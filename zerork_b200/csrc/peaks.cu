// peaks.cu -- FP64 roofline denominators measured on the running GPU.
//
// The rate kernels are FP64 SIMT work dominated by exponentials; the HBM
// and BF16 peaks of the machine say nothing about that pipe, so the library
// measures (a) dependent-chain-free FP64 FMA throughput and (b) double
// precision exp() throughput, each over a few hundred milliseconds.
#include <cuda_runtime.h>

#include "../../include/zerork_b200_diag.h"
#include "capi_internal.h"

namespace {

__global__ void fma_kernel(double *out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-3, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
  double x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 12345.678) out[0] = s;  // keep the chains alive
}

__global__ void exp_kernel(double *out, int iters) {
  double a0 = -1e-3 * threadIdx.x, a1 = a0 - 0.1, a2 = a0 - 0.2, a3 = a0 - 0.3;
  double s = 0.0;
  for (int i = 0; i < iters; ++i) {
    s += exp(a0) + exp(a1) + exp(a2) + exp(a3);
    a0 -= 1e-7; a1 -= 1e-7; a2 -= 1e-7; a3 -= 1e-7;
  }
  if (s == 12345.678) out[0] = s;
}

}  // namespace

extern "C" int zrk_measure_fp64(double *fma_gflops, double *exp_gps) {
  using namespace zrk;
  if (!fma_gflops || !exp_gps) return set_error(2, "null argument");
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  double *d = nullptr;
  cudaError_t e = cudaMalloc(&d, 64);
  if (e != cudaSuccess) return cuda_error(e, "cudaMalloc");
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  const int blocks = sms * 8, threads = 256;
  float ms = 0.f;
  const int fiters = 4096;
  fma_kernel<<<blocks, threads>>>(d, 64, 0.999999, 1e-9);  // warm-up
  cudaEventRecord(t0);
  fma_kernel<<<blocks, threads>>>(d, fiters, 0.999999, 1e-9);
  cudaEventRecord(t1);
  cudaEventSynchronize(t1);
  cudaEventElapsedTime(&ms, t0, t1);
  *fma_gflops = 2.0 * 64.0 * fiters * (double)blocks * threads / (ms * 1e-3) / 1e9;
  const int eiters = 1024;
  exp_kernel<<<blocks, threads>>>(d, 16);
  cudaEventRecord(t0);
  exp_kernel<<<blocks, threads>>>(d, eiters);
  cudaEventRecord(t1);
  cudaEventSynchronize(t1);
  cudaEventElapsedTime(&ms, t0, t1);
  *exp_gps = 4.0 * eiters * (double)blocks * threads / (ms * 1e-3) / 1e9;
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  e = cudaGetLastError();
  cudaFree(d);
  if (e != cudaSuccess) return cuda_error(e, "fp64 peak kernels");
  return 0;
}
