// fp64_peak.cu — FP64 FMA throughput microbenchmark (libdsp_bench.so).
//
// The driver-measured peaks cover HBM and BF16 only; the solver kernels are
// FP64-bound, so this kernel measures the FP64 FMA roofline on the same GPU:
// 8 independent FMA chains per thread, 8 CTAs of 256 threads per SM, timed
// with CUDA events.  Used by bench.py for the roofline denominator.
#include <cuda_runtime.h>

#include <cstdint>

#include "dsp_device.cuh"

__global__ void __launch_bounds__(256) dfma_chains(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = (threadIdx.x + k) * 1e-3;
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 12345.678) out[blockIdx.x * blockDim.x + threadIdx.x] = s;  // keeps the chains live
}

extern "C" double dsp_bench_fp64_tflops(int device, int repeats) {
  if (cudaSetDevice(device) != cudaSuccess) return -1.0;
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const int blocks = sms * 8, threads = 256, iters = 4096;
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  dfma_chains<<<blocks, threads>>>(out, 64, 0.999999, 1e-7);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < (repeats > 0 ? repeats : 5); ++r) {
    cudaEventRecord(e0);
    dfma_chains<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  return flops / (best * 1e-3) / 1e12;
}

// Check of the solver's branch-free reciprocal (dsp::rcp_newton, used for the
// pivots of the boundary-value kernel) against CUDA's division on n values:
// y[k] = rcp_newton(x[k]), q[k] = 1 / x[k] (device arrays).  Returns 0 or the
// CUDA error code.
__global__ void rcp_check_kernel(const double* x, double* y, double* q, int n) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  y[k] = dsp::rcp_newton(x[k]);
  q[k] = 1.0 / x[k];
}

extern "C" int dsp_bench_rcp_check(const double* x, double* y, double* q, int n) {
  if (n <= 0) return 0;
  rcp_check_kernel<<<(n + 255) / 256, 256>>>(x, y, q, n);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  return (int)e;
}
