// nrgpu_probe.cu -- FP64 FMA throughput probe for the roofline denominator.
// The available peak list has no FP64 figure, so it is measured here on the
// same GPU and clocks as the kernels it normalises: independent FMA chains,
// 8 per thread, enough resident warps to hide the FMA latency.
#include "nrgpu_common.cuh"

namespace {
__global__ void __launch_bounds__(256) fma_chains(double *out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-3, x2 = x0 + 2e-3, x3 = x0 + 3e-3;
  double x4 = x0 + 4e-3, x5 = x0 + 5e-3, x6 = x0 + 6e-3, x7 = x0 + 7e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 12345.678) out[blockIdx.x] = s;  // keeps the chains alive
}
}  // namespace

// measured FP64 FLOP/s (2 per FMA) of the current device; *ms = kernel time
extern "C" int nrgpu_probe_fp64_peak(int iters, double *flops_per_s, float *ms) {
  if (!flops_per_s || !ms || iters < 1) return nrgpu_set_error(NRGPU_ERR_ARG, "bad probe arguments");
  int dev = 0, sms = 0;
  NRGPU_CUDA_TRY(cudaGetDevice(&dev));
  NRGPU_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 8, threads = 256;
  double *out = nullptr;
  NRGPU_CUDA_TRY(cudaMalloc(&out, sizeof(double) * blocks));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fma_chains<<<blocks, threads>>>(out, 8, 1.0000001, 1e-7);  // warm-up
  cudaEventRecord(e0);
  fma_chains<<<blocks, threads>>>(out, iters, 1.0000001, 1e-7);
  cudaEventRecord(e1);
  cudaError_t err = cudaEventSynchronize(e1);
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (err != cudaSuccess) return nrgpu_set_error(NRGPU_ERR_CUDA, "probe: %s", cudaGetErrorString(err));
  const double flops = 2.0 * 8.0 * 16.0 * (double)iters * blocks * threads;
  *flops_per_s = flops / (*ms * 1e-3);
  return NRGPU_OK;
}
