// nrgpu_common.cuh -- shared device helpers of the nrgpu library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/nrgpu.h"

#define NRGPU_NV 24

// minimum resident blocks of 128 threads per SM for the rhs kernels
// (__launch_bounds__): 1 leaves the compiler 255 registers per thread
#ifndef NRGPU_RHS_MINBLOCKS
#define NRGPU_RHS_MINBLOCKS 1
#endif

// 24 device pointers passed by value as a kernel parameter
struct VarPtrs {
  double *p[NRGPU_NV];
};
struct CVarPtrs {
  const double *p[NRGPU_NV];
};

// device-side geometry of one box of a level
struct BoxGeo {
  int m, n, o, noffset;
  double x0, y0, z0;
};

// symmetric index (a,b) -> 0..5 in the order xx xy xz yy yz zz
__host__ __device__ constexpr int sy(int a, int b) {
  return a <= b ? (a == 0 ? b : (a == 1 ? 2 + b : 5)) : (b == 0 ? a : (b == 1 ? 2 + a : 5));
}

static __device__ __forceinline__ double ldg(const double *p) { return __ldg(p); }

// record the first CUDA error of a call sequence
#define NRGPU_CUDA_TRY(expr)                                              \
  do {                                                                    \
    cudaError_t e_ = (expr);                                              \
    if (e_ != cudaSuccess) return nrgpu_set_error(NRGPU_ERR_CUDA, "%s: %s", #expr, \
                                                  cudaGetErrorString(e_)); \
  } while (0)

int nrgpu_set_error(int code, const char *fmt, ...);
