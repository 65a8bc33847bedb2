// nrgpu_fd.cuh -- centred finite-difference numerators of order 2, 4, 6
// (discretize.m:18-71 of the reference: first and second derivative
// stencils, mixed derivatives as the product of two first-derivative
// stencils), shared by the rhs and diagnostic kernels.
#pragma once
#include "nrgpu_common.cuh"

namespace {

// first derivative numerator; the derivative is num / (den1 * h)
template <int ORD>
__device__ __forceinline__ double d1n(const double *__restrict__ f, int x, int s) {
  if (ORD == 2) return ldg(f + x + s) - ldg(f + x - s);
  if (ORD == 4)
    return (ldg(f + x - 2 * s) - ldg(f + x + 2 * s)) + 8.0 * (ldg(f + x + s) - ldg(f + x - s));
  return (ldg(f + x + 3 * s) - ldg(f + x - 3 * s)) + 9.0 * (ldg(f + x - 2 * s) - ldg(f + x + 2 * s)) +
         45.0 * (ldg(f + x + s) - ldg(f + x - s));
}
template <int ORD> __host__ __device__ constexpr double den1() { return ORD == 2 ? 2.0 : ORD == 4 ? 12.0 : 60.0; }
template <int ORD> __host__ __device__ constexpr double den2() { return ORD == 2 ? 1.0 : ORD == 4 ? 12.0 : 180.0; }

// second derivative numerator; the derivative is num / (den2 * h^2)
template <int ORD>
__device__ __forceinline__ double d2n(const double *__restrict__ f, int x, int s) {
  const double c = ldg(f + x);
  if (ORD == 2) return ldg(f + x - s) - 2.0 * c + ldg(f + x + s);
  if (ORD == 4)
    return 16.0 * (ldg(f + x - s) + ldg(f + x + s)) - (ldg(f + x - 2 * s) + ldg(f + x + 2 * s)) - 30.0 * c;
  return 2.0 * (ldg(f + x - 3 * s) + ldg(f + x + 3 * s)) - 27.0 * (ldg(f + x - 2 * s) + ldg(f + x + 2 * s)) +
         270.0 * (ldg(f + x - s) + ldg(f + x + s)) - 490.0 * c;
}

// mixed derivative numerator: product of two first-derivative stencils
// (discretize.m:68-71); the derivative is num / (den1^2 * h1 * h2)
template <int ORD>
__device__ __forceinline__ double d11n(const double *__restrict__ f, int x, int s1, int s2) {
  if (ORD == 2) return d1n<2>(f, x + s1, s2) - d1n<2>(f, x - s1, s2);
  if (ORD == 4)
    return (d1n<4>(f, x - 2 * s1, s2) - d1n<4>(f, x + 2 * s1, s2)) +
           8.0 * (d1n<4>(f, x + s1, s2) - d1n<4>(f, x - s1, s2));
  return (d1n<6>(f, x + 3 * s1, s2) - d1n<6>(f, x - 3 * s1, s2)) +
         9.0 * (d1n<6>(f, x - 2 * s1, s2) - d1n<6>(f, x + 2 * s1, s2)) +
         45.0 * (d1n<6>(f, x + s1, s2) - d1n<6>(f, x - s1, s2));
}

// ---- FP32 variants (the mixed-precision option) -------------------------------
// The taps enter as differences to the centre value, formed in FP64 and
// rounded to FP32; the weighted sums run in FP32 and the result returns to
// FP64.  A stencil's weights sum to zero (first and second derivative,
// Kreiss-Oliger), so the centre-relative form is the same linear combination;
// what changes is only the rounding of the taps and of the sum.
__device__ __forceinline__ float tapf(const double *__restrict__ f, int x, int k, int s, double c) {
  return (float)(ldg(f + x + k * s) - c);
}

template <int ORD>
__device__ __forceinline__ double d1n_f(const double *__restrict__ f, int x, int s) {
  const double c = ldg(f + x);
  float r;
  if (ORD == 2) r = tapf(f, x, 1, s, c) - tapf(f, x, -1, s, c);
  else if (ORD == 4)
    r = (tapf(f, x, -2, s, c) - tapf(f, x, 2, s, c)) + 8.0f * (tapf(f, x, 1, s, c) - tapf(f, x, -1, s, c));
  else
    r = (tapf(f, x, 3, s, c) - tapf(f, x, -3, s, c)) + 9.0f * (tapf(f, x, -2, s, c) - tapf(f, x, 2, s, c)) +
        45.0f * (tapf(f, x, 1, s, c) - tapf(f, x, -1, s, c));
  return (double)r;
}

template <int ORD>
__device__ __forceinline__ double d2n_f(const double *__restrict__ f, int x, int s) {
  const double c = ldg(f + x);
  float r;
  if (ORD == 2) r = tapf(f, x, -1, s, c) + tapf(f, x, 1, s, c);
  else if (ORD == 4)
    r = 16.0f * (tapf(f, x, -1, s, c) + tapf(f, x, 1, s, c)) - (tapf(f, x, -2, s, c) + tapf(f, x, 2, s, c));
  else
    r = 2.0f * (tapf(f, x, -3, s, c) + tapf(f, x, 3, s, c)) - 27.0f * (tapf(f, x, -2, s, c) + tapf(f, x, 2, s, c)) +
        270.0f * (tapf(f, x, -1, s, c) + tapf(f, x, 1, s, c));
  return (double)r;
}

// mixed derivative: the taps relative to the point's own value
template <int ORD>
__device__ __forceinline__ float d1n_rel(const double *__restrict__ f, int x, int s, double c) {
  if (ORD == 2) return (float)(ldg(f + x + s) - c) - (float)(ldg(f + x - s) - c);
  if (ORD == 4)
    return ((float)(ldg(f + x - 2 * s) - c) - (float)(ldg(f + x + 2 * s) - c)) +
           8.0f * ((float)(ldg(f + x + s) - c) - (float)(ldg(f + x - s) - c));
  return ((float)(ldg(f + x + 3 * s) - c) - (float)(ldg(f + x - 3 * s) - c)) +
         9.0f * ((float)(ldg(f + x - 2 * s) - c) - (float)(ldg(f + x + 2 * s) - c)) +
         45.0f * ((float)(ldg(f + x + s) - c) - (float)(ldg(f + x - s) - c));
}

template <int ORD>
__device__ __forceinline__ double d11n_f(const double *__restrict__ f, int x, int s1, int s2) {
  const double c = ldg(f + x);
  float r;
  if (ORD == 2) r = d1n_rel<2>(f, x + s1, s2, c) - d1n_rel<2>(f, x - s1, s2, c);
  else if (ORD == 4)
    r = (d1n_rel<4>(f, x - 2 * s1, s2, c) - d1n_rel<4>(f, x + 2 * s1, s2, c)) +
        8.0f * (d1n_rel<4>(f, x + s1, s2, c) - d1n_rel<4>(f, x - s1, s2, c));
  else
    r = (d1n_rel<6>(f, x + 3 * s1, s2, c) - d1n_rel<6>(f, x - 3 * s1, s2, c)) +
        9.0f * (d1n_rel<6>(f, x - 2 * s1, s2, c) - d1n_rel<6>(f, x + 2 * s1, s2, c)) +
        45.0f * (d1n_rel<6>(f, x + s1, s2, c) - d1n_rel<6>(f, x - s1, s2, c));
  return (double)r;
}

// precision-dispatched numerators: P = 0 FP64, P = 2 FP32 stencils
template <int ORD, int P>
__device__ __forceinline__ double d1p(const double *__restrict__ f, int x, int s) {
  return P >= 2 ? d1n_f<ORD>(f, x, s) : d1n<ORD>(f, x, s);
}
template <int ORD, int P>
__device__ __forceinline__ double d2p(const double *__restrict__ f, int x, int s) {
  return P >= 2 ? d2n_f<ORD>(f, x, s) : d2n<ORD>(f, x, s);
}
template <int ORD, int P>
__device__ __forceinline__ double d11p(const double *__restrict__ f, int x, int s1, int s2) {
  return P >= 2 ? d11n_f<ORD>(f, x, s1, s2) : d11n<ORD>(f, x, s1, s2);
}

}  // namespace
