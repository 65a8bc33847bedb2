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

}  // namespace
