// nrgpu_adm.cu -- ADM diagnostics on the device (sm_100a), FP64:
//   nrgpu_to_adm            bssn_to_adm_vl (bssn.c:132-197) / z4_to_adm_vl
//                           (z4.c:93-124): g = psi^4 g~, K = psi^4 A~ + K g/3
//   nrgpu_adm_constraints   adm_constraints_N (spec adm_constraints_N.m:14-143,
//                           usepsi = 0, no matter) with the optional
//                           normalised constraints (plain / term by term)
//   nrgpu_norms             bampi_allreduce_norm2 / _normInf (reduce.c:41-131,
//                           209-266): RMS and max |u| over the flag-0 points
// One thread per point; the constraint kernel keeps the 72 derivatives of a
// point in registers and contracts them in the order of the spec.  The
// reductions are two-pass and fixed-order, so a norm is bit-reproducible
// from run to run.
#include <cfloat>

#include "nrgpu_level.cuh"
#include "nrgpu_fd.cuh"

namespace {

struct AdmIn {
  const double *p[12];  // g11 g12 g13 g22 g23 g33 K11 ... K33
};
struct AdmOut {
  double *p[12];
};
struct ConOut {
  double *p[8];  // ham mom1 mom2 mom3 [normham normmom1 normmom2 normmom3]
};
struct ConfIn {
  const double *p[14];  // g~ (6), chi, A~ (6), K
};

__global__ void to_adm_kernel(ConfIn u, AdmOut adm, double oochipsipower, int np) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const double psi = pow(ldg(u.p[6] + i), oochipsipower);
  const double psi4 = pow(psi, 4.0);
  const double trK = ldg(u.p[13] + i);
#pragma unroll
  for (int n = 0; n < 6; ++n) {
    const double g = psi4 * ldg(u.p[n] + i);
    adm.p[n][i] = g;
    adm.p[6 + n][i] = psi4 * ldg(u.p[7 + n] + i) + 1.0 / 3.0 * trK * g;
  }
}

// ---- constraints of one point -----------------------------------------------
template <int ORD, int MODE>
__device__ __forceinline__ void con_point(const AdmIn &A, int x, const int st[3], const double h[3],
                                          double out[8]) {
  double g[6], K[6], dg[3][6], dK[3][6], dd[6][6];
  const double i1[3] = {1.0 / (den1<ORD>() * h[0]), 1.0 / (den1<ORD>() * h[1]), 1.0 / (den1<ORD>() * h[2])};
#pragma unroll
  for (int v = 0; v < 6; ++v) {
    g[v] = ldg(A.p[v] + x);
    K[v] = ldg(A.p[6 + v] + x);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      dg[c][v] = d1n<ORD>(A.p[v], x, st[c]) * i1[c];
      dK[c][v] = d1n<ORD>(A.p[6 + v], x, st[c]) * i1[c];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b)
        dd[sy(a, b)][v] = a == b ? d2n<ORD>(A.p[v], x, st[a]) / (den2<ORD>() * h[a] * h[a])
                                 : d11n<ORD>(A.p[v], x, st[a], st[b]) / (den1<ORD>() * h[a] * den1<ORD>() * h[b]);
  }
  const double det = g[0] * (g[3] * g[5] - g[4] * g[4]) - g[1] * (g[1] * g[5] - g[2] * g[4]) +
                     g[2] * (g[1] * g[4] - g[2] * g[3]);
  const double idet = 1.0 / det;
  double gi[6];
  gi[0] = (g[3] * g[5] - g[4] * g[4]) * idet;
  gi[1] = (g[2] * g[4] - g[1] * g[5]) * idet;
  gi[2] = (g[1] * g[4] - g[2] * g[3]) * idet;
  gi[3] = (g[0] * g[5] - g[2] * g[2]) * idet;
  gi[4] = (g[1] * g[2] - g[0] * g[4]) * idet;
  gi[5] = (g[0] * g[3] - g[1] * g[1]) * idet;
  // connection, first kind gd[c][ab] and second kind gu[c][ab]
  double gd[3][6], gu[3][6];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) gd[c][sy(a, b)] = 0.5 * (dg[a][sy(b, c)] + dg[b][sy(a, c)] - dg[c][sy(a, b)]);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int ab = 0; ab < 6; ++ab)
      gu[c][ab] = gi[sy(c, 0)] * gd[0][ab] + gi[sy(c, 1)] * gd[1][ab] + gi[sy(c, 2)] * gd[2][ab];
  // Ricci scalar (and the term-by-term pieces): R[a,b] for a <= b, weight 2
  // off the diagonal; the piece RB[a,b] is ginv[c,d] deldelg[b,c,a,d], the
  // index order of the generated code (adm_constraints_N.c:4660-4700)
  double R = 0, RA = 0, RB = 0, RC = 0, RD = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      const double w = (a == b ? 1.0 : 2.0) * gi[sy(a, b)];
      double r = 0, ra = 0, rb = 0, rc = 0, rd = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const double gcd = gi[sy(c, d)];
          double cc = 0, dn = 0;
#pragma unroll
          for (int e = 0; e < 3; ++e) {
            cc += gu[e][sy(a, c)] * gd[e][sy(b, d)];
            dn -= gu[e][sy(a, b)] * gd[e][sy(c, d)];
          }
          r += gcd * (0.5 * (-dd[sy(c, d)][sy(a, b)] - dd[sy(a, b)][sy(c, d)] + dd[sy(a, c)][sy(b, d)] +
                             dd[sy(b, c)][sy(a, d)]) +
                      cc + dn);
          if (MODE == 2) {
            ra -= gcd * dd[sy(c, d)][sy(a, b)];
            rb += gcd * dd[sy(b, c)][sy(a, d)];
            rc += gcd * cc;
            rd += gcd * dn;
          }
        }
      R += w * r;
      if (MODE == 2) {
        RA += w * ra;
        RB += w * rb;
        RC += w * rc;
        RD += w * rd;
      }
    }
  // extrinsic curvature
  double Kud[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
      Kud[a][b] = gi[sy(a, 0)] * K[sy(0, b)] + gi[sy(a, 1)] * K[sy(1, b)] + gi[sy(a, 2)] * K[sy(2, b)];
  const double trK = Kud[0][0] + Kud[1][1] + Kud[2][2];
  double KK = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) KK += Kud[a][b] * Kud[b][a];
  // covariant derivative of K; the term-by-term pieces B and C both take the
  // value -gamma[d,a,b] K[d,c] of the generated code (b <= c)
  double cK[3][6], cKB[3][6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = b; c < 3; ++c) {
        double sb = 0, sd = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          sb -= gu[d][sy(a, b)] * K[sy(d, c)];
          sd -= gu[d][sy(a, c)] * K[sy(b, d)];
        }
        cKB[a][sy(b, c)] = sb;
        cK[a][sy(b, c)] = dK[a][sy(b, c)] + sb + sd;
      }
  double cdK[3][6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int bc = 0; bc < 6; ++bc)
      cdK[a][bc] = gi[sy(a, 0)] * cK[0][bc] + gi[sy(a, 1)] * cK[1][bc] + gi[sy(a, 2)] * cK[2][bc];
  out[0] = R + trK * trK - KK;
  double mu[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double s = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) s += gi[sy(a, b)] * cdK[c][sy(b, c)] - gi[sy(b, c)] * cdK[a][sy(b, c)];
    mu[a] = s;
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) out[1 + a] = g[sy(a, 0)] * mu[0] + g[sy(a, 1)] * mu[1] + g[sy(a, 2)] * mu[2];
  if (MODE == 0) return;
  double den = MODE == 2 ? fabs(RA) + fabs(RB) + fabs(RC) + fabs(RD) + trK * trK + fabs(KK)
                         : fabs(R) + trK * trK + fabs(KK);
  out[4] = den <= 0.0 ? 0.0 : out[0] / den;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (MODE == 2) {
      double cA = 0, cB = 0, tA = 0, tB = 0;
#pragma unroll
      for (int p = 0; p < 3; ++p)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          cA += gi[sy(p, q)] * dK[p][sy(a, q)];
          cB += gi[sy(p, q)] * cKB[p][sy(a, q)];
          tA += gi[sy(p, q)] * dK[a][sy(p, q)];
          tB += gi[sy(p, q)] * cKB[a][sy(p, q)];
        }
      den = fabs(cA) + 2.0 * fabs(cB) + fabs(tA) + 2.0 * fabs(tB);
    } else {
      double s1 = 0, s2 = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c) s1 += cdK[c][sy(a, c)];
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) s2 += gi[sy(b, c)] * cK[a][sy(b, c)];
      den = fabs(s1) + fabs(s2);
    }
    out[5 + a] = den <= 0.0 ? 0.0 : out[1 + a] / den;
  }
}

__device__ __forceinline__ int ladder_c(int order, int d) {
  if (order == 2 || d == 1) return 2;
  if (order == 4 || d == 2) return 4;
  return 6;
}

// one thread per point of the box interior; flag-0 points only
// (forinnerpoints_ijk, bam_amr_loops_box.h:138)
template <int MODE>
__global__ void __launch_bounds__(128) adm_constraints_kernel(AdmIn A, ConOut C, BoxGeo box,
                                                             const int *__restrict__ boundary, int order,
                                                             double dx, double dy, double dz, int *status) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > box.m - 2 || j > box.n - 2 || k > box.o - 2) return;
  const int x = box.noffset + i + box.m * (j + box.n * k);
  if (__ldg(boundary + x) != 0) return;
  int d = min(min(i, j), k);
  d = min(d, min(min(box.m - 1 - i, box.n - 1 - j), box.o - 1 - k));
  const int st[3] = {1, box.m, box.m * box.n};
  const double h[3] = {dx, dy, dz};
  double out[8];
  const int ord = ladder_c(order, d);
  if (ord == 2) con_point<2, MODE>(A, x, st, h, out);
  else if (ord == 4) con_point<4, MODE>(A, x, st, h, out);
  else con_point<6, MODE>(A, x, st, h, out);
  if (!isfinite(out[0])) atomicOr(status, 1);
  const int nout = MODE ? 8 : 4;
#pragma unroll
  for (int v = 0; v < nout; ++v) C.p[v][x] = out[v];
}

// ---- norms ------------------------------------------------------------------
constexpr int kRedBlocks = 296;  // 2 blocks per SM of the 148
constexpr int kRedThreads = 256;
constexpr int kMaxNormVars = 32;

struct NormIn {
  const double *p[kMaxNormVars];
};

// pass 1: block b of variable v writes (sum u^2, max |u|) of its grid-stride
// share of the flag-0 points to part[v][b]
__global__ void __launch_bounds__(kRedThreads) norm_partial_kernel(NormIn V, const int *__restrict__ boundary,
                                                                   int np, double2 *part) {
  const int v = blockIdx.y;
  const double *u = V.p[v];
  double s = 0.0, mx = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    if (__ldg(boundary + i) != 0) continue;
    const double x = ldg(u + i);
    s += x * x;
    mx = fmax(mx, fabs(x));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  __shared__ double ss[kRedThreads / 32], sm[kRedThreads / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) { ss[w] = s; sm[w] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int q = 0; q < kRedThreads / 32; ++q) { a += ss[q]; b = fmax(b, sm[q]); }
    part[v * kRedBlocks + blockIdx.x] = make_double2(a, b);
  }
}

// pass 2: one warp per variable folds the kRedBlocks partials in a fixed order
__global__ void norm_final_kernel(const double2 *part, double ninner, double *res, int nv) {
  const int v = blockIdx.x;
  if (v >= nv) return;
  double s = 0.0, mx = 0.0;
  for (int b = threadIdx.x; b < kRedBlocks; b += 32) {
    const double2 q = part[v * kRedBlocks + b];
    s += q.x;
    mx = fmax(mx, q.y);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_down_sync(0xffffffffu, s, o);
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  if (threadIdx.x == 0) {
    res[2 * v] = sqrt(s / ninner);
    res[2 * v + 1] = mx;
  }
}

}  // namespace

extern "C" int nrgpu_to_adm(nrgpu_level *L, const double *const *u, double *const *adm, double chipsipower,
                            void *stream) {
  if (!L || !u || !adm || chipsipower == 0.0) return nrgpu_set_error(NRGPU_ERR_ARG, "bad arguments");
  ConfIn ci;
  AdmOut ao;
  for (int v = 0; v < 14; ++v) {
    if (!u[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null u[%d]", v);
    ci.p[v] = u[v];
  }
  for (int v = 0; v < 12; ++v) {
    if (!adm[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null adm[%d]", v);
    ao.p[v] = adm[v];
  }
  NRGPU_CUDA_TRY(cudaSetDevice(L->device));
  to_adm_kernel<<<(L->npoints + 255) / 256, 256, 0, (cudaStream_t)stream>>>(ci, ao, 1.0 / chipsipower,
                                                                              L->npoints);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_adm_constraints(nrgpu_level *L, const double *const *adm, double *const *con,
                                     int order_centered, int mode, void *stream) {
  if (!L || !adm || !con) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  if (order_centered != 2 && order_centered != 4 && order_centered != 6)
    return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "order_centered %d", order_centered);
  if (mode < NRGPU_CON_PLAIN || mode > NRGPU_CON_TERMBYTERM)
    return nrgpu_set_error(NRGPU_ERR_ARG, "constraint mode %d", mode);
  AdmIn A;
  ConOut C;
  for (int v = 0; v < 12; ++v) {
    if (!adm[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null adm[%d]", v);
    A.p[v] = adm[v];
  }
  const int nout = mode ? 8 : 4;
  for (int v = 0; v < 8; ++v) {
    C.p[v] = v < nout ? con[v] : nullptr;
    if (v < nout && !con[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null con[%d]", v);
  }
  NRGPU_CUDA_TRY(cudaSetDevice(L->device));
  const cudaStream_t st = (cudaStream_t)stream;
  for (int b = 0; b < L->nboxes; ++b) {
    const BoxGeo &bx = L->hbox[b];
    if (bx.m < 3 || bx.n < 3 || bx.o < 3) continue;
    const dim3 blk(32, 4, 1);
    const dim3 grd((bx.m - 2 + 31) / 32, (bx.n - 2 + 3) / 4, bx.o - 2);
    if (mode == NRGPU_CON_PLAIN)
      adm_constraints_kernel<0><<<grd, blk, 0, st>>>(A, C, bx, L->d_boundary, order_centered, L->dx, L->dy,
                                                     L->dz, L->d_status);
    else if (mode == NRGPU_CON_NORMALIZED)
      adm_constraints_kernel<1><<<grd, blk, 0, st>>>(A, C, bx, L->d_boundary, order_centered, L->dx, L->dy,
                                                     L->dz, L->d_status);
    else
      adm_constraints_kernel<2><<<grd, blk, 0, st>>>(A, C, bx, L->d_boundary, order_centered, L->dx, L->dy,
                                                     L->dz, L->d_status);
    NRGPU_CUDA_TRY(cudaGetLastError());
  }
  return NRGPU_OK;
}

extern "C" int nrgpu_norms(nrgpu_level *L, const double *const *vars, int nvars, double *norm2, double *norminf,
                           void *stream) {
  if (!L || !vars || nvars < 1 || nvars > kMaxNormVars || !norm2 || !norminf)
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad arguments (1 <= nvars <= %d)", kMaxNormVars);
  NormIn V;
  for (int v = 0; v < kMaxNormVars; ++v) V.p[v] = v < nvars ? vars[v] : nullptr;
  for (int v = 0; v < nvars; ++v)
    if (!vars[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null vars[%d]", v);
  NRGPU_CUDA_TRY(cudaSetDevice(L->device));
  if (L->ninner == 0) {
    for (int v = 0; v < nvars; ++v) {
      norm2[v] = -1.0;
      norminf[v] = -1.7976931348623157e308;
    }
    return NRGPU_OK;
  }
  if (!L->d_red) {
    const size_t bytes = sizeof(double2) * kRedBlocks * kMaxNormVars + sizeof(double) * 2 * kMaxNormVars;
    if (cudaMalloc(&L->d_red, bytes) != cudaSuccess) {
      L->d_red = nullptr;
      cudaGetLastError();
      return nrgpu_set_error(NRGPU_ERR_NOMEM, "reduction buffer of %zu bytes", bytes);
    }
  }
  double2 *part = (double2 *)L->d_red;
  double *res = (double *)(part + kRedBlocks * kMaxNormVars);
  const cudaStream_t st = (cudaStream_t)stream;
  norm_partial_kernel<<<dim3(kRedBlocks, nvars), kRedThreads, 0, st>>>(V, L->d_boundary, L->npoints, part);
  NRGPU_CUDA_TRY(cudaGetLastError());
  norm_final_kernel<<<nvars, 32, 0, st>>>(part, (double)L->ninner, res, nvars);
  NRGPU_CUDA_TRY(cudaGetLastError());
  double h[2 * kMaxNormVars];
  NRGPU_CUDA_TRY(cudaMemcpyAsync(h, res, sizeof(double) * 2 * nvars, cudaMemcpyDeviceToHost, st));
  NRGPU_CUDA_TRY(cudaStreamSynchronize(st));
  for (int v = 0; v < nvars; ++v) {
    norm2[v] = h[2 * v];
    norminf[v] = h[2 * v + 1];
  }
  return NRGPU_OK;
}

// ---- 0d output ---------------------------------------------------------------
// write_level_0d (utility/output/output0d.c:28-116) through bampi_allreduce
// (main/bampi/reduce.c:37-135) on one rank: over the flag-0 points, per
// variable the maximum, the minimum, the RMS (the list's norm2 times
// sqrt(nvars)), the maximum of |u| and the sum times dx^3.  Two passes as
// for the norms: block partials, then a fixed-order fold, so the results do
// not depend on scheduling.
constexpr int kRed0d = 5;

__global__ void __launch_bounds__(kRedThreads) red0d_partial_kernel(NormIn V, const int *__restrict__ boundary,
                                                                    int np, double *part) {
  const int v = blockIdx.y;
  const double *u = V.p[v];
  double mx = -DBL_MAX, mn = DBL_MAX, s = 0.0, s2 = 0.0, ma = -DBL_MAX;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < np; i += gridDim.x * blockDim.x) {
    if (__ldg(boundary + i) != 0) continue;
    const double x = ldg(u + i);
    mx = fmax(mx, x);
    mn = fmin(mn, x);
    s += x;
    s2 += x * x;
    ma = fmax(ma, fabs(x));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
    s += __shfl_down_sync(0xffffffffu, s, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
    ma = fmax(ma, __shfl_down_sync(0xffffffffu, ma, o));
  }
  __shared__ double w5[kRed0d][kRedThreads / 32];
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    w5[0][w] = mx; w5[1][w] = mn; w5[2][w] = s; w5[3][w] = s2; w5[4][w] = ma;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 1; q < kRedThreads / 32; ++q) {
      mx = fmax(mx, w5[0][q]); mn = fmin(mn, w5[1][q]); s += w5[2][q]; s2 += w5[3][q]; ma = fmax(ma, w5[4][q]);
    }
    double *o = part + (size_t)kRed0d * (v * kRedBlocks + blockIdx.x);
    o[0] = mx; o[1] = mn; o[2] = s; o[3] = s2; o[4] = ma;
  }
}

// the norm as bampi_allreduce_norm2 and write_level_0d form it: the count n
// is nvars x inner points (reduce.c:79-90, :215-216), the RMS sqrt(s2 / n)
// times sqrt(nvars) (output0d.c:71-75); the integral times pow(dx, 3) (:86-89)
__global__ void red0d_final_kernel(const double *part, double ninner, double dx3, double *res, int nv) {
  const int v = blockIdx.x;
  if (v >= nv) return;
  double mx = -DBL_MAX, mn = DBL_MAX, s = 0.0, s2 = 0.0, ma = -DBL_MAX;
  for (int b = threadIdx.x; b < kRedBlocks; b += 32) {
    const double *q = part + (size_t)kRed0d * (v * kRedBlocks + b);
    mx = fmax(mx, q[0]); mn = fmin(mn, q[1]); s += q[2]; s2 += q[3]; ma = fmax(ma, q[4]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, o));
    mn = fmin(mn, __shfl_down_sync(0xffffffffu, mn, o));
    s += __shfl_down_sync(0xffffffffu, s, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
    ma = fmax(ma, __shfl_down_sync(0xffffffffu, ma, o));
  }
  if (threadIdx.x == 0) {
    double *r = res + kRed0d * v;
    r[0] = mx;
    r[1] = mn;
    const double n = (double)nv * ninner;
    r[2] = (n > 0 ? sqrt(s2 / n) : -1.0) * sqrt((double)nv);
    r[3] = ma;
    r[4] = s * dx3;
  }
}

extern "C" int nrgpu_output0d(nrgpu_level *L, const double *const *vars, int nvars, double *out, void *stream) {
  if (!L || !vars || nvars < 1 || nvars > kMaxNormVars || !out)
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad arguments (1 <= nvars <= %d)", kMaxNormVars);
  NormIn V;
  for (int v = 0; v < kMaxNormVars; ++v) V.p[v] = v < nvars ? vars[v] : nullptr;
  for (int v = 0; v < nvars; ++v)
    if (!vars[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null vars[%d]", v);
  NRGPU_CUDA_TRY(cudaSetDevice(L->device));
  if (!L->d_red0d) {
    const size_t bytes = sizeof(double) * kRed0d * (kRedBlocks + 1) * kMaxNormVars;
    if (cudaMalloc(&L->d_red0d, bytes) != cudaSuccess) {
      L->d_red0d = nullptr;
      cudaGetLastError();
      return nrgpu_set_error(NRGPU_ERR_NOMEM, "0d reduction buffer of %zu bytes", bytes);
    }
  }
  double *part = L->d_red0d;
  double *res = part + (size_t)kRed0d * kRedBlocks * kMaxNormVars;
  const cudaStream_t st = (cudaStream_t)stream;
  red0d_partial_kernel<<<dim3(kRedBlocks, nvars), kRedThreads, 0, st>>>(V, L->d_boundary, L->npoints, part);
  NRGPU_CUDA_TRY(cudaGetLastError());
  red0d_final_kernel<<<nvars, 32, 0, st>>>(part, (double)L->ninner, pow(L->dx, 3), res, nvars);
  NRGPU_CUDA_TRY(cudaGetLastError());
  NRGPU_CUDA_TRY(cudaMemcpyAsync(out, res, sizeof(double) * kRed0d * nvars, cudaMemcpyDeviceToHost, st));
  NRGPU_CUDA_TRY(cudaStreamSynchronize(st));
  return NRGPU_OK;
}
