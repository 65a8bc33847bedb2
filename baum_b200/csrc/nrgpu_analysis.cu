// nrgpu_analysis.cu -- analysis quantities on the device (sm_100a), FP64:
//   nrgpu_adm_mass_integrands  the eight integrands of ADM_mass
//                              (projects/ADM_mass/ADM_mass.c:11-225): the ADM
//                              mass (adm_mass_integrand.c), its conformal-
//                              factor version (adm_mass_integrand_chi.c) and
//                              the linear and angular momentum
//                              (adm_pj_integrand.c), at the flag-0 points
//   nrgpu_sphere_integral      integral_over_sphere_Simpson (utility/
//                              NumericUtils/Integral_over_sphere.c:197-357):
//                              Simpson weights in theta and phi, the values
//                              at the sphere points by Lagrange interpolation
//                              (interpolate_xyz_local_minimal, utility/
//                              interpolate/interpolate.c:633-676)
// The integrands take the first derivatives of the metric and of chi with
// the 2nd-order centred stencil, whatever order_centered is, as the
// reference's integrands do.  With the 3-metric g, its inverse g^-1,
// N = x / |x| and R = |x| they are
//   mass       g^jk (d_j g_ik - d_i g_jk) N^i R^2 sqrt(det g) / (16 pi)
//   mass(chi)  (d_i chi N^i) R^2 / (8 pi chi^(5/4))
//   P_m        v_m R^2 sqrt(det g) / (8 pi),  v_m = g^jk N_j K_km - N_m K
//   J_m        eps_mlq x^l v_q R^2 sqrt(det g) / (8 pi)
// The sphere points and Simpson weights are formed on the host with the
// reference's arithmetic and its C library's sin and cos; the device
// interpolates each point (one thread per point, sums over z, then y, then
// x, every operation rounded separately, as interpolate_TriN); the host adds
// the weighted values in the reference's order.
#include <math.h>
#include <vector>

#include "nrgpu_level.cuh"

namespace {

constexpr double kPi = 3.1415926535897932;  // PI of adm_mass_integrand*.c
constexpr double kEps = 1e-10;              // dequaleps (main/main/bam_main.h:19)
constexpr int kMaxOrder = 8;

struct MassIn {
  const double *g[6], *K[6], *trK, *chi;
};
struct MassOut {
  double *p[8];  // mass, mass(chi), Px, Py, Pz, Jx, Jy, Jz
};

// one thread per point of one box; flag-0 points only (forinnerpoints_ijk,
// main/amr/bam_amr_loops_box.h:70-71; forinner19 of adm_pj_integrand.c)
__global__ void __launch_bounds__(128) adm_mass_kernel(MassIn A, MassOut O, BoxGeo box,
                                                      const int *__restrict__ boundary, double dx, double dy,
                                                      double dz) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nb = (long)box.m * box.n * box.o;
  if (t >= nb) return;
  const long x = box.noffset + t;
  if (__ldg(boundary + x) != 0) return;
  const int i = (int)(t % box.m), j = (int)((t / box.m) % box.n), k = (int)(t / ((long)box.m * box.n));
  const long st[3] = {1, box.m, (long)box.m * box.n};
  const double oo2h[3] = {1 / (2 * dx), 1 / (2 * dy), 1 / (2 * dz)};
  double g[6], dg[3][6], K[6];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    const double *f = A.g[c];
    g[c] = f[x];
    K[c] = A.K[c][x];
#pragma unroll
    for (int d = 0; d < 3; ++d) dg[d][c] = oo2h[d] * (-f[x - st[d]] + f[x + st[d]]);
  }
  double dchi[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) dchi[d] = oo2h[d] * (-A.chi[x - st[d]] + A.chi[x + st[d]]);
  const double det = 2. * g[1] * g[2] * g[4] + g[0] * g[3] * g[5] - g[5] * g[1] * g[1] - g[3] * g[2] * g[2] -
                     g[0] * g[4] * g[4];
  const double idet = 1 / det;
  double gi[6];
  gi[0] = idet * (g[3] * g[5] - g[4] * g[4]);
  gi[1] = idet * (g[2] * g[4] - g[1] * g[5]);
  gi[2] = idet * (-(g[2] * g[3]) + g[1] * g[4]);
  gi[3] = idet * (g[0] * g[5] - g[2] * g[2]);
  gi[4] = idet * (g[1] * g[2] - g[0] * g[4]);
  gi[5] = idet * (g[0] * g[3] - g[1] * g[1]);
  const double xc[3] = {box.x0 + i * dx, box.y0 + j * dy, box.z0 + k * dz};
  const double R = sqrt(xc[0] * xc[0] + xc[1] * xc[1] + xc[2] * xc[2]);
  const double N[3] = {xc[0] / R, xc[1] / R, xc[2] / R};
  const double area = R * R * sqrt(det);
  // mass: g^jk (d_j g_ik - d_i g_jk) N^i
  double s = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      double t2 = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) t2 += (dg[a][sy(c, b)] - dg[c][sy(a, b)]) * N[c];
      s += gi[sy(a, b)] * t2;
    }
  O.p[0][x] = 0.0625 * s * area / kPi;
  O.p[1][x] = 0.125 * (dchi[0] * N[0] + dchi[1] * N[1] + dchi[2] * N[2]) * (R * R) / (kPi * pow(A.chi[x], 1.25));
  // v_m = g^jk N_j K_km - N_m K
  double v[3];
#pragma unroll
  for (int m = 0; m < 3; ++m) {
    double w = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) w += gi[sy(a, b)] * N[a] * K[sy(b, m)];
    v[m] = w - N[m] * A.trK[x];
  }
  const double f8 = 0.125 * area / kPi;
  O.p[2][x] = v[0] * f8;
  O.p[3][x] = v[1] * f8;
  O.p[4][x] = v[2] * f8;
  O.p[5][x] = (xc[1] * v[2] - xc[2] * v[1]) * f8;
  O.p[6][x] = (xc[2] * v[0] - xc[0] * v[2]) * f8;
  O.p[7][x] = (xc[0] * v[1] - xc[1] * v[0]) * f8;
}

__device__ __forceinline__ bool dless(double a, double b) { return a < __dsub_rn(b, kEps); }
__device__ __forceinline__ bool dequal(double a, double b) { return !(dless(a, b) || dless(b, a)); }

// coefficients_lagrange_N (utility/interpolate/lagrange.c:13-27) about the
// cube's first node
__device__ void lagrange_c(int n, double x, double xmin, double h, double *c) {
  for (int i = 0; i < n; i++) {
    double d = 1.0;
    for (int j = 0; j < n; j++)
      if (j != i)
        d = __dmul_rn(d, __ddiv_rn(__dsub_rn(__dsub_rn(x, xmin), __dmul_rn((double)j, h)),
                                   __dmul_rn((double)(i - j), h)));
    c[i] = d;
  }
}

__device__ __forceinline__ double dot_rn(int n, const double *c, const double *u) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s = __dadd_rn(s, __dmul_rn(c[i], u[i]));
  return s;
}

__device__ int node_index(double c, double x0, double h, int n) {
  const int i = (int)floor(__dadd_rn(__ddiv_rn(__dsub_rn(c, x0), h), 0.5));
  if (i < 0 || i >= n || !dequal(c, __dadd_rn(x0, __dmul_rn((double)i, h)))) return -1;
  return i;
}

struct SphereArgs {
  const BoxGeo *box;
  int nboxes, order;
  double o[3], h[3];
  const double *f;
  const double *xyz;  // [3 np]
  double *val;        // [np]
  int *ok;            // [np]
  int np;
};

// one thread per sphere point: the cube's first node is the node at
// floor((x - xmin + eps)/h) - (order-1)/2 from the level's lower corner; the
// first box holding it must hold the whole cube, else the point is not
// found (find_one_point_box, interpolate_fillindexcube)
__global__ void sphere_interp_kernel(SphereArgs A) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= A.np) return;
  const double p[3] = {A.xyz[3 * q], A.xyz[3 * q + 1], A.xyz[3 * q + 2]};
  const int a = A.order, nh = (a - 1) / 2;
  double xc[3];
  for (int d = 0; d < 3; d++)
    xc[d] = __dadd_rn(A.o[d], __dmul_rn(A.h[d], floor(__ddiv_rn(__dadd_rn(__dsub_rn(p[d], A.o[d]), kEps), A.h[d])) -
                                                      (double)nh));
  A.ok[q] = 0;
  A.val[q] = 0.0;
  for (int b = 0; b < A.nboxes; b++) {
    const BoxGeo B = A.box[b];
    const int i = node_index(xc[0], B.x0, A.h[0], B.m);
    const int j = node_index(xc[1], B.y0, A.h[1], B.n);
    const int k = node_index(xc[2], B.z0, A.h[2], B.o);
    if (i < 0 || j < 0 || k < 0) continue;
    if (i + a > B.m || j + a > B.n || k + a > B.o) return;
    double cz[kMaxOrder], cy[kMaxOrder], cx[kMaxOrder], w[kMaxOrder], vv[kMaxOrder][kMaxOrder], line[kMaxOrder];
    lagrange_c(a, p[2], xc[2], A.h[2], cz);
    for (int ii = 0; ii < a; ii++)
      for (int jj = 0; jj < a; jj++) {
        for (int kk = 0; kk < a; kk++)
          line[kk] = A.f[(long)B.noffset + (i + ii) + (long)B.m * (j + jj) + (long)B.m * B.n * (k + kk)];
        vv[ii][jj] = dot_rn(a, cz, line);
      }
    lagrange_c(a, p[1], xc[1], A.h[1], cy);
    for (int ii = 0; ii < a; ii++) w[ii] = dot_rn(a, cy, vv[ii]);
    lagrange_c(a, p[0], xc[0], A.h[0], cx);
    A.val[q] = dot_rn(a, cx, w);
    A.ok[q] = 1;
    return;
  }
}

}  // namespace

extern "C" int nrgpu_adm_mass_integrands(nrgpu_level *L, const double *const *gK, const double *trK, const double *chi,
                                         double *const *out, void *stream) {
  if (!L || !gK || !trK || !chi || !out) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  MassIn A;
  MassOut O;
  for (int c = 0; c < 6; ++c) {
    A.g[c] = gK[c];
    A.K[c] = gK[6 + c];
    if (!A.g[c] || !A.K[c]) return nrgpu_set_error(NRGPU_ERR_ARG, "null metric or curvature pointer %d", c);
  }
  A.trK = trK;
  A.chi = chi;
  for (int v = 0; v < 8; ++v) {
    O.p[v] = out[v];
    if (!out[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null output pointer %d", v);
  }
  const cudaStream_t st = (cudaStream_t)stream;
  for (int b = 0; b < L->nboxes; ++b) {
    const BoxGeo &B = L->hbox[b];
    const long nb = (long)B.m * B.n * B.o;
    adm_mass_kernel<<<(unsigned)((nb + 127) / 128), 128, 0, st>>>(A, O, B, L->d_boundary, L->dx, L->dy, L->dz);
  }
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_sphere_integral(nrgpu_level *L, const double *f, double x0, double y0, double z0, double r,
                                     int ntheta, int nphi, int order, double *result, void *stream) {
  if (!L || !f || !result) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  if (ntheta < 1 || ntheta % 2 == 0) return nrgpu_set_error(NRGPU_ERR_ARG, "ntheta %d: an odd number of circles", ntheta);
  if (nphi < 2 || nphi % 2) return nrgpu_set_error(NRGPU_ERR_ARG, "nphi %d: an even number of points", nphi);
  if (order < 2 || order > kMaxOrder) return nrgpu_set_error(NRGPU_ERR_ARG, "interpolation order %d", order);
  // the sphere part covered by the grid and the symmetry factor
  // (Integral_over_sphere.c:233-268)
  double dtheta, dphi, symfactor;
  switch (L->symmetry) {
    case 0: dtheta = kPi / (ntheta + 1); dphi = 2.0 * kPi / nphi; symfactor = 1; break;
    case 4: dtheta = kPi / (2 * (ntheta + 1)); dphi = 2.0 * kPi / nphi; symfactor = 2; break;  // bitant
    case 6: dtheta = kPi / (2 * (ntheta + 1)); dphi = kPi / nphi; symfactor = 4; break;        // qreflect
    case 7: dtheta = kPi / (2 * (ntheta + 1)); dphi = kPi / (2 * nphi); symfactor = 8; break;  // octant
    default: return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "sphere integral on symmetry %d", L->symmetry);
  }
  std::vector<double> ct(ntheta + 2), cp(nphi + 2);
  for (int i = 1; i <= ntheta - 2; i += 2) {
    ct[i] = 2;
    ct[i + 1] = 1;
  }
  ct[ntheta] = 2;
  ct[ntheta + 1] = 0.5;
  cp[1] = 0.5;
  for (int i = 2; i <= nphi; i += 2) {
    cp[i] = 2;
    cp[i + 1] = 1;
  }
  cp[nphi + 1] = 0.5;
  const int np = (ntheta + 1) * (nphi + 1);
  std::vector<double> xyz(3 * (size_t)np), c(np);
  int n = 0;
  for (int i = 1; i <= ntheta + 1; i++) {
    const double theta = i * dtheta, sint = sin(theta), cost = cos(theta);
    for (int j = 1; j <= nphi + 1; j++) {
      const double phi = (j - 1) * dphi;
      c[n] = 4 * dtheta * dphi / 9 * ct[i] * cp[j] * sint;
      xyz[3 * n] = x0 + r * sint * cos(phi);
      xyz[3 * n + 1] = y0 + r * sint * sin(phi);
      xyz[3 * n + 2] = z0 + r * cost;
      n++;
    }
  }
  SphereArgs A;
  A.box = L->d_box;
  A.nboxes = L->nboxes;
  A.order = order;
  A.h[0] = L->dx;
  A.h[1] = L->dy;
  A.h[2] = L->dz;
  A.o[0] = L->hbox[0].x0;
  A.o[1] = L->hbox[0].y0;
  A.o[2] = L->hbox[0].z0;
  for (int b = 1; b < L->nboxes; b++) {
    A.o[0] = fmin(A.o[0], L->hbox[b].x0);
    A.o[1] = fmin(A.o[1], L->hbox[b].y0);
    A.o[2] = fmin(A.o[2], L->hbox[b].z0);
  }
  A.f = f;
  A.np = np;
  double *d_xyz = nullptr, *d_val = nullptr;
  int *d_ok = nullptr;
  const cudaStream_t st = (cudaStream_t)stream;
  int e = NRGPU_OK;
  if (cudaMalloc(&d_xyz, sizeof(double) * 3 * np) != cudaSuccess ||
      cudaMalloc(&d_val, sizeof(double) * np) != cudaSuccess || cudaMalloc(&d_ok, sizeof(int) * np) != cudaSuccess) {
    cudaGetLastError();
    e = nrgpu_set_error(NRGPU_ERR_NOMEM, "sphere points");
  }
  std::vector<double> val(np);
  std::vector<int> ok(np);
  if (!e && cudaMemcpyAsync(d_xyz, xyz.data(), sizeof(double) * 3 * np, cudaMemcpyHostToDevice, st) != cudaSuccess)
    e = nrgpu_set_error(NRGPU_ERR_CUDA, "sphere points upload");
  if (!e) {
    A.xyz = d_xyz;
    A.val = d_val;
    A.ok = d_ok;
    sphere_interp_kernel<<<(np + 127) / 128, 128, 0, st>>>(A);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(val.data(), d_val, sizeof(double) * np, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaMemcpyAsync(ok.data(), d_ok, sizeof(int) * np, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
      e = nrgpu_set_error(NRGPU_ERR_CUDA, "sphere interpolation");
  }
  cudaFree(d_xyz);
  cudaFree(d_val);
  cudaFree(d_ok);
  if (e) return e;
  // the weighted values summed in point order; a point off the level makes
  // the integral 0 (Integral_over_sphere.c:333-343)
  double sum = 0;
  for (int q = 0; q < np; q++) {
    if (!ok[q]) {
      *result = 0;
      return NRGPU_OK;
    }
    sum += c[q] * val[q];
  }
  *result = sum * symfactor;
  return NRGPU_OK;
}
