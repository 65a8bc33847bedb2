// nrgpu_analysis.cu -- analysis quantities on the device (sm_100a), FP64:
//   nrgpu_adm_mass_integrands  the eight integrands of ADM_mass
//                              (projects/ADM_mass/ADM_mass.c:11-225): the ADM
//                              mass (adm_mass_integrand.c), its conformal-
//                              factor version (adm_mass_integrand_chi.c) and
//                              the linear and angular momentum
//                              (adm_pj_integrand.c), at the flag-0 points
//   nrgpu_psi4                 rpsi4, ipsi4 and Csqr of curvature_invariants_N
//                              (projects/Invariants), rescaled by r
//   nrgpu_psi4_modes           the spin-weight -2 modes of compute_modes
//                              (Invariants.c:367-540) on spheres
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
#include "nrgpu_fd.cuh"

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

// ---- Psi4 and the square of the Weyl tensor ---------------------------------
// curvature_invariants_N (projects/Invariants/curvature_invariants_N.m:
// 14-208; the C code is generated from it): from the ADM metric and
// curvature, the lapse and the shift at a flag-0 point,
//   3-Ricci R_ab (MTW conventions) from the metric's first and second
//   derivatives, the 3-Riemann tensor from R_ab (three dimensions),
//   Riemm_abcd = R_abcd + K_ac K_bd - K_ad K_bc,
//   Riemm_abc  = -(d_c K_ab - d_b K_ac + G^d_ab K_cd - G^d_ac K_bd),
//   Riemm_ab   = R_ab + K K_ab - K_ac g^cd K_db,
//   Csqr = g^ac g^bd (E_ab E_cd - B_ab B_cd), E = Riemm_ab,
//          B_ab = -g_ac eps^cef Riemm_bef / (2 sqrt(det g)),
// the tetrad (Gram-Schmidt on the azimuthal, radial and their cross
// vectors, or the flat Kinnersley tetrad), and
//   psi4 = -(Riemm_abcd r^a r^c - 2 Riemm_bcd r^c + Riemm_bd)
//          (mb^b mb^d) / 2                       (gauss_codacci_mainardi
//                                                 standard), or
//   psi4 = -(Riemm_abcd n^a n^c + 2 Riemm_bcd n^0 n^c + Riemm_bd n^0 n^0)
//          (mb^b mb^d)                           (flat),
// with mb = m - i m_imag conjugated as the reference's rmb, imb.
// Derivatives at order_centered with the order ladder near box faces (2nd
// order one point in, 4th two points in), as the constraints.
struct Psi4In {
  const double *p[16];  // g (6), K (6), alpha, beta (3)
};
struct Psi4Out {
  double *rpsi4, *ipsi4, *csqr;  // csqr may be null
};
struct Psi4Opt {
  int kinnersley, flat, csqr;
  double x0, y0, z0;
};

__device__ __forceinline__ double eps3(int a, int b, int c) {
  return (double)((a - b) * (b - c) * (c - a)) * 0.5;
}

template <int ORD>
__device__ void psi4_point(const Psi4In &A, long x, const long st[3], const double h[3], const double xc[3],
                           const Psi4Opt &O, double out[3]) {
  double g[6], K[6], dg[3][6], dK[3][6], dd[6][6];
  const double i1[3] = {1.0 / (den1<ORD>() * h[0]), 1.0 / (den1<ORD>() * h[1]), 1.0 / (den1<ORD>() * h[2])};
#pragma unroll
  for (int v = 0; v < 6; ++v) {
    g[v] = ldg(A.p[v] + x);
    K[v] = ldg(A.p[6 + v] + x);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      dg[c][v] = d1n<ORD>(A.p[v], (int)x, (int)st[c]) * i1[c];
      dK[c][v] = d1n<ORD>(A.p[6 + v], (int)x, (int)st[c]) * i1[c];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b)
        dd[sy(a, b)][v] = a == b ? d2n<ORD>(A.p[v], (int)x, (int)st[a]) / (den2<ORD>() * h[a] * h[a])
                                 : d11n<ORD>(A.p[v], (int)x, (int)st[a], (int)st[b]) /
                                       (den1<ORD>() * h[a] * den1<ORD>() * h[b]);
  }
  // inverse metric by the adjugate over det = g_1c adj_1c
  double adj[6];
  adj[0] = g[3] * g[5] - g[4] * g[4];
  adj[1] = g[2] * g[4] - g[1] * g[5];
  adj[2] = g[1] * g[4] - g[2] * g[3];
  adj[3] = g[0] * g[5] - g[2] * g[2];
  adj[4] = g[1] * g[2] - g[0] * g[4];
  adj[5] = g[0] * g[3] - g[1] * g[1];
  const double detg = g[0] * adj[0] + g[1] * adj[1] + g[2] * adj[2];
  double gi[6];
#pragma unroll
  for (int v = 0; v < 6; ++v) gi[v] = adj[v] / detg;
  // connection of the first kind gd[c][ab] and the second kind gu[c][ab]
  double gd[3][6], gu[3][6];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) gd[c][sy(a, b)] = 0.5 * (dg[b][sy(a, c)] + dg[a][sy(b, c)] - dg[c][sy(a, b)]);
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int ab = 0; ab < 6; ++ab)
      gu[c][ab] = gi[sy(c, 0)] * gd[0][ab] + gi[sy(c, 1)] * gd[1][ab] + gi[sy(c, 2)] * gd[2][ab];
  // Ricci tensor and scalar
  double Ric[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double r = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          double q = 0.5 * (-dd[sy(c, d)][sy(a, b)] - dd[sy(a, b)][sy(c, d)] + dd[sy(a, c)][sy(b, d)] +
                            dd[sy(b, c)][sy(a, d)]);
#pragma unroll
          for (int e = 0; e < 3; ++e) q += gu[e][sy(a, c)] * gd[e][sy(b, d)] - gu[e][sy(a, b)] * gd[e][sy(c, d)];
          r += gi[sy(c, d)] * q;
        }
      Ric[sy(a, b)] = r;
    }
  double Rs = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) Rs += gi[sy(a, b)] * Ric[sy(a, b)];
  double trK = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) trK += gi[sy(a, b)] * K[sy(a, b)];
  // Riemm_ab and Riemm_abc (the electric part and the Codazzi term)
  double R2[3][3], R3[3][3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      double kk = 0;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) kk += K[sy(a, c)] * gi[sy(c, d)] * K[sy(d, b)];
      R2[a][b] = Ric[sy(a, b)] + trK * K[sy(a, b)] - kk;
    }
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double t = dK[c][sy(a, b)] - dK[b][sy(a, c)];
#pragma unroll
        for (int d = 0; d < 3; ++d) t += gu[d][sy(a, b)] * K[sy(c, d)] - gu[d][sy(a, c)] * K[sy(b, d)];
        R3[a][b][c] = -t;
      }
  // 4-Riemann contracted with a vector u on its 1st and 3rd index:
  // Riemm_abcd u^a u^c with R_abcd from the Ricci tensor
  auto riem4uu = [&](const double u[3], double M[3][3]) {
    double gu_[3], Ru[3], Ku[3];
    double S = 0, Ru2 = 0, Ku2 = 0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      gu_[b] = g[sy(b, 0)] * u[0] + g[sy(b, 1)] * u[1] + g[sy(b, 2)] * u[2];
      Ru[b] = Ric[sy(b, 0)] * u[0] + Ric[sy(b, 1)] * u[1] + Ric[sy(b, 2)] * u[2];
      Ku[b] = K[sy(b, 0)] * u[0] + K[sy(b, 1)] * u[1] + K[sy(b, 2)] * u[2];
    }
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      S += gu_[b] * u[b];
      Ru2 += Ru[b] * u[b];
      Ku2 += Ku[b] * u[b];
    }
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int d = 0; d < 3; ++d)
        M[b][d] = S * Ric[sy(b, d)] + g[sy(b, d)] * Ru2 - 0.5 * Rs * S * g[sy(b, d)] - gu_[d] * Ru[b] -
                  gu_[b] * Ru[d] + 0.5 * Rs * gu_[d] * gu_[b] + Ku2 * K[sy(b, d)] - Ku[d] * Ku[b];
  };
  const double sq = sqrt(detg);
  if (O.csqr) {
    // Csqr
    double B[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        double t = 0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int e = 0; e < 3; ++e)
#pragma unroll
            for (int f = 0; f < 3; ++f)
              if (e != f && c != e && c != f) t += g[sy(a, c)] * eps3(c, e, f) * R3[b][e][f];
        B[a][b] = -0.5 / sq * t;
      }
    double cs = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int d = 0; d < 3; ++d)
            cs += gi[sy(a, c)] * gi[sy(b, d)] * (R2[a][b] * R2[c][d] - B[a][b] * B[c][d]);
    out[2] = cs;
  }
  // coordinates about the sphere origin and the tetrad
  const double X = xc[0] - O.x0, Y = xc[1] - O.y0, Z = xc[2] - O.z0;
  const double r = sqrt(X * X + Y * Y + Z * Z);
  double vr[3] = {0, 0, 0}, rm[3], im[3], n[3], n0;
  const double tf = 1 / sqrt(2.0);
  if (O.kinnersley) {
    const double ct = Z / r, stt = sqrt(1 - (Z / r) * (Z / r));
    const double cp = X / (r * stt), sp = Y / (r * stt);
    n0 = 0.5;
    n[0] = -0.5 * stt * cp;
    n[1] = -0.5 * stt * sp;
    n[2] = -0.5 * ct;
    rm[0] = tf * ct * cp;
    rm[1] = tf * ct * sp;
    rm[2] = -tf * stt;
    im[0] = -tf * sp;
    im[1] = tf * cp;
    im[2] = 0;
  } else {
    double v1[3] = {-Y, X, 0}, v2[3] = {X, Y, Z}, v3[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double t = 0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double cr = 0;
#pragma unroll
        for (int b = 0; b < 3; ++b)
#pragma unroll
          for (int c = 0; c < 3; ++c)
            if (b != c && d != b && d != c) cr += eps3(d, b, c) * v1[b] * v2[c];
        t += gi[sy(a, d)] * cr;
      }
      v3[a] = sq * t;
    }
    auto dotg = [&](const double *p, const double *q) {
      double s2 = 0;
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) s2 += p[a] * q[b] * g[sy(a, b)];
      return s2;
    };
    const double w11 = sqrt(dotg(v1, v1));
    for (int a = 0; a < 3; ++a) v1[a] /= w11;
    const double w12 = dotg(v1, v2);
    for (int a = 0; a < 3; ++a) v2[a] -= v1[a] * w12;
    const double w22 = sqrt(dotg(v2, v2));
    for (int a = 0; a < 3; ++a) v2[a] /= w22;
    const double w13 = dotg(v1, v3), w23 = dotg(v2, v3);
    for (int a = 0; a < 3; ++a) v3[a] -= v1[a] * w13 + v2[a] * w23;
    const double w33 = sqrt(dotg(v3, v3));
    for (int a = 0; a < 3; ++a) v3[a] /= w33;
    const double al = ldg(A.p[12] + x);
    n0 = tf / al;
    for (int a = 0; a < 3; ++a) {
      vr[a] = v2[a];
      n[a] = tf * (-ldg(A.p[13 + a] + x) / al - v2[a]);
      rm[a] = tf * v3[a];
      im[a] = tf * v1[a];
    }
  }
  // mb = rm - i im: rmb = rm, imb = -im
  double Xbd[3][3], M4[3][3];
  const double *u = O.flat ? n : vr;
  riem4uu(u, M4);
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double m3 = R3[b][0][d] * u[0] + R3[b][1][d] * u[1] + R3[b][2][d] * u[2];
      Xbd[b][d] = O.flat ? M4[b][d] + 2 * m3 * n0 + R2[b][d] * n0 * n0 : M4[b][d] - 2 * m3 + R2[b][d];
    }
  double re = 0, imv = 0;
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      re += Xbd[b][d] * (rm[b] * rm[d] - im[b] * im[d]);
      imv += Xbd[b][d] * (rm[b] * (-im[d]) + (-im[b]) * rm[d]);
    }
  const double f = O.flat ? -1.0 : -0.5;
  out[0] = f * re;
  out[1] = f * imv;
}

__device__ __forceinline__ int ladder_o(int order, int d) {
  if (order == 2 || d == 1) return 2;
  if (order == 4 || d == 2) return 4;
  return 6;
}

__global__ void __launch_bounds__(128) psi4_kernel(Psi4In A, Psi4Out O, Psi4Opt opt, BoxGeo box,
                                                  const int *__restrict__ boundary, int order, double dx, double dy,
                                                  double dz, int *status) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nb = (long)box.m * box.n * box.o;
  if (t >= nb) return;
  const long x = box.noffset + t;
  if (__ldg(boundary + x) != 0) return;
  const int i = (int)(t % box.m), j = (int)((t / box.m) % box.n), k = (int)(t / ((long)box.m * box.n));
  int d = min(min(i, j), k);
  d = min(d, min(min(box.m - 1 - i, box.n - 1 - j), box.o - 1 - k));
  const long st[3] = {1, box.m, (long)box.m * box.n};
  const double h[3] = {dx, dy, dz};
  const double xc[3] = {box.x0 + i * dx, box.y0 + j * dy, box.z0 + k * dz};
  double out[3];
  const int ord = ladder_o(order, d);
  if (ord == 2) psi4_point<2>(A, x, st, h, xc, opt, out);
  else if (ord == 4) psi4_point<4>(A, x, st, h, xc, opt, out);
  else psi4_point<6>(A, x, st, h, xc, opt, out);
  if (!isfinite(out[0]) || !isfinite(out[1])) atomicOr(status, 1);
  O.rpsi4[x] = out[0];
  O.ipsi4[x] = out[1];
  if (O.csqr) O.csqr[x] = out[2];
}

// rescale_psi4 (Invariants.c:263-284): psi4 times the distance to the
// sphere origin at every point
__global__ void rescale_psi4_kernel(double *rp, double *ip, BoxGeo box, double dx, double dy, double dz, double x0,
                                    double y0, double z0) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nb = (long)box.m * box.n * box.o;
  if (t >= nb) return;
  const long x = box.noffset + t;
  const int i = (int)(t % box.m), j = (int)((t / box.m) % box.n), k = (int)(t / ((long)box.m * box.n));
  const double X = box.x0 + i * dx - x0, Y = box.y0 + j * dy - y0, Z = box.z0 + k * dz - z0;
  const double r = sqrt(X * X + Y * Y + Z * Z);
  rp[x] *= r;
  ip[x] *= r;
}

// the spin-weight -2 spherical harmonic -2Y_lm (theta, phi) by the Wigner
// d-function sum of Ajith et al., "Data formats for numerical relativity
// waves" (arXiv:0709.0093, eqs. II.7-II.8): sqrt((2l+1)/4pi) d^l_{m,2}(theta)
// e^{i m phi}, the convention of the reference's precomputed table
// (SphericalHarmonics_precomp.c:235-442)
__device__ double factorial_d(int n) {
  double f = 1;
  for (int i = 2; i <= n; i++) f *= i;
  return f;
}
__device__ void sYlm_m2(int l, int m, double phi, double theta, double *re, double *im) {
  const double c = cos(0.5 * theta), s = sin(0.5 * theta);
  const int k1 = m - 2 > 0 ? m - 2 : 0, k2 = l + m < l - 2 ? l + m : l - 2;
  const double pre = sqrt(factorial_d(l + m) * factorial_d(l - m) * factorial_d(l + 2) * factorial_d(l - 2));
  double d = 0;
  for (int k = k1; k <= k2; k++) {
    const double den = factorial_d(l + m - k) * factorial_d(l - 2 - k) * factorial_d(k) * factorial_d(k + 2 - m);
    d += ((k & 1) ? -1.0 : 1.0) * pre / den * pow(c, 2 * l + m - 2 - 2 * k) * pow(s, 2 * k + 2 - m);
  }
  const double a = sqrt((2 * l + 1) / (4 * kPi)) * d;
  *re = a * cos(m * phi);
  *im = a * sin(m * phi);
}

// compute_modes (Invariants.c:367-452): the integrand of mode (l, m) at
// every point, conj(Y) psi4 with phi = atan(y/x) (+ pi for x < 0) and
// cos(theta) = z/r about the sphere origin
__global__ void mode_integrand_kernel(const double *__restrict__ rp, const double *__restrict__ ip, double *outR,
                                      double *outI, BoxGeo box, double dx, double dy, double dz, double x0,
                                      double y0, double z0, int l, int m) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nb = (long)box.m * box.n * box.o;
  if (t >= nb) return;
  const long x = box.noffset + t;
  const int i = (int)(t % box.m), j = (int)((t / box.m) % box.n), k = (int)(t / ((long)box.m * box.n));
  const double X = box.x0 + i * dx - x0, Y = box.y0 + j * dy - y0, Z = box.z0 + k * dz - z0;
  const double r = sqrt(X * X + Y * Y + Z * Z);
  const double ct = Z / r;
  const double phi = X >= 0 ? atan(Y / X) : kPi + atan(Y / X);
  double yr, yi;
  sYlm_m2(l, m, phi, acos(ct), &yr, &yi);
  outR[x] = yr * rp[x] + yi * ip[x];
  outI[x] = yr * ip[x] - yi * rp[x];
}

}  // namespace

extern "C" int nrgpu_sphere_integral(nrgpu_level *L, const double *f, double x0, double y0, double z0, double r,
                                     int ntheta, int nphi, int order, double *result, void *stream);

extern "C" int nrgpu_psi4_modes(nrgpu_level *L, const double *rpsi4, const double *ipsi4, const double *origin,
                                int lmin, int lmax, const double *radii, int nr, int ntheta, int nphi, int order,
                                double *out, void *stream) {
  if (!L || !rpsi4 || !ipsi4 || !radii || !out || nr < 1) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  if (lmin < 2 || lmax < lmin || lmax > 12) return nrgpu_set_error(NRGPU_ERR_ARG, "modes l = %d..%d (2..12)", lmin, lmax);
  if (L->symmetry) return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "mode decomposition on a symmetry grid");
  const double o[3] = {origin ? origin[0] : 0.0, origin ? origin[1] : 0.0, origin ? origin[2] : 0.0};
  const cudaStream_t st = (cudaStream_t)stream;
  double *buf = nullptr;
  if (cudaMalloc(&buf, sizeof(double) * 2 * (size_t)L->npoints) != cudaSuccess) {
    cudaGetLastError();
    return nrgpu_set_error(NRGPU_ERR_NOMEM, "mode integrands");
  }
  cudaMemsetAsync(buf, 0, sizeof(double) * 2 * (size_t)L->npoints, st);
  const int lnum = lmax - lmin + 1, mnum = 2 * lmax + 1;
  int e = NRGPU_OK;
  for (int l = lmin; l <= lmax && !e; l++)
    for (int m = l; m >= -l && !e; m--) {
      for (int b = 0; b < L->nboxes; ++b) {
        const BoxGeo &B = L->hbox[b];
        const long nb = (long)B.m * B.n * B.o;
        mode_integrand_kernel<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(
            rpsi4, ipsi4, buf, buf + L->npoints, B, L->dx, L->dy, L->dz, o[0], o[1], o[2], l, m);
      }
      if (cudaGetLastError() != cudaSuccess) e = nrgpu_set_error(NRGPU_ERR_CUDA, "mode integrand");
      for (int n = 0; n < nr && !e; n++) {
        double *dst = out + 2 * ((size_t)n * lnum * mnum + (size_t)(l - lmin) * mnum + (m + l));
        if ((e = nrgpu_sphere_integral(L, buf, o[0], o[1], o[2], radii[n], ntheta, nphi, order, dst, stream)))
          break;
        e = nrgpu_sphere_integral(L, buf + L->npoints, o[0], o[1], o[2], radii[n], ntheta, nphi, order, dst + 1,
                                  stream);
      }
    }
  cudaStreamSynchronize(st);
  cudaFree(buf);
  return e;
}

extern "C" int nrgpu_psi4(nrgpu_level *L, const double *const *gK, const double *alpha, const double *const *beta,
                          int order_centered, int kinnersley, int flat, const double *origin, double *rpsi4,
                          double *ipsi4, double *csqr, void *stream) {
  if (!L || !gK || !alpha || !beta || !rpsi4 || !ipsi4) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  if (order_centered != 2 && order_centered != 4 && order_centered != 6)
    return nrgpu_set_error(NRGPU_ERR_ARG, "order_centered %d", order_centered);
  Psi4In A;
  for (int c = 0; c < 12; ++c) {
    A.p[c] = gK[c];
    if (!gK[c]) return nrgpu_set_error(NRGPU_ERR_ARG, "null metric or curvature pointer %d", c);
  }
  A.p[12] = alpha;
  for (int c = 0; c < 3; ++c) {
    A.p[13 + c] = beta[c];
    if (!beta[c]) return nrgpu_set_error(NRGPU_ERR_ARG, "null shift pointer %d", c);
  }
  Psi4Out O = {rpsi4, ipsi4, csqr};
  Psi4Opt opt = {kinnersley ? 1 : 0, flat ? 1 : 0, csqr ? 1 : 0, origin ? origin[0] : 0.0,
                 origin ? origin[1] : 0.0, origin ? origin[2] : 0.0};
  const cudaStream_t st = (cudaStream_t)stream;
  for (int b = 0; b < L->nboxes; ++b) {
    const BoxGeo &B = L->hbox[b];
    const long nb = (long)B.m * B.n * B.o;
    psi4_kernel<<<(unsigned)((nb + 127) / 128), 128, 0, st>>>(A, O, opt, B, L->d_boundary, order_centered, L->dx,
                                                              L->dy, L->dz, L->d_status);
  }
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_psi4_rescale(nrgpu_level *L, double *rpsi4, double *ipsi4, const double *origin, void *stream) {
  if (!L || !rpsi4 || !ipsi4) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  const double o[3] = {origin ? origin[0] : 0.0, origin ? origin[1] : 0.0, origin ? origin[2] : 0.0};
  const cudaStream_t st = (cudaStream_t)stream;
  for (int b = 0; b < L->nboxes; ++b) {
    const BoxGeo &B = L->hbox[b];
    const long nb = (long)B.m * B.n * B.o;
    rescale_psi4_kernel<<<(unsigned)((nb + 255) / 256), 256, 0, st>>>(rpsi4, ipsi4, B, L->dx, L->dy, L->dz, o[0],
                                                                     o[1], o[2]);
  }
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

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
