// nrgpu_z4bg_cpbc.cu -- the CPBC2 box boundary of Z4c (sm_100a, FP64):
// z4_boundary_box (projects/z4/z4_boundary_box.m:14-420; the C code is
// generated from it), written in tensor form.  At each point one inside a
// box face (boundaryNaway(1)): the outward face normal s (give_cube_normal,
// utility/boundary/normals.c:14-48, the diagonal of an edge or corner),
// normalised with the physical inverse metric chi g~^-1; the 2+1 projectors
// q; the lapse and shift speeds; the conformal and full Ricci tensors; and
// the rhs of Khat, Theta, A_ab (its ss, sA, qq and trace-free AB parts) and
// G^a (its s and A parts) from the constraint-preserving and gauge
// conditions.  Derivatives by the 2nd-order centred stencils of the spec's
// del and deldel.  The guards of the spec are kept: chi below
// z4_chi_div_floor is raised to it, a determinant inverse below 1e-5 is
// taken as 1, and a normal of squared length below 1e-5 is normalised
// with the flat metric.  The shift-driver terms carry z4_shiftdriver times
// z4_bc_use_eta (default no: zero); this build takes the default.
#include "nrgpu_level.cuh"

namespace {

constexpr int NV = NRGPU_Z4_NVARS;

struct Vars {
  double *p[NV];
};

struct Cpbc {
  double kappa1, kappa2, chiDivFloor, chipsipower, shiftdriver;
};

// the rhs of A (6), Khat, G (3) and Theta at the point x of a box with
// strides st, local indices idx, largest indices mx and coordinates X, Y, Z
__host__ __device__ inline void cpbc_point(double *const *cur, long x, const long st[3], const double h[3],
                                           const int idx[3], const int mx[3], double X, double Y, double Z,
                                           const Cpbc &P, double out[11]) {
  auto V = [&](int v, long o) { return cur[v][x + o]; };
  auto d1 = [&](int v, int a) { return (1 / (2 * h[a])) * (-V(v, -st[a]) + V(v, st[a])); };
  auto d2 = [&](int v, int a, int b) {
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    if (a == b) return (1 / (h[a] * h[a])) * (-2. * V(v, 0) + V(v, -st[a]) + V(v, st[a]));
    return (1 / (4 * h[a] * h[b])) *
           (V(v, -st[a] - st[b]) - V(v, st[a] - st[b]) - V(v, -st[a] + st[b]) + V(v, st[a] + st[b]));
  };
  // symmetric tensors keep their a <= b components (the generated code
  // stores only those)
  auto mirror = [](double(&m)[3][3]) {
    m[1][0] = m[0][1];
    m[2][0] = m[0][2];
    m[2][1] = m[1][2];
  };
  // state
  double g[3][3], A[3][3], G[3], beta[3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      g[a][b] = V(sy(a, b), 0);
      A[a][b] = V(7 + sy(a, b), 0);
    }
  for (int a = 0; a < 3; ++a) {
    G[a] = V(14 + a, 0);
    beta[a] = V(19 + a, 0);
  }
  const double chi = V(6, 0), Khat = V(13, 0), Theta = V(17, 0), alpha = V(18, 0);
  // derivatives
  double da[3], dda[3][3], db[3][3], ddb[3][3][3], dchi[3], ddchi[3][3], dg[3][3][3], ddg[3][3][3][3];
  double dKhat[3], dA[3][3][3], dG[3][3], dTheta[3];
  for (int a = 0; a < 3; ++a) {
    da[a] = d1(18, a);
    dchi[a] = d1(6, a);
    dKhat[a] = d1(13, a);
    dTheta[a] = d1(17, a);
    for (int b = 0; b < 3; ++b) {
      dda[a][b] = d2(18, a, b);
      ddchi[a][b] = d2(6, a, b);
      db[a][b] = d1(19 + b, a);
      dG[a][b] = d1(14 + b, a);
      for (int c2 = 0; c2 < 3; ++c2) {
        ddb[a][b][c2] = d2(19 + c2, a, b);
        dg[a][b][c2] = d1(sy(b, c2), a);
        dA[a][b][c2] = d1(7 + sy(b, c2), a);
        for (int e = 0; e < 3; ++e) ddg[a][b][c2][e] = d2(sy(c2, e), a, b);
      }
    }
  }
  // normal
  double shat[3], sn = 0;
  for (int a = 0; a < 3; ++a) {
    shat[a] = idx[a] == mx[a] - 1 ? 1.0 : (idx[a] == 1 ? -1.0 : 0.0);
    sn += shat[a] * shat[a];
  }
  const double oos = 1. / sqrt(sn);
  for (int a = 0; a < 3; ++a) shat[a] *= oos;
  const double r = sqrt(X * X + Y * Y + Z * Z);
  const double chig = chi < P.chiDivFloor ? P.chiDivFloor : chi;
  // inverse conformal metric
  const double adj[6] = {g[1][1] * g[2][2] - g[1][2] * g[1][2], g[0][2] * g[1][2] - g[0][1] * g[2][2],
                         g[0][1] * g[1][2] - g[0][2] * g[1][1], g[0][0] * g[2][2] - g[0][2] * g[0][2],
                         g[0][1] * g[0][2] - g[0][0] * g[1][2], g[0][0] * g[1][1] - g[0][1] * g[0][1]};
  double detginv = 1 / (2. * g[0][1] * g[0][2] * g[1][2] + g[0][0] * g[1][1] * g[2][2] -
                         g[2][2] * (g[0][1] * g[0][1]) - g[1][1] * (g[0][2] * g[0][2]) -
                         g[0][0] * (g[1][2] * g[1][2]));
  if (detginv < 0.00001) detginv = 1.0;
  double gi[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) gi[a][b] = detginv * adj[sy(a, b)];
  double Gi[3][3];  // ADMginv
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) Gi[a][b] = chig * gi[a][b];
  double mod = 0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) mod += Gi[a][b] * shat[a] * shat[b];
  if (mod < 0.00001) mod = shat[0] * shat[0] + shat[1] * shat[1] + shat[2] * shat[2];
  const double oom = 1 / sqrt(mod);
  double sd[3], su[3];
  for (int a = 0; a < 3; ++a) sd[a] = oom * shat[a];
  for (int a = 0; a < 3; ++a) su[a] = Gi[a][0] * sd[0] + Gi[a][1] * sd[1] + Gi[a][2] * sd[2];
  double qud[3][3], qdd[3][3], quu[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      qud[a][b] = (a == b ? 1.0 : 0.0) - su[a] * sd[b];
      qdd[a][b] = g[a][b] / chig - sd[a] * sd[b];
      quu[a][b] = Gi[a][b] - su[a] * su[b];
    }
  mirror(qdd);
  mirror(quu);
  const double muL = 2 / alpha, muS = 1 / chig;
  const double vbetas = 2 * sqrt(muS / 3), vbetaA = sqrt(muS), smuL = sqrt(muL);
  const double K = Khat + 2 * Theta;
  double dK[3];
  for (int a = 0; a < 3; ++a) dK[a] = dKhat[a] + 2 * dTheta[a];
  // connection of the conformal metric: gdo[c][a][b] = G_cab, gam[c][a][b]
  double gdo[3][3][3], gam[3][3][3];
  for (int cc = 0; cc < 3; ++cc)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) gdo[cc][a][b] = 0.5 * (dg[a][b][cc] + dg[b][a][cc] - dg[cc][a][b]);
  for (int cc = 0; cc < 3; ++cc)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double t = 0;
        for (int d = 0; d < 3; ++d) t += gi[cc][d] * gdo[d][a][b];
        gam[cc][a][b] = t;
      }
  double Gfg[3];
  for (int a = 0; a < 3; ++a) {
    double t = 0;
    for (int b = 0; b < 3; ++b)
      for (int cc = 0; cc < 3; ++cc) t += gi[b][cc] * gam[a][b][cc];
    Gfg[a] = t;
  }
  // dGfromgdu[a][b]
  double dGfg[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double t = 0;
      for (int cc = 0; cc < 3; ++cc)
        for (int d = 0; d < 3; ++d)
          for (int e = 0; e < 3; ++e) t += gi[b][cc] * gi[d][e] * ddg[a][d][e][cc];
      for (int cc = 0; cc < 3; ++cc)
        for (int d = 0; d < 3; ++d)
          for (int e = 0; e < 3; ++e)
            for (int f = 0; f < 3; ++f)
              for (int g2 = 0; g2 < 3; ++g2)
                t -= (gi[b][cc] * gi[d][f] * gi[e][g2] + gi[b][e] * gi[g2][cc] * gi[d][f]) * dg[g2][e][f] *
                     dg[a][cc][d];
      dGfg[a][b] = t;
    }
  // Ricci tensor of the conformal metric
  double R[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double t = 0;
      for (int cc = 0; cc < 3; ++cc)
        for (int d = 0; d < 3; ++d) {
          double u = -0.5 * ddg[cc][d][a][b];
          for (int e = 0; e < 3; ++e)
            u += gam[e][cc][a] * gdo[b][e][d] + gam[e][cc][b] * gdo[a][e][d] + gam[e][a][d] * gdo[e][cc][b];
          t += gi[cc][d] * u;
        }
      double w = 0;
      for (int cc = 0; cc < 3; ++cc)
        w += g[cc][a] * dG[b][cc] + g[cc][b] * dG[a][cc] + Gfg[cc] * (gdo[a][b][cc] + gdo[b][a][cc]);
      R[a][b] = t + 0.5 * w;
    }
  mirror(R);
  // conformal factor terms
  const double oocp = 1 / P.chipsipower;
  const double fphi = oocp * log(chig);
  const double psim4 = exp(-4 * fphi);
  double df[3], ddf[3][3], cddf[3][3];
  for (int a = 0; a < 3; ++a) df[a] = oocp * dchi[a] / chig;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) ddf[a][b] = oocp * ddchi[a][b] / chig - P.chipsipower * df[a] * df[b];
  mirror(ddf);
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double t = ddf[a][b];
      for (int cc = 0; cc < 3; ++cc) t -= gam[cc][a][b] * df[cc];
      cddf[a][b] = t;
    }
  mirror(cddf);
  double trcddf = 0, dfdf = 0, dfda = 0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      trcddf += gi[a][b] * cddf[a][b];
      dfdf += gi[a][b] * df[a] * df[b];
      dfda += gi[a][b] * df[a] * da[b];
    }
  double Rf[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b)
      Rf[a][b] = R[a][b] + 4 * df[a] * df[b] - 2 * cddf[a][b] - 2 * g[a][b] * trcddf - 4 * g[a][b] * dfdf;
  mirror(Rf);
  double Rhat = 0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) Rhat += gi[a][b] * Rf[a][b];
  Rhat *= psim4;
  // second covariant derivative of the lapse (the generated code stores
  // its a > b components in the ordered slots, z4_boundary_box.m:446, so
  // the tensor is symmetric)
  double cdda[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) {
      double t = dda[a][b];
      for (int cc = 0; cc < 3; ++cc) t -= gam[cc][a][b] * da[cc];
      cdda[a][b] = t - 2 * (df[a] * da[b] + df[b] * da[a] - g[a][b] * dfda);
    }
  mirror(cdda);
  double trcdda = 0;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) trcdda += gi[a][b] * cdda[a][b];
  trcdda *= psim4;
  // A products and derivatives
  double AA[3][3], Ai[3][3], cdA[3][3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double t = 0, u = 0;
      for (int cc = 0; cc < 3; ++cc)
        for (int d = 0; d < 3; ++d) {
          t += gi[cc][d] * A[a][cc] * A[d][b];
          u += gi[a][cc] * gi[b][d] * A[cc][d];
        }
      AA[a][b] = t;
      Ai[a][b] = u;
    }
  mirror(Ai);
  for (int cc = 0; cc < 3; ++cc)
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        double t = dA[cc][a][b];
        for (int d = 0; d < 3; ++d) t -= gam[d][cc][a] * A[b][d] + gam[d][cc][b] * A[a][d];
        cdA[cc][a][b] = t;
      }
  for (int cc = 0; cc < 3; ++cc) mirror(cdA[cc]);
  const double divb = db[0][0] + db[1][1] + db[2][2], tdb = 2. / 3 * divb;
  double lieg[3][3], lieA[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) {
      double t = -g[a][b] * tdb, u = -A[a][b] * tdb;
      for (int cc = 0; cc < 3; ++cc) {
        t += beta[cc] * dg[cc][a][b] + db[a][cc] * g[b][cc] + db[b][cc] * g[a][cc];
        u += beta[cc] * dA[cc][a][b] + db[a][cc] * A[b][cc] + db[b][cc] * A[a][cc];
      }
      lieg[a][b] = t;
      lieA[a][b] = u;
    }
  mirror(lieg);
  mirror(lieA);
  double DKhat = 0, DK = 0, DTheta = 0, bdKhat = 0, bdTheta = 0;
  for (int a = 0; a < 3; ++a) {
    DKhat += su[a] * dKhat[a];
    DK += su[a] * dK[a];
    DTheta += su[a] * dTheta[a];
    bdKhat += beta[a] * dKhat[a];
    bdTheta += beta[a] * dTheta[a];
  }
  const double lienKhat = -smuL * DKhat - smuL * Khat / r;
  const double lienTheta = -(DTheta + Theta / r) - P.kappa1 * (2 + P.kappa2) * Theta;
  const double rKhat = bdKhat + alpha * lienKhat;
  const double rTheta = alpha * lienTheta + bdTheta;
  // G^a, s part
  double rGams = 0;
  {
    double dGaa = dG[0][0] + dG[1][1] + dG[2][2], sbdG = 0, t1 = 0, t2 = 0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        sbdG += sd[b] * beta[a] * dG[a][b];
        for (int cc = 0; cc < 3; ++cc) {
          t1 += quu[a][b] * sd[cc] * ddb[a][b][cc];
          t2 += su[a] * qud[b][cc] * ddb[a][b][cc];
        }
      }
    rGams = -vbetas * dGaa + sbdG + 2 * P.shiftdriver / sqrt(3.) / vbetaA * divb + t1 / chig - t2 / chig +
            4 * alpha * smuL / (3 * (vbetas + smuL)) * DKhat / chig + 2 * alpha / (3 * (vbetas + 1)) * DTheta / chig;
  }
  // A, ss part
  double rACss;
  {
    double t = 0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        for (int cc = 0; cc < 3; ++cc) t += 2 * su[b] * gi[cc][a] * cdA[cc][a][b] - 3 * su[a] * gi[b][cc] * dchi[cc] * A[a][b] / chig;
    t += -4. / 3 * DK + 2 * DTheta;
    for (int a = 0; a < 3; ++a) t -= P.kappa1 * chig * sd[a] * (G[a] - Gfg[a]);
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        t += 2. / 3 * chig * su[a] * sd[b] * (dG[a][b] - dGfg[a][b]) - 1. / 3 * chig * qud[a][b] * (dG[a][b] - dGfg[a][b]);
    double u = 0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        u += su[a] * su[b] *
             (psim4 * (-cdda[a][b] + alpha * Rf[a][b]) - 1. / 3 * g[a][b] * (-trcdda + alpha * Rhat) +
              alpha * (K * A[a][b] - 2 * AA[a][b]) + lieA[a][b]);
    rACss = -alpha * chig * t + u;
  }
  double rACqq = -rACss;
  for (int a = 0; a < 3; ++a)
    for (int b = 0; b < 3; ++b) rACqq += chig * Ai[a][b] * (-2 * alpha * A[a][b] + lieg[a][b]);
  // G^a, A part
  double rGamA[3];
  for (int k = 0; k < 3; ++k) {
    double t = 0;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        t += -vbetaA * (su[a] * qud[k][b] * dG[a][b] - quu[k][a] * sd[b] * dG[a][b] / chig);
        t += P.shiftdriver / (chig * vbetaA) * (su[a] * qud[k][b] * db[a][b] - sd[a] * quu[k][b] * db[b][a]);
        t += qud[k][b] * beta[a] * dG[a][b];
        for (int cc = 0; cc < 3; ++cc)
          t += quu[a][b] * qud[k][cc] * ddb[a][b][cc] / chig + 4 * su[b] * sd[cc] * quu[k][a] * ddb[a][b][cc] / 3 / chig +
               qud[b][cc] * quu[k][a] * ddb[a][b][cc] / 3 / chig;
      }
    for (int a = 0; a < 3; ++a)
      t += -4 * alpha * quu[k][a] * dKhat[a] / 3 / chig - 2 * alpha * quu[k][a] * dTheta[a] / 3 / chig;
    rGamA[k] = t;
  }
  // A, sA part
  double rACsA[3];
  for (int a = 0; a < 3; ++a) {
    double t = 0, u = 0;
    for (int d = 0; d < 3; ++d) {
      for (int b = 0; b < 3; ++b)
        for (int cc = 0; cc < 3; ++cc)
          t += gi[b][cc] * qud[d][a] * cdA[b][cc][d] - 3 * qud[d][a] * gi[b][cc] * A[b][d] * dchi[cc] / (2 * chi);
      t += -2. / 3 * qud[d][a] * dK[d] + qud[d][a] * dTheta[d];
      t -= P.kappa1 * chig * qdd[d][a] * (G[d] - Gfg[d]) / 2;
      for (int b = 0; b < 3; ++b) {
        t += -qud[d][a] * su[b] * Rf[b][d] + chig * su[b] * qdd[d][a] * (dG[b][d] - dGfg[b][d]) / 2;
        u += -chig * qud[d][a] * su[b] * cdda[b][d] + alpha * su[b] * qud[d][a] * (A[b][d] * K - 2 * AA[b][d]) +
             su[b] * qud[d][a] * lieA[b][d];
      }
    }
    rACsA[a] = -alpha * chig * t + u;
  }
  // A, trace-free AB part, and the full rhs of A
  double rA[3][3];
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) {
      double t = 0;
      for (int cc = 0; cc < 3; ++cc)
        for (int d = 0; d < 3; ++d) {
          const double qp = (qud[cc][a] * qud[d][b] + qud[cc][b] * qud[d][a] - quu[cc][d] * qdd[a][b]) / 2;
          double inner = 0, sdchi = 0;
          for (int e = 0; e < 3; ++e) {
            inner += su[e] * cdA[e][cc][d] - 0.5 * su[e] * cdA[cc][d][e] - 0.5 * su[e] * cdA[d][cc][e] +
                     1 / (4 * chig) * su[e] * A[e][cc] * dchi[d] + 1 / (4 * chig) * su[e] * A[e][d] * dchi[cc];
            sdchi += su[e] * dchi[e];
          }
          inner -= 1 / (2 * chig) * A[cc][d] * sdchi;
          t += qp * (-alpha * inner - chig * cdda[cc][d] - alpha * AA[cc][d] + 2. / 3 * alpha * K * A[cc][d] +
                     lieA[cc][d]);
        }
      double v = t + sd[a] * sd[b] * rACss + qdd[a][b] / 2 * rACqq;
      for (int k = 0; k < 3; ++k) v += (qud[k][a] * sd[b] + qud[k][b] * sd[a]) * rACsA[k];
      rA[a][b] = v;
    }
  double rG[3];
  for (int a = 0; a < 3; ++a) {
    double t = su[a] * rGams;
    for (int k = 0; k < 3; ++k) t += qud[a][k] * rGamA[k];
    rG[a] = t;
  }
  for (int a = 0; a < 3; ++a)
    for (int b = a; b < 3; ++b) out[sy(a, b)] = rA[a][b];
  out[6] = rKhat;
  for (int a = 0; a < 3; ++a) out[7 + a] = rG[a];
  out[10] = rTheta;
}

__global__ void __launch_bounds__(64) cpbc_kernel(Vars cur, Vars nw, Vars pre, double c,
                                                 const FlagPoint *__restrict__ lad, int nlad,
                                                 const BoxGeo *__restrict__ box, double dx, double dy, double dz,
                                                 Cpbc P) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nlad) return;
  const FlagPoint F = lad[q];
  const BoxGeo B = box[F.box];
  const long x = F.ijk;
  const long st[3] = {1, B.m, (long)B.m * B.n};
  const double h[3] = {dx, dy, dz};
  const int idx[3] = {F.i, F.j, F.k}, mx[3] = {B.m - 1, B.n - 1, B.o - 1};
  double out[11];
  cpbc_point(cur.p, x, st, h, idx, mx, B.x0 + F.i * dx, B.y0 + F.j * dy, B.z0 + F.k * dz, P, out);
  for (int v = 0; v < 11; ++v) nw.p[7 + v][x] = c != 0.0 ? pre.p[7 + v][x] + c * out[v] : out[v];
}

}  // namespace

int nrgpu_z4_cpbc_launch(nrgpu_level *L, double *const *ucur, double *const *unew, double *const *upre, double c,
                         const nrgpu_z4_params *p, cudaStream_t st) {
  Vars cu, nw, pr;
  for (int v = 0; v < NV; ++v) {
    cu.p[v] = ucur[v];
    nw.p[v] = unew[v];
    pr.p[v] = upre[v];
  }
  const Cpbc P = {p->kappa1, p->kappa2, p->chiDivFloor, p->chipsipower, 0.0};
  // the distance-1 segment of the ladder: the inner points one inside a box face
  const int n = L->nladder[1] - L->nladder[0];
  if (n > 0)
    cpbc_kernel<<<(n + 63) / 64, 64, 0, st>>>(cu, nw, pr, c, L->d_ladder + L->nladder[0], n, L->d_box, L->dx, L->dy,
                                             L->dz, P);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}
