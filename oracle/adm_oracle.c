/* adm_oracle.c -- CPU restatement of the reference's ADM diagnostics.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/ (through oracle/oracle.py) as
 * the checker of the CUDA path; the product never links or calls it.
 *
 * Restates, FP64, point by point:
 *   bssn_to_adm_vl / z4_to_adm_vl (bssn.c:132-197, z4.c:93-124):
 *     psi = chi^(1/chipsipower), g = psi^4 g~, K_ij = psi^4 A~_ij + K g_ij/3
 *     on every point of the level
 *   adm_constraints_N (spec adm_constraints_N.m:14-143, generated
 *     adm_constraints_N.c:22-5382) with usepsi = 0 and no matter, on the
 *     points of every box whose boundary flag is 0 (forinnerpoints_ijk,
 *     bam_amr_loops_box.h:138), centred order from the distance ladder
 *     (order 2 one point from the box edge, 4 two points away, then the
 *     requested order), plus the normalised constraints (plain and
 *     term-by-term denominators)
 *   bampi_allreduce_norm2 / _normInf (reduce.c:41-131, 209-266): RMS and
 *     max |u| over the points with boundary flag 0
 * The derivative stencils are the centred ones of discretize.m:18-71
 * (first derivative, second derivative, mixed = product of two first
 * derivative stencils).  Parity against the reference binary is pinned by
 * tests/test_adm_oracle_pin.py on tests/golden/*_con.npz.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include "../include/nrgpu.h"

static const double W1[3][7] = {{0, 0, -1, 0, 1, 0, 0},
                                {0, 1, -8, 0, 8, -1, 0},
                                {-1, 9, -45, 0, 45, -9, 1}};
static const double D1[3] = {2, 12, 60};
static const double W2[3][7] = {{0, 0, 1, -2, 1, 0, 0},
                                {0, -1, 16, -30, 16, -1, 0},
                                {2, -27, 270, -490, 270, -27, 2}};
static const double D2[3] = {1, 12, 180};
/* symmetric index pairs in the order xx xy xz yy yz zz */
static const int S[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

static double fd1(const double *f, long ijk, long s, double h, int o)
{
  double a = 0;
  for (int n = -3; n <= 3; n++)
    if (W1[o][n + 3] != 0) a += W1[o][n + 3] * f[ijk + n * s];
  return a / (D1[o] * h);
}

static double fd2(const double *f, long ijk, long s, double h, int o)
{
  double a = 0;
  for (int n = -3; n <= 3; n++)
    if (W2[o][n + 3] != 0) a += W2[o][n + 3] * f[ijk + n * s];
  return a / (D2[o] * h * h);
}

static double fd11(const double *f, long ijk, long s1, long s2, double h1, double h2, int o)
{
  double a = 0;
  for (int p = -3; p <= 3; p++) {
    if (W1[o][p + 3] == 0) continue;
    for (int q = -3; q <= 3; q++)
      if (W1[o][q + 3] != 0) a += W1[o][p + 3] * W1[o][q + 3] * f[ijk + p * s1 + q * s2];
  }
  return a / (D1[o] * h1 * D1[o] * h2);
}

int oracle_to_adm(const nrgpu_level_desc *L, const double *const *u, double *const *adm, double chipsipower)
{
  long np = L->npoints;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < np; i++) {
    double psi = pow(u[6][i], 1.0 / chipsipower);
    double psi4 = pow(psi, 4.0);
    for (int n = 0; n < 6; n++) {
      adm[n][i] = psi4 * u[n][i];
      adm[6 + n][i] = psi4 * u[7 + n][i] + 1.0 / 3.0 * u[13][i] * adm[n][i];
    }
  }
  return 0;
}

/* mode: 0 ham/mom only; 1 also normalised with the plain denominators;
 * 2 also normalised with the term-by-term denominators */
static void constraint_point(const double *const *adm, long ijk, const long st[3], const double h[3], int o,
                             int mode, double *out)
{
  double g[6], K[6], dg[3][6], dK[3][6], ddg[6][6];
  for (int v = 0; v < 6; v++) {
    g[v] = adm[v][ijk];
    K[v] = adm[6 + v][ijk];
    for (int c = 0; c < 3; c++) {
      dg[c][v] = fd1(adm[v], ijk, st[c], h[c], o);
      dK[c][v] = fd1(adm[6 + v], ijk, st[c], h[c], o);
    }
    for (int a = 0; a < 3; a++)
      for (int b = a; b < 3; b++)
        ddg[S[a][b]][v] = a == b ? fd2(adm[v], ijk, st[a], h[a], o)
                                 : fd11(adm[v], ijk, st[a], st[b], h[a], h[b], o);
  }
  /* inverse metric */
  double det = g[0] * (g[3] * g[5] - g[4] * g[4]) - g[1] * (g[1] * g[5] - g[2] * g[4]) +
               g[2] * (g[1] * g[4] - g[2] * g[3]);
  double idet = 1.0 / det, gi[6];
  gi[0] = (g[3] * g[5] - g[4] * g[4]) * idet;
  gi[1] = (g[2] * g[4] - g[1] * g[5]) * idet;
  gi[2] = (g[1] * g[4] - g[2] * g[3]) * idet;
  gi[3] = (g[0] * g[5] - g[2] * g[2]) * idet;
  gi[4] = (g[1] * g[2] - g[0] * g[4]) * idet;
  gi[5] = (g[0] * g[3] - g[1] * g[1]) * idet;
#define GI(a, b) gi[S[a][b]]
#define G(a, b) g[S[a][b]]
#define KK(a, b) K[S[a][b]]
  /* Christoffel symbols, first kind gd[c][ab] and second kind gu[c][ab] */
  double gd[3][6], gu[3][6];
  for (int c = 0; c < 3; c++)
    for (int a = 0; a < 3; a++)
      for (int b = a; b < 3; b++)
        gd[c][S[a][b]] = 0.5 * (dg[a][S[b][c]] + dg[b][S[a][c]] - dg[c][S[a][b]]);
  for (int c = 0; c < 3; c++)
    for (int ab = 0; ab < 6; ab++) {
      double s = 0;
      for (int d = 0; d < 3; d++) s += GI(c, d) * gd[d][ab];
      gu[c][ab] = s;
    }
  /* Ricci tensor, its trace and the term-by-term pieces; every R[a,b] is
   * evaluated for a <= b and stands for R[b,a] too.  The spec declares the
   * pieces symmetric, which RB[a,b] = ginv[c,d] deldelg[a,c,b,d] is not; the
   * generated code (adm_constraints_N.c:4660-4700) stores, for a <= b,
   * ginv[c,d] deldelg[b,c,a,d], and so does this restatement */
  double Rt = 0, RA = 0, RB = 0, RC = 0, RD = 0;
  for (int a = 0; a < 3; a++)
    for (int b = a; b < 3; b++) {
      const double w = a == b ? 1.0 : 2.0;
      double r = 0, ra = 0, rb = 0, rc = 0, rd = 0;
      for (int c = 0; c < 3; c++)
        for (int d = 0; d < 3; d++) {
          double gcd = GI(c, d);
          double cc = 0, dd = 0;
          for (int e = 0; e < 3; e++) {
            cc += gu[e][S[a][c]] * gd[e][S[b][d]];
            dd -= gu[e][S[a][b]] * gd[e][S[c][d]];
          }
          r += gcd * (0.5 * (-ddg[S[c][d]][S[a][b]] - ddg[S[a][b]][S[c][d]] + ddg[S[a][c]][S[b][d]] +
                             ddg[S[b][c]][S[a][d]]) +
                      cc + dd);
          ra -= gcd * ddg[S[c][d]][S[a][b]];
          rb += gcd * ddg[S[b][c]][S[a][d]];
          rc += gcd * cc;
          rd += gcd * dd;
        }
      Rt += w * GI(a, b) * r;
      RA += w * GI(a, b) * ra;
      RB += w * GI(a, b) * rb;
      RC += w * GI(a, b) * rc;
      RD += w * GI(a, b) * rd;
    }
  /* extrinsic curvature terms */
  double Kud[3][3], trK = 0, KudKud = 0;
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) {
      double s = 0;
      for (int c = 0; c < 3; c++) s += GI(a, c) * KK(c, b);
      Kud[a][b] = s;
    }
  for (int a = 0; a < 3; a++) trK += Kud[a][a];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) KudKud += Kud[a][b] * Kud[b][a];
  /* covariant derivative of K; its term-by-term pieces B and C are stored
   * for b <= c and read back symmetrically.  In the generated code
   * (adm_constraints_N.c:4907-5330) the piece codelKC[a,b,c] =
   * -gamma[d,a,c] K[b,d] comes out as -gamma[d,a,b] K[c,d], the same value
   * as codelKB[a,b,c]; that is what is restated here */
  double cK[3][6], cKB[3][6], cKC[3][6], cdK[3][6];
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++)
      for (int c = b; c < 3; c++) {
        double sb = 0, sc = 0, sd = 0;
        for (int d = 0; d < 3; d++) {
          sb -= gu[d][S[a][b]] * KK(d, c);
          sc -= gu[d][S[a][b]] * KK(c, d);
          sd -= gu[d][S[a][c]] * KK(b, d);
        }
        cKB[a][S[b][c]] = sb;
        cKC[a][S[b][c]] = sc;
        cK[a][S[b][c]] = dK[a][S[b][c]] + sb + sd;
      }
  for (int a = 0; a < 3; a++)
    for (int bc = 0; bc < 6; bc++) {
      double s = 0;
      for (int d = 0; d < 3; d++) s += GI(a, d) * cK[d][bc];
      cdK[a][bc] = s;
    }
  out[0] = Rt + trK * trK - KudKud;
  double momu[3];
  for (int a = 0; a < 3; a++) {
    double s = 0;
    for (int b = 0; b < 3; b++)
      for (int c = 0; c < 3; c++) s += GI(a, b) * cdK[c][S[b][c]] - GI(b, c) * cdK[a][S[b][c]];
    momu[a] = s;
  }
  for (int a = 0; a < 3; a++) out[1 + a] = G(a, 0) * momu[0] + G(a, 1) * momu[1] + G(a, 2) * momu[2];
  if (!mode) return;
  double den;
  if (mode == 2)
    den = fabs(RA) + fabs(RB) + fabs(RC) + fabs(RD) + trK * trK + fabs(KudKud);
  else
    den = fabs(Rt) + trK * trK + fabs(KudKud);
  out[4] = den <= 0.0 ? 0.0 : out[0] / den;
  for (int a = 0; a < 3; a++) {
    if (mode == 2) {
      /* cdKd*[b] = ginv[a,c] piece[a,b,c]; codelTrK*[a] = ginv[b,c] piece[a,b,c] */
      double cA = 0, cB = 0, cC = 0, tA = 0, tB = 0, tC = 0;
      for (int p = 0; p < 3; p++)
        for (int q = 0; q < 3; q++) {
          cA += GI(p, q) * dK[p][S[a][q]];
          cB += GI(p, q) * cKB[p][S[a][q]];
          cC += GI(p, q) * cKC[p][S[a][q]];
          tA += GI(p, q) * dK[a][S[p][q]];
          tB += GI(p, q) * cKB[a][S[p][q]];
          tC += GI(p, q) * cKC[a][S[p][q]];
        }
      den = fabs(cA) + fabs(cB) + fabs(cC) + fabs(tA) + fabs(tB) + fabs(tC);
    } else {
      double s1 = 0, s2 = 0;
      for (int c = 0; c < 3; c++) s1 += cdK[c][S[a][c]];
      for (int b = 0; b < 3; b++)
        for (int c = 0; c < 3; c++) s2 += GI(b, c) * cK[a][S[b][c]];
      den = fabs(s1) + fabs(s2);
    }
    out[5 + a] = den <= 0.0 ? 0.0 : out[1 + a] / den;
  }
#undef GI
#undef G
#undef KK
}

int oracle_adm_constraints(const nrgpu_level_desc *L, const double *const *adm, double *const *con,
                           int order_centered, int mode)
{
  const double h[3] = {L->dx, L->dy, L->dz};
  if (order_centered != 2 && order_centered != 4 && order_centered != 6) return -1;
  for (int b = 0; b < L->nboxes; b++) {
    int m = L->box[b].m, n = L->box[b].n, o = L->box[b].o;
    long off = L->box[b].noffset, npb = (long)m * n * o;
    const long st[3] = {1, m, (long)m * n};
#pragma omp parallel for schedule(static)
    for (long q = 0; q < npb; q++) {
      int k = (int)(q / ((long)m * n)), j = (int)((q / m) % n), i = (int)(q % m);
      long ijk = off + q;
      if (L->boundary[ijk]) continue;
      int d = i < j ? i : j;
      d = d < k ? d : k;
      if (m - 1 - i < d) d = m - 1 - i;
      if (n - 1 - j < d) d = n - 1 - j;
      if (o - 1 - k < d) d = o - 1 - k;
      int ord = (order_centered == 2 || d == 1) ? 2 : (order_centered == 4 || d == 2) ? 4 : 6;
      double out[8];
      constraint_point(adm, ijk, st, h, ord / 2 - 1, mode, out);
      int nout = mode ? 8 : 4;
      for (int v = 0; v < nout; v++) con[v][ijk] = out[v];
    }
  }
  return 0;
}

/* RMS (norm2) and max |u| (normInf) of each variable over the flag-0 points */
int oracle_norms(const nrgpu_level_desc *L, const double *const *v, int nv, double *norm2, double *norminf)
{
  for (int q = 0; q < nv; q++) {
    double s = 0, mx = 0;
    long n = 0;
    for (long i = 0; i < L->npoints; i++) {
      if (L->boundary[i]) continue;
      double x = v[q][i];
      s += x * x;
      if (fabs(x) > mx) mx = fabs(x);
      n++;
    }
    norm2[q] = n ? sqrt(s / n) : -1;
    norminf[q] = n ? mx : -DBL_MAX;
  }
  return 0;
}
