/* nr_oracle.c -- CPU restatement of the reference's BSSN evolution hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * it (as oracle/liboracle.so through oracle/oracle.py).  Nothing in the
 * product links it, and the product never falls back to it.
 *
 * It restates, in plain C99 + OpenMP, FP64, point by point:
 *   bssn_rhs_movpunc_N   (spec bssn_rhs_movpunc_N.m:18-461; generated
 *                         bssn_rhs_movpunc_N.c:27-15516), non-shell branch
 *   set_boundary_rot_rad (radiative.c:105-300) with rot = 0
 *   set_boundary_symmetry (symmetry.c:93-140), reflections only
 *   bssn_algcon          (bssn_algcon.c:25-230)
 *   evolve_rk_rk4        (rk.c:220-257) with vladd/vladdto (variables.c:650,721)
 * Finite-difference weights follow discretize.m:18-50 (centred),
 * discretize.m:44-50 + :132-139 (Kreiss-Oliger) and the lopsided advection
 * tables with their edge shifting (bam_amr_advection.h:28-192).
 * Its parity against the reference binary (oracle/_ref/bam) is pinned by
 * tests/test_oracle_pin.py on golden dumps in tests/golden/.
 *
 * Compile as C (oracle) or, with -DORACLE_COUNT_FLOPS, as C++ with a
 * counting scalar type to obtain the algorithmic FLOPs per point.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "../include/nrgpu.h"

#ifdef ORACLE_COUNT_FLOPS
#include "flopcount.h"
typedef fcdouble real;
#define RLOG(x) fc_log(x)
#define REXP(x) fc_exp(x)
#define RPOW(x, y) fc_pow(x, y)
#define RVAL(x) fc_val(x)
#define OMP_FOR
#define GV(x) ((real)(x))
#else
typedef double real;
#define RLOG(x) log(x)
#define REXP(x) exp(x)
#define RPOW(x, y) pow(x, y)
#define RVAL(x) (x)
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#define GV(x) (x)
#endif

enum { G11, G12, G13, G22, G23, G33, CHI, A11, A12, A13, A22, A23, A33, KK, GA1, GA2, GA3,
       ALPHA, BETA1, BETA2, BETA3, BB1, BB2, BB3, NV = 24 };
/* symmetric index (a,b) -> 0..5 in the order xx xy xz yy yz zz */
static const int SY[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};

/* ---- finite-difference weights (numerator tables) ----------------------- */
/* centred first derivative weights on offsets -h..h, divided by (den*dx) */
static const double C1W2[3] = {-1, 0, 1};                      /* /2  */
static const double C1W4[5] = {1, -8, 0, 8, -1};               /* /12 */
static const double C1W6[7] = {-1, 9, -45, 0, 45, -9, 1};      /* /60 */
/* centred second derivative, divided by (den*dx^2) */
static const double C2W2[3] = {1, -2, 1};                      /* /1   */
static const double C2W4[5] = {-1, 16, -30, 16, -1};           /* /12  */
static const double C2W6[7] = {2, -27, 270, -490, 270, -27, 2};/* /180 */
/* lopsided advection rows: row r = stencil shifted by r (see adv_dir) */
static const double ADV2[3][3] = {{3, -4, 1}, {1, 0, -1}, {-1, 4, -3}};         /* /2 */
static const double ADV4[5][5] = {{25, -48, 36, -16, 3}, {3, 10, -18, 6, -1},
                                  {-1, 8, 0, -8, 1}, {1, -6, 18, -10, -3},
                                  {-3, 16, -36, 48, -25}};                     /* /12 */
static const double ADV6[7][7] = {{147, -360, 450, -400, 225, -72, 10},
                                  {10, 77, -150, 100, -50, 15, -2},
                                  {-2, 24, 35, -80, 30, -8, 1},
                                  {1, -9, 45, 0, -45, 9, -1},
                                  {-1, 8, -30, 80, -35, -24, 2},
                                  {2, -15, 50, -100, 150, -77, -10},
                                  {-10, 72, -225, 400, -450, 360, -147}};     /* /60 */
/* Kreiss-Oliger: undivided 4th / 6th differences */
static const double KO4[5] = {1, -4, 6, -4, 1};
static const double KO6[7] = {1, -6, 15, -20, 15, -6, 1};

typedef struct {
  const double *const *u;  /* 24 fields */
  long ijk;
  long s[3];               /* strides in x, y, z */
  double h[3];
} pt_t;

static real d1(const double *f, long ijk, long s, double h, int ord)
{
  int r = ord / 2, n;
  const double *w = ord == 2 ? C1W2 : ord == 4 ? C1W4 : C1W6;
  double den = ord == 2 ? 2 : ord == 4 ? 12 : 60;
  real acc = 0;
  for (n = -r; n <= r; n++)
    if (w[n + r] != 0) acc += w[n + r] * GV(f[ijk + n * s]);
  return acc / (den * h);
}

static real d2(const double *f, long ijk, long s, double h, int ord)
{
  int r = ord / 2, n;
  const double *w = ord == 2 ? C2W2 : ord == 4 ? C2W4 : C2W6;
  double den = ord == 2 ? 1 : ord == 4 ? 12 : 180;
  real acc = 0;
  for (n = -r; n <= r; n++) acc += w[n + r] * GV(f[ijk + n * s]);
  return acc / (den * h * h);
}

/* mixed second derivative = product of two first-derivative stencils
 * (discretize.m:68-71, findif2) */
static real d11(const double *f, long ijk, long s1, long s2, double h1, double h2, int ord)
{
  int r = ord / 2, a, b;
  const double *w = ord == 2 ? C1W2 : ord == 4 ? C1W4 : C1W6;
  double den = ord == 2 ? 2 : ord == 4 ? 12 : 60;
  real acc = 0;
  for (a = -r; a <= r; a++) {
    if (w[a + r] == 0) continue;
    for (b = -r; b <= r; b++) {
      if (w[b + r] == 0) continue;
      acc += (w[a + r] * w[b + r]) * GV(f[ijk + a * s1 + b * s2]);
    }
  }
  return acc / (den * h1 * den * h2);
}

/* advection tap set of one direction (bam_amr_advection.h:72-192):
 * index i in [0, imax], weight wx = beta/dx, order q, lopsidedness lop. */
typedef struct { int nt; long off[7]; real c[7]; } adv_t;
static void adv_dir(adv_t *a, int i, int imax, real wx, int q, int lop, long s)
{
  int rst, offset, n;
  double wsign;
  const double *row;
  double den;
  if (q == 2) lop = 0;
  rst = q - lop;
  if (wx < 0) { wsign = -1; offset = (i >= rst) ? 0 : rst - i; }
  else if (wx > 0) { wsign = 1; offset = (imax - i >= rst) ? 0 : rst - (imax - i); }
  else { wsign = 0; offset = 0; }
  offset += lop;
  row = q == 2 ? ADV2[offset] : q == 4 ? ADV4[offset] : ADV6[offset];
  den = q == 2 ? 2 : q == 4 ? 12 : 60;
  a->nt = q + 1;
  for (n = 0; n <= q; n++) {
    a->off[n] = (long)(wsign * (n - offset)) * s;
    a->c[n] = -wsign * wx * (row[n] / den);
  }
}

static real adv_apply(const adv_t a[3], const double *f, long ijk)
{
  real acc = 0;
  int d, n;
  for (d = 0; d < 3; d++)
    for (n = 0; n < a[d].nt; n++) acc += a[d].c[n] * GV(f[ijk + a[d].off[n]]);
  return acc;
}

static real ko(const double *f, long ijk, const long s[3], const double h[3], int ord)
{
  int r = ord / 2, d, n;
  const double *w = ord == 4 ? KO4 : KO6;
  real acc = 0;
  for (d = 0; d < 3; d++) {
    real t = 0;
    for (n = -r; n <= r; n++) t += w[n + r] * GV(f[ijk + n * s[d]]);
    acc += t / h[d];
  }
  /* dissipation4 carries a minus sign, dissipation6 a plus (discretize.m:132-137) */
  return ord == 4 ? -acc : acc;
}

static int ladder(int order, int d)
{
  if (order == 2 || d == 1) return 2;
  if (order == 4 || d == 2) return 4;
  if (order == 6 || d == 3) return 6;
  return 0;
}

/* one inner point of bssn_rhs_movpunc_N; writes the 24 rhs values to r */
static int bssn_point(const double *const *u, long ijk, int i, int j, int k, int imax, int jmax,
                      int kmax, long di, long dj, long dk, const double h[3],
                      const nrgpu_bssn_params *p, real r[NV])
{
  const long s[3] = {di, dj, dk};
  int a, b, c, d, e, ord, aord;
  int dist = i;
  if (j < dist) dist = j;
  if (k < dist) dist = k;
  if (imax - i < dist) dist = imax - i;
  if (jmax - j < dist) dist = jmax - j;
  if (kmax - k < dist) dist = kmax - k;
  ord = ladder(p->order_centered, dist);
  aord = ladder(p->order_advection, dist);
  if (!ord || !aord) return -1;

  real g[6], A[6], Gv[3], beta[3], B[3];
  real alpha = u[ALPHA][ijk], chi = u[CHI][ijk], K = u[KK][ijk];
  for (a = 0; a < 6; a++) { g[a] = u[G11 + a][ijk]; A[a] = u[A11 + a][ijk]; }
  for (a = 0; a < 3; a++) {
    Gv[a] = u[GA1 + a][ijk]; beta[a] = u[BETA1 + a][ijk]; B[a] = u[BB1 + a][ijk];
  }

  /* centred derivatives */
  real da[3], dda[6], db[3][3], ddb[6][3], delg[3][6], deldelg[6][6], delG[3][3], dK[3],
      dA[3][6], dchi[3], ddchi[6];
  for (a = 0; a < 3; a++) {
    da[a] = d1(u[ALPHA], ijk, s[a], h[a], ord);
    dK[a] = d1(u[KK], ijk, s[a], h[a], ord);
    dchi[a] = d1(u[CHI], ijk, s[a], h[a], ord);
    for (c = 0; c < 3; c++) {
      db[a][c] = d1(u[BETA1 + c], ijk, s[a], h[a], ord);
      delG[a][c] = d1(u[GA1 + c], ijk, s[a], h[a], ord);
    }
    for (c = 0; c < 6; c++) {
      delg[a][c] = d1(u[G11 + c], ijk, s[a], h[a], ord);
      dA[a][c] = d1(u[A11 + c], ijk, s[a], h[a], ord);
    }
  }
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      int ab = SY[a][b];
      if (a == b) {
        dda[ab] = d2(u[ALPHA], ijk, s[a], h[a], ord);
        ddchi[ab] = d2(u[CHI], ijk, s[a], h[a], ord);
        for (c = 0; c < 3; c++) ddb[ab][c] = d2(u[BETA1 + c], ijk, s[a], h[a], ord);
        for (c = 0; c < 6; c++) deldelg[ab][c] = d2(u[G11 + c], ijk, s[a], h[a], ord);
      } else {
        dda[ab] = d11(u[ALPHA], ijk, s[a], s[b], h[a], h[b], ord);
        ddchi[ab] = d11(u[CHI], ijk, s[a], s[b], h[a], h[b], ord);
        for (c = 0; c < 3; c++) ddb[ab][c] = d11(u[BETA1 + c], ijk, s[a], s[b], h[a], h[b], ord);
        for (c = 0; c < 6; c++)
          deldelg[ab][c] = d11(u[G11 + c], ijk, s[a], s[b], h[a], h[b], ord);
      }
    }

  /* advection, weights w = beta/dx (bssn_rhs_movpunc_N.m:126) */
  adv_t av[3];
  {
    const int idx[3] = {i, j, k}, mx[3] = {imax, jmax, kmax};
    const int lop = aord == 6 ? p->advection_lopsided6 : p->advection_lopsided;
    for (a = 0; a < 3; a++) adv_dir(&av[a], idx[a], mx[a], beta[a] / h[a], aord, lop, s[a]);
  }
  real lieg[6], lieA[6], lieK, liechi, liealpha, advG[3], advbeta[3], advB[3];
  for (a = 0; a < 6; a++) {
    lieg[a] = adv_apply(av, u[G11 + a], ijk);
    lieA[a] = adv_apply(av, u[A11 + a], ijk);
  }
  lieK = adv_apply(av, u[KK], ijk);
  liechi = adv_apply(av, u[CHI], ijk);
  liealpha = adv_apply(av, u[ALPHA], ijk);
  for (a = 0; a < 3; a++) {
    advG[a] = adv_apply(av, u[GA1 + a], ijk);
    advbeta[a] = adv_apply(av, u[BETA1 + a], ijk);
    advB[a] = adv_apply(av, u[BB1 + a], ijk);
  }

  /* inverse conformal metric */
  real detg = g[0] * g[3] * g[5] + 2 * g[1] * g[2] * g[4] - g[0] * g[4] * g[4] - g[3] * g[2] * g[2] -
              g[5] * g[1] * g[1];
  real detginv = 1 / detg;
  real ginv[6];
  ginv[0] = detginv * (g[3] * g[5] - g[4] * g[4]);
  ginv[1] = detginv * (g[2] * g[4] - g[1] * g[5]);
  ginv[2] = detginv * (g[1] * g[4] - g[2] * g[3]);
  ginv[3] = detginv * (g[0] * g[5] - g[2] * g[2]);
  ginv[4] = detginv * (g[1] * g[2] - g[0] * g[4]);
  ginv[5] = detginv * (g[0] * g[3] - g[1] * g[1]);
#define GI(x, y) ginv[SY[x][y]]
#define GG(x, y) g[SY[x][y]]
#define AAi(x, y) A[SY[x][y]]

  /* connection: gammado[c][ab] = 1/2 (d_a g_bc + d_b g_ac - d_c g_ab) */
  real gammado[3][6], gamma[3][6], Gfromg[3];
  for (c = 0; c < 3; c++)
    for (a = 0; a < 3; a++)
      for (b = a; b < 3; b++)
        gammado[c][SY[a][b]] = 0.5 * (delg[a][SY[b][c]] + delg[b][SY[a][c]] - delg[c][SY[a][b]]);
  for (c = 0; c < 3; c++)
    for (a = 0; a < 6; a++) {
      real t = 0;
      for (d = 0; d < 3; d++) t += GI(c, d) * gammado[d][a];
      gamma[c][a] = t;
    }
  for (a = 0; a < 3; a++) {
    real t = 0;
    for (b = 0; b < 3; b++)
      for (c = 0; c < 3; c++) t += GI(b, c) * gamma[a][SY[b][c]];
    Gfromg[a] = t;
  }
#define GAM(x, y, z) gamma[x][SY[y][z]]
#define GDO(x, y, z) gammado[x][SY[y][z]]

  /* Ricci tensor of the conformal metric */
  real Rab[6];
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      real t = 0;
      for (c = 0; c < 3; c++)
        for (d = 0; d < 3; d++) {
          real q = -0.5 * deldelg[SY[c][d]][SY[a][b]];
          for (e = 0; e < 3; e++)
            q += GAM(e, c, a) * GDO(b, e, d) + GAM(e, c, b) * GDO(a, e, d) +
                 GAM(e, a, d) * GDO(e, c, b);
          t += GI(c, d) * q;
        }
      real t2 = 0;
      for (c = 0; c < 3; c++)
        t2 += GG(c, a) * delG[b][c] + GG(c, b) * delG[a][c] +
              Gfromg[c] * (GDO(a, b, c) + GDO(b, a, c));
      Rab[SY[a][b]] = t + 0.5 * t2;
    }

  /* conformal factor */
  real chiguarded = chi;
  if (chiguarded < p->chiDivFloor) chiguarded = p->chiDivFloor;
  real oochipsipower = 1 / p->chipsipower;
  real f = oochipsipower * RLOG(chiguarded);
  real df[3], ddf[6], cddf[6];
  for (a = 0; a < 3; a++) df[a] = oochipsipower * dchi[a] / chiguarded;
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++)
      ddf[SY[a][b]] = oochipsipower * ddchi[SY[a][b]] / chiguarded - p->chipsipower * df[a] * df[b];
  real psim2 = REXP(-2 * f), psim4 = REXP(-4 * f);
  (void)psim2;
  real trcddf = 0, dfdf = 0, dfda = 0;
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      real t = ddf[SY[a][b]];
      for (c = 0; c < 3; c++) t -= GAM(c, a, b) * df[c];
      cddf[SY[a][b]] = t;
    }
  for (a = 0; a < 3; a++)
    for (b = 0; b < 3; b++) {
      trcddf += GI(a, b) * cddf[SY[a][b]];
      dfdf += GI(a, b) * df[a] * df[b];
      dfda += GI(a, b) * df[a] * da[b];
    }
  real Rphi[6], cdda[6];
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      int ab = SY[a][b];
      Rphi[ab] = 4 * df[a] * df[b] - 2 * cddf[ab] - 2 * g[ab] * trcddf - 4 * g[ab] * dfdf;
      real t = dda[ab];
      for (c = 0; c < 3; c++) t -= GAM(c, a, b) * da[c];
      cdda[ab] = t - 2 * (df[a] * da[b] + df[b] * da[a] - g[ab] * dfda);
    }
  real trcdda = 0;
  for (a = 0; a < 3; a++)
    for (b = 0; b < 3; b++) trcdda += GI(a, b) * cdda[SY[a][b]];
  trcdda = psim4 * trcdda;

  /* K zero option */
  K = K * p->forceKzerofactor;
  for (a = 0; a < 3; a++) dK[a] = dK[a] * p->forceKzerofactor;

  /* trace-free extrinsic curvature */
  real AAab[6], Ainv[6], AAs = 0, divAinv[3];
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      real t = 0, t2 = 0;
      for (c = 0; c < 3; c++)
        for (d = 0; d < 3; d++) {
          t += GI(c, d) * AAi(a, c) * AAi(d, b);
          t2 += GI(a, c) * GI(b, d) * AAi(c, d);
        }
      AAab[SY[a][b]] = t;
      Ainv[SY[a][b]] = t2;
    }
  for (a = 0; a < 3; a++)
    for (b = 0; b < 3; b++) AAs += GI(a, b) * AAab[SY[a][b]];
  for (a = 0; a < 3; a++) {
    real t = 0;
    for (b = 0; b < 3; b++) t += (2.0 / 3.0) * GI(a, b) * dK[b] - 6 * Ainv[SY[a][b]] * df[b];
    for (b = 0; b < 3; b++)
      for (c = 0; c < 3; c++) t -= GAM(a, b, c) * Ainv[SY[b][c]];
    divAinv[a] = t;
  }
  real Rsc = AAs - 2 * K * K / 3;

  /* shift terms */
  real divbeta = db[0][0] + db[1][1] + db[2][2];
  real totdivbeta = (2.0 / 3.0) * divbeta;
  real ootddivbeta[3];
  for (a = 0; a < 3; a++)
    ootddivbeta[a] = (1.0 / 3.0) * (ddb[SY[a][0]][0] + ddb[SY[a][1]][1] + ddb[SY[a][2]][2]);
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      int ab = SY[a][b];
      real tg = lieg[ab] - g[ab] * totdivbeta, tA = lieA[ab] - A[ab] * totdivbeta;
      for (c = 0; c < 3; c++) {
        tg += db[a][c] * GG(b, c) + db[b][c] * GG(a, c);
        tA += db[a][c] * AAi(b, c) + db[b][c] * AAi(a, c);
      }
      lieg[ab] = tg;
      lieA[ab] = tA;
    }
  liechi = liechi + (p->chipsipower / 6) * chiguarded * divbeta;
  real pseudolieG[3];
  for (a = 0; a < 3; a++) {
    real t = 0;
    for (b = 0; b < 3; b++)
      for (c = 0; c < 3; c++) t += GI(b, c) * ddb[SY[b][c]][a];
    for (b = 0; b < 3; b++) t += GI(a, b) * ootddivbeta[b] - Gfromg[b] * db[b][a];
    pseudolieG[a] = t + Gfromg[a] * totdivbeta + advG[a];
  }

  /* right-hand sides */
  real rg[6], rA[6], rG[3], rK, rchi;
  for (a = 0; a < 6; a++) {
    rg[a] = -2 * alpha * A[a] + lieg[a];
    rA[a] = psim4 * (-cdda[a] + alpha * (Rab[a] + Rphi[a])) -
            (1.0 / 3.0) * g[a] * (-trcdda + alpha * Rsc) + alpha * (K * A[a] - 2 * AAab[a]) + lieA[a];
  }
  for (a = 0; a < 3; a++) {
    real t = 0;
    for (b = 0; b < 3; b++) t += Ainv[SY[a][b]] * da[b];
    rG[a] = -2 * t - 2 * alpha * divAinv[a] + pseudolieG[a];
  }
  rK = -trcdda + alpha * (AAs + K * K / 3) + lieK;
  rchi = (-p->chipsipower / 6) * chiguarded * alpha * K + liechi;

  /* gauge */
  real falpha = p->oploglapse * p->lapseharmonicf + p->oploglapse2 * 8.0 / (3 * (3 - alpha)) +
                p->harmoniclapse * alpha;
  real ralpha = p->oplogwithshift * liealpha - falpha * alpha * K;
  real betaF = p->shiftgammacoeff * RPOW(alpha, p->shiftalphapower);
  real alphaG = RPOW(alpha, p->shiftGalphapower);
  real rbeta[3], rB[3];
  for (a = 0; a < 3; a++) {
    rbeta[a] = (p->gamma2factor + p->gamma0factor * betaF) * p->withB * B[a] +
               p->withShiftadv * advbeta[a] +
               (1 - p->withB) * (p->shiftgammacoeff * alphaG * Gv[a] - p->shiftdriver * beta[a]);
    rB[a] = p->withB * ((p->gamma0factor + p->gamma2factor * betaF) * (rG[a] - p->withGadv * advG[a]) -
                        p->shiftdriver * B[a] + p->withBadv * advB[a]);
  }

  /* Kreiss-Oliger dissipation, only where the full stencil fits */
  if ((p->order_dissipation == 4 && dist >= 2) || (p->order_dissipation == 6 && dist >= 3)) {
    const int od = p->order_dissipation;
    const double df_ = p->dissfactor;
    for (a = 0; a < 6; a++) {
      rg[a] += df_ * ko(u[G11 + a], ijk, s, h, od);
      rA[a] += df_ * ko(u[A11 + a], ijk, s, h, od);
    }
    for (a = 0; a < 3; a++) rG[a] += df_ * ko(u[GA1 + a], ijk, s, h, od);
    rK += df_ * ko(u[KK], ijk, s, h, od);
    rchi += df_ * ko(u[CHI], ijk, s, h, od);
  }

  for (a = 0; a < 6; a++) { r[G11 + a] = rg[a]; r[A11 + a] = rA[a]; }
  r[CHI] = rchi;
  r[KK] = p->forceKzerofactor * rK;
  for (a = 0; a < 3; a++) {
    r[GA1 + a] = rG[a];
    r[BETA1 + a] = rbeta[a];
    r[BB1 + a] = rB[a];
  }
  r[ALPHA] = ralpha;
  return 0;
#undef GI
#undef GG
#undef AAi
#undef GAM
#undef GDO
}

/* linear update with the reference's algebraic fixes for c != 0
 * (bssn_rhs_movpunc_N.m:432-450) */
static void addlinear(double *const *unew, double *const *upre, long ijk, double c,
                      const real r[NV], const nrgpu_bssn_params *p)
{
  double n[NV];
  int v;
  for (v = 0; v < NV; v++) n[v] = upre[v][ijk] + c * RVAL(r[v]);
  n[KK] = p->forceKzerofactor * (upre[KK][ijk] + c * RVAL(r[KK]));
  double *g = n + G11, *A = n + A11;
  double detg = g[0] * g[3] * g[5] + 2 * g[1] * g[2] * g[4] - g[0] * g[4] * g[4] -
                g[3] * g[2] * g[2] - g[5] * g[1] * g[1];
  double detnginv = 1 / detg;
  if (p->subtractA) {
    double gi[6];
    gi[0] = (g[3] * g[5] - g[4] * g[4]);
    gi[1] = (g[2] * g[4] - g[1] * g[5]);
    gi[2] = (g[1] * g[4] - g[2] * g[3]);
    gi[3] = (g[0] * g[5] - g[2] * g[2]);
    gi[4] = (g[1] * g[2] - g[0] * g[4]);
    gi[5] = (g[0] * g[3] - g[1] * g[1]);
    double trA = detnginv * (gi[0] * A[0] + gi[3] * A[3] + gi[5] * A[5] +
                             2 * (gi[1] * A[1] + gi[2] * A[2] + gi[4] * A[4]));
    double aux = -trA / 3;
    for (v = 0; v < 6; v++) A[v] += aux * g[v];
  }
  if (p->normalizedetg) {
    double aux = pow(detnginv, 1.0 / 3.0);
    for (v = 0; v < 6; v++) g[v] *= aux;
  }
  for (v = 0; v < NV; v++) unew[v][ijk] = n[v];
}

static int box_of(const nrgpu_level_desc *L, int b, int *m, int *n, int *o)
{
  *m = L->box[b].m; *n = L->box[b].n; *o = L->box[b].o;
  return L->box[b].noffset;
}

/* bssn_rhs_movpunc_N over the inner points of a level */
int oracle_bssn_rhs(const nrgpu_level_desc *L, double *const *unew, double *const *upre, double c,
                    double *const *ucur, const nrgpu_bssn_params *p)
{
  int b, err = 0;
  const double h[3] = {L->dx, L->dy, L->dz};
  for (b = 0; b < L->nboxes; b++) {
    int m, n, o;
    long off = box_of(L, b, &m, &n, &o);
    long np = (long)m * n * o, q;
    OMP_FOR
    for (q = 0; q < np; q++) {
      int k = (int)(q / ((long)m * n)), j = (int)((q / m) % n), i = (int)(q % m);
      long ijk = off + q;
      real r[NV];
      int v;
      if (L->boundary[ijk]) continue;
      if (bssn_point((const double *const *)ucur, ijk, i, j, k, m - 1, n - 1, o - 1, 1, m,
                     (long)m * n, h, p, r)) {
        err = -1;
        continue;
      }
      if (c == 0.0)
        for (v = 0; v < NV; v++) unew[v][ijk] = RVAL(r[v]);
      else
        addlinear(unew, upre, ijk, c, r, p);
    }
  }
  return err;
}

/* computedel of radiative.c:19-42, neighbours clipped to the box as in
 * set_nbinds_check_13 (bam_amr_loops_box.h:331-395) */
static double computedel(const double *var, double vx, long ccc, long mcc, long Mcc, long pcc,
                         long Pcc)
{
#define CEN(p_, m_) (var[p_] - var[m_])
#define RGT(c_, p_, P_) (4 * var[p_] - var[P_] - 3 * var[c_])
#define LFT(c_, m_, M_) (3 * var[c_] + var[M_] - 4 * var[m_])
  if (vx > 0) {
    if (Mcc != ccc) return LFT(ccc, mcc, Mcc);
    if (mcc != ccc) return CEN(pcc, mcc);
    return RGT(ccc, pcc, Pcc);
  } else if (vx < 0) {
    if (Pcc != ccc) return RGT(ccc, pcc, Pcc);
    if (mcc != ccc) return CEN(pcc, mcc);
    return LFT(ccc, mcc, Mcc);
  } else {
    if (pcc != ccc && mcc != ccc) return CEN(pcc, mcc);
    if (mcc == ccc) return RGT(ccc, pcc, Pcc);
    return LFT(ccc, mcc, Mcc);
  }
#undef CEN
#undef RGT
#undef LFT
}

/* VarSymmetry (variables.c) of the evolved variables, from their AddVar
 * index strings: g~ and A~ "ij+ji" (xx xy xz yy yz zz), Gamma~, beta and B
 * "I", the rest scalars; the sign of variable v under the reflection of
 * axis dir.  Z4c lists put Theta before alpha. */
static double var_parity(int nv, int v, int dir)
{
  static const int ij[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  int beta = nv == NV ? 18 : 19, B = nv == NV ? 21 : 22;
  if (v < 6) return (ij[v][0] == dir ? -1.0 : 1.0) * (ij[v][1] == dir ? -1.0 : 1.0);
  if (v >= 7 && v < 13) return (ij[v - 7][0] == dir ? -1.0 : 1.0) * (ij[v - 7][1] == dir ? -1.0 : 1.0);
  if (v >= 14 && v < 17) return v - 14 == dir ? -1.0 : 1.0;
  if (v >= beta && v < beta + 3) return v - beta == dir ? -1.0 : 1.0;
  if (v >= B && v < B + 3) return v - B == dir ? -1.0 : 1.0;
  return 1.0;
}

/* set_boundary_symmetry (symmetry.c:93-140) for the reflections of the
 * level's mask, x then y then z, each by set_boundary_reflection_one
 * (symmetry.c:28-82): on every box whose lower bound is negative, the
 * nneg = (int)(1 - lo/h) planes below zero take sign * the value of plane
 * 2 nneg - 1 - n */
static void symmetry_nv(const nrgpu_level_desc *L, int nv, double *const *u)
{
  for (int dir = 0; dir < 3; dir++) {
    if (!(L->symmetry >> dir & 1)) continue;
    double h = dir == 0 ? L->dx : (dir == 1 ? L->dy : L->dz);
    for (int b = 0; b < L->nboxes; b++) {
      const nrgpu_box *bx = &L->box[b];
      double lo = dir == 0 ? bx->x0 : (dir == 1 ? bx->y0 : bx->z0);
      int nneg = (int)(1 - lo / h), nmax = 2 * nneg - 1;
      int n3[3] = {bx->m, bx->n, bx->o};
      long st[3] = {1, bx->m, (long)bx->m * bx->n};
      int a1 = dir == 0 ? 1 : 0, a2 = dir == 2 ? 1 : 2;
      if (nneg <= 0) continue;
      for (int v = 0; v < nv; v++) {
        double sg = var_parity(nv, v, dir);
        for (int p2 = 0; p2 < n3[a2]; p2++)
          for (int p1 = 0; p1 < n3[a1]; p1++) {
            long base = bx->noffset + p1 * st[a1] + p2 * st[a2];
            for (int n = 0; n < nneg; n++) u[v][base + n * st[dir]] = sg * u[v][base + (nmax - n) * st[dir]];
          }
      }
    }
  }
}

/* set_boundary_rot_rad (radiative.c:105) without rotation, nv variables,
 * then set_boundary_symmetry on unew (boundary.c:221) */
static int boundary_rad_nv(const nrgpu_level_desc *L, int nv, double *const *unew, double *const *upre,
                           double c, double *const *ucur, const double *bvar0, const double *bspeed);
static int boundary_nv(const nrgpu_level_desc *L, int nv, double *const *unew, double *const *upre,
                       double c, double *const *ucur, const double *bvar0, const double *bspeed)
{
  int e = boundary_rad_nv(L, nv, unew, upre, c, ucur, bvar0, bspeed);
  symmetry_nv(L, nv, unew);
  return e;
}

static int boundary_rad_nv(const nrgpu_level_desc *L, int nv, double *const *unew, double *const *upre,
                           double c, double *const *ucur, const double *bvar0, const double *bspeed)
{
  int b;
  const double oo2d[3] = {1 / (2 * L->dx), 1 / (2 * L->dy), 1 / (2 * L->dz)};
  for (b = 0; b < L->nboxes; b++) {
    int m, n, o;
    long off = box_of(L, b, &m, &n, &o);
    long np = (long)m * n * o, q;
    OMP_FOR
    for (q = 0; q < np; q++) {
      int k = (int)(q / ((long)m * n)), j = (int)((q / m) % n), i = (int)(q % m);
      long ijk = off + q, di = 1, dj = m, dk = (long)m * n;
      int v;
      if (L->boundary[ijk] != NRGPU_PHYBOUND) continue;
      long ccc = ijk;
      long mcc = i > 0 ? ijk - di : ijk, pcc = i + 1 < m ? ijk + di : ijk;
      long cmc = j > 0 ? ijk - dj : ijk, cpc = j + 1 < n ? ijk + dj : ijk;
      long ccm = k > 0 ? ijk - dk : ijk, ccp = k + 1 < o ? ijk + dk : ijk;
      long Mcc = i > 1 ? mcc - di : ccc, Pcc = i + 2 < m ? pcc + di : ccc;
      long cMc = j > 1 ? cmc - dj : ccc, cPc = j + 2 < n ? cpc + dj : ccc;
      long ccM = k > 1 ? ccm - dk : ccc, ccP = k + 2 < o ? ccp + dk : ccc;
      double x = L->box[b].x0 + i * L->dx, y = L->box[b].y0 + j * L->dy,
             z = L->box[b].z0 + k * L->dz;
      double rr = sqrt(x * x + y * y + z * z);
      for (v = 0; v < nv; v++) {
        const double *var = ucur[v];
        double vv = bspeed[v], var0 = bvar0[v];
        double Wx = vv * x / rr, Wy = vv * y / rr, Wz = vv * z / rr;
        double delx = computedel(var, Wx, ccc, mcc, Mcc, pcc, Pcc);
        double dely = computedel(var, Wy, ccc, cmc, cMc, cpc, cPc);
        double delz = computedel(var, Wz, ccc, ccm, ccM, ccp, ccP);
        double rhs = -vv * (var[ccc] - var0) / rr;
        rhs += -(Wx * delx * oo2d[0] + Wy * dely * oo2d[1] + Wz * delz * oo2d[2]);
        unew[v][ijk] = (c != 0.0) ? upre[v][ijk] + c * rhs : rhs;
      }
    }
  }
  return 0;
}

int oracle_bssn_boundary(const nrgpu_level_desc *L, double *const *unew, double *const *upre,
                         double c, double *const *ucur, const nrgpu_bssn_params *p)
{
  return boundary_nv(L, NV, unew, upre, c, ucur, p->bc_var0, p->bc_speed);
}

/* bssn_algcon (bssn_algcon.c:25) on all points */
int oracle_bssn_algcon(const nrgpu_level_desc *L, double *const *u, const nrgpu_bssn_params *p)
{
  long q, np = L->npoints;
  OMP_FOR
  for (q = 0; q < np; q++) {
    double g[6], A[6];
    int v;
    for (v = 0; v < 6; v++) { g[v] = u[G11 + v][q]; A[v] = u[A11 + v][q]; }
    double detg = g[0] * g[3] * g[5] + 2 * g[1] * g[2] * g[4] - g[0] * g[4] * g[4] -
                  g[3] * g[2] * g[2] - g[5] * g[1] * g[1];
    if (p->normalizedetg) {
      double eps = detg - 1, aux;
      if (fabs(eps) < 1e-12) aux = 1 - eps / 3;
      else aux = pow(detg, -1.0 / 3.0);
      for (v = 0; v < 6; v++) g[v] *= aux;
      detg = g[0] * g[3] * g[5] + 2 * g[1] * g[2] * g[4] - g[0] * g[4] * g[4] -
             g[3] * g[2] * g[2] - g[5] * g[1] * g[1];
    }
    if (p->subtractA) {
      double detginv = 1 / detg;
      double gi[6];
      gi[0] = (g[3] * g[5] - g[4] * g[4]);
      gi[1] = (g[2] * g[4] - g[1] * g[5]);
      gi[2] = (g[1] * g[4] - g[2] * g[3]);
      gi[3] = (g[0] * g[5] - g[2] * g[2]);
      gi[4] = (g[1] * g[2] - g[0] * g[4]);
      gi[5] = (g[0] * g[3] - g[1] * g[1]);
      double trA = detginv * (gi[0] * A[0] + gi[3] * A[3] + gi[5] * A[5] +
                              2 * (gi[1] * A[1] + gi[2] * A[2] + gi[4] * A[4]));
      double aux = -trA / 3;
      for (v = 0; v < 6; v++) A[v] += aux * g[v];
    }
    for (v = 0; v < 6; v++) { u[G11 + v][q] = g[v]; u[A11 + v][q] = A[v]; }
  }
  return 0;
}

/* r = a x + b y over all points (vladd, variables.c:650) */
static void vladd_nv(long np, int nv, double *const *r, double a, double *const *x, double b,
                     double *const *y)
{
  int v;
  for (v = 0; v < nv; v++) {
    long q;
    OMP_FOR
    for (q = 0; q < np; q++) r[v][q] = a * x[v][q] + b * y[v][q];
  }
}

static void vladd(long np, double *const *r, double a, double *const *x, double b,
                  double *const *y)
{
  vladd_nv(np, NV, r, a, x, b, y);
}

static int rhs_stage(const nrgpu_level_desc *L, double *const *r, double *const *upre,
                     double *const *ucur, const nrgpu_bssn_params *p)
{
  int e = oracle_bssn_rhs(L, r, upre, 0.0, ucur, p);
  oracle_bssn_boundary(L, r, upre, 0.0, ucur, p);
  return e;
}

/* evolve_rk_rk4 (rk.c:220-257) + algcon, u updated in place */
/* the four RK4 stages of evolve_rk_rk4 (rk.c:220-257) without the
 * algebraic constraints that bssn_algcon_wrapper applies afterwards */
int oracle_bssn_rk4_stages(const nrgpu_level_desc *L, double *const *u, double dt,
                           const nrgpu_bssn_params *p)
{
  long np = L->npoints;
  double *buf = (double *)malloc(sizeof(double) * 3 * NV * np);
  double *P[NV], *R[NV], *V[NV];
  int v, e = 0;
  if (!buf) return -4;
  for (v = 0; v < NV; v++) {
    P[v] = buf + (0 * NV + v) * np;
    R[v] = buf + (1 * NV + v) * np;
    V[v] = buf + (2 * NV + v) * np;
    memcpy(P[v], u[v], sizeof(double) * np);
    /* the reference leaves boundary-flagged non-physical points of the
     * rhs untouched; start the rhs from zero */
    memset(R[v], 0, sizeof(double) * np);
  }
  e |= rhs_stage(L, R, P, u, p);       /* r = f(u_c) with u_c == u_p */
  vladd(np, u, 1.0, u, dt / 6, R);     /* u_c += dt/6 r */
  vladd(np, V, 1.0, P, dt / 2, R);     /* v = u_p + dt/2 r */
  e |= rhs_stage(L, R, P, V, p);
  vladd(np, u, 1.0, u, dt / 3, R);
  vladd(np, V, 1.0, P, dt / 2, R);
  e |= rhs_stage(L, R, P, V, p);
  vladd(np, u, 1.0, u, dt / 3, R);
  vladd(np, V, 1.0, P, dt, R);
  e |= rhs_stage(L, R, P, V, p);
  vladd(np, u, 1.0, u, dt / 6, R);
  free(buf);
  return e;
}

int oracle_bssn_rk4_step(const nrgpu_level_desc *L, double *const *u, double dt,
                         const nrgpu_bssn_params *p)
{
  int e = oracle_bssn_rk4_stages(L, u, dt, p);
  oracle_bssn_algcon(L, u, p);
  return e;
}

int oracle_bssn_evolve(const nrgpu_level_desc *L, double *const *u, double dt, int nsteps,
                       const nrgpu_bssn_params *p)
{
  int s, e = 0;
  for (s = 0; s < nsteps; s++) e |= oracle_bssn_rk4_step(L, u, dt, p);
  return e;
}

#ifdef ORACLE_COUNT_FLOPS
fc_counts g_fc;
/* FLOPs and transcendental calls of one inner point at distance >= 3 from the
 * box edge (full order, advection with a non-zero shift, dissipation on) */
extern "C" void oracle_count_point(const nrgpu_level_desc *L, double *const *u, int i, int j, int k,
                                   const nrgpu_bssn_params *p, long long *flops, long long *transc)
{
  const double h[3] = {L->dx, L->dy, L->dz};
  int m = L->box[0].m, n = L->box[0].n, o = L->box[0].o;
  long ijk = i + (long)m * (j + (long)n * k);
  real r[NV];
  g_fc.flops = g_fc.transc = 0;
  bssn_point((const double *const *)u, ijk, i, j, k, m - 1, n - 1, o - 1, 1, m, (long)m * n, h, p, r);
  *flops = g_fc.flops;
  *transc = g_fc.transc;
}
#endif

/* ======================================================================
 * Z4c: z4_rhs_movpunc_N (spec z4_rhs_movpunc_N.m:18-520, non-shell branch,
 * useNPTs = 0), boundary = set_boundary (z4.c:248), algcon z4_algcon
 * (identical operations to bssn_algcon on g~ and A~).
 * Variables: g11..g33 chi A11..A33 Khat G1..G3 Theta alpha beta1..3 B1..3.
 * ====================================================================== */
enum { ZG11, ZCHI = 6, ZA11 = 7, ZKHAT = 13, ZGA1 = 14, ZTHETA = 17, ZALPHA = 18, ZBETA1 = 19,
       ZBB1 = 22, ZNV = 25 };

static int z4_point(const double *const *u, long ijk, int i, int j, int k, int imax, int jmax,
                    int kmax, long di, long dj, long dk, const double h[3],
                    const nrgpu_z4_params *p, real r[ZNV])
{
  const long s[3] = {di, dj, dk};
  int a, b, c, d, e, ord, aord;
  int dist = i;
  if (j < dist) dist = j;
  if (k < dist) dist = k;
  if (imax - i < dist) dist = imax - i;
  if (jmax - j < dist) dist = jmax - j;
  if (kmax - k < dist) dist = kmax - k;
  ord = ladder(p->order_centered, dist);
  aord = ladder(p->order_advection, dist);
  if (!ord || !aord || p->useNPTs) return -1;

  real g[6], A[6], Gv[3], beta[3], B[3];
  real alpha = u[ZALPHA][ijk], chi = u[ZCHI][ijk], Khat = u[ZKHAT][ijk], Theta = u[ZTHETA][ijk];
  for (a = 0; a < 6; a++) { g[a] = u[ZG11 + a][ijk]; A[a] = u[ZA11 + a][ijk]; }
  for (a = 0; a < 3; a++) {
    Gv[a] = u[ZGA1 + a][ijk]; beta[a] = u[ZBETA1 + a][ijk]; B[a] = u[ZBB1 + a][ijk];
  }

  real da[3], dda[6], db[3][3], ddb[6][3], delg[3][6], deldelg[6][6], delG[3][3], dKhat[3],
      dchi[3], ddchi[6], dTheta[3];
  for (a = 0; a < 3; a++) {
    da[a] = d1(u[ZALPHA], ijk, s[a], h[a], ord);
    dKhat[a] = d1(u[ZKHAT], ijk, s[a], h[a], ord);
    dchi[a] = d1(u[ZCHI], ijk, s[a], h[a], ord);
    dTheta[a] = d1(u[ZTHETA], ijk, s[a], h[a], ord);
    for (c = 0; c < 3; c++) {
      db[a][c] = d1(u[ZBETA1 + c], ijk, s[a], h[a], ord);
      delG[a][c] = d1(u[ZGA1 + c], ijk, s[a], h[a], ord);
    }
    for (c = 0; c < 6; c++) delg[a][c] = d1(u[ZG11 + c], ijk, s[a], h[a], ord);
  }
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      int ab = SY[a][b];
      if (a == b) {
        dda[ab] = d2(u[ZALPHA], ijk, s[a], h[a], ord);
        ddchi[ab] = d2(u[ZCHI], ijk, s[a], h[a], ord);
        for (c = 0; c < 3; c++) ddb[ab][c] = d2(u[ZBETA1 + c], ijk, s[a], h[a], ord);
        for (c = 0; c < 6; c++) deldelg[ab][c] = d2(u[ZG11 + c], ijk, s[a], h[a], ord);
      } else {
        dda[ab] = d11(u[ZALPHA], ijk, s[a], s[b], h[a], h[b], ord);
        ddchi[ab] = d11(u[ZCHI], ijk, s[a], s[b], h[a], h[b], ord);
        for (c = 0; c < 3; c++) ddb[ab][c] = d11(u[ZBETA1 + c], ijk, s[a], s[b], h[a], h[b], ord);
        for (c = 0; c < 6; c++)
          deldelg[ab][c] = d11(u[ZG11 + c], ijk, s[a], s[b], h[a], h[b], ord);
      }
    }

  adv_t av[3];
  {
    const int idx[3] = {i, j, k}, mx[3] = {imax, jmax, kmax};
    const int lop = aord == 6 ? p->advection_lopsided6 : p->advection_lopsided;
    for (a = 0; a < 3; a++) adv_dir(&av[a], idx[a], mx[a], beta[a] / h[a], aord, lop, s[a]);
  }
  real lieg[6], lieA[6], lieKhat, liechi, liealpha, advG[3], advbeta[3], advB[3], advTheta;
  for (a = 0; a < 6; a++) {
    lieg[a] = adv_apply(av, u[ZG11 + a], ijk);
    lieA[a] = adv_apply(av, u[ZA11 + a], ijk);
  }
  lieKhat = adv_apply(av, u[ZKHAT], ijk);
  liechi = adv_apply(av, u[ZCHI], ijk);
  liealpha = adv_apply(av, u[ZALPHA], ijk);
  advTheta = adv_apply(av, u[ZTHETA], ijk);
  for (a = 0; a < 3; a++) {
    advG[a] = adv_apply(av, u[ZGA1 + a], ijk);
    advbeta[a] = adv_apply(av, u[ZBETA1 + a], ijk);
    advB[a] = adv_apply(av, u[ZBB1 + a], ijk);
  }

  real K = Khat + 2 * Theta;
  real detg = g[0] * g[3] * g[5] + 2 * g[1] * g[2] * g[4] - g[0] * g[4] * g[4] - g[3] * g[2] * g[2] -
              g[5] * g[1] * g[1];
  real detginv = 1 / detg;
  real ginv[6];
  ginv[0] = detginv * (g[3] * g[5] - g[4] * g[4]);
  ginv[1] = detginv * (g[2] * g[4] - g[1] * g[5]);
  ginv[2] = detginv * (g[1] * g[4] - g[2] * g[3]);
  ginv[3] = detginv * (g[0] * g[5] - g[2] * g[2]);
  ginv[4] = detginv * (g[1] * g[2] - g[0] * g[4]);
  ginv[5] = detginv * (g[0] * g[3] - g[1] * g[1]);
#define GI(x, y) ginv[SY[x][y]]
#define GG(x, y) g[SY[x][y]]
#define AAi(x, y) A[SY[x][y]]
  real gammado[3][6], gamma[3][6], Gfromg[3];
  for (c = 0; c < 3; c++)
    for (a = 0; a < 3; a++)
      for (b = a; b < 3; b++)
        gammado[c][SY[a][b]] = 0.5 * (delg[a][SY[b][c]] + delg[b][SY[a][c]] - delg[c][SY[a][b]]);
  for (c = 0; c < 3; c++)
    for (a = 0; a < 6; a++) {
      real t = 0;
      for (d = 0; d < 3; d++) t += GI(c, d) * gammado[d][a];
      gamma[c][a] = t;
    }
  for (a = 0; a < 3; a++) {
    real t = 0;
    for (b = 0; b < 3; b++)
      for (c = 0; c < 3; c++) t += GI(b, c) * gamma[a][SY[b][c]];
    Gfromg[a] = t;
  }
#define GAM(x, y, z) gamma[x][SY[y][z]]
#define GDO(x, y, z) gammado[x][SY[y][z]]
  real Rab[6];
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      real t = 0, t2 = 0;
      for (c = 0; c < 3; c++)
        for (d = 0; d < 3; d++) {
          real q = -0.5 * deldelg[SY[c][d]][SY[a][b]];
          for (e = 0; e < 3; e++)
            q += GAM(e, c, a) * GDO(b, e, d) + GAM(e, c, b) * GDO(a, e, d) + GAM(e, a, d) * GDO(e, c, b);
          t += GI(c, d) * q;
        }
      for (c = 0; c < 3; c++)
        t2 += GG(c, a) * delG[b][c] + GG(c, b) * delG[a][c] + Gfromg[c] * (GDO(a, b, c) + GDO(b, a, c));
      Rab[SY[a][b]] = t + 0.5 * t2;
    }

  real chiguarded = chi;
  if (chiguarded < p->chiDivFloor) chiguarded = p->chiDivFloor;
  real oochipsipower = 1 / p->chipsipower;
  real f = oochipsipower * RLOG(chiguarded);
  real psim4 = REXP(-4 * f);
  real df[3], ddf[6], cddf[6];
  for (a = 0; a < 3; a++) df[a] = oochipsipower * dchi[a] / chiguarded;
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++)
      ddf[SY[a][b]] = oochipsipower * ddchi[SY[a][b]] / chiguarded - p->chipsipower * df[a] * df[b];
  real trcddf = 0, dfdf = 0, dfda = 0;
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      real t = ddf[SY[a][b]];
      for (c = 0; c < 3; c++) t -= GAM(c, a, b) * df[c];
      cddf[SY[a][b]] = t;
    }
  for (a = 0; a < 3; a++)
    for (b = 0; b < 3; b++) {
      trcddf += GI(a, b) * cddf[SY[a][b]];
      dfdf += GI(a, b) * df[a] * df[b];
      dfda += GI(a, b) * df[a] * da[b];
    }
  real Rphi[6], cdda[6];
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      int ab = SY[a][b];
      Rphi[ab] = 4 * df[a] * df[b] - 2 * cddf[ab] - 2 * g[ab] * trcddf - 4 * g[ab] * dfdf;
      real t = dda[ab];
      for (c = 0; c < 3; c++) t -= GAM(c, a, b) * da[c];
      cdda[ab] = t - 2 * (df[a] * da[b] + df[b] * da[a] - g[ab] * dfda);
    }
  real trcdda = 0;
  for (a = 0; a < 3; a++)
    for (b = 0; b < 3; b++) trcdda += GI(a, b) * cdda[SY[a][b]];
  trcdda = psim4 * trcdda;

  real AAab[6], Ainv[6], cAA = 0, divAinv[3];
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      real t = 0, t2 = 0;
      for (c = 0; c < 3; c++)
        for (d = 0; d < 3; d++) {
          t += GI(c, d) * AAi(a, c) * AAi(d, b);
          t2 += GI(a, c) * GI(b, d) * AAi(c, d);
        }
      AAab[SY[a][b]] = t;
      Ainv[SY[a][b]] = t2;
    }
  for (a = 0; a < 3; a++)
    for (b = 0; b < 3; b++) cAA += GI(a, b) * AAab[SY[a][b]];
  for (a = 0; a < 3; a++) {
    real t = 0;
    for (b = 0; b < 3; b++)
      for (c = 0; c < 3; c++) t += GAM(a, b, c) * Ainv[SY[b][c]];
    for (b = 0; b < 3; b++)
      t += -1.5 * Ainv[SY[a][b]] * dchi[b] / chiguarded -
           (1.0 / 3.0) * GI(a, b) * (2 * dKhat[b] + dTheta[b]);
    divAinv[a] = t;
  }
  real Rhat = 0;
  for (a = 0; a < 3; a++)
    for (b = 0; b < 3; b++) Rhat += GI(a, b) * (Rab[SY[a][b]] + Rphi[SY[a][b]]);
  Rhat = psim4 * Rhat;
  real Hhat = Rhat + 2 * K * K / 3 - cAA;

  real divbeta = db[0][0] + db[1][1] + db[2][2];
  real totdivbeta = (2.0 / 3.0) * divbeta;
  real ootddivbeta[3];
  for (a = 0; a < 3; a++)
    ootddivbeta[a] = (1.0 / 3.0) * (ddb[SY[a][0]][0] + ddb[SY[a][1]][1] + ddb[SY[a][2]][2]);
  for (a = 0; a < 3; a++)
    for (b = a; b < 3; b++) {
      int ab = SY[a][b];
      real tg = lieg[ab] - g[ab] * totdivbeta, tA = lieA[ab] - A[ab] * totdivbeta;
      for (c = 0; c < 3; c++) {
        tg += db[a][c] * GG(b, c) + db[b][c] * GG(a, c);
        tA += db[a][c] * AAi(b, c) + db[b][c] * AAi(a, c);
      }
      lieg[ab] = tg;
      lieA[ab] = tA;
    }
  liechi = liechi + (p->chipsipower / 6) * chiguarded * divbeta;
  real pseudolieG[3];
  for (a = 0; a < 3; a++) {
    real t = 0;
    for (b = 0; b < 3; b++)
      for (c = 0; c < 3; c++) t += GI(b, c) * ddb[SY[b][c]][a];
    for (b = 0; b < 3; b++) t += GI(a, b) * ootddivbeta[b] - Gfromg[b] * db[b][a];
    pseudolieG[a] = t + Gfromg[a] * totdivbeta + advG[a];
  }

  real rg[6], rA[6], rG[3], rKhat, rchi, rTheta;
  for (a = 0; a < 6; a++) {
    rg[a] = -2 * alpha * A[a] + lieg[a];
    rA[a] = psim4 * (-cdda[a] + alpha * (Rab[a] + Rphi[a])) - (1.0 / 3.0) * g[a] * (-trcdda + alpha * Rhat) +
            alpha * (K * A[a] - 2 * AAab[a]) + lieA[a];
  }
  for (a = 0; a < 3; a++) {
    real t = 0;
    for (b = 0; b < 3; b++) t += Ainv[SY[a][b]] * da[b];
    rG[a] = -2 * t + 2 * alpha * divAinv[a] - 2 * alpha * p->kappa1 * (Gv[a] - Gfromg[a]) + pseudolieG[a];
  }
  rKhat = -trcdda + alpha * (cAA + K * K / 3) + lieKhat + p->kappa1 * (1 - p->kappa2) * alpha * Theta;
  rchi = (-p->chipsipower / 6) * chiguarded * alpha * K + liechi;
  rTheta = (alpha * (Hhat / 2 - (2 + p->kappa2) * p->kappa1 * Theta) + advTheta) * p->zeroThetaRHS;

  real falpha = p->oploglapse * p->lapseharmonicf + p->oploglapse2 * 8.0 / (3 * (3 - alpha)) +
                p->harmoniclapse * alpha;
  real ralpha = p->oplogwithshift * liealpha - falpha * alpha * Khat;
  real rbeta[3], rB[3];
  if (p->withB != 0) {
    real betaF = p->shiftgammacoeff * RPOW(alpha, p->shiftalphapower);
    for (a = 0; a < 3; a++) {
      rbeta[a] = (p->gamma2factor + p->gamma0factor * betaF) * B[a] + p->withShiftadv * advbeta[a];
      rB[a] = (p->gamma0factor + p->gamma2factor * betaF) * (rG[a] - p->withGadv * advG[a]) -
              p->shiftdriver * B[a] + p->withBadv * advB[a];
    }
  } else {
    for (a = 0; a < 3; a++) {
      rB[a] = 0;
      rbeta[a] = Gv[a] + p->withShiftadv * advbeta[a] - p->shiftdriver * beta[a];
    }
  }

  if ((p->order_dissipation == 4 && dist >= 2) || (p->order_dissipation == 6 && dist >= 3)) {
    const int od = p->order_dissipation;
    const double e_ = p->dissfactor;
    for (a = 0; a < 6; a++) {
      rg[a] += e_ * ko(u[ZG11 + a], ijk, s, h, od);
      rA[a] += e_ * ko(u[ZA11 + a], ijk, s, h, od);
    }
    for (a = 0; a < 3; a++) {
      rG[a] += e_ * ko(u[ZGA1 + a], ijk, s, h, od);
      rbeta[a] += e_ * ko(u[ZBETA1 + a], ijk, s, h, od);
      rB[a] += e_ * ko(u[ZBB1 + a], ijk, s, h, od);
    }
    rKhat += e_ * ko(u[ZKHAT], ijk, s, h, od);
    rchi += e_ * ko(u[ZCHI], ijk, s, h, od);
    rTheta += e_ * ko(u[ZTHETA], ijk, s, h, od);
    ralpha += e_ * ko(u[ZALPHA], ijk, s, h, od);
  }

  for (a = 0; a < 6; a++) { r[ZG11 + a] = rg[a]; r[ZA11 + a] = rA[a]; }
  r[ZCHI] = rchi;
  r[ZKHAT] = rKhat;
  r[ZTHETA] = rTheta;
  r[ZALPHA] = ralpha;
  for (a = 0; a < 3; a++) {
    r[ZGA1 + a] = rG[a];
    r[ZBETA1 + a] = rbeta[a];
    r[ZBB1 + a] = rB[a];
  }
  return 0;
#undef GI
#undef GG
#undef AAi
#undef GAM
#undef GDO
}

static void z4_addlinear(double *const *unew, double *const *upre, long ijk, double c, const real r[ZNV],
                         const nrgpu_z4_params *p)
{
  double n[ZNV];
  int v;
  for (v = 0; v < ZNV; v++) n[v] = upre[v][ijk] + c * RVAL(r[v]);
  double *g = n + ZG11, *A = n + ZA11;
  double detg = g[0] * g[3] * g[5] + 2 * g[1] * g[2] * g[4] - g[0] * g[4] * g[4] -
                g[3] * g[2] * g[2] - g[5] * g[1] * g[1];
  double detnginv = 1 / detg;
  if (p->subtractA) {
    double gi[6];
    gi[0] = (g[3] * g[5] - g[4] * g[4]);
    gi[1] = (g[2] * g[4] - g[1] * g[5]);
    gi[2] = (g[1] * g[4] - g[2] * g[3]);
    gi[3] = (g[0] * g[5] - g[2] * g[2]);
    gi[4] = (g[1] * g[2] - g[0] * g[4]);
    gi[5] = (g[0] * g[3] - g[1] * g[1]);
    double trA = detnginv * (gi[0] * A[0] + gi[3] * A[3] + gi[5] * A[5] +
                             2 * (gi[1] * A[1] + gi[2] * A[2] + gi[4] * A[4]));
    double aux = -trA / 3;
    for (v = 0; v < 6; v++) A[v] += aux * g[v];
  }
  if (p->normalizedetg) {
    double aux = pow(detnginv, 1.0 / 3.0);
    for (v = 0; v < 6; v++) g[v] *= aux;
  }
  for (v = 0; v < ZNV; v++) unew[v][ijk] = n[v];
}

int oracle_z4_rhs(const nrgpu_level_desc *L, double *const *unew, double *const *upre, double c,
                  double *const *ucur, const nrgpu_z4_params *p)
{
  int b, err = 0;
  const double h[3] = {L->dx, L->dy, L->dz};
  for (b = 0; b < L->nboxes; b++) {
    int m, n, o;
    long off = box_of(L, b, &m, &n, &o);
    long np = (long)m * n * o, q;
    OMP_FOR
    for (q = 0; q < np; q++) {
      int k = (int)(q / ((long)m * n)), j = (int)((q / m) % n), i = (int)(q % m);
      long ijk = off + q;
      real r[ZNV];
      int v;
      if (L->boundary[ijk]) continue;
      if (z4_point((const double *const *)ucur, ijk, i, j, k, m - 1, n - 1, o - 1, 1, m, (long)m * n, h, p, r)) {
        err = -1;
        continue;
      }
      if (c == 0.0)
        for (v = 0; v < ZNV; v++) unew[v][ijk] = RVAL(r[v]);
      else
        z4_addlinear(unew, upre, ijk, c, r, p);
    }
  }
  return err;
}

int oracle_z4_boundary(const nrgpu_level_desc *L, double *const *unew, double *const *upre, double c,
                       double *const *ucur, const nrgpu_z4_params *p)
{
  return boundary_nv(L, ZNV, unew, upre, c, ucur, p->bc_var0, p->bc_speed);
}

/* z4_algcon on the g~ and A~ of a Z4c list: same operations as bssn_algcon */
void oracle_z4_algcon(const nrgpu_level_desc *L, double *const *u, const nrgpu_z4_params *p)
{
  nrgpu_bssn_params q;
  double *bl[NV];
  int v;
  memset(&q, 0, sizeof q);
  q.subtractA = p->subtractA;
  q.normalizedetg = p->normalizedetg;
  for (v = 0; v < NV; v++) bl[v] = u[v];  /* g at 0..5, A at 7..12 in both lists */
  oracle_bssn_algcon(L, bl, &q);
}

int oracle_z4_rk4_stages(const nrgpu_level_desc *L, double *const *u, double dt, const nrgpu_z4_params *p)
{
  long np = L->npoints;
  double *buf = (double *)malloc(sizeof(double) * 3 * ZNV * np);
  double *P[ZNV], *R[ZNV], *V[ZNV];
  int v, e = 0;
  if (!buf) return -4;
  for (v = 0; v < ZNV; v++) {
    P[v] = buf + (0 * ZNV + v) * np;
    R[v] = buf + (1 * ZNV + v) * np;
    V[v] = buf + (2 * ZNV + v) * np;
    memcpy(P[v], u[v], sizeof(double) * np);
    memset(R[v], 0, sizeof(double) * np);
  }
#define ZSTAGE(cur)                                   \
  e |= oracle_z4_rhs(L, R, P, 0.0, cur, p);           \
  oracle_z4_boundary(L, R, P, 0.0, cur, p);
  ZSTAGE(u);
  vladd_nv(np, ZNV, u, 1.0, u, dt / 6, R);
  vladd_nv(np, ZNV, V, 1.0, P, dt / 2, R);
  ZSTAGE(V);
  vladd_nv(np, ZNV, u, 1.0, u, dt / 3, R);
  vladd_nv(np, ZNV, V, 1.0, P, dt / 2, R);
  ZSTAGE(V);
  vladd_nv(np, ZNV, u, 1.0, u, dt / 3, R);
  vladd_nv(np, ZNV, V, 1.0, P, dt, R);
  ZSTAGE(V);
  vladd_nv(np, ZNV, u, 1.0, u, dt / 6, R);
#undef ZSTAGE
  free(buf);
  return e;
}

int oracle_z4_rk4_step(const nrgpu_level_desc *L, double *const *u, double dt, const nrgpu_z4_params *p)
{
  int e = oracle_z4_rk4_stages(L, u, dt, p);
  oracle_z4_algcon(L, u, p);
  return e;
}

int oracle_z4_evolve(const nrgpu_level_desc *L, double *const *u, double dt, int nsteps, const nrgpu_z4_params *p)
{
  int s, e = 0;
  for (s = 0; s < nsteps; s++) e |= oracle_z4_rk4_step(L, u, dt, p);
  return e;
}

#ifdef ORACLE_COUNT_FLOPS
/* the same for the Z4c rhs */
extern "C" void oracle_count_z4_point(const nrgpu_level_desc *L, double *const *u, int i, int j, int k,
                                      const nrgpu_z4_params *p, long long *flops, long long *transc)
{
  const double h[3] = {L->dx, L->dy, L->dz};
  int m = L->box[0].m, n = L->box[0].n, o = L->box[0].o;
  long ijk = i + (long)m * (j + (long)n * k);
  real r[25];
  g_fc.flops = g_fc.transc = 0;
  z4_point((const double *const *)u, ijk, i, j, k, m - 1, n - 1, o - 1, 1, m, (long)m * n, h, p, r);
  *flops = g_fc.flops;
  *transc = g_fc.transc;
}
#endif
