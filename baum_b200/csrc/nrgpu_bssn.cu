// nrgpu_bssn.cu -- BSSN right-hand side, radiative boundary, algebraic
// constraints and the fused RK4 stages for B200 (sm_100a), FP64.
//
// The physics is the reference's bssn_rhs_movpunc_N (spec
// bssn_rhs_movpunc_N.m:18-461), computed per inner point in one thread:
//   centred FD of order 2/4/6 with the reference's order ladder near box
//   edges (bssn_rhs_movpunc_N.m:32-110, boundaryNaway bam_amr_loops_box.h:215),
//   lopsided advection with edge-shifted stencils (bam_amr_advection.h:72-192),
//   BSSN algebra + 1+log / Gamma-driver gauge (bssn_rhs_movpunc_N.m:218-346),
//   Kreiss-Oliger dissipation where the full stencil fits (:351-372).
// The order of work inside a thread is chosen for register pressure, not the
// reference's: each group of derivatives is consumed right after it is formed
// (connection -> Ricci -> conformal factor -> lapse -> A -> shift), and the
// advection and dissipation sums are added at the end, so that the 24 rhs
// accumulators are the only long-lived state.  Algebraically this is the
// reference's expression; it differs from it only in rounding.
#include <cstdio>
#include <cstring>
#include <mutex>
#include "nrgpu_level.cuh"
#include "nrgpu_fd.cuh"
#include "nrgpu_tma.cuh"

namespace {

enum { G11 = 0, CHI = 6, A11 = 7, KK = 13, GA1 = 14, ALPHA = 17, BETA1 = 18, BB1 = 21 };

// lopsided advection rows (numerators), row r = stencil shifted by r
// (bam_amr_advection.h:28-66); denominators 2, 12, 60
__constant__ double kAdv2[3][3] = {{3, -4, 1}, {1, 0, -1}, {-1, 4, -3}};
__constant__ double kAdv4[5][5] = {{25, -48, 36, -16, 3}, {3, 10, -18, 6, -1}, {-1, 8, 0, -8, 1},
                                   {1, -6, 18, -10, -3}, {-3, 16, -36, 48, -25}};
__constant__ double kAdv6[7][7] = {{147, -360, 450, -400, 225, -72, 10}, {10, 77, -150, 100, -50, 15, -2},
                                   {-2, 24, 35, -80, 30, -8, 1},        {1, -9, 45, 0, -45, 9, -1},
                                   {-1, 8, -30, 80, -35, -24, 2},       {2, -15, 50, -100, 150, -77, -10},
                                   {-10, 72, -225, 400, -450, 360, -147}};

struct AdvDir {
  int base;     // offset of tap 0 relative to the point
  int step;     // +-stride between taps (0 when the shift is zero)
  int row;      // stencil row
};

// direction setup of set_advectionN_onedir (bam_amr_advection.h:72-192)
__device__ __forceinline__ AdvDir adv_dir(int i, int imax, double w, int q, int lop, int s) {
  AdvDir a;
  int rst = q - lop, offset, wsign;
  if (w < 0) { wsign = -1; offset = (i >= rst) ? 0 : rst - i; }
  else if (w > 0) { wsign = 1; offset = (imax - i >= rst) ? 0 : rst - (imax - i); }
  else { wsign = 0; offset = 0; }
  offset += lop;
  a.row = offset;
  a.step = wsign * s;
  a.base = -offset * wsign * s;
  return a;
}

template <int Q>
__device__ __forceinline__ double adv_sum(const double *__restrict__ f, int x, const AdvDir ad[3],
                                          const double cw[3]) {
  double acc = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double t = 0.0;
    const int p0 = x + ad[d].base;
#pragma unroll
    for (int n = 0; n <= Q; ++n) {
      const double c = Q == 2 ? kAdv2[ad[d].row][n] : Q == 4 ? kAdv4[ad[d].row][n] : kAdv6[ad[d].row][n];
      t += c * ldg(f + p0 + n * ad[d].step);
    }
    acc += cw[d] * t;
  }
  return acc;
}

// Kreiss-Oliger: sum over directions of undivided differences / h
template <int OD>
__device__ __forceinline__ double ko_sum(const double *__restrict__ f, int x, const int st[3],
                                         const double ooh[3]) {
  double acc = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int s = st[d];
    double t;
    if (OD == 4)
      t = 6.0 * ldg(f + x) - 4.0 * (ldg(f + x - s) + ldg(f + x + s)) + (ldg(f + x - 2 * s) + ldg(f + x + 2 * s));
    else
      t = (ldg(f + x - 3 * s) + ldg(f + x + 3 * s)) - 6.0 * (ldg(f + x - 2 * s) + ldg(f + x + 2 * s)) +
          15.0 * (ldg(f + x - s) + ldg(f + x + s)) - 20.0 * ldg(f + x);
    acc += ooh[d] * t;
  }
  return OD == 4 ? -acc : acc;
}

// Kreiss-Oliger with FP32 sums of centre-relative taps (the weights sum to
// zero); P = 0 keeps FP64
template <int OD, int P>
__device__ __forceinline__ double ko_p(const double *__restrict__ f, int x, const int st[3], const double ooh[3]) {
  if (P == 0) return ko_sum<OD>(f, x, st, ooh);
  const double c = ldg(f + x);
  double acc = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int s = st[d];
    float t;
    if (OD == 4)
      t = -4.0f * (tapf(f, x, -1, s, c) + tapf(f, x, 1, s, c)) + (tapf(f, x, -2, s, c) + tapf(f, x, 2, s, c));
    else
      t = (tapf(f, x, -3, s, c) + tapf(f, x, 3, s, c)) - 6.0f * (tapf(f, x, -2, s, c) + tapf(f, x, 2, s, c)) +
          15.0f * (tapf(f, x, -1, s, c) + tapf(f, x, 1, s, c));
    acc += ooh[d] * (double)t;
  }
  return OD == 4 ? -acc : acc;
}

struct PointCtx {
  int ijk, i, j, k, imax, jmax, kmax, dist;
  int st[3];
  double h[3];
};

// ---- the per-point right-hand side -------------------------------------------
template <int ORD, int CSY = 0, int CSZ = 0>
__device__ __forceinline__ void bssn_point(const CVarPtrs &U, const PointCtx &P,
                                           const nrgpu_bssn_params &p, double r[NRGPU_NV]) {
  const int x = P.ijk;
  // strides: compile-time when the box size is known, so taps fold into
  // immediate load offsets
#define STR(c_) ((c_) == 0 ? 1 : (CSY > 0 ? ((c_) == 1 ? CSY : CSZ) : P.st[(c_)]))
  const double o1[3] = {1.0 / (den1<ORD>() * P.h[0]), 1.0 / (den1<ORD>() * P.h[1]),
                        1.0 / (den1<ORD>() * P.h[2])};

  double g[6], A[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) { g[a] = ldg(U.p[G11 + a] + x); A[a] = ldg(U.p[A11 + a] + x); }
  const double alpha = ldg(U.p[ALPHA] + x);
  const double chi = ldg(U.p[CHI] + x);
  double K = ldg(U.p[KK] + x);

  // inverse conformal metric
  const double detg = g[0] * g[3] * g[5] + 2.0 * g[1] * g[2] * g[4] - g[0] * g[4] * g[4] -
                      g[3] * g[2] * g[2] - g[5] * g[1] * g[1];
  const double detginv = 1.0 / detg;
  double gi[6];
  gi[0] = detginv * (g[3] * g[5] - g[4] * g[4]);
  gi[1] = detginv * (g[2] * g[4] - g[1] * g[5]);
  gi[2] = detginv * (g[1] * g[4] - g[2] * g[3]);
  gi[3] = detginv * (g[0] * g[5] - g[2] * g[2]);
  gi[4] = detginv * (g[1] * g[2] - g[0] * g[4]);
  gi[5] = detginv * (g[0] * g[3] - g[1] * g[1]);

  // Ricci tensor of the conformal metric.  Its -1/2 ginv^cd d_c d_d g_ab
  // part (folded over the symmetric pair c, d): with compile-time strides it
  // comes first, so that its stencil loads have no connection values live
  // beside them; with run-time strides after the connection terms
  double Rt[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) Rt[a] = 0.0;
  auto ricci_dd = [&]() {
    const double o2[3] = {1.0 / (den2<ORD>() * P.h[0] * P.h[0]), 1.0 / (den2<ORD>() * P.h[1] * P.h[1]),
                          1.0 / (den2<ORD>() * P.h[2] * P.h[2])};
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int d = c; d < 3; ++d) {
        const double w = (c == d ? -0.5 : -1.0) * gi[sy(c, d)] * (c == d ? o2[c] : o1[c] * o1[d]);
#pragma unroll
        for (int a = 0; a < 6; ++a) {
          const double dd = c == d ? d2n<ORD>(U.p[G11 + a], x, STR(c))
                                   : d11n<ORD>(U.p[G11 + a], x, STR(c), STR(d));
          Rt[a] += w * dd;
        }
      }
  };
  constexpr bool kDdFirst = CSY > 0;
  if constexpr (kDdFirst) ricci_dd();

  // connection: gdo[c][ab] = 1/2 (d_a g_bc + d_b g_ac - d_c g_ab), gam = ginv gdo
  double gdo[3][6], gam[3][6], Gfg[3];
  {
    double dg[3][6];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int a = 0; a < 6; ++a) dg[c][a] = o1[c] * d1n<ORD>(U.p[G11 + a], x, STR(c));
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = a; b < 3; ++b)
          gdo[c][sy(a, b)] = 0.5 * (dg[a][sy(b, c)] + dg[b][sy(a, c)] - dg[c][sy(a, b)]);
  }
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int a = 0; a < 6; ++a)
      gam[c][a] = gi[sy(c, 0)] * gdo[0][a] + gi[sy(c, 1)] * gdo[1][a] + gi[sy(c, 2)] * gdo[2][a];
#pragma unroll
  for (int a = 0; a < 3; ++a)
    Gfg[a] = gi[0] * gam[a][0] + gi[3] * gam[a][3] + gi[5] * gam[a][5] +
             2.0 * (gi[1] * gam[a][1] + gi[2] * gam[a][2] + gi[4] * gam[a][4]);

  // the connection terms of the Ricci tensor plus, later, the chi part
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double t = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          double q = 0.0;
#pragma unroll
          for (int e = 0; e < 3; ++e)
            q += gam[e][sy(c, a)] * gdo[b][sy(e, d)] + gam[e][sy(c, b)] * gdo[a][sy(e, d)] +
                 gam[e][sy(a, d)] * gdo[e][sy(c, b)];
          t += gi[sy(c, d)] * q;
        }
      Rt[sy(a, b)] += t;
    }
  if constexpr (!kDdFirst) ricci_dd();
  {
    // 1/2 (g_ca d_b G^c + g_cb d_a G^c + G^c (gdo_abc + gdo_bac))
    double dG[3][3];
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) dG[b][c] = o1[b] * d1n<ORD>(U.p[GA1 + c], x, STR(b));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        double t2 = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
          t2 += g[sy(c, a)] * dG[b][c] + g[sy(c, b)] * dG[a][c] +
                Gfg[c] * (gdo[a][sy(b, c)] + gdo[b][sy(a, c)]);
        Rt[sy(a, b)] += 0.5 * t2;
      }
  }

  // conformal factor chi = psi^chipsipower
  double chig = chi;
  if (chig < p.chiDivFloor) chig = p.chiDivFloor;
  const double oocp = 1.0 / p.chipsipower;
  const double f = oocp * log(chig);
  const double psim4 = exp(-4.0 * f);
  double df[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) df[a] = oocp * (o1[a] * d1n<ORD>(U.p[CHI], x, STR(a))) / chig;
  double dfdf = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) dfdf += gi[sy(a, b)] * df[a] * df[b];
  {
    const double o2[3] = {1.0 / (den2<ORD>() * P.h[0] * P.h[0]), 1.0 / (den2<ORD>() * P.h[1] * P.h[1]),
                          1.0 / (den2<ORD>() * P.h[2] * P.h[2])};
    double cddf[6];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        const double ddchi = a == b ? o2[a] * d2n<ORD>(U.p[CHI], x, STR(a))
                                    : o1[a] * o1[b] * d11n<ORD>(U.p[CHI], x, STR(a), STR(b));
        double t = oocp * ddchi / chig - p.chipsipower * df[a] * df[b];
        t -= gam[0][sy(a, b)] * df[0] + gam[1][sy(a, b)] * df[1] + gam[2][sy(a, b)] * df[2];
        cddf[sy(a, b)] = t;
      }
    const double trcddf = gi[0] * cddf[0] + gi[3] * cddf[3] + gi[5] * cddf[5] +
                          2.0 * (gi[1] * cddf[1] + gi[2] * cddf[2] + gi[4] * cddf[4]);
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        const int ab = sy(a, b);
        Rt[ab] += 4.0 * df[a] * df[b] - 2.0 * cddf[ab] - 2.0 * g[ab] * trcddf - 4.0 * g[ab] * dfdf;
      }
  }

  // derivatives of the lapse
  double da[3], cdda[6];
#pragma unroll
  for (int a = 0; a < 3; ++a) da[a] = o1[a] * d1n<ORD>(U.p[ALPHA], x, STR(a));
  {
    const double o2[3] = {1.0 / (den2<ORD>() * P.h[0] * P.h[0]), 1.0 / (den2<ORD>() * P.h[1] * P.h[1]),
                          1.0 / (den2<ORD>() * P.h[2] * P.h[2])};
    double dfda = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = 0; b < 3; ++b) dfda += gi[sy(a, b)] * df[a] * da[b];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        const int ab = sy(a, b);
        double t = a == b ? o2[a] * d2n<ORD>(U.p[ALPHA], x, STR(a))
                          : o1[a] * o1[b] * d11n<ORD>(U.p[ALPHA], x, STR(a), STR(b));
        t -= gam[0][ab] * da[0] + gam[1][ab] * da[1] + gam[2][ab] * da[2];
        cdda[ab] = t - 2.0 * (df[a] * da[b] + df[b] * da[a] - g[ab] * dfda);
      }
  }
  const double trcdda = psim4 * (gi[0] * cdda[0] + gi[3] * cdda[3] + gi[5] * cdda[5] +
                                 2.0 * (gi[1] * cdda[1] + gi[2] * cdda[2] + gi[4] * cdda[4]));

  K = K * p.forceKzerofactor;

  // trace-free extrinsic curvature
  double AAab[6], Ainv[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double t = 0.0, t2 = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          t += gi[sy(c, d)] * A[sy(a, c)] * A[sy(d, b)];
          t2 += gi[sy(a, c)] * gi[sy(b, d)] * A[sy(c, d)];
        }
      AAab[sy(a, b)] = t;
      Ainv[sy(a, b)] = t2;
    }
  const double AAs = gi[0] * AAab[0] + gi[3] * AAab[3] + gi[5] * AAab[5] +
                     2.0 * (gi[1] * AAab[1] + gi[2] * AAab[2] + gi[4] * AAab[4]);
  const double Rsc = AAs - 2.0 * K * K / 3.0;

  // rhs of g~ and A~ (advection added later)
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    r[G11 + a] = -2.0 * alpha * A[a];
    r[A11 + a] = psim4 * (-cdda[a] + alpha * Rt[a]) - (1.0 / 3.0) * g[a] * (-trcdda + alpha * Rsc) +
                 alpha * (K * A[a] - 2.0 * AAab[a]);
  }
  r[KK] = -trcdda + alpha * (AAs + K * K / 3.0);

  // rhs of Gamma~ without advection: -2 Ainv da - 2 alpha divAinv + shift terms
  double rG[3];
  {
    double dK[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) dK[a] = p.forceKzerofactor * (o1[a] * d1n<ORD>(U.p[KK], x, STR(a)));
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double t = 0.0, s = 0.0;
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        t += (2.0 / 3.0) * gi[sy(a, b)] * dK[b] - 6.0 * Ainv[sy(a, b)] * df[b];
        s += Ainv[sy(a, b)] * da[b];
      }
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) t -= gam[a][sy(b, c)] * Ainv[sy(b, c)];
      rG[a] = -2.0 * s - 2.0 * alpha * t;
    }
  }

  // shift terms: Lie-derivative corrections and pseudo-Lie of Gamma~
  {
    const double o2[3] = {1.0 / (den2<ORD>() * P.h[0] * P.h[0]), 1.0 / (den2<ORD>() * P.h[1] * P.h[1]),
                          1.0 / (den2<ORD>() * P.h[2] * P.h[2])};
    double db[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) db[a][c] = o1[a] * d1n<ORD>(U.p[BETA1 + c], x, STR(a));
    const double divbeta = db[0][0] + db[1][1] + db[2][2];
    const double totdivbeta = (2.0 / 3.0) * divbeta;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        const int ab = sy(a, b);
        double tg = -g[ab] * totdivbeta, tA = -A[ab] * totdivbeta;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          tg += db[a][c] * g[sy(b, c)] + db[b][c] * g[sy(a, c)];
          tA += db[a][c] * A[sy(b, c)] + db[b][c] * A[sy(a, c)];
        }
        r[G11 + ab] += tg;
        r[A11 + ab] += tA;
      }
    r[CHI] = (p.chipsipower / 6.0) * chig * divbeta - (p.chipsipower / 6.0) * chig * alpha * K;
    // ddb[bc][a] = d_b d_c beta^a
    double trddb[3] = {0.0, 0.0, 0.0};   // g^bc d_b d_c beta^a
    double divdb[3] = {0.0, 0.0, 0.0};   // d_a d_b beta^b
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = b; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double dd = b == c ? o2[b] * d2n<ORD>(U.p[BETA1 + a], x, STR(b))
                                   : o1[b] * o1[c] * d11n<ORD>(U.p[BETA1 + a], x, STR(b), STR(c));
          trddb[a] += (b == c ? 1.0 : 2.0) * gi[sy(b, c)] * dd;
          // d_b d_c beta^a contributes to divdb[b] when c == a and to divdb[c] when b == a
          if (c == a) divdb[b] += dd;
          if (b == a && b != c) divdb[c] += dd;
        }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double t = trddb[a];
#pragma unroll
      for (int b = 0; b < 3; ++b) t += gi[sy(a, b)] * ((1.0 / 3.0) * divdb[b]) - Gfg[b] * db[b][a];
      rG[a] += t + Gfg[a] * totdivbeta;
    }
  }

  // gauge
  const double falpha = p.oploglapse * p.lapseharmonicf + p.oploglapse2 * 8.0 / (3.0 * (3.0 - alpha)) +
                        p.harmoniclapse * alpha;
  r[ALPHA] = -falpha * alpha * K;
  const double betaF = p.shiftgammacoeff * pow(alpha, p.shiftalphapower);
  const double bfac = p.gamma0factor + p.gamma2factor * betaF;
  const double alphaG = p.shiftgammacoeff * pow(alpha, p.shiftGalphapower);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double Ba = ldg(U.p[BB1 + a] + x), ba = ldg(U.p[BETA1 + a] + x), Ga = ldg(U.p[GA1 + a] + x);
    r[BETA1 + a] = (p.gamma2factor + p.gamma0factor * betaF) * p.withB * Ba +
                   (1.0 - p.withB) * (alphaG * Ga - p.shiftdriver * ba);
    r[BB1 + a] = p.withB * (bfac * rG[a] - p.shiftdriver * Ba);
    r[GA1 + a] = rG[a];
  }

  // advection beta^i d_i u with lopsided stencils (weights w = beta/dx)
  {
    const int lop = ORD == 2 ? 0 : (ORD == 6 ? p.advection_lopsided6 : p.advection_lopsided);
    const int idx[3] = {P.i, P.j, P.k}, mx[3] = {P.imax, P.jmax, P.kmax};
    AdvDir ad[3];
    double cw[3];
    const double oad = 1.0 / den1<ORD>();
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double w = ldg(U.p[BETA1 + d] + x) / P.h[d];
      ad[d] = adv_dir(idx[d], mx[d], w, ORD, lop, STR(d));
      const int ws = w < 0 ? -1 : (w > 0 ? 1 : 0);
      cw[d] = -ws * w * oad;
    }
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      r[G11 + a] += adv_sum<ORD>(U.p[G11 + a], x, ad, cw);
      r[A11 + a] += adv_sum<ORD>(U.p[A11 + a], x, ad, cw);
    }
    r[KK] += adv_sum<ORD>(U.p[KK], x, ad, cw);
    r[CHI] += adv_sum<ORD>(U.p[CHI], x, ad, cw);
    r[ALPHA] += p.oplogwithshift * adv_sum<ORD>(U.p[ALPHA], x, ad, cw);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double aG = adv_sum<ORD>(U.p[GA1 + a], x, ad, cw);
      r[GA1 + a] += aG;
      r[BB1 + a] += p.withB * (bfac * (1.0 - p.withGadv) * aG +
                               p.withBadv * adv_sum<ORD>(U.p[BB1 + a], x, ad, cw));
      r[BETA1 + a] += p.withShiftadv * adv_sum<ORD>(U.p[BETA1 + a], x, ad, cw);
    }
  }

  // Kreiss-Oliger dissipation where the full stencil fits
  if ((p.order_dissipation == 4 && P.dist >= 2) || (p.order_dissipation == 6 && P.dist >= 3)) {
    const double ooh[3] = {1.0 / P.h[0], 1.0 / P.h[1], 1.0 / P.h[2]};
    const int kst[3] = {STR(0), STR(1), STR(2)};
    const double e = p.dissfactor;
    if (p.order_dissipation == 6) {
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        r[G11 + a] += e * ko_sum<6>(U.p[G11 + a], x, kst, ooh);
        r[A11 + a] += e * ko_sum<6>(U.p[A11 + a], x, kst, ooh);
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) r[GA1 + a] += e * ko_sum<6>(U.p[GA1 + a], x, kst, ooh);
      r[KK] += e * ko_sum<6>(U.p[KK], x, kst, ooh);
      r[CHI] += e * ko_sum<6>(U.p[CHI], x, kst, ooh);
    } else {
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        r[G11 + a] += e * ko_sum<4>(U.p[G11 + a], x, kst, ooh);
        r[A11 + a] += e * ko_sum<4>(U.p[A11 + a], x, kst, ooh);
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) r[GA1 + a] += e * ko_sum<4>(U.p[GA1 + a], x, kst, ooh);
      r[KK] += e * ko_sum<4>(U.p[KK], x, kst, ooh);
      r[CHI] += e * ko_sum<4>(U.p[CHI], x, kst, ooh);
    }
  }
  r[KK] *= p.forceKzerofactor;
#undef STR
}

// ---- epilogues ----------------------------------------------------------------
// a hint that the line holding p will be read soon: fetched into L2, no
// register written (PTX prefetch.global.L2)
__device__ __forceinline__ void l2_prefetch(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

enum { EPI_RHS = 0, EPI_ADDLINEAR = 1, EPI_RK = 2 };

// EPI_RK accumulator modes: ACC_ADD acc += wacc rhs; ACC_INIT acc = upre +
// wacc rhs (the first stage, so that the step needs no copy of u); ACC_FINAL
// out = acc + wacc rhs (the last stage writes u from the accumulator)
enum { ACC_ADD = 0, ACC_INIT = 1, ACC_FINAL = 2 };

struct Epilogue {
  int mode;
  double c;        // EPI_ADDLINEAR: unew = upre + c rhs
  double wacc;     // EPI_RK: acc += wacc * rhs
  double cv;       // EPI_RK: vout = upre + cv * rhs (when has_v)
  int has_v;
  int accmode;     // EPI_RK: ACC_ADD / ACC_INIT / ACC_FINAL
};

__device__ __forceinline__ void det_trace_fix(double n[NRGPU_NV], const nrgpu_bssn_params &p) {
  double *g = n + G11, *A = n + A11;
  const double detg = g[0] * g[3] * g[5] + 2.0 * g[1] * g[2] * g[4] - g[0] * g[4] * g[4] -
                      g[3] * g[2] * g[2] - g[5] * g[1] * g[1];
  const double detnginv = 1.0 / detg;
  if (p.subtractA) {
    const double gi0 = g[3] * g[5] - g[4] * g[4], gi1 = g[2] * g[4] - g[1] * g[5],
                 gi2 = g[1] * g[4] - g[2] * g[3], gi3 = g[0] * g[5] - g[2] * g[2],
                 gi4 = g[1] * g[2] - g[0] * g[4], gi5 = g[0] * g[3] - g[1] * g[1];
    const double trA = detnginv * (gi0 * A[0] + gi3 * A[3] + gi5 * A[5] + 2.0 * (gi1 * A[1] + gi2 * A[2] + gi4 * A[4]));
    const double aux = -trA / 3.0;
#pragma unroll
    for (int v = 0; v < 6; ++v) A[v] += aux * g[v];
  }
  if (p.normalizedetg) {
    const double aux = cbrt(detnginv);
#pragma unroll
    for (int v = 0; v < 6; ++v) g[v] *= aux;
  }
}

__device__ __forceinline__ void store(const double r[NRGPU_NV], int x, const VarPtrs &out, const CVarPtrs &pre,
                                      const VarPtrs &acc, const Epilogue &E, const nrgpu_bssn_params &p) {
  if (E.mode == EPI_RHS) {
#pragma unroll
    for (int v = 0; v < NRGPU_NV; ++v) out.p[v][x] = r[v];
  } else if (E.mode == EPI_ADDLINEAR) {
    double n[NRGPU_NV];
#pragma unroll
    for (int v = 0; v < NRGPU_NV; ++v) n[v] = ldg(pre.p[v] + x) + E.c * r[v];
    n[KK] = p.forceKzerofactor * n[KK];
    det_trace_fix(n, p);
#pragma unroll
    for (int v = 0; v < NRGPU_NV; ++v) out.p[v][x] = n[v];
  } else if (E.accmode == ACC_FINAL) {
#pragma unroll
    for (int v = 0; v < NRGPU_NV; ++v) out.p[v][x] = acc.p[v][x] + E.wacc * r[v];
  } else if (E.accmode == ACC_INIT) {
#pragma unroll
    for (int v = 0; v < NRGPU_NV; ++v) {
      const double u0 = ldg(pre.p[v] + x);
      acc.p[v][x] = u0 + E.wacc * r[v];
      if (E.has_v) out.p[v][x] = u0 + E.cv * r[v];
    }
  } else {
#pragma unroll
    for (int v = 0; v < NRGPU_NV; ++v) {
      acc.p[v][x] += E.wacc * r[v];
      if (E.has_v) out.p[v][x] = ldg(pre.p[v] + x) + E.cv * r[v];
    }
  }
}

__device__ __forceinline__ int ladder(int order, int d) {
  if (order == 2 || d == 1) return 2;
  if (order == 4 || d == 2) return 4;
  if (order == 6 || d == 3) return 6;
  return 0;
}

// ---- kernels ----------------------------------------------------------------
// one thread per point of the box interior (i,j,k in [1, m-2]); inner points
// (flag 0) only, the flagged ones are handled by bssn_flagged_kernel
// CSY, CSZ: the box strides dj = m and dk = m n when known at compile time
// (0 = read them from the box)
// the input lists are read at in.x + i + in.y (j + in.z k): the box itself,
// or its staged copy (as for z4_rhs_kernel); the outputs, the previous
// state and the flags at the box's own index
template <int CSY = 0, int CSZ = 0, int ORD = 4, int MINB = NRGPU_RHS_MINBLOCKS>
__global__ void __launch_bounds__(256, MINB) bssn_rhs_kernel(CVarPtrs U, VarPtrs out, CVarPtrs pre, VarPtrs acc,
                                                      Epilogue E, const nrgpu_bssn_params p, BoxGeo box,
                                                      const int *__restrict__ boundary, double dx, double dy,
                                                      double dz, int *status, int k0, int k1, int3 in) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = k0 + blockIdx.z * blockDim.z + threadIdx.z;
  if (i > box.m - 2 || j > box.n - 2 || k > k1) return;
  PointCtx P;
  P.i = i; P.j = j; P.k = k;
  P.imax = box.m - 1; P.jmax = box.n - 1; P.kmax = box.o - 1;
  P.st[0] = 1; P.st[1] = box.m; P.st[2] = box.m * box.n;
  const int xo = box.noffset + i + box.m * (j + box.n * k);
  P.ijk = in.x + i + in.y * (j + in.z * k);
  if (__ldg(boundary + xo) != 0) return;
  P.h[0] = dx; P.h[1] = dy; P.h[2] = dz;
  int d = min(min(i, j), k);
  d = min(d, min(min(P.imax - i, P.jmax - j), P.kmax - k));
  // points nearer the faces than the full stencil reaches take a lower
  // order (the ladder): bssn_ladder_kernel computes them
  if (d < ORD / 2) return;
  P.dist = d;
  // the point's own values of every input list, which its stencils and its
  // neighbours' stencils read one field after another: all their lines
  // requested from DRAM at once
#pragma unroll
  for (int v = 0; v < NRGPU_NV; ++v) l2_prefetch(U.p[v] + P.ijk);
  // the RK epilogue reads the accumulator and the previous state at the
  // end; ask L2 for their lines now, so that those loads do not wait on DRAM
  if (E.mode == EPI_RK) {
#pragma unroll
    for (int v = 0; v < NRGPU_NV; ++v) {
      if (E.accmode != ACC_INIT) l2_prefetch(acc.p[v] + xo);
      if (E.accmode == ACC_INIT || E.has_v) l2_prefetch(pre.p[v] + xo);
    }
  }
  double r[NRGPU_NV];
  bssn_point<ORD, CSY, CSZ>(U, P, p, r);
  double s = 0.0;
#pragma unroll
  for (int v = 0; v < NRGPU_NV; ++v) s += r[v];
  if (!isfinite(s)) atomicOr(status, 1);
  store(r, xo, out, pre, acc, E, p);
}

// planes klo..khi of a box's nv input lists into the staging buffer with
// strides (1, P, P P): field v at pad + v fs, point (i, j, k) at
// i + P (j + P k)
template <class CP>
__global__ void pad_copy_kernel(CP U, double *__restrict__ pad, BoxGeo box, int P, long fs, int klo, int khi) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long mn = (long)box.m * box.n;
  if (t >= mn * (khi - klo + 1)) return;
  const int v = blockIdx.y;
  const int i = (int)(t % box.m), j = (int)((t / box.m) % box.n), k = klo + (int)(t / mn);
  pad[v * fs + i + (long)P * (j + (long)P * k)] = ldg(U.p[v] + box.noffset + i + mn * k + (long)box.m * j);
}

// the points of the order ladder (flag 0, within 2 of a box face, sorted by
// that distance; the launch covers those below the full order's reach):
// 2nd order one point in, 4th two points in for 6th-order runs, as
// boundaryNaway/boundaryNormore select them (bam_amr_loops_box.h:215-220); a
// flag-0 point on a face has no stencil at all and is refused
__global__ void bssn_ladder_kernel(CVarPtrs U, VarPtrs out, CVarPtrs pre, VarPtrs acc, Epilogue E,
                                   const nrgpu_bssn_params p, const FlagPoint *__restrict__ pts, int n,
                                   const BoxGeo *__restrict__ boxes, double dx, double dy, double dz, int *status,
                                   int k0, int k1) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const FlagPoint fp = pts[t];
  if (fp.k < k0 || fp.k > k1) return;
  const BoxGeo b = boxes[fp.box];
  PointCtx P;
  P.i = fp.i; P.j = fp.j; P.k = fp.k;
  P.imax = b.m - 1; P.jmax = b.n - 1; P.kmax = b.o - 1;
  P.st[0] = 1; P.st[1] = b.m; P.st[2] = b.m * b.n;
  P.ijk = fp.ijk;
  P.h[0] = dx; P.h[1] = dy; P.h[2] = dz;
  P.dist = fp.flag;
  const int oc = ladder(p.order_centered, P.dist);
  if (oc == 0 || oc != ladder(p.order_advection, P.dist)) {
    atomicOr(status + 1, 1);
    return;
  }
  if (oc == p.order_centered) return;
  double r[NRGPU_NV];
  if (oc == 2) bssn_point<2>(U, P, p, r);
  else bssn_point<4>(U, P, p, r);
  double s = 0.0;
#pragma unroll
  for (int v = 0; v < NRGPU_NV; ++v) s += r[v];
  if (!isfinite(s)) atomicOr(status, 1);
  store(r, P.ijk, out, pre, acc, E, p);
}

// computedel of radiative.c:19-42 on clipped neighbours
__device__ __forceinline__ double computedel(const double *__restrict__ v, double w, int ccc, int mcc, int Mcc,
                                             int pcc, int Pcc) {
  if (w > 0) {
    if (Mcc != ccc) return 3.0 * ldg(v + ccc) + ldg(v + Mcc) - 4.0 * ldg(v + mcc);
    if (mcc != ccc) return ldg(v + pcc) - ldg(v + mcc);
    return 4.0 * ldg(v + pcc) - ldg(v + Pcc) - 3.0 * ldg(v + ccc);
  } else if (w < 0) {
    if (Pcc != ccc) return 4.0 * ldg(v + pcc) - ldg(v + Pcc) - 3.0 * ldg(v + ccc);
    if (mcc != ccc) return ldg(v + pcc) - ldg(v + mcc);
    return 3.0 * ldg(v + ccc) + ldg(v + Mcc) - 4.0 * ldg(v + mcc);
  } else {
    if (pcc != ccc && mcc != ccc) return ldg(v + pcc) - ldg(v + mcc);
    if (mcc == ccc) return 4.0 * ldg(v + pcc) - ldg(v + Pcc) - 3.0 * ldg(v + ccc);
    return 3.0 * ldg(v + ccc) + ldg(v + Mcc) - 4.0 * ldg(v + mcc);
  }
}

// one thread per (flagged point, variable): radiative rhs on PHYBOUND points
// (set_boundary_rot_rad, radiative.c:105-300, rot = 0); other flags have a
// zero rhs, which in the RK epilogue leaves acc unchanged and sets vout = pre
__global__ void bssn_flagged_kernel(CVarPtrs U, VarPtrs out, CVarPtrs pre, VarPtrs acc, Epilogue E,
                                    const nrgpu_bssn_params p, const FlagPoint *__restrict__ pts, int npts,
                                    const BoxGeo *__restrict__ boxes, double dx, double dy, double dz) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * NRGPU_NV) return;
  const int v = t % NRGPU_NV;
  const FlagPoint fp = pts[t / NRGPU_NV];
  const int ccc = fp.ijk;
  if (fp.flag != NRGPU_PHYBOUND) {
    if (E.mode == EPI_RK) {
      if (E.accmode == ACC_INIT) acc.p[v][ccc] = ldg(pre.p[v] + ccc);
      else if (E.accmode == ACC_FINAL) out.p[v][ccc] = acc.p[v][ccc];
      if (E.has_v) out.p[v][ccc] = ldg(pre.p[v] + ccc);
    }
    return;
  }
  const BoxGeo b = boxes[fp.box];
  const int i = fp.i, j = fp.j, k = fp.k;
  const int di = 1, dj = b.m, dk = b.m * b.n;
  const int mcc = i > 0 ? ccc - di : ccc, pcc = i + 1 < b.m ? ccc + di : ccc;
  const int cmc = j > 0 ? ccc - dj : ccc, cpc = j + 1 < b.n ? ccc + dj : ccc;
  const int ccm = k > 0 ? ccc - dk : ccc, ccp = k + 1 < b.o ? ccc + dk : ccc;
  const int Mcc = i > 1 ? mcc - di : ccc, Pcc = i + 2 < b.m ? pcc + di : ccc;
  const int cMc = j > 1 ? cmc - dj : ccc, cPc = j + 2 < b.n ? cpc + dj : ccc;
  const int ccM = k > 1 ? ccm - dk : ccc, ccP = k + 2 < b.o ? ccp + dk : ccc;
  const double xx = b.x0 + i * dx, yy = b.y0 + j * dy, zz = b.z0 + k * dz;
  const double rr = sqrt(xx * xx + yy * yy + zz * zz);
  const double vv = p.bc_speed[v], var0 = p.bc_var0[v];
  const double *var = U.p[v];
  const double Wx = vv * xx / rr, Wy = vv * yy / rr, Wz = vv * zz / rr;
  const double delx = computedel(var, Wx, ccc, mcc, Mcc, pcc, Pcc);
  const double dely = computedel(var, Wy, ccc, cmc, cMc, cpc, cPc);
  const double delz = computedel(var, Wz, ccc, ccm, ccM, ccp, ccP);
  double rhs = -vv * (ldg(var + ccc) - var0) / rr;
  rhs += -(Wx * delx * (1.0 / (2.0 * dx)) + Wy * dely * (1.0 / (2.0 * dy)) + Wz * delz * (1.0 / (2.0 * dz)));
  if (E.mode == EPI_RHS) out.p[v][ccc] = rhs;
  else if (E.mode == EPI_ADDLINEAR) out.p[v][ccc] = ldg(pre.p[v] + ccc) + E.c * rhs;
  else if (E.accmode == ACC_FINAL) out.p[v][ccc] = acc.p[v][ccc] + E.wacc * rhs;
  else if (E.accmode == ACC_INIT) {
    const double u0 = ldg(pre.p[v] + ccc);
    acc.p[v][ccc] = u0 + E.wacc * rhs;
    if (E.has_v) out.p[v][ccc] = u0 + E.cv * rhs;
  } else {
    acc.p[v][ccc] += E.wacc * rhs;
    if (E.has_v) out.p[v][ccc] = ldg(pre.p[v] + ccc) + E.cv * rhs;
  }
}

// bssn_algcon (bssn_algcon.c:25-230) on the points q0 <= q < q1
__global__ void bssn_algcon_kernel(VarPtrs u, int q0, int q1, int subtractA, int normalizedetg) {
  const int q = q0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= q1) return;
  double g[6], A[6];
#pragma unroll
  for (int v = 0; v < 6; ++v) { g[v] = u.p[G11 + v][q]; A[v] = u.p[A11 + v][q]; }
  double detg = g[0] * g[3] * g[5] + 2.0 * g[1] * g[2] * g[4] - g[0] * g[4] * g[4] - g[3] * g[2] * g[2] -
                g[5] * g[1] * g[1];
  if (normalizedetg) {
    const double eps = detg - 1.0;
    const double aux = fabs(eps) < 1e-12 ? 1.0 - eps / 3.0 : 1.0 / cbrt(detg);
#pragma unroll
    for (int v = 0; v < 6; ++v) g[v] *= aux;
    detg = g[0] * g[3] * g[5] + 2.0 * g[1] * g[2] * g[4] - g[0] * g[4] * g[4] - g[3] * g[2] * g[2] -
           g[5] * g[1] * g[1];
  }
  if (subtractA) {
    const double detginv = 1.0 / detg;
    const double gi0 = g[3] * g[5] - g[4] * g[4], gi1 = g[2] * g[4] - g[1] * g[5],
                 gi2 = g[1] * g[4] - g[2] * g[3], gi3 = g[0] * g[5] - g[2] * g[2],
                 gi4 = g[1] * g[2] - g[0] * g[4], gi5 = g[0] * g[3] - g[1] * g[1];
    const double trA = detginv * (gi0 * A[0] + gi3 * A[3] + gi5 * A[5] + 2.0 * (gi1 * A[1] + gi2 * A[2] + gi4 * A[4]));
    const double aux = -trA / 3.0;
#pragma unroll
    for (int v = 0; v < 6; ++v) A[v] += aux * g[v];
  }
#pragma unroll
  for (int v = 0; v < 6; ++v) { u.p[G11 + v][q] = g[v]; u.p[A11 + v][q] = A[v]; }
}

// r = a x + b y for n variables (vladd, variables.c:650)
__global__ void vladd_kernel(VarPtrs r, CVarPtrs xv, CVarPtrs yv, double a, double b, int nvars, int npoints) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)nvars * npoints) return;
  const int v = (int)(t / npoints), q = (int)(t % npoints);
  double s = 0.0;
  if (a != 0.0) s = a * xv.p[v][q];
  if (b != 0.0) s += b * yv.p[v][q];
  r.p[v][q] = s;
}

// copy 24 variables (vlcopy, variables.c:575)
__global__ void vlcopy_kernel(VarPtrs dst, CVarPtrs src, int npoints) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)NRGPU_NV * npoints) return;
  const int v = (int)(t / npoints), q = (int)(t % npoints);
  dst.p[v][q] = src.p[v][q];
}


#include "nrgpu_z4.cuh"
#include "nrgpu_bssn_tile.cuh"

}  // namespace

// set_boundary_symmetry (symmetry.c:93-140) as one pass over the symmetry
// ghosts: each takes its mirror image's value times the variable's parity
// under the reflected axes (the reference reflects axis after axis; the
// product of the parities gives the same values, negation being exact)
struct SymVars {
  double *p[NRGPU_Z4_NVARS];
};
struct SymParity {
  signed char s[NRGPU_Z4_NVARS][3];
};
__global__ void symmetry_kernel(SymVars u, int nv, SymParity par, const SymPoint *__restrict__ pts, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nv) return;
  const int v = t % nv;
  const SymPoint sp = pts[t / nv];
  int sign = 1;
#pragma unroll
  for (int a = 0; a < 3; ++a)
    if (sp.mask >> a & 1) sign *= par.s[v][a];
  const double x = u.p[v][sp.src];
  u.p[v][sp.dst] = sign < 0 ? -x : x;
}

// ---- host side ----------------------------------------------------------------
// the RK-stage updates of the fused epilogue (store(), EPI_RK) from a stored
// rhs list, at every point: the unfused stages of a symmetry grid
__global__ void rk_update_kernel(SymVars r, SymVars out, SymVars pre, SymVars acc, Epilogue E, int nv, long np) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= np * nv) return;
  const int v = (int)(t / np);
  const long x = t - (long)v * np;
  const double rv = r.p[v][x];
  if (E.accmode == ACC_FINAL) {
    out.p[v][x] = acc.p[v][x] + E.wacc * rv;
  } else if (E.accmode == ACC_INIT) {
    const double u0 = pre.p[v][x];
    acc.p[v][x] = u0 + E.wacc * rv;
    if (E.has_v) out.p[v][x] = u0 + E.cv * rv;
  } else {
    acc.p[v][x] += E.wacc * rv;
    if (E.has_v) out.p[v][x] = pre.p[v][x] + E.cv * rv;
  }
}

// the rhs list of a symmetry grid's unfused stages (first use, zeroed: points
// without a rhs keep 0, as the reference's evolution lists do)
static int sym_rhs_list(nrgpu_level *L, int nv, SymVars *R) {
  const size_t np = (size_t)L->npoints;
  if (!L->rsym) {
    if (cudaMalloc(&L->rsym, sizeof(double) * NRGPU_Z4_NVARS * np) != cudaSuccess) {
      L->rsym = nullptr;
      cudaGetLastError();
      return nrgpu_set_error(NRGPU_ERR_NOMEM, "symmetry rhs list of %zu points", np);
    }
    NRGPU_CUDA_TRY(cudaMemset(L->rsym, 0, sizeof(double) * NRGPU_Z4_NVARS * np));
  }
  for (int v = 0; v < NRGPU_Z4_NVARS; ++v) R->p[v] = v < nv ? L->rsym + v * np : nullptr;
  return NRGPU_OK;
}

static SymVars sym_vars(double *const *u, int nv) {
  SymVars S;
  for (int v = 0; v < NRGPU_Z4_NVARS; ++v) S.p[v] = v < nv ? u[v] : nullptr;
  return S;
}

// the parity of each variable of a system under x -> -x, y -> -y, z -> -z:
// VarSymmetry (variables.c) of the AddVar index strings, "ij+ji" for g~ and
// A~ (xx xy xz yy yz zz), "I" for Gamma~, beta and B, scalars otherwise
static SymParity parity_table(int system) {
  SymParity P;
  const int nv = system == NRGPU_SYSTEM_BSSN ? NRGPU_NV : NRGPU_Z4_NVARS;
  static const int ij[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  // first variable of g~, A~, Gamma~, beta, B in each list
  const int g = 0, A = 7, G = 14, beta = system == NRGPU_SYSTEM_BSSN ? 18 : 19,
            B = system == NRGPU_SYSTEM_BSSN ? 21 : 22;
  for (int v = 0; v < NRGPU_Z4_NVARS; ++v)
    for (int a = 0; a < 3; ++a) P.s[v][a] = 1;
  for (int v = 0; v < nv; ++v)
    for (int a = 0; a < 3; ++a) {
      int s = 1;
      if (v >= g && v < g + 6) s = (ij[v - g][0] == a ? -1 : 1) * (ij[v - g][1] == a ? -1 : 1);
      else if (v >= A && v < A + 6) s = (ij[v - A][0] == a ? -1 : 1) * (ij[v - A][1] == a ? -1 : 1);
      else if (v >= G && v < G + 3) s = v - G == a ? -1 : 1;
      else if (v >= beta && v < beta + 3) s = v - beta == a ? -1 : 1;
      else if (v >= B && v < B + 3) s = v - B == a ? -1 : 1;
      P.s[v][a] = (signed char)s;
    }
  return P;
}

int nrgpu_level_symmetry(nrgpu_level *L, double *const *u, int system, cudaStream_t st) {
  if (!L->nsym) return NRGPU_OK;
  const int nv = system == NRGPU_SYSTEM_BSSN ? NRGPU_NV : NRGPU_Z4_NVARS;
  SymVars U;
  for (int v = 0; v < NRGPU_Z4_NVARS; ++v) U.p[v] = v < nv ? u[v] : nullptr;
  const long n = (long)L->nsym * nv;
  symmetry_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(U, nv, parity_table(system), L->d_sym, L->nsym);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

static int check_params(const nrgpu_bssn_params *p) {
  if (!p) return nrgpu_set_error(NRGPU_ERR_ARG, "null parameters");
  if (p->order_centered != 2 && p->order_centered != 4 && p->order_centered != 6)
    return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "order_centered %d not in {2,4,6}", p->order_centered);
  if (p->order_advection != p->order_centered)
    return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "order_advection %d != order_centered %d",
                           p->order_advection, p->order_centered);
  if (p->order_dissipation != 0 && p->order_dissipation != 4 && p->order_dissipation != 6)
    return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "order_dissipation %d not in {0,4,6}", p->order_dissipation);
  if (p->advection_lopsided < 0 || p->advection_lopsided > 2 || p->advection_lopsided6 < 0 ||
      p->advection_lopsided6 > 3)
    return nrgpu_set_error(NRGPU_ERR_ARG, "advection lopsidedness out of range");
  return NRGPU_OK;
}

static int fill_ptrs(VarPtrs *vp, double *const *src, const char *what) {
  if (!src) return nrgpu_set_error(NRGPU_ERR_ARG, "null %s list", what);
  for (int v = 0; v < NRGPU_NV; ++v) {
    if (!src[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null %s[%d]", what, v);
    vp->p[v] = src[v];
  }
  return NRGPU_OK;
}

static CVarPtrs cptrs(const VarPtrs &v) {
  CVarPtrs c;
  for (int i = 0; i < NRGPU_NV; ++i) c.p[i] = v.p[i];
  return c;
}

// ---- tensor maps of the staged tiles ----------------------------------------
// cuTensorMapEncodeTiled from the driver, looked up once (no link-time
// dependency on libcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn tma_encoder() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)f;
  });
  return fn;
}

// the maps of the last few (variable list, box) pairs a level launched on
struct TmaCacheEntry {
  const double *key[NRGPU_Z4_NVARS];
  int box, nv, valid;
  CUtensorMap m[NRGPU_Z4_NVARS];
};
struct TmaCache {
  int next;
  TmaCacheEntry e[8];
};

// one 3-D map per variable over box b of the level: (m, n, o) FP64 points,
// boxes of kBX x kBY x kBZ, zero fill outside the array
static int tma_maps(nrgpu_level *L, int b, const double *const *ptr, int nv, const CUtensorMap **out) {
  if (!L->tma_cache) {
    L->tma_cache = calloc(1, sizeof(TmaCache));
    if (!L->tma_cache) return nrgpu_set_error(NRGPU_ERR_NOMEM, "tensor-map cache");
  }
  TmaCache *C = (TmaCache *)L->tma_cache;
  for (int q = 0; q < 8; ++q) {
    TmaCacheEntry &E = C->e[q];
    if (!E.valid || E.box != b || E.nv != nv) continue;
    bool same = true;
    for (int v = 0; v < nv && same; ++v) same = E.key[v] == ptr[v];
    if (same) {
      *out = E.m;
      return NRGPU_OK;
    }
  }
  EncodeTiledFn enc = tma_encoder();
  if (!enc) return nrgpu_set_error(NRGPU_ERR_CUDA, "cuTensorMapEncodeTiled not available from the driver");
  TmaCacheEntry &E = C->e[C->next];
  C->next = (C->next + 1) % 8;
  E.valid = 0;
  const BoxGeo &bx = L->hbox[b];
  const cuuint64_t dims[3] = {(cuuint64_t)bx.m, (cuuint64_t)bx.n, (cuuint64_t)bx.o};
  const cuuint64_t strides[2] = {(cuuint64_t)bx.m * 8, (cuuint64_t)bx.m * bx.n * 8};
  const cuuint32_t box[3] = {kBX, kBY, kBZ}, es[3] = {1, 1, 1};
  for (int v = 0; v < nv; ++v) {
    const CUresult r = enc(&E.m[v], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, (void *)(ptr[v] + bx.noffset), dims, strides,
                           box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return nrgpu_set_error(NRGPU_ERR_CUDA, "cuTensorMapEncodeTiled: error %d", (int)r);
    E.key[v] = ptr[v];
  }
  E.box = b;
  E.nv = nv;
  E.valid = 1;
  *out = E.m;
  return NRGPU_OK;
}

// whether the staged-tile kernel covers box b with these parameters: runs of
// order 4 or 6 whose full-order taps stay within the halo of 3 (lopsided
// advection shifted by 1 or 2 at 4th order, centred 6th-order advection;
// the ladder points are computed apart), row and plane strides and every
// field's start on 16-byte boundaries (the copy engine's rule)
static bool tile_eligible(const nrgpu_level *L, int b, const double *const *ptr, int nv, int order, int lop,
                          int lop6) {
  const BoxGeo &bx = L->hbox[b];
  if (bx.m < 3 || bx.n < 3 || bx.o < 3 || (bx.m & 1)) return false;
  if (order == 2 || (order == 4 && (lop < 1 || lop > 2)) || (order == 6 && lop6 != 3)) return false;
  for (int v = 0; v < nv; ++v)
    if (((uintptr_t)(ptr[v] + bx.noffset)) & 15) return false;
  return true;
}

static int launch_bssn_tile(nrgpu_level *L, int b, const CUtensorMap *maps, const CVarPtrs &U, const VarPtrs &out,
                            const CVarPtrs &pre, const VarPtrs &acc, const Epilogue &E, const nrgpu_bssn_params &p,
                            cudaStream_t st, int k0, int k1) {
  const BoxGeo &bx = L->hbox[b];
  BssnMaps M;
  memcpy(M.m, maps, sizeof M.m);
  const int ntiles = ((bx.m - 2 + kTX - 1) / kTX) * ((bx.n - 2 + kTY - 1) / kTY) * ((k1 - k0 + kTZ) / kTZ);
  // L->tile 1: one block per tile; 2: the persistent form, one block per SM
  const bool pers = L->tile == 2;
  const int grid = pers ? (ntiles < L->nsm ? ntiles : L->nsm) : ntiles;
  static std::once_flag attr;
  std::call_once(attr, [] {
    cudaFuncSetAttribute(bssn_rhs_tile_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmem);
    cudaFuncSetAttribute(bssn_rhs_tile_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTileSmem);
    cudaFuncSetAttribute(bssn_rhs_tile_persistent_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kTileSmem);
    cudaFuncSetAttribute(bssn_rhs_tile_persistent_kernel<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)kTileSmem);
  });
#define NR_TILE_LAUNCH(K_)                                                                                     \
  K_<<<grid, kTileThreads, kTileSmem, st>>>(M, U, out, pre, acc, E, p, bx, L->d_boundary, L->dx, L->dy, L->dz, \
                                            L->d_status, k0, k1)
  if (p.order_centered <= 4) {
    if (pers) NR_TILE_LAUNCH(bssn_rhs_tile_persistent_kernel<4>);
    else NR_TILE_LAUNCH(bssn_rhs_tile_kernel<4>);
  } else {
    if (pers) NR_TILE_LAUNCH(bssn_rhs_tile_persistent_kernel<6>);
    else NR_TILE_LAUNCH(bssn_rhs_tile_kernel<6>);
  }
#undef NR_TILE_LAUNCH
  return NRGPU_OK;
}

// launch the interior and flagged kernels of one rhs evaluation
// (kb <= k <= ke: the planes of the interior launch, whole boxes by default)
static int launch_rhs(nrgpu_level *L, const CVarPtrs &U, const VarPtrs &out, const CVarPtrs &pre, const VarPtrs &acc,
                      const Epilogue &E, const nrgpu_bssn_params &p, cudaStream_t st, bool interior, bool flagged,
                      int kb = 1, int ke = 1 << 30) {
  // with both parts, the boundary kernel runs on the level's side stream,
  // launched after the interior kernel so that its blocks fill the
  // interior kernel's last wave; they write disjoint points
  const bool fork = interior && flagged && L->nflagpts > 0;
  if (fork) {
    int e = nrgpu_level_side(L);
    if (e) return e;
    NRGPU_CUDA_TRY(cudaEventRecord(L->ev_fork, st));
    NRGPU_CUDA_TRY(cudaStreamWaitEvent(L->side, L->ev_fork, 0));
  }
  if (interior) {
    // the staging buffer of off-size boxes, allocated here unless a graph
    // is being captured (the refinement driver allocates it beforehand)
    if (!L->pad_tried) {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) nrgpu_level_pad(L);
      cudaGetLastError();
    }
    for (int b = 0; b < L->nboxes; ++b) {
      const BoxGeo &bx = L->hbox[b];
      if (bx.m < 3 || bx.n < 3 || bx.o < 3) continue;
      const int k0 = max(kb, 1), k1 = min(ke, bx.o - 2);
      if (k1 < k0) continue;
      if (L->tile && tile_eligible(L, b, U.p, NRGPU_NV, p.order_centered, p.advection_lopsided,
                                   p.advection_lopsided6)) {
        const CUtensorMap *maps = nullptr;
        int e = tma_maps(L, b, U.p, NRGPU_NV, &maps);
        if (e) return e;
        if ((e = launch_bssn_tile(L, b, maps, U, out, pre, acc, E, p, st, k0, k1))) return e;
        continue;
      }
      // the block shape of the level (32 x 4 x 1, or what nrgpu_level_autotune
      // measured fastest for this box); 128 or 256 threads, one point each
      const dim3 blk(L->blk[0], L->blk[1], L->blk[2]);
      const dim3 grd((bx.m - 2 + blk.x - 1) / blk.x, (bx.n - 2 + blk.y - 1) / blk.y, (k1 - k0 + blk.z) / blk.z);
      // box strides as compile-time constants (every stencil tap becomes one
      // load with an immediate offset) for the box sizes of kPadSizes; a box
      // of another size up to the largest is staged into the level's padding
      // buffer with the strides of the next one (as for Z4c); run-time
      // strides otherwise; one kernel per stencil order
      const int ord = p.order_centered;
      CVarPtrs In = U;
      int3 in = make_int3(bx.noffset, bx.m, bx.n);
      int P = ord >= 4 && bx.m == bx.n ? bx.m : 0;
      const int Q = ord >= 4 ? nrgpu_pad_size(bx.m, bx.n) : 0;
      if (Q && L->pad) {
        const long fs = (long)Q * Q * bx.o;
        P = 0;
        if ((size_t)(NRGPU_NV * fs) <= L->pad_doubles) {
          // the planes the launch's stencils reach (a launch on some planes:
          // the host-buffer step's slabs)
          const int H = max(max(p.order_advection, p.order_centered / 2 + 1), p.order_dissipation / 2 + 1);
          const int klo = max(0, k0 - H), khi = min(bx.o - 1, k1 + H);
          const long nb = (long)bx.m * bx.n * (khi - klo + 1);
          pad_copy_kernel<<<dim3((unsigned)((nb + 255) / 256), NRGPU_NV), 256, 0, st>>>(U, L->pad, bx, Q, fs, klo,
                                                                                        khi);
          for (int v = 0; v < NRGPU_NV; ++v) In.p[v] = L->pad + v * fs;
          in = make_int3(0, Q, Q);
          P = Q;
        }
      }
#define NR_BSSN_LDG(CSY_, CSZ_, ORD_)                                                                          \
  bssn_rhs_kernel<CSY_, CSZ_, ORD_><<<grd, blk, 0, st>>>(In, out, pre, acc, E, p, bx, L->d_boundary, L->dx, L->dy, \
                                                        L->dz, L->d_status, k0, k1, in)
#define NR_BSSN_SIZE(M_)                          \
  else if (P == M_ && ord == 4) NR_BSSN_LDG(M_, M_ * M_, 4); \
  else if (P == M_ && ord == 6) NR_BSSN_LDG(M_, M_ * M_, 6);
      if (false) {
      }
      NR_BSSN_SIZE(66) NR_BSSN_SIZE(72) NR_BSSN_SIZE(104) NR_BSSN_SIZE(136) NR_BSSN_SIZE(162) NR_BSSN_SIZE(168)
      NR_BSSN_SIZE(194)
      else if (ord == 2) bssn_rhs_kernel<0, 0, 2><<<grd, blk, 0, st>>>(U, out, pre, acc, E, p, bx, L->d_boundary,
                                                                       L->dx, L->dy, L->dz, L->d_status, k0, k1,
                                                                       make_int3(bx.noffset, bx.m, bx.n));
      else if (ord == 4) bssn_rhs_kernel<0, 0, 4><<<grd, blk, 0, st>>>(U, out, pre, acc, E, p, bx, L->d_boundary,
                                                                       L->dx, L->dy, L->dz, L->d_status, k0, k1,
                                                                       make_int3(bx.noffset, bx.m, bx.n));
      else bssn_rhs_kernel<0, 0, 6><<<grd, blk, 0, st>>>(U, out, pre, acc, E, p, bx, L->d_boundary, L->dx, L->dy,
                                                         L->dz, L->d_status, k0, k1, make_int3(bx.noffset, bx.m, bx.n));
#undef NR_BSSN_SIZE
#undef NR_BSSN_LDG
    }
    // the ladder points of all boxes (beside the interior kernel)
    const int nlad = L->nladder[p.order_centered / 2 - 1];
    if (nlad > 0)
      bssn_ladder_kernel<<<(nlad + 127) / 128, 128, 0, fork ? L->side : st>>>(
          U, out, pre, acc, E, p, L->d_ladder, nlad, L->d_box, L->dx, L->dy, L->dz, L->d_status, kb, ke);
  }
  if (flagged && L->nflagpts > 0) {
    const int n = L->nflagpts * NRGPU_NV;
    bssn_flagged_kernel<<<(n + 255) / 256, 256, 0, fork ? L->side : st>>>(U, out, pre, acc, E, p, L->d_flagpts,
                                                                           L->nflagpts, L->d_box, L->dx, L->dy,
                                                                           L->dz);
  }
  if (fork) {
    NRGPU_CUDA_TRY(cudaEventRecord(L->ev_join, L->side));
    NRGPU_CUDA_TRY(cudaStreamWaitEvent(st, L->ev_join, 0));
  }
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_bssn_rhs(nrgpu_level *L, double *const *unew, double *const *upre, double c,
                              double *const *ucur, const nrgpu_bssn_params *p, void *stream) {
  if (!L) return nrgpu_set_error(NRGPU_ERR_ARG, "null level");
  int e;
  if ((e = check_params(p))) return e;
  VarPtrs n, pr, cu;
  if ((e = fill_ptrs(&n, unew, "unew")) || (e = fill_ptrs(&cu, ucur, "ucur"))) return e;
  if (c != 0.0) {
    if ((e = fill_ptrs(&pr, upre, "upre"))) return e;
  } else {
    pr = cu;
  }
  Epilogue E = {c != 0.0 ? EPI_ADDLINEAR : EPI_RHS, c, 0.0, 0.0, 0};
  return launch_rhs(L, cptrs(cu), n, cptrs(pr), n, E, *p, (cudaStream_t)stream, true, false);
}

extern "C" int nrgpu_bssn_boundary(nrgpu_level *L, double *const *unew, double *const *upre, double c,
                                   double *const *ucur, const nrgpu_bssn_params *p, void *stream) {
  if (!L) return nrgpu_set_error(NRGPU_ERR_ARG, "null level");
  if (!p) return nrgpu_set_error(NRGPU_ERR_ARG, "null parameters");
  int e;
  VarPtrs n, pr, cu;
  if ((e = fill_ptrs(&n, unew, "unew")) || (e = fill_ptrs(&cu, ucur, "ucur"))) return e;
  if (c != 0.0) {
    if ((e = fill_ptrs(&pr, upre, "upre"))) return e;
  } else {
    pr = cu;
  }
  Epilogue E = {c != 0.0 ? EPI_ADDLINEAR : EPI_RHS, c, 0.0, 0.0, 0};
  if ((e = launch_rhs(L, cptrs(cu), n, cptrs(pr), n, E, *p, (cudaStream_t)stream, false, true))) return e;
  return nrgpu_level_symmetry(L, unew, NRGPU_SYSTEM_BSSN, (cudaStream_t)stream);
}

extern "C" int nrgpu_bssn_algcon(nrgpu_level *L, double *const *u, const nrgpu_bssn_params *p, void *stream) {
  if (!L || !p) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  int e;
  VarPtrs uu;
  if ((e = fill_ptrs(&uu, u, "u"))) return e;
  bssn_algcon_kernel<<<(L->npoints + 255) / 256, 256, 0, (cudaStream_t)stream>>>(uu, 0, L->npoints, p->subtractA,
                                                                                  p->normalizedetg);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_vladd(nrgpu_level *L, int nvars, double *const *r, double a, double *const *x, double b,
                           double *const *y, void *stream) {
  if (!L || !r || nvars < 1 || nvars > NRGPU_NV) return nrgpu_set_error(NRGPU_ERR_ARG, "bad vladd arguments");
  VarPtrs rr = {}, xx = {}, yy = {};
  for (int v = 0; v < nvars; ++v) {
    rr.p[v] = r[v];
    if (a != 0.0) {
      if (!x || !x[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null x");
      xx.p[v] = x[v];
    }
    if (b != 0.0) {
      if (!y || !y[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null y");
      yy.p[v] = y[v];
    }
  }
  const long n = (long)nvars * L->npoints;
  vladd_kernel<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(rr, cptrs(xx), cptrs(yy), a, b, nvars,
                                                                              L->npoints);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

int nrgpu_level_scratch(nrgpu_level *L, double **out);

// The RK4 step of rk.c:220-257 without a copy of u: u itself is the stage
// input of stage 1 and the "P" of every stage (only read until stage 4);
// stage 1 initialises the accumulator A = u + dt/6 r1, stages 2-3 add to it,
// and stage 4 writes u = A + dt/6 r4.  Per point the floating-point
// operations are those of P + c r and u += w r in the reference's order.
struct RkLists {
  VarPtrs U, A, V1, V2;
};

static RkLists rk_lists(const VarPtrs &U, double *scr, long np) {
  RkLists R;
  R.U = U;
  for (int v = 0; v < NRGPU_NV; ++v) {
    R.A.p[v] = scr + (0 * NRGPU_NV + v) * np;
    R.V1.p[v] = scr + (1 * NRGPU_NV + v) * np;
    R.V2.p[v] = scr + (2 * NRGPU_NV + v) * np;
  }
  return R;
}

// stage sg (0..3) of the step, on the planes kb..ke of the interior and/or
// the flagged points
// the epilogue of RK4 stage sg (rk.c:231-255: weights dt/6, dt/3, dt/3,
// dt/6 into u, dt/2, dt/2, dt into the next stage input)
static Epilogue stage_epilogue(int sg, double dt) {
  switch (sg) {
    case 0: return Epilogue{EPI_RK, 0.0, dt / 6, dt / 2, 1, ACC_INIT};
    case 1: return Epilogue{EPI_RK, 0.0, dt / 3, dt / 2, 1, ACC_ADD};
    case 2: return Epilogue{EPI_RK, 0.0, dt / 3, dt, 1, ACC_ADD};
    default: return Epilogue{EPI_RK, 0.0, dt / 6, 0.0, 0, ACC_FINAL};
  }
}

static int rk_stage_parts(nrgpu_level *L, const RkLists &R, int sg, double dt, const nrgpu_bssn_params &p,
                          cudaStream_t st, bool interior, bool flagged, int kb, int ke) {
  const CVarPtrs cU = cptrs(R.U);
  const Epilogue E = stage_epilogue(sg, dt);
  switch (sg) {
    case 0: return launch_rhs(L, cU, R.V1, cU, R.A, E, p, st, interior, flagged, kb, ke);
    case 1: return launch_rhs(L, cptrs(R.V1), R.V2, cU, R.A, E, p, st, interior, flagged, kb, ke);
    case 2: return launch_rhs(L, cptrs(R.V2), R.V1, cU, R.A, E, p, st, interior, flagged, kb, ke);
    default: return launch_rhs(L, cptrs(R.V1), R.U, cU, R.A, E, p, st, interior, flagged, kb, ke);
  }
}

// a stage, or part of one; after a whole stage the symmetry ghosts of its
// output (the next stage's input, or u after the last) are reflected, which
// gives the reference's values: it reflects the rhs (set_boundary), and the
// RK updates are linear
static int rk_stage(nrgpu_level *L, const RkLists &R, int sg, double dt, const nrgpu_bssn_params &p,
                    cudaStream_t st, bool interior, bool flagged, int kb = 1, int ke = 1 << 30) {
  if (!L->nsym) return rk_stage_parts(L, R, sg, dt, p, st, interior, flagged, kb, ke);
  // a symmetry grid: the reference's order, unfused: the rhs of the stage
  // input, its radiative boundary and its reflection (set_boundary,
  // boundary.c:221), then the updates of evolve_rk_rk4 at every point
  const VarPtrs &in = sg == 0 ? R.U : (sg == 2 ? R.V2 : R.V1);
  const VarPtrs &out = sg == 0 || sg == 2 ? R.V1 : (sg == 1 ? R.V2 : R.U);
  const Epilogue E = stage_epilogue(sg, dt);
  SymVars RS;
  int e = sym_rhs_list(L, NRGPU_NV, &RS);
  if (e) return e;
  VarPtrs Rp;
  for (int v = 0; v < NRGPU_NV; ++v) Rp.p[v] = RS.p[v];
  const Epilogue Er = {EPI_RHS, 0.0, 0.0, 0.0, 0, 0};
  if ((e = launch_rhs(L, cptrs(in), Rp, cptrs(in), Rp, Er, p, st, true, true))) return e;
  if ((e = nrgpu_level_symmetry(L, Rp.p, NRGPU_SYSTEM_BSSN, st))) return e;
  const long n = (long)NRGPU_NV * L->npoints;
  rk_update_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(RS, sym_vars(out.p, NRGPU_NV),
                                                                sym_vars(R.U.p, NRGPU_NV), sym_vars(R.A.p, NRGPU_NV),
                                                                E, NRGPU_NV, L->npoints);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

// fused RK4 (rk.c:220-257): stage s reads V_in, adds w_s*r to u and writes
// V_out = P + c_s*r; both the interior and the flagged kernels do it
// the four RK4 stages of evolve_rk_rk4 (rk.c:220-257) without the algebraic
// constraints; the mesh-refinement driver puts the time interpolation between
int nrgpu_bssn_rk4_stages(nrgpu_level *L, double *const *u, double dt, const nrgpu_bssn_params *p,
                          cudaStream_t st) {
  if (!L) return nrgpu_set_error(NRGPU_ERR_ARG, "null level");
  int e;
  if ((e = check_params(p))) return e;
  VarPtrs U;
  if ((e = fill_ptrs(&U, u, "u"))) return e;
  double *scr = nullptr;
  if ((e = nrgpu_level_scratch(L, &scr))) return e;
  RkLists R = rk_lists(U, scr, L->npoints);
  for (int sg = 0; sg < 4; ++sg)
    if ((e = rk_stage(L, R, sg, dt, *p, st, true, true))) return e;
  return NRGPU_OK;
}

extern "C" int nrgpu_bssn_rk4_step(nrgpu_level *L, double *const *u, double dt, const nrgpu_bssn_params *p,
                                   void *stream) {
  int e = nrgpu_bssn_rk4_stages(L, u, dt, p, (cudaStream_t)stream);
  if (e) return e;
  return nrgpu_bssn_algcon(L, u, p, stream);
}

// ---- steps on host buffers ------------------------------------------------------
// The state crosses PCIe once up before the first step and once down after
// the last.  On a single-box level the box is cut into NRGPU_HOST_SLABS z
// slabs: stage 1 of the first step runs on the planes of a slab as soon as
// the uploads cover its stencils (H planes past it), so the upload of the
// later slabs overlaps it; stage 4 of the last step, and the algebraic
// constraints, run slab by slab after the flagged points, and each slab's
// download overlaps the work on the slabs after it.  The per-point
// arithmetic is that of nrgpu_bssn_rk4_step.
static int host_streams(nrgpu_level *L) {
  if (L->hs_comp) return NRGPU_OK;
  // blocking streams: ordered after earlier work on the legacy default stream
  NRGPU_CUDA_TRY(cudaStreamCreate(&L->hs_copy));
  NRGPU_CUDA_TRY(cudaStreamCreate(&L->hs_comp));
  for (int q = 0; q < NRGPU_HOST_SLABS; ++q) {
    NRGPU_CUDA_TRY(cudaEventCreateWithFlags(&L->hev_in[q], cudaEventDisableTiming));
    NRGPU_CUDA_TRY(cudaEventCreateWithFlags(&L->hev_out[q], cudaEventDisableTiming));
  }
  return NRGPU_OK;
}

// planes [off, off + n) of the 24 variables between the device state (pitch
// np) and the host arrays: one 2D copy when the host arrays lie at one
// pitch (hpitch > 0 bytes: a (24, np) array or rows of a larger one), else
// one copy per variable (each cudaMemcpyAsync costs a few microseconds, so
// the slabs are only used with the 2D form)
static int copy_planes(double *dev, double *const *host, long hpitch, long np, long off, long n, bool up,
                       cudaStream_t st) {
  const cudaMemcpyKind kind = up ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
  if (hpitch > 0) {
    double *h0 = host[0] + off, *d0 = dev + off;
    if (cudaMemcpy2DAsync(up ? (void *)d0 : (void *)h0, up ? np * sizeof(double) : (size_t)hpitch,
                          up ? (const void *)h0 : (const void *)d0, up ? (size_t)hpitch : np * sizeof(double),
                          n * sizeof(double), NRGPU_NV, kind, st) != cudaSuccess)
      return nrgpu_set_error(NRGPU_ERR_CUDA, "%s of planes", up ? "upload" : "download");
    return NRGPU_OK;
  }
  for (int v = 0; v < NRGPU_NV; ++v) {
    double *h = host[v] + off, *d = dev + v * np + off;
    if (cudaMemcpyAsync(up ? (void *)d : (void *)h, up ? (const void *)h : (const void *)d, sizeof(double) * n, kind,
                        st) != cudaSuccess)
      return nrgpu_set_error(NRGPU_ERR_CUDA, "%s of variable %d", up ? "upload" : "download", v);
  }
  return NRGPU_OK;
}

// the common pitch in bytes of the host arrays, or 0
static long host_pitch(double *const *host, long np) {
  const long pb = (long)((const char *)host[1] - (const char *)host[0]);
  if (pb < np * (long)sizeof(double) || pb >= (1L << 31) || pb % sizeof(double)) return 0;
  for (int v = 2; v < NRGPU_NV; ++v)
    if ((const char *)host[v] - (const char *)host[0] != pb * v) return 0;
  return pb;
}

extern "C" int nrgpu_bssn_evolve_host(nrgpu_level *L, double *const *host_u, int nsteps, double dt,
                                      const nrgpu_bssn_params *p) {
  if (!L || !host_u || nsteps < 0) return nrgpu_set_error(NRGPU_ERR_ARG, "bad arguments");
  int e;
  if ((e = check_params(p))) return e;
  for (int v = 0; v < NRGPU_NV; ++v)
    if (!host_u[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null host_u[%d]", v);
  const long np = L->npoints;
  if (!L->hoststate && cudaMalloc(&L->hoststate, sizeof(double) * NRGPU_NV * np) != cudaSuccess) {
    L->hoststate = nullptr;
    cudaGetLastError();
    return nrgpu_set_error(NRGPU_ERR_NOMEM, "state of %ld points", np);
  }
  double *scr = nullptr;
  if ((e = nrgpu_level_scratch(L, &scr))) return e;
  if ((e = host_streams(L))) return e;
  const cudaStream_t cs = L->hs_copy, ks = L->hs_comp;
  VarPtrs U;
  for (int v = 0; v < NRGPU_NV; ++v) U.p[v] = L->hoststate + v * np;
  const RkLists R = rk_lists(U, scr, np);

  // slabs of ps planes; H = the stencils' reach in planes
  const BoxGeo &b0 = L->hbox[0];
  const long hp = host_pitch(host_u, np);
  const bool pipe = L->nboxes == 1 && b0.o >= 2 * NRGPU_HOST_SLABS && nsteps > 0 && hp > 0 && !L->nsym;
  const int ps = pipe ? (b0.o + NRGPU_HOST_SLABS - 1) / NRGPU_HOST_SLABS : b0.o;
  const int ns = pipe ? (b0.o + ps - 1) / ps : 1;
  const long mn = pipe ? (long)b0.m * b0.n : 0;
  const int H = max(max(p->order_advection, p->order_centered / 2 + 1), p->order_dissipation / 2 + 1);

  // upload (whole state when not pipelined)
  for (int q = 0; q < ns && !e; ++q) {
    const long off = pipe ? q * ps * mn : 0, n = pipe ? min(ps, b0.o - q * ps) * mn : np;
    if (!(e = copy_planes(L->hoststate, host_u, hp, np, off, n, true, cs)))
      if (cudaEventRecord(L->hev_in[q], cs) != cudaSuccess) e = nrgpu_set_error(NRGPU_ERR_CUDA, "event");
  }
  if (!e && nsteps == 0) e = copy_planes(L->hoststate, host_u, hp, np, 0, np, false, cs);

  int waited = -1;  // last upload slab the compute stream has waited for
  for (int t = 0; t < nsteps && !e; ++t) {
    const bool first = t == 0, last = t == nsteps - 1;
    // stage 1
    if (first && pipe) {
      for (int q = 0; q < ns && !e; ++q) {
        const int kb = q * ps, ke = min(b0.o, kb + ps) - 1;
        const int need = min(ns - 1, min(b0.o - 1, ke + H) / ps);
        for (; waited < need; ++waited) cudaStreamWaitEvent(ks, L->hev_in[waited + 1], 0);
        e = rk_stage(L, R, 0, dt, *p, ks, true, false, kb, ke);
      }
      for (; waited < ns - 1; ++waited) cudaStreamWaitEvent(ks, L->hev_in[waited + 1], 0);
      if (!e) e = rk_stage(L, R, 0, dt, *p, ks, false, true);
    } else {
      if (first) cudaStreamWaitEvent(ks, L->hev_in[0], 0);
      e = rk_stage(L, R, 0, dt, *p, ks, true, true);
    }
    for (int sg = 1; sg < 3 && !e; ++sg) e = rk_stage(L, R, sg, dt, *p, ks, true, true);
    if (e) break;
    // stage 4 and the algebraic constraints; the download
    if (last && pipe) {
      e = rk_stage(L, R, 3, dt, *p, ks, false, true);
      for (int q = 0; q < ns && !e; ++q) {
        const int kb = q * ps, ke = min(b0.o, kb + ps) - 1;
        if ((e = rk_stage(L, R, 3, dt, *p, ks, true, false, kb, ke))) break;
        const int q0 = (int)(kb * mn), q1 = (int)((ke + 1) * mn);
        bssn_algcon_kernel<<<(unsigned)((q1 - q0 + 255) / 256), 256, 0, ks>>>(U, q0, q1, p->subtractA,
                                                                              p->normalizedetg);
        if (cudaEventRecord(L->hev_out[q], ks) != cudaSuccess || cudaStreamWaitEvent(cs, L->hev_out[q], 0))
          e = nrgpu_set_error(NRGPU_ERR_CUDA, "event");
        else
          e = copy_planes(L->hoststate, host_u, hp, np, kb * mn, (ke + 1 - kb) * mn, false, cs);
      }
    } else {
      if (!(e = rk_stage(L, R, 3, dt, *p, ks, true, true))) {
        bssn_algcon_kernel<<<(unsigned)((np + 255) / 256), 256, 0, ks>>>(U, 0, (int)np, p->subtractA,
                                                                        p->normalizedetg);
        if (last) {
          if (cudaEventRecord(L->hev_out[0], ks) != cudaSuccess || cudaStreamWaitEvent(cs, L->hev_out[0], 0))
            e = nrgpu_set_error(NRGPU_ERR_CUDA, "event");
          else
            e = copy_planes(L->hoststate, host_u, hp, np, 0, np, false, cs);
        }
      }
    }
  }
  const cudaError_t c1 = cudaStreamSynchronize(ks), c2 = cudaStreamSynchronize(cs);
  if (!e && (c1 != cudaSuccess || c2 != cudaSuccess || cudaGetLastError() != cudaSuccess))
    e = nrgpu_set_error(NRGPU_ERR_CUDA, "host-buffer step: %s", cudaGetErrorString(c1 != cudaSuccess ? c1 : c2));
  return e;
}

// ---- allocation-free RK4 step -------------------------------------------------
// For callers that cannot allocate device memory themselves (a host code that
// runs inside a memory pool it does not own, or under a policy that forbids
// cudaMalloc after start-up): the RK4 step of one box with its three scratch
// lists in a fixed device array that the library image carries.
//
// Limit: NRGPU_NOALLOC_MAX_POINTS points per box (m*n*o), i.e.
// 3 * 24 * 16384 doubles = 9 MiB of device memory held by every GPU that
// loads the library, until the process exits.  All calls share the array:
// calls that overlap on the GPU (different streams, or host threads using the
// same device) race on it and must be serialised by the caller.
// g_noalloc_status collects, over all calls since it was last read, bit 0 of
// word 0 for a non-finite rhs and word 1 for an inner point without room for
// its stencil; nrgpu_bssn_noalloc_status reads and clears it.
#define NRGPU_NOALLOC_MAX_POINTS 16384
static __device__ __align__(256) double g_noalloc_scratch[3 * NRGPU_NV * NRGPU_NOALLOC_MAX_POINTS];
static __device__ __align__(256) int g_noalloc_status[4];

namespace {

// interior of a single box whose outer layer is the physical boundary
// (flag.c:23-36): every point with 1 <= i,j,k <= size-2 is an inner point
__global__ void __launch_bounds__(128) bssn_rhs_box_kernel(CVarPtrs U, VarPtrs out, CVarPtrs pre, VarPtrs acc,
                                                          Epilogue E, const nrgpu_bssn_params p, BoxGeo box,
                                                          double dx, double dy, double dz, int *status) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = 1 + blockIdx.z;
  if (i > box.m - 2 || j > box.n - 2 || k > box.o - 2) return;
  PointCtx P;
  P.i = i; P.j = j; P.k = k;
  P.imax = box.m - 1; P.jmax = box.n - 1; P.kmax = box.o - 1;
  P.st[0] = 1; P.st[1] = box.m; P.st[2] = box.m * box.n;
  P.ijk = box.noffset + i + box.m * (j + box.n * k);
  P.h[0] = dx; P.h[1] = dy; P.h[2] = dz;
  int d = min(min(i, j), k);
  d = min(d, min(min(P.imax - i, P.jmax - j), P.kmax - k));
  P.dist = d;
  const int oc = ladder(p.order_centered, d);
  if (oc == 0 || oc != ladder(p.order_advection, d)) {
    atomicOr(status + 1, 1);
    return;
  }
  double r[NRGPU_NV];
  if (oc == 2) bssn_point<2>(U, P, p, r);
  else if (oc == 4) bssn_point<4>(U, P, p, r);
  else bssn_point<6>(U, P, p, r);
  double s = 0.0;
#pragma unroll
  for (int v = 0; v < NRGPU_NV; ++v) s += r[v];
  if (!isfinite(s)) atomicOr(status, 1);
  store(r, P.ijk, out, pre, acc, E, p);
}

// radiative rhs on the outer layer of a single box, one thread per
// (point, variable); interior points return at once
__global__ void bssn_surface_kernel(CVarPtrs U, VarPtrs out, CVarPtrs pre, VarPtrs acc, Epilogue E,
                                    const nrgpu_bssn_params p, BoxGeo b, double dx, double dy, double dz) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long np = (long)b.m * b.n * b.o;
  if (t >= np * NRGPU_NV) return;
  const int v = (int)(t % NRGPU_NV);
  const int q = (int)(t / NRGPU_NV);
  const int i = q % b.m, j = (q / b.m) % b.n, k = q / (b.m * b.n);
  if (i > 0 && j > 0 && k > 0 && i < b.m - 1 && j < b.n - 1 && k < b.o - 1) return;
  const int ccc = b.noffset + q;
  const int di = 1, dj = b.m, dk = b.m * b.n;
  const int mcc = i > 0 ? ccc - di : ccc, pcc = i + 1 < b.m ? ccc + di : ccc;
  const int cmc = j > 0 ? ccc - dj : ccc, cpc = j + 1 < b.n ? ccc + dj : ccc;
  const int ccm = k > 0 ? ccc - dk : ccc, ccp = k + 1 < b.o ? ccc + dk : ccc;
  const int Mcc = i > 1 ? mcc - di : ccc, Pcc = i + 2 < b.m ? pcc + di : ccc;
  const int cMc = j > 1 ? cmc - dj : ccc, cPc = j + 2 < b.n ? cpc + dj : ccc;
  const int ccM = k > 1 ? ccm - dk : ccc, ccP = k + 2 < b.o ? ccp + dk : ccc;
  const double xx = b.x0 + i * dx, yy = b.y0 + j * dy, zz = b.z0 + k * dz;
  const double rr = sqrt(xx * xx + yy * yy + zz * zz);
  const double vv = p.bc_speed[v], var0 = p.bc_var0[v];
  const double *var = U.p[v];
  const double Wx = vv * xx / rr, Wy = vv * yy / rr, Wz = vv * zz / rr;
  const double delx = computedel(var, Wx, ccc, mcc, Mcc, pcc, Pcc);
  const double dely = computedel(var, Wy, ccc, cmc, cMc, cpc, cPc);
  const double delz = computedel(var, Wz, ccc, ccm, ccM, ccp, ccP);
  double rhs = -vv * (ldg(var + ccc) - var0) / rr;
  rhs += -(Wx * delx * (1.0 / (2.0 * dx)) + Wy * dely * (1.0 / (2.0 * dy)) + Wz * delz * (1.0 / (2.0 * dz)));
  acc.p[v][ccc] += E.wacc * rhs;
  if (E.has_v) out.p[v][ccc] = ldg(pre.p[v] + ccc) + E.cv * rhs;
}

}  // namespace

// device addresses of the static arrays, looked up once per device (under a
// lock, so that host threads making their first call at once do not race);
// a cudaDeviceReset between calls reloads the module and is not supported
static double *g_noalloc_ptr[64];
static int *g_noalloc_status_ptr[64];
static std::mutex g_noalloc_setup;

static int noalloc_setup(int *dev_out) {
  int dev = 0;
  NRGPU_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return nrgpu_set_error(NRGPU_ERR_ARG, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_setup);
  if (!g_noalloc_ptr[dev]) {
    // set-up on the first call on this device, with this device current
    void *sp = nullptr, *st = nullptr;
    NRGPU_CUDA_TRY(cudaGetSymbolAddress(&sp, g_noalloc_scratch));
    NRGPU_CUDA_TRY(cudaGetSymbolAddress(&st, g_noalloc_status));
    g_noalloc_status_ptr[dev] = (int *)st;
    g_noalloc_ptr[dev] = (double *)sp;
  }
  *dev_out = dev;
  return NRGPU_OK;
}

extern "C" int nrgpu_bssn_rk4_step_noalloc(const nrgpu_box *box, double dx, double dy, double dz,
                                           double *const *u, double dt, const nrgpu_bssn_params *p,
                                           void *stream) {
  if (!box) return nrgpu_set_error(NRGPU_ERR_ARG, "null box");
  int e;
  if ((e = check_params(p))) return e;
  VarPtrs U;
  if ((e = fill_ptrs(&U, u, "u"))) return e;
  if (box->m < 3 || box->n < 3 || box->o < 3 || box->noffset != 0)
    return nrgpu_set_error(NRGPU_ERR_ARG, "box must be at least 3^3 points with noffset 0");
  const long np = (long)box->m * box->n * box->o;
  if (np > NRGPU_NOALLOC_MAX_POINTS)
    return nrgpu_set_error(NRGPU_ERR_ARG, "box of %ld points exceeds the allocation-free limit of %d points", np,
                           NRGPU_NOALLOC_MAX_POINTS);
  if (!(dx > 0.0) || !(dy > 0.0) || !(dz > 0.0)) return nrgpu_set_error(NRGPU_ERR_ARG, "grid spacing must be > 0");
  int dev = 0;
  if ((e = noalloc_setup(&dev))) return e;
  double *scr = g_noalloc_ptr[dev];
  int *status = g_noalloc_status_ptr[dev];
  cudaStream_t s = (cudaStream_t)stream;
  VarPtrs P, V1, V2;
  for (int v = 0; v < NRGPU_NV; ++v) {
    P.p[v] = scr + (0 * NRGPU_NV + v) * np;
    V1.p[v] = scr + (1 * NRGPU_NV + v) * np;
    V2.p[v] = scr + (2 * NRGPU_NV + v) * np;
  }
  const BoxGeo bx{box->m, box->n, box->o, 0, box->x0, box->y0, box->z0};
  vlcopy_kernel<<<(unsigned)((NRGPU_NV * np + 255) / 256), 256, 0, s>>>(P, cptrs(U), (int)np);
  const CVarPtrs cP = cptrs(P);
  const Epilogue Es[4] = {{EPI_RK, 0.0, dt / 6, dt / 2, 1},
                          {EPI_RK, 0.0, dt / 3, dt / 2, 1},
                          {EPI_RK, 0.0, dt / 3, dt, 1},
                          {EPI_RK, 0.0, dt / 6, 0.0, 0}};
  const CVarPtrs ins[4] = {cP, cptrs(V1), cptrs(V2), cptrs(V1)};
  const VarPtrs outs[4] = {V1, V2, V1, V2};
  const dim3 blk(32, 4, 1), grd((box->m - 2 + 31) / 32, (box->n - 2 + 3) / 4, box->o - 2);
  const unsigned sgrid = (unsigned)((np * NRGPU_NV + 255) / 256);
  for (int st = 0; st < 4; ++st) {
    bssn_rhs_box_kernel<<<grd, blk, 0, s>>>(ins[st], outs[st], cP, U, Es[st], *p, bx, dx, dy, dz, status);
    bssn_surface_kernel<<<sgrid, 256, 0, s>>>(ins[st], outs[st], cP, U, Es[st], *p, bx, dx, dy, dz);
  }
  bssn_algcon_kernel<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(U, 0, (int)np, p->subtractA, p->normalizedetg);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

// the status of the allocation-free step: read on the caller's stream, then
// cleared; allocates nothing
extern "C" int nrgpu_bssn_noalloc_status(int *flag, void *stream) {
  if (!flag) return nrgpu_set_error(NRGPU_ERR_ARG, "null flag");
  int dev = 0, e;
  if ((e = noalloc_setup(&dev))) return e;
  int *status = g_noalloc_status_ptr[dev];
  cudaStream_t s = (cudaStream_t)stream;
  int h[2] = {0, 0};
  NRGPU_CUDA_TRY(cudaMemcpyAsync(h, status, sizeof h, cudaMemcpyDeviceToHost, s));
  NRGPU_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof h, s));
  NRGPU_CUDA_TRY(cudaStreamSynchronize(s));
  *flag = h[0] ? 1 : 0;
  if (h[1]) return nrgpu_set_error(NRGPU_ERR_ARG, "an inner point had no room for its stencil");
  return NRGPU_OK;
}

// ---- Z4c ---------------------------------------------------------------------
static int z4_check_params(const nrgpu_z4_params *p) {
  if (!p) return nrgpu_set_error(NRGPU_ERR_ARG, "null parameters");
  if (p->order_centered != 2 && p->order_centered != 4 && p->order_centered != 6)
    return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "order_centered %d not in {2,4,6}", p->order_centered);
  if (p->order_advection != p->order_centered)
    return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "order_advection %d != order_centered %d", p->order_advection,
                           p->order_centered);
  if (p->order_dissipation != 0 && p->order_dissipation != 4 && p->order_dissipation != 6)
    return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "order_dissipation %d not in {0,4,6}", p->order_dissipation);
  if (p->useNPTs) return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "z4_useNPTs = yes is not supported");
  if (p->precision < 0 || p->precision > 2) return nrgpu_set_error(NRGPU_ERR_ARG, "precision %d", p->precision);
  if (p->boundary < 0 || p->boundary > 2) return nrgpu_set_error(NRGPU_ERR_ARG, "boundary %d", p->boundary);
  if (p->advection_lopsided < 0 || p->advection_lopsided > 2 || p->advection_lopsided6 < 0 ||
      p->advection_lopsided6 > 3)
    return nrgpu_set_error(NRGPU_ERR_ARG, "advection lopsidedness out of range");
  return NRGPU_OK;
}

static int z4_fill(ZVarPtrs *vp, double *const *src, const char *what) {
  if (!src) return nrgpu_set_error(NRGPU_ERR_ARG, "null %s list", what);
  for (int v = 0; v < ZNV; ++v) {
    if (!src[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null %s[%d]", what, v);
    vp->p[v] = src[v];
  }
  return NRGPU_OK;
}
static ZCVarPtrs z4_c(const ZVarPtrs &v) {
  ZCVarPtrs c;
  for (int i = 0; i < ZNV; ++i) c.p[i] = v.p[i];
  return c;
}

// FP64 interior launch with compile-time strides for the box sizes of the
// workloads (66, 162, the finer levels of the batched refinement step, and
// 194, the coarsest level of the full form's grid).  A box of another size
// up to 194 points per side is staged first into the level's padding
// buffer with the strides of the next such size (nrgpu_level_pad), whose
// kernel then reads it: with run-time strides the kernel's tap addresses
// take registers of their own, it spills, and it runs about half as fast.
// Generic strides remain for larger boxes; one kernel per stencil order.
template <int ORD>
static void z4_interior_fp64(const ZCVarPtrs &U, const ZVarPtrs &out, const ZCVarPtrs &pre, const ZVarPtrs &acc,
                             const Epilogue &E, const nrgpu_z4_params &p, const BoxGeo &bx, nrgpu_level *L, dim3 grd,
                             dim3 blk, cudaStream_t st) {
#define NRGPU_Z4_FIXED(M_)                                                                                   \
  if (P == M_) {                                                                                             \
    z4_rhs_kernel<M_, M_ * M_, 0, ORD><<<grd, blk, 0, st>>>(In, out, pre, acc, E, p, bx, L->d_boundary, L->dx, \
                                                            L->dy, L->dz, L->d_status, 1, bx.o - 2, in);     \
    return;                                                                                                  \
  }
  if constexpr (ORD >= 4) {
    ZCVarPtrs In = U;
    int3 in = make_int3(bx.noffset, bx.m, bx.n);
    int P = bx.m == bx.n ? bx.m : 0;  // a kernel of its own, if one below matches
    const int Q = nrgpu_pad_size(bx.m, bx.n);
    if (Q && L->pad) {
      P = Q;
      const long fs = (long)P * P * bx.o;
      if ((size_t)(NRGPU_Z4_NVARS * fs) <= L->pad_doubles) {
        const long nb = (long)bx.m * bx.n * bx.o;
        pad_copy_kernel<<<dim3((unsigned)((nb + 255) / 256), NRGPU_Z4_NVARS), 256, 0, st>>>(U, L->pad, bx, P, fs, 0,
                                                                                              bx.o - 1);
        for (int v = 0; v < NRGPU_Z4_NVARS; ++v) In.p[v] = L->pad + v * fs;
        in = make_int3(0, P, P);
      } else {
        P = 0;
      }
    }
    NRGPU_Z4_FIXED(162) NRGPU_Z4_FIXED(168) NRGPU_Z4_FIXED(136) NRGPU_Z4_FIXED(104) NRGPU_Z4_FIXED(72)
    NRGPU_Z4_FIXED(66) NRGPU_Z4_FIXED(194)
  }
#undef NRGPU_Z4_FIXED
  z4_rhs_kernel<0, 0, 0, ORD><<<grd, blk, 0, st>>>(U, out, pre, acc, E, p, bx, L->d_boundary, L->dx, L->dy, L->dz,
                                                   L->d_status, 1, bx.o - 2, make_int3(bx.noffset, bx.m, bx.n));
}

// the FP32-stencil options (precision 1, 2): the 162^3 box of the
// precision sweep with compile-time strides, generic strides otherwise
template <int PREC>
static void z4_interior_prec(const ZCVarPtrs &U, const ZVarPtrs &out, const ZCVarPtrs &pre, const ZVarPtrs &acc,
                             const Epilogue &E, const nrgpu_z4_params &p, const BoxGeo &bx, nrgpu_level *L, dim3 grd,
                             dim3 blk, cudaStream_t st) {
#define NR_Z4P(CSY_, CSZ_, ORD_)                                                                               \
  z4_rhs_kernel<CSY_, CSZ_, PREC, ORD_><<<grd, blk, 0, st>>>(U, out, pre, acc, E, p, bx, L->d_boundary, L->dx, \
                                                             L->dy, L->dz, L->d_status, 1, bx.o - 2,       \
                                                             make_int3(bx.noffset, bx.m, bx.n))
  if (p.order_centered == 6 && bx.m == 162 && bx.n == 162) NR_Z4P(162, 162 * 162, 6);
  else if (p.order_centered == 6) NR_Z4P(0, 0, 6);
  else if (p.order_centered == 4) NR_Z4P(0, 0, 4);
  else NR_Z4P(0, 0, 2);
#undef NR_Z4P
}

// the box size of a level that the queue kernel can run: all boxes m x m
// in x and y with m a compile-time-stride size, at 4th or 6th order, FP64,
// more than one box; 0 otherwise
static int z4_queue_size(const nrgpu_level *L, const nrgpu_z4_params &p) {
  if (L->nboxes < 2 || p.precision || p.order_centered < 4) return 0;
  const int m = L->hbox[0].m;
  for (int b = 0; b < L->nboxes; ++b)
    if (L->hbox[b].m != m || L->hbox[b].n != m || L->hbox[b].o != L->hbox[0].o) return 0;
  for (int c : kPadSizes)
    if (c == m) return m;
  return 0;
}

// the interior of all boxes of the level by z4_rhs_queue_kernel
static int z4_queue_launch(nrgpu_level *L, int m, const ZCVarPtrs &U, const ZVarPtrs &out, const ZCVarPtrs &pre,
                           const ZVarPtrs &acc, const Epilogue &E, const nrgpu_z4_params &p, cudaStream_t st) {
  const BoxGeo &b0 = L->hbox[0];
  const dim3 blk(L->blk[0], L->blk[1], L->blk[2]);
  const int3 tiles = make_int3((b0.m - 2 + blk.x - 1) / blk.x, (b0.n - 2 + blk.y - 1) / blk.y,
                               (b0.o - 2 + blk.z - 1) / blk.z);
  const int total = tiles.x * tiles.y * tiles.z * L->nboxes;
  // resident blocks: one or two per SM at 255 registers; more would wait
  const int per_sm = blk.x * blk.y * blk.z <= 128 ? 2 : 1;
  const int grid = min(total, L->nsm * per_sm);
  int *counter = L->d_status + 2;
  NRGPU_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(int), st));
#define NR_Z4Q(M_, O_)                                                                                               \
  z4_rhs_queue_kernel<M_, M_ * M_, O_><<<grid, blk, 0, st>>>(U, out, pre, acc, E, p, L->d_box, L->nboxes, tiles,       \
                                                             L->d_boundary, L->dx, L->dy, L->dz, L->d_status, counter)
#define NR_Z4Q_SIZE(M_)                                    \
  if (m == M_) {                                           \
    if (p.order_centered == 4) NR_Z4Q(M_, 4);              \
    else NR_Z4Q(M_, 6);                                    \
  }
  NR_Z4Q_SIZE(66) NR_Z4Q_SIZE(72) NR_Z4Q_SIZE(104) NR_Z4Q_SIZE(136) NR_Z4Q_SIZE(162) NR_Z4Q_SIZE(168)
  NR_Z4Q_SIZE(194)
#undef NR_Z4Q_SIZE
#undef NR_Z4Q
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

static int z4_launch(nrgpu_level *L, const ZCVarPtrs &U, const ZVarPtrs &out, const ZCVarPtrs &pre,
                     const ZVarPtrs &acc, const Epilogue &E, const nrgpu_z4_params &p, cudaStream_t st, bool interior,
                     bool flagged) {
  // the boundary kernel beside the interior kernel, as in launch_rhs
  const bool fork = interior && flagged && L->nflagpts > 0;
  if (fork) {
    int e = nrgpu_level_side(L);
    if (e) return e;
    NRGPU_CUDA_TRY(cudaEventRecord(L->ev_fork, st));
    NRGPU_CUDA_TRY(cudaStreamWaitEvent(L->side, L->ev_fork, 0));
  }
  if (interior) {
    // the staging buffer of off-size boxes, allocated here unless a graph
    // is being captured (the refinement driver allocates it beforehand)
    if (!L->pad_tried) {
      cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
      if (cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone) nrgpu_level_pad(L);
      cudaGetLastError();
    }
    // all boxes in one persistent launch (nrgpu_level_queue), or one launch per box
    const int qm = L->queue ? z4_queue_size(L, p) : 0;
    if (qm) {
      int e = z4_queue_launch(L, qm, U, out, pre, acc, E, p, st);
      if (e) return e;
    }
    for (int b = 0; b < L->nboxes && !qm; ++b) {
      const BoxGeo &bx = L->hbox[b];
      if (bx.m < 3 || bx.n < 3 || bx.o < 3) continue;
      // the block shape of the level (32 x 4 x 1, or what nrgpu_level_autotune
      // measured fastest for this box); 128 or 256 threads, one point each
      const dim3 blk(L->blk[0], L->blk[1], L->blk[2]);
      const dim3 grd((bx.m - 2 + blk.x - 1) / blk.x, (bx.n - 2 + blk.y - 1) / blk.y, (bx.o - 2 + blk.z - 1) / blk.z);
      if (p.precision == 1) z4_interior_prec<1>(U, out, pre, acc, E, p, bx, L, grd, blk, st);
      else if (p.precision == 2) z4_interior_prec<2>(U, out, pre, acc, E, p, bx, L, grd, blk, st);
      else if (p.order_centered == 2) z4_interior_fp64<2>(U, out, pre, acc, E, p, bx, L, grd, blk, st);
      else if (p.order_centered == 4) z4_interior_fp64<4>(U, out, pre, acc, E, p, bx, L, grd, blk, st);
      else z4_interior_fp64<6>(U, out, pre, acc, E, p, bx, L, grd, blk, st);
    }
    // the ladder points of all boxes (beside the interior kernel)
    const int nlad = L->nladder[p.order_centered / 2 - 1];
    if (nlad > 0) {
      const cudaStream_t ls = fork ? L->side : st;
      const unsigned g = (unsigned)((nlad + 127) / 128);
#define NR_Z4L(P_)                                                                                                   \
  z4_ladder_kernel<P_><<<g, 128, 0, ls>>>(U, out, pre, acc, E, p, L->d_ladder, nlad, L->d_box, L->dx, L->dy, L->dz, \
                                          L->d_status, 1, 1 << 30)
      if (p.precision == 1) NR_Z4L(1);
      else if (p.precision == 2) NR_Z4L(2);
      else NR_Z4L(0);
#undef NR_Z4L
    }
  }
  if (flagged && L->nflagpts > 0) {
    const int n = L->nflagpts * ZNV;
    z4_flagged_kernel<<<(n + 255) / 256, 256, 0, fork ? L->side : st>>>(U, out, pre, acc, E, p, L->d_flagpts,
                                                                         L->nflagpts, L->d_box, L->dx, L->dy, L->dz);
  }
  if (fork) {
    NRGPU_CUDA_TRY(cudaEventRecord(L->ev_join, L->side));
    NRGPU_CUDA_TRY(cudaStreamWaitEvent(st, L->ev_join, 0));
  }
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_z4_rhs(nrgpu_level *L, double *const *unew, double *const *upre, double c, double *const *ucur,
                            const nrgpu_z4_params *p, void *stream) {
  if (!L) return nrgpu_set_error(NRGPU_ERR_ARG, "null level");
  int e;
  if ((e = z4_check_params(p))) return e;
  ZVarPtrs n, pr, cu;
  if ((e = z4_fill(&n, unew, "unew")) || (e = z4_fill(&cu, ucur, "ucur"))) return e;
  if (c != 0.0) {
    if ((e = z4_fill(&pr, upre, "upre"))) return e;
  } else {
    pr = cu;
  }
  // the background boundary extrapolates the state onto the boundary first
  if (p->boundary && (e = nrgpu_z4_background_extrapolate(L, ucur, (cudaStream_t)stream))) return e;
  Epilogue E = {c != 0.0 ? EPI_ADDLINEAR : EPI_RHS, c, 0.0, 0.0, 0};
  return z4_launch(L, z4_c(cu), n, z4_c(pr), n, E, *p, (cudaStream_t)stream, true, false);
}

extern "C" int nrgpu_z4_boundary(nrgpu_level *L, double *const *unew, double *const *upre, double c,
                                 double *const *ucur, const nrgpu_z4_params *p, void *stream) {
  if (!L || !p) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  int e;
  ZVarPtrs n, pr, cu;
  if ((e = z4_fill(&n, unew, "unew")) || (e = z4_fill(&cu, ucur, "ucur"))) return e;
  if (c != 0.0) {
    if ((e = z4_fill(&pr, upre, "upre"))) return e;
  } else {
    pr = cu;
  }
  if (p->boundary) return nrgpu_z4_background_boundary(L, unew, upre, c, ucur, p, (cudaStream_t)stream);
  Epilogue E = {c != 0.0 ? EPI_ADDLINEAR : EPI_RHS, c, 0.0, 0.0, 0};
  if ((e = z4_launch(L, z4_c(cu), n, z4_c(pr), n, E, *p, (cudaStream_t)stream, false, true))) return e;
  return nrgpu_level_symmetry(L, unew, NRGPU_SYSTEM_Z4C, (cudaStream_t)stream);
}

// evolve_rk_rk4 (rk.c:220) for the Z4c list + z4_algcon_wrapper (z4.c:49)
int nrgpu_z4_rk4_stages(nrgpu_level *L, double *const *u, double dt, const nrgpu_z4_params *p, cudaStream_t st) {
  if (!L) return nrgpu_set_error(NRGPU_ERR_ARG, "null level");
  int e;
  if ((e = z4_check_params(p))) return e;
  if (p->boundary) return nrgpu_z4_rk4_background(L, u, dt, p, st);
  ZVarPtrs U;
  if ((e = z4_fill(&U, u, "u"))) return e;
  double *scr = nullptr;
  if ((e = nrgpu_level_scratch(L, &scr))) return e;
  // the RK4 step without a copy of u, as for BSSN (rk_stage): u is the
  // stage-1 input and "P"; A accumulates; stage 4 writes u = A + dt/6 r4
  ZVarPtrs A, V1, V2;
  const size_t np = (size_t)L->npoints;
  for (int v = 0; v < ZNV; ++v) {
    A.p[v] = scr + (0 * ZNV + v) * np;
    V1.p[v] = scr + (1 * ZNV + v) * np;
    V2.p[v] = scr + (2 * ZNV + v) * np;
  }
  const ZCVarPtrs cU = z4_c(U);
  const Epilogue E1 = {EPI_RK, 0.0, dt / 6, dt / 2, 1, ACC_INIT};
  const Epilogue E2 = {EPI_RK, 0.0, dt / 3, dt / 2, 1, ACC_ADD};
  const Epilogue E3 = {EPI_RK, 0.0, dt / 3, dt, 1, ACC_ADD};
  const Epilogue E4 = {EPI_RK, 0.0, dt / 6, 0.0, 0, ACC_FINAL};
  if (L->nsym) {
    // a symmetry grid: rhs, radiative boundary and reflection of the rhs,
    // then the updates at every point (as for BSSN, rk_stage)
    SymVars RS;
    if ((e = sym_rhs_list(L, ZNV, &RS))) return e;
    ZVarPtrs Rp;
    for (int v = 0; v < ZNV; ++v) Rp.p[v] = RS.p[v];
    const Epilogue Er = {EPI_RHS, 0.0, 0.0, 0.0, 0, 0};
    const ZVarPtrs *ins[4] = {&U, &V1, &V2, &V1}, *outs[4] = {&V1, &V2, &V1, &U};
    for (int sg = 0; sg < 4; ++sg) {
      if ((e = z4_launch(L, z4_c(*ins[sg]), Rp, z4_c(*ins[sg]), Rp, Er, *p, st, true, true))) return e;
      if ((e = nrgpu_level_symmetry(L, Rp.p, NRGPU_SYSTEM_Z4C, st))) return e;
      const long n = (long)ZNV * L->npoints;
      rk_update_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(RS, sym_vars(outs[sg]->p, ZNV), sym_vars(U.p, ZNV),
                                                                    sym_vars(A.p, ZNV), stage_epilogue(sg, dt), ZNV,
                                                                    L->npoints);
      NRGPU_CUDA_TRY(cudaGetLastError());
    }
    return NRGPU_OK;
  }
  if ((e = z4_launch(L, cU, V1, cU, A, E1, *p, st, true, true))) return e;
  if ((e = z4_launch(L, z4_c(V1), V2, cU, A, E2, *p, st, true, true))) return e;
  if ((e = z4_launch(L, z4_c(V2), V1, cU, A, E3, *p, st, true, true))) return e;
  if ((e = z4_launch(L, z4_c(V1), U, cU, A, E4, *p, st, true, true))) return e;
  return NRGPU_OK;
}

// z4_algcon (z4_algcon.c:22): the operations of bssn_algcon on g~ and A~
int nrgpu_z4_algcon(nrgpu_level *L, double *const *u, const nrgpu_z4_params *p, cudaStream_t st) {
  VarPtrs gA;
  for (int v = 0; v < NRGPU_NV; ++v) gA.p[v] = u[v];  // g~ 0..5 and A~ 7..12 as in BSSN
  bssn_algcon_kernel<<<(L->npoints + 255) / 256, 256, 0, st>>>(gA, 0, L->npoints, p->subtractA,
                                                                p->normalizedetg);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_z4_rk4_step(nrgpu_level *L, double *const *u, double dt, const nrgpu_z4_params *p,
                                 void *stream) {
  int e = nrgpu_z4_rk4_stages(L, u, dt, p, (cudaStream_t)stream);
  if (e) return e;
  return nrgpu_z4_algcon(L, u, p, (cudaStream_t)stream);
}

// ---- block-shape autotuner (no counterpart in the reference) -------------------
// The rhs kernels compute one point per thread in 128-thread blocks; which
// x extent (8 .. 128) runs fastest depends on the box size and the order.
// The tuner times each shape on a flat state in the level's own scratch
// (user data untouched), keeps the fastest in the level, and returns it.
namespace {
__global__ void flat_state_kernel(double *base, int nv, long np, int alpha) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)nv * np) return;
  const int v = (int)(t / np);
  base[t] = (v == 0 || v == 3 || v == 5 || v == 6 || v == alpha) ? 1.0 : 0.0;
}
}  // namespace

extern "C" int nrgpu_level_autotune(nrgpu_level *L, int system, const void *params, void *stream, int *best_block) {
  if (!L || !params || (system != NRGPU_SYSTEM_BSSN && system != NRGPU_SYSTEM_Z4C))
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad autotune arguments");
  int e;
  if (system == NRGPU_SYSTEM_BSSN && (e = check_params((const nrgpu_bssn_params *)params))) return e;
  if (system == NRGPU_SYSTEM_Z4C && (e = z4_check_params((const nrgpu_z4_params *)params))) return e;
  double *scr = nullptr;
  if ((e = nrgpu_level_scratch(L, &scr))) return e;
  const cudaStream_t st = (cudaStream_t)stream;
  const long np = L->npoints;
  const int nv = system == NRGPU_SYSTEM_BSSN ? NRGPU_NV : ZNV;
  flat_state_kernel<<<(unsigned)((nv * np + 255) / 256), 256, 0, st>>>(scr, nv, np,
                                                                       system == NRGPU_SYSTEM_BSSN ? 17 : 18);
  NRGPU_CUDA_TRY(cudaGetLastError());
  const Epilogue E = {EPI_RHS, 0.0, 0.0, 0.0, 0};
  cudaEvent_t ev0, ev1;
  NRGPU_CUDA_TRY(cudaEventCreate(&ev0));
  NRGPU_CUDA_TRY(cudaEventCreate(&ev1));
  // 128- and 256-thread shapes, flat (x, y) and with a z extent.  The
  // kernels wait on L1/L2: the larger and the more cubic the block, the
  // smaller its stencil halo per point, so more taps hit in L1 (a 256-thread
  // block at 255 registers is one block per SM, the same 8 warps as two
  // 128-thread blocks)
  static const int cand[][3] = {{32, 4, 1}, {64, 2, 1}, {16, 8, 1}, {8, 16, 1}, {128, 1, 1}, {16, 4, 2},
                                {8, 8, 2},  {32, 2, 2}, {8, 4, 4},  {4, 8, 4}, {16, 2, 4},  {4, 4, 8},
                                {64, 4, 1}, {32, 8, 1}, {16, 8, 2}, {32, 4, 2}, {16, 4, 4}, {8, 8, 4},
                                {64, 2, 2}, {128, 2, 1}};
  const int ncand = (int)(sizeof cand / sizeof cand[0]);
  float best = 1e30f;
  int bb = 0;
  for (int c = 0; c < ncand && !e; ++c) {
    for (int a = 0; a < 3; ++a) L->blk[a] = cand[c][a];
    for (int rep = 0; rep < 4 && !e; ++rep) {
      if (rep == 1) cudaEventRecord(ev0, st);
      if (system == NRGPU_SYSTEM_BSSN) {
        VarPtrs P, O;
        for (int v = 0; v < NRGPU_NV; ++v) {
          P.p[v] = scr + (long)v * np;
          O.p[v] = scr + (long)(ZNV + v) * np;
        }
        e = launch_rhs(L, cptrs(P), O, cptrs(P), O, E, *(const nrgpu_bssn_params *)params, st, true, false);
      } else {
        ZVarPtrs P, O;
        for (int v = 0; v < ZNV; ++v) {
          P.p[v] = scr + (long)v * np;
          O.p[v] = scr + (long)(ZNV + v) * np;
        }
        e = z4_launch(L, z4_c(P), O, z4_c(P), O, E, *(const nrgpu_z4_params *)params, st, true, false);
      }
    }
    cudaEventRecord(ev1, st);
    cudaEventSynchronize(ev1);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    if (ms < best) {
      best = ms;
      bb = c;
    }
  }
  for (int q = 0; q < 3; ++q) L->blk[q] = cand[bb][q];
  // the staged-tile kernel (BSSN) against the fastest shape
  L->tile = 0;
  if (!e && system == NRGPU_SYSTEM_BSSN) {
    const nrgpu_bssn_params &bp = *(const nrgpu_bssn_params *)params;
    VarPtrs P, O;
    for (int v = 0; v < NRGPU_NV; ++v) {
      P.p[v] = scr + (long)v * np;
      O.p[v] = scr + (long)(ZNV + v) * np;
    }
    bool elig = true;
    for (int b = 0; b < L->nboxes; ++b)
      elig = elig && tile_eligible(L, b, P.p, NRGPU_NV, bp.order_centered, bp.advection_lopsided,
                                   bp.advection_lopsided6);
    int pick = 0;
    for (int mode = 1; mode <= 2 && elig && !e; ++mode) {
      L->tile = mode;
      for (int rep = 0; rep < 4 && !e; ++rep) {
        if (rep == 1) cudaEventRecord(ev0, st);
        e = launch_rhs(L, cptrs(P), O, cptrs(P), O, E, bp, st, true, false);
      }
      cudaEventRecord(ev1, st);
      cudaEventSynchronize(ev1);
      float ms = 0;
      cudaEventElapsedTime(&ms, ev0, ev1);
      if (!e && ms < best) {
        best = ms;
        pick = mode;
      }
    }
    L->tile = pick;
  }
  // the box work-queue kernel (Z4c levels of several equal boxes) against
  // one launch per box with the fastest shape
  L->queue = 0;
  if (!e && system == NRGPU_SYSTEM_Z4C && z4_queue_size(L, *(const nrgpu_z4_params *)params)) {
    const nrgpu_z4_params &zp = *(const nrgpu_z4_params *)params;
    ZVarPtrs P, O;
    for (int v = 0; v < ZNV; ++v) {
      P.p[v] = scr + (long)v * np;
      O.p[v] = scr + (long)(ZNV + v) * np;
    }
    L->queue = 1;
    for (int rep = 0; rep < 4 && !e; ++rep) {
      if (rep == 1) cudaEventRecord(ev0, st);
      e = z4_launch(L, z4_c(P), O, z4_c(P), O, E, zp, st, true, false);
    }
    cudaEventRecord(ev1, st);
    cudaEventSynchronize(ev1);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    if (e || ms >= best) L->queue = 0;
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  for (int q = 0; q < 3; ++q)
    if (best_block) best_block[q] = L->tile ? 0 : cand[bb][q];
  if (e) return e;
  NRGPU_CUDA_TRY(cudaStreamSynchronize(st));
  return NRGPU_OK;
}

extern "C" int nrgpu_level_block(nrgpu_level *L, int bx, int by, int bz) {
  auto pow2 = [](int v) { return v >= 1 && v <= 256 && (v & (v - 1)) == 0; };
  if (!L || !pow2(bx) || !pow2(by) || !pow2(bz) || (bx * by * bz != 128 && bx * by * bz != 256))
    return nrgpu_set_error(NRGPU_ERR_ARG, "block %d x %d x %d (powers of two, 128 or 256 threads)", bx, by, bz);
  L->blk[0] = bx; L->blk[1] = by; L->blk[2] = bz;
  L->tile = 0;
  return NRGPU_OK;
}

extern "C" int nrgpu_level_queue(nrgpu_level *L, int on) {
  if (!L) return nrgpu_set_error(NRGPU_ERR_ARG, "null level");
  if (on > 1) return nrgpu_set_error(NRGPU_ERR_ARG, "queue mode %d (0, 1)", on);
  if (on >= 0) L->queue = on;
  return L->queue;
}

extern "C" int nrgpu_level_tile(nrgpu_level *L, int on) {
  if (!L) return nrgpu_set_error(NRGPU_ERR_ARG, "null level");
  if (on > 2) return nrgpu_set_error(NRGPU_ERR_ARG, "staged-tile mode %d (0, 1, 2)", on);
  if (on >= 0) L->tile = on;
  return L->tile;
}

extern "C" int nrgpu_level_get_block(nrgpu_level *L, int *block) {
  if (!L || !block) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  for (int q = 0; q < 3; ++q) block[q] = L->blk[q];
  return NRGPU_OK;
}
