// nrgpu_z4.cuh -- Z4c right-hand side on B200 (included inside the anonymous
// namespace of nrgpu_bssn.cu; shares its stencil, advection, dissipation and
// boundary helpers).
//
// The physics is the reference's z4_rhs_movpunc_N (spec
// z4_rhs_movpunc_N.m:18-520) without shells and without the non-principal
// terms (z4_useNPTs = no): K = Khat + 2 Theta, the Theta equation with the
// constraint-damping kappa1/kappa2, the hatted Hamiltonian constraint in the
// trace of A~, Gamma~ damping -2 alpha kappa1 (G - G(g)), the Z4c shift
// equations, and Kreiss-Oliger dissipation on all 25 fields.  As for BSSN,
// one thread computes one inner point, derivative groups are consumed as
// soon as they are formed, and advection/dissipation are added last.

enum { ZG11 = 0, ZCHI = 6, ZA11 = 7, ZKHAT = 13, ZGA1 = 14, ZTHETA = 17, ZALPHA = 18, ZBETA1 = 19, ZBB1 = 22 };
constexpr int ZNV = NRGPU_Z4_NVARS;

struct ZVarPtrs {
  double *p[ZNV];
};
struct ZCVarPtrs {
  const double *p[ZNV];
};

template <int ORD, int CSY = 0, int CSZ = 0, int PREC = 0>
__device__ __forceinline__ void z4_point(const ZCVarPtrs &U, const PointCtx &P, const nrgpu_z4_params &p,
                                         double r[ZNV]) {
  const int x = P.ijk;
#define ZSTR(c_) ((c_) == 0 ? 1 : (CSY > 0 ? ((c_) == 1 ? CSY : CSZ) : P.st[(c_)]))
  const double o1[3] = {1.0 / (den1<ORD>() * P.h[0]), 1.0 / (den1<ORD>() * P.h[1]),
                        1.0 / (den1<ORD>() * P.h[2])};
  const double o2[3] = {1.0 / (den2<ORD>() * P.h[0] * P.h[0]), 1.0 / (den2<ORD>() * P.h[1] * P.h[1]),
                        1.0 / (den2<ORD>() * P.h[2] * P.h[2])};

  double g[6], A[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) { g[a] = ldg(U.p[ZG11 + a] + x); A[a] = ldg(U.p[ZA11 + a] + x); }
  const double alpha = ldg(U.p[ZALPHA] + x);
  const double chi = ldg(U.p[ZCHI] + x);
  const double Khat = ldg(U.p[ZKHAT] + x);
  const double Theta = ldg(U.p[ZTHETA] + x);
  const double K = Khat + 2.0 * Theta;

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

  // Ricci tensor R_ab.  Its -1/2 g^cd d_c d_d g_ab part: with compile-time
  // strides it comes first, so that its many stencil loads have no
  // connection values live beside them (the 6th-order kernel then keeps
  // almost everything in registers); with run-time strides, whose tap
  // addresses take registers of their own, after the connection terms
  double Rt[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) Rt[a] = 0.0;
  auto ricci_dd = [&]() {
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int d = c; d < 3; ++d) {
        const double w = (c == d ? -0.5 : -1.0) * gi[sy(c, d)] * (c == d ? o2[c] : o1[c] * o1[d]);
#pragma unroll
        for (int a = 0; a < 6; ++a) {
          const double dd = c == d ? d2p<ORD, PREC>(U.p[ZG11 + a], x, ZSTR(c))
                                   : d11p<ORD, PREC>(U.p[ZG11 + a], x, ZSTR(c), ZSTR(d));
          Rt[a] += w * dd;
        }
      }
  };
  constexpr bool kDdFirst = CSY > 0;
  if constexpr (kDdFirst) ricci_dd();

  // connection
  double gdo[3][6], gam[3][6], Gfg[3];
  {
    double dg[3][6];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int a = 0; a < 6; ++a) dg[c][a] = o1[c] * d1p<ORD, PREC>(U.p[ZG11 + a], x, ZSTR(c));
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

  // the connection terms of R_ab (+ the chi part below)
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
    double dG[3][3];
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) dG[b][c] = o1[b] * d1p<ORD, PREC>(U.p[ZGA1 + c], x, ZSTR(b));
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        double t2 = 0.0;
#pragma unroll
        for (int c = 0; c < 3; ++c)
          t2 += g[sy(c, a)] * dG[b][c] + g[sy(c, b)] * dG[a][c] + Gfg[c] * (gdo[a][sy(b, c)] + gdo[b][sy(a, c)]);
        Rt[sy(a, b)] += 0.5 * t2;
      }
  }

  // conformal factor
  double chig = chi;
  if (chig < p.chiDivFloor) chig = p.chiDivFloor;
  const double oocp = 1.0 / p.chipsipower;
  const double psim4 = exp(-4.0 * (oocp * log(chig)));
  double df[3], dchic[3];  // dchic = d chi / chiguarded
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double dc = o1[a] * d1p<ORD, PREC>(U.p[ZCHI], x, ZSTR(a));
    df[a] = oocp * dc / chig;
    dchic[a] = dc / chig;
  }
  double dfdf = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) dfdf += gi[sy(a, b)] * df[a] * df[b];
  {
    double cddf[6];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int b = a; b < 3; ++b) {
        const double ddchi = a == b ? o2[a] * d2p<ORD, PREC>(U.p[ZCHI], x, ZSTR(a))
                                    : o1[a] * o1[b] * d11p<ORD, PREC>(U.p[ZCHI], x, ZSTR(a), ZSTR(b));
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
  const double Rhat = psim4 * (gi[0] * Rt[0] + gi[3] * Rt[3] + gi[5] * Rt[5] +
                               2.0 * (gi[1] * Rt[1] + gi[2] * Rt[2] + gi[4] * Rt[4]));

  // lapse
  double da[3], cdda[6];
#pragma unroll
  for (int a = 0; a < 3; ++a) da[a] = o1[a] * d1p<ORD, PREC>(U.p[ZALPHA], x, ZSTR(a));
  {
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
        double t = a == b ? o2[a] * d2p<ORD, PREC>(U.p[ZALPHA], x, ZSTR(a))
                          : o1[a] * o1[b] * d11p<ORD, PREC>(U.p[ZALPHA], x, ZSTR(a), ZSTR(b));
        t -= gam[0][ab] * da[0] + gam[1][ab] * da[1] + gam[2][ab] * da[2];
        cdda[ab] = t - 2.0 * (df[a] * da[b] + df[b] * da[a] - g[ab] * dfda);
      }
  }
  const double trcdda = psim4 * (gi[0] * cdda[0] + gi[3] * cdda[3] + gi[5] * cdda[5] +
                                 2.0 * (gi[1] * cdda[1] + gi[2] * cdda[2] + gi[4] * cdda[4]));

  // trace-free curvature
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
  const double cAA = gi[0] * AAab[0] + gi[3] * AAab[3] + gi[5] * AAab[5] +
                     2.0 * (gi[1] * AAab[1] + gi[2] * AAab[2] + gi[4] * AAab[4]);
  const double Hhat = Rhat + 2.0 * K * K / 3.0 - cAA;

#pragma unroll
  for (int a = 0; a < 6; ++a) {
    r[ZG11 + a] = -2.0 * alpha * A[a];
    r[ZA11 + a] = psim4 * (-cdda[a] + alpha * Rt[a]) - (1.0 / 3.0) * g[a] * (-trcdda + alpha * Rhat) +
                  alpha * (K * A[a] - 2.0 * AAab[a]);
  }
  r[ZKHAT] = -trcdda + alpha * (cAA + K * K / 3.0) + p.kappa1 * (1.0 - p.kappa2) * alpha * Theta;
  r[ZTHETA] = alpha * (Hhat / 2.0 - (2.0 + p.kappa2) * p.kappa1 * Theta) * p.zeroThetaRHS;

  // Gamma~ without advection: -2 Ainv da + 2 alpha divAinv - 2 alpha kappa1 (G - G(g))
  double rG[3];
  {
    double dKhat[3], dTheta[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      dKhat[a] = o1[a] * d1p<ORD, PREC>(U.p[ZKHAT], x, ZSTR(a));
      dTheta[a] = o1[a] * d1p<ORD, PREC>(U.p[ZTHETA], x, ZSTR(a));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      double dv = 0.0, s = 0.0;
#pragma unroll
      for (int b = 0; b < 3; ++b)
#pragma unroll
        for (int c = 0; c < 3; ++c) dv += gam[a][sy(b, c)] * Ainv[sy(b, c)];
#pragma unroll
      for (int b = 0; b < 3; ++b) {
        dv += -1.5 * Ainv[sy(a, b)] * dchic[b] - (1.0 / 3.0) * gi[sy(a, b)] * (2.0 * dKhat[b] + dTheta[b]);
        s += Ainv[sy(a, b)] * da[b];
      }
      const double Ga = ldg(U.p[ZGA1 + a] + x);
      rG[a] = -2.0 * s + 2.0 * alpha * dv - 2.0 * alpha * p.kappa1 * (Ga - Gfg[a]);
    }
  }

  // shift: Lie-derivative terms and pseudo-Lie of Gamma~
  {
    double db[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c) db[a][c] = o1[a] * d1p<ORD, PREC>(U.p[ZBETA1 + c], x, ZSTR(a));
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
        r[ZG11 + ab] += tg;
        r[ZA11 + ab] += tA;
      }
    r[ZCHI] = (-p.chipsipower / 6.0) * chig * alpha * K + (p.chipsipower / 6.0) * chig * divbeta;
    double trddb[3] = {0.0, 0.0, 0.0}, divdb[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = b; c < 3; ++c)
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double dd = b == c ? o2[b] * d2p<ORD, PREC>(U.p[ZBETA1 + a], x, ZSTR(b))
                                   : o1[b] * o1[c] * d11p<ORD, PREC>(U.p[ZBETA1 + a], x, ZSTR(b), ZSTR(c));
          trddb[a] += (b == c ? 1.0 : 2.0) * gi[sy(b, c)] * dd;
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
  r[ZALPHA] = -falpha * alpha * Khat;
  const double betaF = p.shiftgammacoeff * pow(alpha, p.shiftalphapower);
  const double bfac = p.gamma0factor + p.gamma2factor * betaF;
  const bool withB = p.withB != 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const double Ba = ldg(U.p[ZBB1 + a] + x);
    if (withB) {
      r[ZBETA1 + a] = (p.gamma2factor + p.gamma0factor * betaF) * Ba;
      r[ZBB1 + a] = bfac * rG[a] - p.shiftdriver * Ba;
    } else {
      r[ZBETA1 + a] = ldg(U.p[ZGA1 + a] + x) - p.shiftdriver * ldg(U.p[ZBETA1 + a] + x);
      r[ZBB1 + a] = 0.0;
    }
    r[ZGA1 + a] = rG[a];
  }

  // advection
  {
    const int lop = ORD == 2 ? 0 : (ORD == 6 ? p.advection_lopsided6 : p.advection_lopsided);
    const int idx[3] = {P.i, P.j, P.k}, mx[3] = {P.imax, P.jmax, P.kmax};
    AdvDir ad[3];
    double cw[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double w = ldg(U.p[ZBETA1 + d] + x) / P.h[d];
      ad[d] = adv_dir(idx[d], mx[d], w, ORD, lop, ZSTR(d));
      const int ws = w < 0 ? -1 : (w > 0 ? 1 : 0);
      cw[d] = -ws * w * (1.0 / den1<ORD>());
    }
#pragma unroll
    for (int a = 0; a < 6; ++a) {
      r[ZG11 + a] += adv_sum<ORD>(U.p[ZG11 + a], x, ad, cw);
      r[ZA11 + a] += adv_sum<ORD>(U.p[ZA11 + a], x, ad, cw);
    }
    r[ZKHAT] += adv_sum<ORD>(U.p[ZKHAT], x, ad, cw);
    r[ZCHI] += adv_sum<ORD>(U.p[ZCHI], x, ad, cw);
    r[ZTHETA] += p.zeroThetaRHS * adv_sum<ORD>(U.p[ZTHETA], x, ad, cw);
    r[ZALPHA] += p.oplogwithshift * adv_sum<ORD>(U.p[ZALPHA], x, ad, cw);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double aG = adv_sum<ORD>(U.p[ZGA1 + a], x, ad, cw);
      r[ZGA1 + a] += aG;
      r[ZBETA1 + a] += p.withShiftadv * adv_sum<ORD>(U.p[ZBETA1 + a], x, ad, cw);
      if (withB) r[ZBB1 + a] += bfac * (1.0 - p.withGadv) * aG + p.withBadv * adv_sum<ORD>(U.p[ZBB1 + a], x, ad, cw);
    }
  }

  // Kreiss-Oliger on all 25 fields
  if ((p.order_dissipation == 4 && P.dist >= 2) || (p.order_dissipation == 6 && P.dist >= 3)) {
    const double ooh[3] = {1.0 / P.h[0], 1.0 / P.h[1], 1.0 / P.h[2]};
    const int kst[3] = {ZSTR(0), ZSTR(1), ZSTR(2)};
    const double e = p.dissfactor;
    if (p.order_dissipation == 6) {
#pragma unroll
      for (int v = 0; v < ZNV; ++v) r[v] += e * ko_p<6, PREC>(U.p[v], x, kst, ooh);
    } else {
#pragma unroll
      for (int v = 0; v < ZNV; ++v) r[v] += e * ko_p<4, PREC>(U.p[v], x, kst, ooh);
    }
  }
#undef ZSTR
}

__device__ __forceinline__ void z4_store(const double r[ZNV], int x, const ZVarPtrs &out, const ZCVarPtrs &pre,
                                         const ZVarPtrs &acc, const Epilogue &E, const nrgpu_z4_params &p) {
  if (E.mode == EPI_RHS) {
#pragma unroll
    for (int v = 0; v < ZNV; ++v) out.p[v][x] = r[v];
  } else if (E.mode == EPI_ADDLINEAR) {
    double n[ZNV];
#pragma unroll
    for (int v = 0; v < ZNV; ++v) n[v] = ldg(pre.p[v] + x) + E.c * r[v];
    nrgpu_bssn_params q;  // only subtractA / normalizedetg are read
    q.subtractA = p.subtractA;
    q.normalizedetg = p.normalizedetg;
    det_trace_fix(n, q);  // g~ at 0..5 and A~ at 7..12 in both lists
#pragma unroll
    for (int v = 0; v < ZNV; ++v) out.p[v][x] = n[v];
  } else if (E.accmode == ACC_FINAL) {
#pragma unroll
    for (int v = 0; v < ZNV; ++v) out.p[v][x] = acc.p[v][x] + E.wacc * r[v];
  } else if (E.accmode == ACC_INIT) {
#pragma unroll
    for (int v = 0; v < ZNV; ++v) {
      const double u0 = ldg(pre.p[v] + x);
      acc.p[v][x] = u0 + E.wacc * r[v];
      if (E.has_v) out.p[v][x] = u0 + E.cv * r[v];
    }
  } else {
#pragma unroll
    for (int v = 0; v < ZNV; ++v) {
      acc.p[v][x] += E.wacc * r[v];
      if (E.has_v) out.p[v][x] = ldg(pre.p[v] + x) + E.cv * r[v];
    }
  }
}

// One inner point (i, j, k) of a box: the input lists U are read at
// in.x + i + in.y (j + in.z k) (the box's own place, or a staged copy of the
// box whose strides are the kernel's compile-time ones, pad_copy_kernel);
// the outputs, the previous state and the flags at the box's own index.
template <int CSY, int CSZ, int PREC, int ORD>
__device__ __forceinline__ void z4_interior_point(int i, int j, int k, const BoxGeo &box, int3 in,
                                                  const ZCVarPtrs &U, const ZVarPtrs &out, const ZCVarPtrs &pre,
                                                  const ZVarPtrs &acc, const Epilogue &E, const nrgpu_z4_params &p,
                                                  const int *__restrict__ boundary, double dx, double dy, double dz,
                                                  int *status) {
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
  // the points of the order ladder are z4_ladder_kernel's
  if (d < ORD / 2) return;
  P.dist = d;
  // the RK epilogue's accumulator and previous state into L2 now (as in
  // bssn_rhs_kernel)
  if (E.mode == EPI_RK) {
#pragma unroll
    for (int v = 0; v < ZNV; ++v) {
      if (E.accmode != ACC_INIT) l2_prefetch(acc.p[v] + xo);
      if (E.accmode == ACC_INIT || E.has_v) l2_prefetch(pre.p[v] + xo);
    }
  }
  double r[ZNV];
  z4_point<ORD, CSY, CSZ, PREC>(U, P, p, r);
  double s = 0.0;
#pragma unroll
  for (int v = 0; v < ZNV; ++v) s += r[v];
  if (!isfinite(s)) atomicOr(status, 1);
  z4_store(r, xo, out, pre, acc, E, p);
}

template <int CSY = 0, int CSZ = 0, int PREC = 0, int ORD = 4>
__global__ void __launch_bounds__(256, NRGPU_RHS_MINBLOCKS) z4_rhs_kernel(ZCVarPtrs U, ZVarPtrs out, ZCVarPtrs pre, ZVarPtrs acc, Epilogue E,
                                                    const nrgpu_z4_params p, BoxGeo box,
                                                    const int *__restrict__ boundary, double dx, double dy, double dz,
                                                    int *status, int k0, int k1, int3 in) {
  const int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
  const int k = k0 + blockIdx.z * blockDim.z + threadIdx.z;
  if (i > box.m - 2 || j > box.n - 2 || k > k1) return;
  z4_interior_point<CSY, CSZ, PREC, ORD>(i, j, k, box, in, U, out, pre, acc, E, p, boundary, dx, dy, dz, status);
}

// The interior of every box of a level in one persistent launch: a queue of
// tiles (the level's block shape) over the boxes, which the blocks take in
// turn from an atomic counter until it runs past the last; each point as in
// z4_rhs_kernel, so the results are those of one launch per box.  For levels
// whose boxes share one size with a compile-time-stride kernel (CSY = m = n):
// the two puncture boxes per level of the full form's finer levels.  No
// block waits on another.
template <int CSY, int CSZ, int ORD>
__global__ void __launch_bounds__(256, NRGPU_RHS_MINBLOCKS)
    z4_rhs_queue_kernel(ZCVarPtrs U, ZVarPtrs out, ZCVarPtrs pre, ZVarPtrs acc, Epilogue E, const nrgpu_z4_params p,
                        const BoxGeo *__restrict__ boxes, int nboxes, int3 tiles, const int *__restrict__ boundary,
                        double dx, double dy, double dz, int *status, int *counter) {
  __shared__ int item;
  const int per_box = tiles.x * tiles.y * tiles.z, total = per_box * nboxes;
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0;
  for (;;) {
    if (lead) item = atomicAdd(counter, 1);
    __syncthreads();
    const int t = item;
    __syncthreads();  // every thread has read item before the next take
    if (t >= total) return;
    const int b = t / per_box, r = t - b * per_box;
    const int tx = r % tiles.x, ty = (r / tiles.x) % tiles.y, tz = r / (tiles.x * tiles.y);
    const BoxGeo box = boxes[b];
    const int i = 1 + tx * blockDim.x + threadIdx.x;
    const int j = 1 + ty * blockDim.y + threadIdx.y;
    const int k = 1 + tz * blockDim.z + threadIdx.z;
    if (i <= box.m - 2 && j <= box.n - 2 && k <= box.o - 2)
      z4_interior_point<CSY, CSZ, 0, ORD>(i, j, k, box, make_int3(box.noffset, box.m, box.n), U, out, pre, acc, E,
                                          p, boundary, dx, dy, dz, status);
  }
}

// the order-ladder points of a level (see bssn_ladder_kernel)
template <int PREC>
__global__ void z4_ladder_kernel(ZCVarPtrs U, ZVarPtrs out, ZCVarPtrs pre, ZVarPtrs acc, Epilogue E,
                                 const nrgpu_z4_params p, const FlagPoint *__restrict__ pts, int n,
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
  double r[ZNV];
  if (oc == 2) z4_point<2, 0, 0, PREC>(U, P, p, r);
  else z4_point<4, 0, 0, PREC>(U, P, p, r);
  double s = 0.0;
#pragma unroll
  for (int v = 0; v < ZNV; ++v) s += r[v];
  if (!isfinite(s)) atomicOr(status, 1);
  z4_store(r, P.ijk, out, pre, acc, E, p);
}

// radiative boundary for the 25 Z4c fields (set_boundary, radiative.c:105)
__global__ void z4_flagged_kernel(ZCVarPtrs U, ZVarPtrs out, ZCVarPtrs pre, ZVarPtrs acc, Epilogue E,
                                  const nrgpu_z4_params p, const FlagPoint *__restrict__ pts, int npts,
                                  const BoxGeo *__restrict__ boxes, double dx, double dy, double dz) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts * ZNV) return;
  const int v = t % ZNV;
  const FlagPoint fp = pts[t / ZNV];
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

