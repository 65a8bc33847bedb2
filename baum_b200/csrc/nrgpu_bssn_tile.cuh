// nrgpu_bssn_tile.cuh -- the BSSN right-hand side over TMA-staged tiles
// (included by nrgpu_bssn.cu inside its anonymous namespace).
//
// The same physics as bssn_point (bssn_rhs_movpunc_N.m:18-461 of the
// reference), reorganised so that every stencil tap comes from shared memory:
//
// * A block of 256 threads computes a tile of 16 x 4 x 4 inner points (one
//   point per thread).  Each field of the input list is staged as one
//   22 x 10 x 10 box (the tile and a halo of 3, enough for 4th-order centred
//   and mixed derivatives, lopsided advection with a shift of 1 or 2 and
//   KO6, and 6th-order centred stencils with the centred 6th-order
//   advection; the points nearer the box faces take lower orders and are
//   left to the ladder kernel) by a single TMA load into a ring of 12 slots of 17.25 KB
//   (207 KB of shared memory, one block per SM).
// * The 24 fields pass through the ring in two rounds, in the order the
//   computation consumes them: round A = g~ (6), Gamma~ (3), chi, alpha, K;
//   round B = beta (3), A~ (6), B (3).  Field f of a round always lands in
//   the same slot, so every shared-memory address is a compile-time offset
//   from one per-thread base.  A slot of round A is refilled with its round
//   B field as soon as all eight warps have released it, so the copies of
//   round B overlap the arithmetic of round A.
// * Each field's advection and Kreiss-Oliger terms are formed while the
//   field is resident (they were the last step of bssn_point); the sums are
//   the same terms, added in a different order.
// * The stencil taps are read through volatile pointers: that keeps the
//   compiler from hoisting hundreds of shared-memory loads ahead of the
//   arithmetic that consumes them (which spills at 255 registers), while
//   each load still issues back to back with the next.
// * Stencil offsets no longer depend on the box: one instance serves every
//   box size.
//
// Points with a non-zero boundary flag or outside the box take part in the
// barrier protocol only.  A wait that runs out of time sets bit 1 of
// status[0] and the thread stops computing.

constexpr int kTX = 16, kTY = 4, kTZ = 4, kTH = 3;
constexpr int kBX = kTX + 2 * kTH, kBY = kTY + 2 * kTH, kBZ = kTZ + 2 * kTH;   // 22 x 10 x 10
constexpr int kTSY = kBX, kTSZ = kBX * kBY;                                    // shared strides
constexpr unsigned kTileBoxBytes = kBX * kBY * kBZ * 8;                        // 17600
constexpr int kSlot = 2208;                                                    // doubles per slot (17664 B)
constexpr int kNSlot = 12;
constexpr int kTileThreads = kTX * kTY * kTZ;
// slots and barriers, plus room to start the slots on a 128-byte boundary
constexpr size_t kTileSmem = (size_t)kNSlot * kSlot * 8 + 2 * kNSlot * 8 + 128;

// the fields of the two rounds, slot by slot (BSSN list order, bssn.c:315-322)
__constant__ int kRoundA[kNSlot] = {G11, G11 + 1, G11 + 2, G11 + 3, G11 + 4, G11 + 5,
                                    GA1, GA1 + 1, GA1 + 2, CHI, ALPHA, KK};
__constant__ int kRoundB[kNSlot] = {BETA1, BETA1 + 1, BETA1 + 2, A11, A11 + 1, A11 + 2,
                                    A11 + 3, A11 + 4, A11 + 5, BB1, BB1 + 1, BB1 + 2};
enum { SL_G = 0, SL_GA = 6, SL_CHI = 9, SL_ALPHA = 10, SL_K = 11, SL_BETA = 0, SL_A = 3, SL_B = 9 };

struct BssnMaps {
  CUtensorMap m[NRGPU_NV];
};

// ---- stencils on a shared-memory tile (c: the point's own value; strides
// are compile-time constants after unrolling) ---------------------------------
typedef const volatile double *tap_t;

template <int ORD>
__device__ __forceinline__ double t_d1(tap_t c, int s) {
  if (ORD == 2) return c[s] - c[-s];
  if (ORD == 4) return (c[-2 * s] - c[2 * s]) + 8.0 * (c[s] - c[-s]);
  return (c[3 * s] - c[-3 * s]) + 9.0 * (c[-2 * s] - c[2 * s]) + 45.0 * (c[s] - c[-s]);
}
template <int ORD>
__device__ __forceinline__ double t_d2(tap_t c, int s) {
  const double c0 = c[0];
  if (ORD == 2) return c[-s] - 2.0 * c0 + c[s];
  if (ORD == 4) return 16.0 * (c[-s] + c[s]) - (c[-2 * s] + c[2 * s]) - 30.0 * c0;
  return 2.0 * (c[-3 * s] + c[3 * s]) - 27.0 * (c[-2 * s] + c[2 * s]) + 270.0 * (c[-s] + c[s]) - 490.0 * c0;
}
template <int ORD>
__device__ __forceinline__ double t_d11(tap_t c, int s1, int s2) {
  if (ORD == 2) return t_d1<2>(c + s1, s2) - t_d1<2>(c - s1, s2);
  if (ORD == 4)
    return (t_d1<4>(c - 2 * s1, s2) - t_d1<4>(c + 2 * s1, s2)) + 8.0 * (t_d1<4>(c + s1, s2) - t_d1<4>(c - s1, s2));
  return (t_d1<6>(c + 3 * s1, s2) - t_d1<6>(c - 3 * s1, s2)) + 9.0 * (t_d1<6>(c - 2 * s1, s2) - t_d1<6>(c + 2 * s1, s2)) +
         45.0 * (t_d1<6>(c + s1, s2) - t_d1<6>(c - s1, s2));
}
__device__ __forceinline__ constexpr int tstr(int d) { return d == 0 ? 1 : (d == 1 ? kTSY : kTSZ); }

template <int Q>
__device__ __forceinline__ double t_adv(tap_t c, const AdvDir ad[3], const double cw[3]) {
  double acc = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double t = 0.0;
    tap_t p0 = c + ad[d].base;
#pragma unroll
    for (int n = 0; n <= Q; ++n) {
      const double w = Q == 2 ? kAdv2[ad[d].row][n] : Q == 4 ? kAdv4[ad[d].row][n] : kAdv6[ad[d].row][n];
      t += w * p0[n * ad[d].step];
    }
    acc += cw[d] * t;
  }
  return acc;
}

template <int OD>
__device__ __forceinline__ double t_ko(tap_t c, const double ooh[3]) {
  double acc = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int s = tstr(d);
    double t;
    if (OD == 4)
      t = 6.0 * c[0] - 4.0 * (c[-s] + c[s]) + (c[-2 * s] + c[2 * s]);
    else
      t = (c[-3 * s] + c[3 * s]) - 6.0 * (c[-2 * s] + c[2 * s]) + 15.0 * (c[-s] + c[s]) - 20.0 * c[0];
    acc += ooh[d] * t;
  }
  return OD == 4 ? -acc : acc;
}

// Kreiss-Oliger term of one field (dissfactor included), 0 where the full
// stencil does not fit
__device__ __forceinline__ double t_kof(tap_t c, const nrgpu_bssn_params &p, const double ooh[3], bool with_ko) {
  if (!with_ko) return 0.0;
  if (p.order_dissipation == 6) return p.dissfactor * t_ko<6>(c, ooh);
  if (p.order_dissipation == 4) return p.dissfactor * t_ko<4>(c, ooh);
  return 0.0;
}

// state carried from group to group within one point
struct TileCarry {
  double gi[6], g[6];
  double gam[3][6], Gfg[3];
  double Rt[6];
  double rg[6];        // advection + KO of g~
  double aG[3], kG[3]; // advection and KO of Gamma~
  double chig, psim4, df[3], rchi;
  double da[3], cdda[6], trcdda, ralpha;
  double dK[3], rK;
};

#define NR_O1 const double o1[3] = {1.0 / (den1<ORD>() * h[0]), 1.0 / (den1<ORD>() * h[1]), 1.0 / (den1<ORD>() * h[2])}
#define NR_O2                                                                                  \
  const double o2[3] = {1.0 / (den2<ORD>() * h[0] * h[0]), 1.0 / (den2<ORD>() * h[1] * h[1]), \
                        1.0 / (den2<ORD>() * h[2] * h[2])}
#define NR_OOH const double ooh[3] = {1.0 / h[0], 1.0 / h[1], 1.0 / h[2]}

// group 1: g~ (slots 0-5): inverse metric, connection, Ricci of g~, the
// second derivatives of g~; advection and KO of g~
template <int ORD>
__device__ __forceinline__ void tg_metric(const double *sb, TileCarry &T, const double h[3], const AdvDir ad[3],
                                          const double cw[3], const nrgpu_bssn_params &p, bool with_ko) {
  NR_O1;
  NR_O2;
#define GS(a_) (tap_t)(sb + (SL_G + (a_)) * kSlot)
  double *g = T.g, *gi = T.gi;
#pragma unroll
  for (int a = 0; a < 6; ++a) g[a] = sb[(SL_G + a) * kSlot];
  const double detg = g[0] * g[3] * g[5] + 2.0 * g[1] * g[2] * g[4] - g[0] * g[4] * g[4] -
                      g[3] * g[2] * g[2] - g[5] * g[1] * g[1];
  const double detginv = 1.0 / detg;
  gi[0] = detginv * (g[3] * g[5] - g[4] * g[4]);
  gi[1] = detginv * (g[2] * g[4] - g[1] * g[5]);
  gi[2] = detginv * (g[1] * g[4] - g[2] * g[3]);
  gi[3] = detginv * (g[0] * g[5] - g[2] * g[2]);
  gi[4] = detginv * (g[1] * g[2] - g[0] * g[4]);
  gi[5] = detginv * (g[0] * g[3] - g[1] * g[1]);
  double gdo[3][6];
  {
    double dg[3][6];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int a = 0; a < 6; ++a) dg[c][a] = o1[c] * t_d1<ORD>(GS(a), tstr(c));
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
      T.gam[c][a] = gi[sy(c, 0)] * gdo[0][a] + gi[sy(c, 1)] * gdo[1][a] + gi[sy(c, 2)] * gdo[2][a];
#pragma unroll
  for (int a = 0; a < 3; ++a)
    T.Gfg[a] = gi[0] * T.gam[a][0] + gi[3] * T.gam[a][3] + gi[5] * T.gam[a][5] +
               2.0 * (gi[1] * T.gam[a][1] + gi[2] * T.gam[a][2] + gi[4] * T.gam[a][4]);
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
            q += T.gam[e][sy(c, a)] * gdo[b][sy(e, d)] + T.gam[e][sy(c, b)] * gdo[a][sy(e, d)] +
                 T.gam[e][sy(a, d)] * gdo[e][sy(c, b)];
          t += gi[sy(c, d)] * q;
        }
      T.Rt[sy(a, b)] = t;
    }
  // G~'s own half of the Ricci term 1/2 G^c (gdo_abc + gdo_bac); the
  // d_a G^c half follows with Gamma~
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double t2 = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) t2 += T.Gfg[c] * (gdo[a][sy(b, c)] + gdo[b][sy(a, c)]);
      T.Rt[sy(a, b)] += 0.5 * t2;
    }
  // -1/2 ginv^cd d_c d_d g_ab, folded over the symmetric pair (c,d)
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int d = c; d < 3; ++d) {
      const double w = (c == d ? -0.5 : -1.0) * gi[sy(c, d)] * (c == d ? o2[c] : o1[c] * o1[d]);
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        const double dd = c == d ? t_d2<ORD>(GS(a), tstr(c)) : t_d11<ORD>(GS(a), tstr(c), tstr(d));
        T.Rt[a] += w * dd;
      }
    }
  NR_OOH;
#pragma unroll
  for (int a = 0; a < 6; ++a) T.rg[a] = t_adv<ORD>(GS(a), ad, cw) + t_kof(GS(a), p, ooh, with_ko);
#undef GS
}

// group 2: Gamma~ (slots 6-8): 1/2 (g_ca d_b G^c + g_cb d_a G^c); advection, KO
template <int ORD>
__device__ __forceinline__ void tg_gamma(const double *sb, TileCarry &T, const double h[3], const AdvDir ad[3],
                                         const double cw[3], const nrgpu_bssn_params &p, bool with_ko) {
  NR_O1;
  double dG[3][3];
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int c = 0; c < 3; ++c) dG[b][c] = o1[b] * t_d1<ORD>((tap_t)(sb + (SL_GA + c) * kSlot), tstr(b));
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      double t2 = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) t2 += T.g[sy(c, a)] * dG[b][c] + T.g[sy(c, b)] * dG[a][c];
      T.Rt[sy(a, b)] += 0.5 * t2;
    }
  NR_OOH;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    tap_t c = (tap_t)(sb + (SL_GA + a) * kSlot);
    T.aG[a] = t_adv<ORD>(c, ad, cw);
    T.kG[a] = t_kof(c, p, ooh, with_ko);
  }
}

// group 3: chi (slot 9): the conformal-factor part of the Ricci tensor
template <int ORD>
__device__ __forceinline__ void tg_chi(const double *sb, TileCarry &T, const double h[3], const AdvDir ad[3],
                                       const double cw[3], const nrgpu_bssn_params &p, bool with_ko) {
  NR_O1;
  NR_O2;
  tap_t c = (tap_t)(sb + SL_CHI * kSlot);
  const double *gi = T.gi, *g = T.g;
  double chig = sb[SL_CHI * kSlot];
  if (chig < p.chiDivFloor) chig = p.chiDivFloor;
  const double oocp = 1.0 / p.chipsipower;
  const double f = oocp * log(chig);
  T.chig = chig;
  T.psim4 = exp(-4.0 * f);
#pragma unroll
  for (int a = 0; a < 3; ++a) T.df[a] = oocp * (o1[a] * t_d1<ORD>(c, tstr(a))) / chig;
  double dfdf = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) dfdf += gi[sy(a, b)] * T.df[a] * T.df[b];
  double cddf[6];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      const double ddchi = a == b ? o2[a] * t_d2<ORD>(c, tstr(a)) : o1[a] * o1[b] * t_d11<ORD>(c, tstr(a), tstr(b));
      double t = oocp * ddchi / chig - p.chipsipower * T.df[a] * T.df[b];
      t -= T.gam[0][sy(a, b)] * T.df[0] + T.gam[1][sy(a, b)] * T.df[1] + T.gam[2][sy(a, b)] * T.df[2];
      cddf[sy(a, b)] = t;
    }
  const double trcddf = gi[0] * cddf[0] + gi[3] * cddf[3] + gi[5] * cddf[5] +
                        2.0 * (gi[1] * cddf[1] + gi[2] * cddf[2] + gi[4] * cddf[4]);
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      const int ab = sy(a, b);
      T.Rt[ab] += 4.0 * T.df[a] * T.df[b] - 2.0 * cddf[ab] - 2.0 * g[ab] * trcddf - 4.0 * g[ab] * dfdf;
    }
  NR_OOH;
  T.rchi = t_adv<ORD>(c, ad, cw) + t_kof(c, p, ooh, with_ko);
}

// group 4: alpha (slot 10): D_a D_b alpha with the conformal correction
template <int ORD>
__device__ __forceinline__ void tg_alpha(const double *sb, TileCarry &T, const double h[3], const AdvDir ad[3],
                                         const double cw[3]) {
  NR_O1;
  NR_O2;
  tap_t c = (tap_t)(sb + SL_ALPHA * kSlot);
  const double *gi = T.gi;
#pragma unroll
  for (int a = 0; a < 3; ++a) T.da[a] = o1[a] * t_d1<ORD>(c, tstr(a));
  double dfda = 0.0;
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b) dfda += gi[sy(a, b)] * T.df[a] * T.da[b];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = a; b < 3; ++b) {
      const int ab = sy(a, b);
      double t = a == b ? o2[a] * t_d2<ORD>(c, tstr(a)) : o1[a] * o1[b] * t_d11<ORD>(c, tstr(a), tstr(b));
      t -= T.gam[0][ab] * T.da[0] + T.gam[1][ab] * T.da[1] + T.gam[2][ab] * T.da[2];
      T.cdda[ab] = t - 2.0 * (T.df[a] * T.da[b] + T.df[b] * T.da[a] - T.g[ab] * dfda);
    }
  T.trcdda = T.psim4 * (gi[0] * T.cdda[0] + gi[3] * T.cdda[3] + gi[5] * T.cdda[5] +
                        2.0 * (gi[1] * T.cdda[1] + gi[2] * T.cdda[2] + gi[4] * T.cdda[4]));
  T.ralpha = t_adv<ORD>(c, ad, cw);
}

// group 5: K (slot 11): its gradient, advection and KO
template <int ORD>
__device__ __forceinline__ void tg_K(const double *sb, TileCarry &T, const double h[3], const AdvDir ad[3],
                                     const double cw[3], const nrgpu_bssn_params &p, bool with_ko) {
  NR_O1;
  tap_t c = (tap_t)(sb + SL_K * kSlot);
#pragma unroll
  for (int a = 0; a < 3; ++a) T.dK[a] = p.forceKzerofactor * (o1[a] * t_d1<ORD>(c, tstr(a)));
  NR_OOH;
  T.rK = t_adv<ORD>(c, ad, cw) + t_kof(c, p, ooh, with_ko);
}

// the terms with A~ at the point and the lapse (before beta); point values
// of fields not resident come from global memory
__device__ __forceinline__ void tg_algebra(TileCarry &T, const nrgpu_bssn_params &p, const CVarPtrs &U, int x,
                                           double r[NRGPU_NV]) {
  const double *gi = T.gi, *g = T.g;
  double A[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) A[a] = ldg(U.p[A11 + a] + x);
  const double alpha = ldg(U.p[ALPHA] + x);
  const double K = ldg(U.p[KK] + x) * p.forceKzerofactor;
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
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    r[G11 + a] = -2.0 * alpha * A[a];
    r[A11 + a] = T.psim4 * (-T.cdda[a] + alpha * T.Rt[a]) - (1.0 / 3.0) * g[a] * (-T.trcdda + alpha * Rsc) +
                 alpha * (K * A[a] - 2.0 * AAab[a]);
  }
  r[KK] = -T.trcdda + alpha * (AAs + K * K / 3.0);
  // -2 Ainv da - 2 alpha divAinv, kept in r[GA] until the shift terms
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double t = 0.0, s = 0.0;
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      t += (2.0 / 3.0) * gi[sy(a, b)] * T.dK[b] - 6.0 * Ainv[sy(a, b)] * T.df[b];
      s += Ainv[sy(a, b)] * T.da[b];
    }
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) t -= T.gam[a][sy(b, c)] * Ainv[sy(b, c)];
    r[GA1 + a] = -2.0 * s - 2.0 * alpha * t;
  }
  r[CHI] = -(p.chipsipower / 6.0) * T.chig * alpha * K;
  const double falpha = p.oploglapse * p.lapseharmonicf + p.oploglapse2 * 8.0 / (3.0 * (3.0 - alpha)) +
                        p.harmoniclapse * alpha;
  r[ALPHA] = -falpha * alpha * K + p.oplogwithshift * T.ralpha;
}

// group 6: beta (slots 0-2 of round B): the Lie-derivative and shift terms,
// the gauge of the shift; r[B] waits for B's advection
template <int ORD>
__device__ __forceinline__ void tg_shift(const double *sb, TileCarry &T, const double h[3], const AdvDir ad[3],
                                         const double cw[3], const nrgpu_bssn_params &p, const CVarPtrs &U, int x,
                                         double r[NRGPU_NV]) {
  NR_O1;
  NR_O2;
  const double *gi = T.gi, *g = T.g;
  double db[3][3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) db[a][c] = o1[a] * t_d1<ORD>((tap_t)(sb + (SL_BETA + c) * kSlot), tstr(a));
  const double divbeta = db[0][0] + db[1][1] + db[2][2];
  const double totdivbeta = (2.0 / 3.0) * divbeta;
  double A[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) A[a] = ldg(U.p[A11 + a] + x);
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
  r[CHI] += (p.chipsipower / 6.0) * T.chig * divbeta;
  double trddb[3] = {0.0, 0.0, 0.0};
  double divdb[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int b = 0; b < 3; ++b)
#pragma unroll
    for (int c = b; c < 3; ++c)
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        tap_t cb = (tap_t)(sb + (SL_BETA + a) * kSlot);
        const double dd = b == c ? o2[b] * t_d2<ORD>(cb, tstr(b)) : o1[b] * o1[c] * t_d11<ORD>(cb, tstr(b), tstr(c));
        trddb[a] += (b == c ? 1.0 : 2.0) * gi[sy(b, c)] * dd;
        if (c == a) divdb[b] += dd;
        if (b == a && b != c) divdb[c] += dd;
      }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double t = trddb[a];
#pragma unroll
    for (int b = 0; b < 3; ++b) t += gi[sy(a, b)] * ((1.0 / 3.0) * divdb[b]) - T.Gfg[b] * db[b][a];
    r[GA1 + a] += t + T.Gfg[a] * totdivbeta;
  }
  const double alpha = ldg(U.p[ALPHA] + x);
  const double betaF = p.shiftgammacoeff * pow(alpha, p.shiftalphapower);
  const double bfac = p.gamma0factor + p.gamma2factor * betaF;
  const double alphaG = p.shiftgammacoeff * pow(alpha, p.shiftGalphapower);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    tap_t cb = (tap_t)(sb + (SL_BETA + a) * kSlot);
    const double Ba = ldg(U.p[BB1 + a] + x), ba = sb[(SL_BETA + a) * kSlot], Ga = ldg(U.p[GA1 + a] + x);
    const double rG = r[GA1 + a];
    r[BETA1 + a] = (p.gamma2factor + p.gamma0factor * betaF) * p.withB * Ba +
                   (1.0 - p.withB) * (alphaG * Ga - p.shiftdriver * ba) + p.withShiftadv * t_adv<ORD>(cb, ad, cw);
    r[BB1 + a] = p.withB * (bfac * rG - p.shiftdriver * Ba) + p.withB * (bfac * (1.0 - p.withGadv) * T.aG[a]);
    r[GA1 + a] = rG + T.aG[a] + T.kG[a];
  }
}

// group 7: A~ (slots 3-8 of round B): its advection and KO; the g~, chi
// and K partials
template <int ORD>
__device__ __forceinline__ void tg_A(const double *sb, TileCarry &T, const double h[3], const AdvDir ad[3],
                                     const double cw[3], const nrgpu_bssn_params &p, bool with_ko,
                                     double r[NRGPU_NV]) {
  NR_OOH;
#pragma unroll
  for (int a = 0; a < 6; ++a) {
    tap_t c = (tap_t)(sb + (SL_A + a) * kSlot);
    r[A11 + a] += t_adv<ORD>(c, ad, cw) + t_kof(c, p, ooh, with_ko);
    r[G11 + a] += T.rg[a];
  }
  r[CHI] += T.rchi;
  r[KK] = (r[KK] + T.rK) * p.forceKzerofactor;
}

// group 8: B (slots 9-11 of round B): its advection
template <int ORD>
__device__ __forceinline__ void tg_B(const double *sb, const AdvDir ad[3], const double cw[3],
                                     const nrgpu_bssn_params &p, double r[NRGPU_NV]) {
#pragma unroll
  for (int a = 0; a < 3; ++a)
    r[BB1 + a] += p.withB * p.withBadv * t_adv<ORD>((tap_t)(sb + (SL_B + a) * kSlot), ad, cw);
}
#undef NR_O1
#undef NR_O2
#undef NR_OOH

// one block per tile (the tiles of planes k0..k1 of one box, x fastest);
// ORD: the run's stencil order, computed where it fits
template <int ORD>
__global__ void __launch_bounds__(kTileThreads, 1)
    bssn_rhs_tile_kernel(const __grid_constant__ BssnMaps maps, CVarPtrs U, VarPtrs out, CVarPtrs pre, VarPtrs acc,
                         Epilogue E, const nrgpu_bssn_params p, BoxGeo box, const int *__restrict__ boundary,
                         double dx, double dy, double dz, int *status, int k0, int k1) {
  extern __shared__ __align__(128) double tsm_raw[];
  // the copy engine writes each box to a 128-byte aligned slot
  double *tsm = tsm_raw + ((128 - (tma::smem_addr(tsm_raw) & 127)) & 127) / 8;
  uint64_t *full = reinterpret_cast<uint64_t *>(tsm + kNSlot * kSlot);
  uint64_t *empty = full + kNSlot;
  const int tid = threadIdx.x, lane = tid & 31;
  const int lx = tid % kTX, ly = (tid / kTX) % kTY, lz = tid / (kTX * kTY);
  const int ntx = (box.m - 2 + kTX - 1) / kTX, nty = (box.n - 2 + kTY - 1) / kTY;
  const int t = blockIdx.x, tx = t % ntx, rr = t / ntx, ty = rr % nty, tz = rr / nty;
  // TMA coordinates of the staged boxes: the tile's first point minus the
  // halo (x is even, so every box starts on a 16-byte boundary)
  const int cx = kTX * tx - 2, cy = kTY * ty - 2, cz = k0 + kTZ * tz - kTH;
  bool ok = true;
  unsigned roundB = 0;   // thread 0: slots whose round-B load was issued
  if (tid == 0) {
    for (int s = 0; s < kNSlot; ++s) {
      tma::mbar_init(&full[s], 1);
      tma::mbar_init(&empty[s], kTileThreads / 32);
    }
    tma::mbar_fence_init();
    for (int s = 0; s < kNSlot; ++s) {
      tma::mbar_arrive_expect_tx(&full[s], kTileBoxBytes);
      tma::load_3d(tsm + s * kSlot, &maps.m[kRoundA[s]], cx, cy, cz, &full[s]);
    }
  }
  __syncthreads();
  auto wait_full = [&](int s0, int s1, unsigned par) {
    for (int s = s0; s < s1; ++s)
      if (ok && !tma::mbar_wait(&full[s], par)) {
        ok = false;
        atomicOr(status, 2);
      }
  };
  // all warps done with slots s0..s1-1 of round A: thread 0 loads their
  // round-B fields
  auto release_refill = [&](int s0, int s1) {
    __syncwarp();
    if (lane == 0)
      for (int s = s0; s < s1; ++s) tma::mbar_arrive(&empty[s]);
    if (tid == 0)
      for (int s = s0; s < s1; ++s) {
        if (ok && !tma::mbar_wait(&empty[s], 0)) {
          ok = false;
          atomicOr(status, 2);
        }
        if (ok) {
          tma::mbar_arrive_expect_tx(&full[s], kTileBoxBytes);
          tma::load_3d(tsm + s * kSlot, &maps.m[kRoundB[s]], cx, cy, cz, &full[s]);
          roundB |= 1u << s;
        }
      }
    __syncwarp();
  };

  const int i = 1 + kTX * tx + lx, j = 1 + kTY * ty + ly, k = k0 + kTZ * tz + lz;
  const int ijk = box.noffset + i + box.m * (j + box.n * k);
  bool act = i <= box.m - 2 && j <= box.n - 2 && k <= k1;
  if (act && __ldg(boundary + ijk) != 0) act = false;
  const int imax = box.m - 1, jmax = box.n - 1, kmax = box.o - 1;
  int d = min(min(i, j), k);
  d = min(d, min(min(imax - i, jmax - j), kmax - k));
  // points nearer the faces than the full stencil reaches: bssn_ladder_kernel
  if (d < ORD / 2) act = false;
  const double h[3] = {dx, dy, dz};
  // lopsided advection directions at this point (shared-memory strides)
  AdvDir ad[3];
  double cw[3];
  if (act) {
    const int lop = ORD == 2 ? 0 : (ORD == 6 ? p.advection_lopsided6 : p.advection_lopsided);
    const int idx[3] = {i, j, k}, mx[3] = {imax, jmax, kmax};
    const double oad = 1.0 / den1<ORD>();
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double w = ldg(U.p[BETA1 + a] + ijk) / h[a];
      ad[a] = adv_dir(idx[a], mx[a], w, ORD, lop, tstr(a));
      const int ws = w < 0 ? -1 : (w > 0 ? 1 : 0);
      cw[a] = -ws * w * oad;
    }
  }
  const bool with_ko = (p.order_dissipation == 4 && d >= 2) || (p.order_dissipation == 6 && d >= 3);
  const double *sb = tsm + (lx + kTH) + kTSY * (ly + kTH) + kTSZ * (lz + kTH);
  TileCarry T;
  double r[NRGPU_NV];
#define NR_TILE_DISPATCH(call_) \
  if (act && ok) {              \
    constexpr int O_ = ORD;     \
    call_;                      \
  }
  // round A
  wait_full(SL_G, SL_G + 6, 0);
  NR_TILE_DISPATCH(tg_metric<O_>(sb, T, h, ad, cw, p, with_ko));
  release_refill(SL_G, SL_G + 6);
  wait_full(SL_GA, SL_GA + 3, 0);
  NR_TILE_DISPATCH(tg_gamma<O_>(sb, T, h, ad, cw, p, with_ko));
  wait_full(SL_CHI, SL_CHI + 1, 0);
  NR_TILE_DISPATCH(tg_chi<O_>(sb, T, h, ad, cw, p, with_ko));
  wait_full(SL_ALPHA, SL_ALPHA + 1, 0);
  NR_TILE_DISPATCH(tg_alpha<O_>(sb, T, h, ad, cw));
  wait_full(SL_K, SL_K + 1, 0);
  NR_TILE_DISPATCH(tg_K<O_>(sb, T, h, ad, cw, p, with_ko));
  release_refill(SL_GA, kNSlot);
  if (act && ok) tg_algebra(T, p, U, ijk, r);
  // round B
  wait_full(SL_BETA, SL_BETA + 3, 1);
  NR_TILE_DISPATCH(tg_shift<O_>(sb, T, h, ad, cw, p, U, ijk, r));
  wait_full(SL_A, SL_A + 6, 1);
  NR_TILE_DISPATCH(tg_A<O_>(sb, T, h, ad, cw, p, with_ko, r));
  wait_full(SL_B, SL_B + 3, 1);
  NR_TILE_DISPATCH(tg_B<O_>(sb, ad, cw, p, r));
#undef NR_TILE_DISPATCH
  if (act && ok) {
    double s = 0.0;
#pragma unroll
    for (int v = 0; v < NRGPU_NV; ++v) s += r[v];
    if (!isfinite(s)) atomicOr(status, 1);
    store(r, ijk, out, pre, acc, E, p);
  }
  // every copy this block issued has landed before it exits (all of them
  // have been waited for unless a wait ran out)
  if (tid == 0)
    for (int s = 0; s < kNSlot; ++s) tma::mbar_wait(&full[s], (roundB >> s) & 1u);
}

// the persistent form: one block per SM computes tiles b, b + gridDim.x,
// ...; the next tile's round A is loaded while this tile's round B is
// consumed.  The grid spacing passes through an empty asm each tile so
// that the compiler recomputes the stencil weights instead of keeping them
// live across the whole loop.
template <int ORD>
__global__ void __launch_bounds__(kTileThreads, 1)
    bssn_rhs_tile_persistent_kernel(const __grid_constant__ BssnMaps maps, CVarPtrs U, VarPtrs out, CVarPtrs pre, VarPtrs acc,
                         Epilogue E, const nrgpu_bssn_params p, BoxGeo box, const int *__restrict__ boundary,
                         double dx, double dy, double dz, int *status, int k0, int k1) {
  extern __shared__ __align__(128) double tsm_raw[];
  double *tsm = tsm_raw + ((128 - (tma::smem_addr(tsm_raw) & 127)) & 127) / 8;
  uint64_t *full = reinterpret_cast<uint64_t *>(tsm + kNSlot * kSlot);
  uint64_t *empty = full + kNSlot;
  const int tid = threadIdx.x, lane = tid & 31;
  const int lx = tid % kTX, ly = (tid / kTX) % kTY, lz = tid / (kTX * kTY);
  const int ntx = (box.m - 2 + kTX - 1) / kTX, nty = (box.n - 2 + kTY - 1) / kTY;
  const int ntiles = ntx * nty * ((k1 - k0 + kTZ) / kTZ);
  bool ok = true;
  unsigned last = 0;   // thread 0: parity of the last load issued into each slot
  auto issue = [&](int s, int f, int tt) {
    const int tx = tt % ntx, rr = tt / ntx, ty = rr % nty, tz = rr / nty;
    tma::mbar_arrive_expect_tx(&full[s], kTileBoxBytes);
    tma::load_3d(tsm + s * kSlot, &maps.m[f], kTX * tx - 2, kTY * ty - 2, k0 + kTZ * tz - kTH, &full[s]);
  };
  if (tid == 0) {
    for (int s = 0; s < kNSlot; ++s) {
      tma::mbar_init(&full[s], 1);
      tma::mbar_init(&empty[s], kTileThreads / 32);
    }
    tma::mbar_fence_init();
    if ((int)blockIdx.x < ntiles)
      for (int s = 0; s < kNSlot; ++s) issue(s, kRoundA[s], blockIdx.x);
  }
  __syncthreads();
  auto wait_full = [&](int s0, int s1, unsigned par) {
    for (int s = s0; s < s1; ++s)
      if (ok && !tma::mbar_wait(&full[s], par)) {
        ok = false;
        atomicOr(status, 2);
      }
  };
  // all warps done with slots s0..s1-1 (phase par): thread 0 loads the
  // next fields into them (round B of this tile, or round A of tile tt)
  auto release_refill = [&](int s0, int s1, unsigned par, bool roundB, int tt) {
    __syncwarp();
    if (lane == 0)
      for (int s = s0; s < s1; ++s) tma::mbar_arrive(&empty[s]);
    if (tid == 0 && tt < ntiles)
      for (int s = s0; s < s1; ++s) {
        if (ok && !tma::mbar_wait(&empty[s], par)) {
          ok = false;
          atomicOr(status, 2);
        }
        if (ok) {
          issue(s, roundB ? kRoundB[s] : kRoundA[s], tt);
          last ^= 1u << s;
        }
      }
    __syncwarp();
  };
  const int co = (lx + kTH) + kTSY * (ly + kTH) + kTSZ * (lz + kTH);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int tn = t + gridDim.x;
    const int tx = t % ntx, rr = t / ntx, ty = rr % nty, tz = rr / nty;
    const int i = 1 + kTX * tx + lx, j = 1 + kTY * ty + ly, k = k0 + kTZ * tz + lz;
    const int ijk = box.noffset + i + box.m * (j + box.n * k);
    bool act = i <= box.m - 2 && j <= box.n - 2 && k <= k1;
    if (act && __ldg(boundary + ijk) != 0) act = false;
    const int imax = box.m - 1, jmax = box.n - 1, kmax = box.o - 1;
    int d = min(min(i, j), k);
    d = min(d, min(min(imax - i, jmax - j), kmax - k));
    if (d < ORD / 2) act = false;
    double h[3] = {dx, dy, dz};
    asm volatile("" : "+d"(h[0]), "+d"(h[1]), "+d"(h[2]));
    AdvDir ad[3];
    double cw[3];
    if (act) {
      const int lop = ORD == 2 ? 0 : (ORD == 6 ? p.advection_lopsided6 : p.advection_lopsided);
      const int idx[3] = {i, j, k}, mx[3] = {imax, jmax, kmax};
      const double oad = 1.0 / den1<ORD>();
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double w = ldg(U.p[BETA1 + a] + ijk) / h[a];
        ad[a] = adv_dir(idx[a], mx[a], w, ORD, lop, tstr(a));
        const int ws = w < 0 ? -1 : (w > 0 ? 1 : 0);
        cw[a] = -ws * w * oad;
      }
    }
    const bool with_ko = (p.order_dissipation == 4 && d >= 2) || (p.order_dissipation == 6 && d >= 3);
    const double *sb = tsm + co;
    TileCarry T;
    double r[NRGPU_NV];
#define NR_TILE_DISPATCH(call_) \
  if (act && ok) {              \
    constexpr int O_ = ORD;     \
    call_;                      \
  }
    wait_full(SL_G, SL_G + 6, 0);
    NR_TILE_DISPATCH(tg_metric<O_>(sb, T, h, ad, cw, p, with_ko));
    release_refill(SL_G, SL_G + 6, 0, true, t);
    wait_full(SL_GA, SL_GA + 3, 0);
    NR_TILE_DISPATCH(tg_gamma<O_>(sb, T, h, ad, cw, p, with_ko));
    wait_full(SL_CHI, SL_CHI + 1, 0);
    NR_TILE_DISPATCH(tg_chi<O_>(sb, T, h, ad, cw, p, with_ko));
    wait_full(SL_ALPHA, SL_ALPHA + 1, 0);
    NR_TILE_DISPATCH(tg_alpha<O_>(sb, T, h, ad, cw));
    wait_full(SL_K, SL_K + 1, 0);
    NR_TILE_DISPATCH(tg_K<O_>(sb, T, h, ad, cw, p, with_ko));
    release_refill(SL_GA, kNSlot, 0, true, t);
    if (act && ok) tg_algebra(T, p, U, ijk, r);
    wait_full(SL_BETA, SL_BETA + 3, 1);
    NR_TILE_DISPATCH(tg_shift<O_>(sb, T, h, ad, cw, p, U, ijk, r));
    release_refill(SL_BETA, SL_BETA + 3, 1, false, tn);
    wait_full(SL_A, SL_A + 6, 1);
    NR_TILE_DISPATCH(tg_A<O_>(sb, T, h, ad, cw, p, with_ko, r));
    release_refill(SL_A, SL_A + 6, 1, false, tn);
    wait_full(SL_B, SL_B + 3, 1);
    NR_TILE_DISPATCH(tg_B<O_>(sb, ad, cw, p, r));
    release_refill(SL_B, kNSlot, 1, false, tn);
#undef NR_TILE_DISPATCH
    if (act && ok) {
      double s = 0.0;
#pragma unroll
      for (int v = 0; v < NRGPU_NV; ++v) s += r[v];
      if (!isfinite(s)) atomicOr(status, 1);
      store(r, ijk, out, pre, acc, E, p);
    }
  }
  if (tid == 0)
    for (int s = 0; s < kNSlot; ++s) tma::mbar_wait(&full[s], ((last >> s) & 1u));
}
