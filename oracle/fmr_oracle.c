/* fmr_oracle.c -- CPU restatement of the reference's fixed mesh refinement
 * around the evolution: refinement flags, Lagrange restriction and
 * prolongation between a level and its child, time interpolation of the
 * parent to the child's half step, and the Berger-Oliger recursion.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/ (through oracle/oracle.py) as
 * the checker of the CUDA path; the product never links or calls it.
 *
 * Restates, FP64, for one or several boxes per level (the single-rank
 * nested-box grid; several boxes where the punctures' boxes do not merge):
 *   setRPflags               flag.c:122-255 (flagprolong on the child,
 *                            flagrestrict on the parent)
 *   restrict_varlist_boxtobox_N / restrict_boxtobox_N
 *                            interpolate_boxtobox_N.c:1055-1370 (bounding
 *                            box of flagrestrict >= 3, N-point Lagrange at
 *                            the midpoint, sweeps z then y then x)
 *   prolong_varlist_boxtobox_N / prolong_boxtobox_N
 *                            interpolate_boxtobox_N.c:585-1054 (bounding box
 *                            of 1 <= flagprolong <= amr_nbuffer minus the
 *                            inner box, tested on the first point of each
 *                            x pair; Lagrange at N/2-1/4 and N/2-3/4)
 *   coefficients_lagrange_N  lagrange.c:13-27
 *   restrict_prolong_evolve  inject.c:116-132 (time-interpolated parent
 *                            unless the levels are aligned in time)
 *   evolve                   evolve.c:292-340,371-380 (time interpolation
 *                            orders 2 and 3 around the RK4 step; the
 *                            algebraic constraints come after it)
 * With several boxes on a level, each fine box pairs with the coarse box
 * that holds it (BAM's box->pr): the flags, the restriction box and the
 * prolongation box are those of the pair (the reference computes them on a
 * ghost parent of each fine box, flag.c:122-255 with
 * interpolate_boxtobox_N.c:870-1370 looping forallboxes(lf)), every pair
 * is restricted before any is prolonged (restrict_prolong_varlist,
 * inject.c:63-100).
 * The Berger-Oliger recursion that strings these together
 * (advance_levelandsublevels, main.c:397-418) is restated in oracle/oracle.py.
 * Every sum runs in the reference's order, so restriction, prolongation and
 * time interpolation are reproduced bit for bit; the evolution itself is
 * nr_oracle.c's.  Pinned by tests/test_fmr_oracle_pin.py against dumps of
 * the reference's own multi-level runs.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "../include/nrgpu.h"

int oracle_bssn_rk4_stages(const nrgpu_level_desc *L, double *const *u, double dt, const nrgpu_bssn_params *p);
int oracle_bssn_algcon(const nrgpu_level_desc *L, double *const *u, const nrgpu_bssn_params *p);
int oracle_z4_rk4_stages(const nrgpu_level_desc *L, double *const *u, double dt, const nrgpu_z4_params *p);
void oracle_z4_algcon(const nrgpu_level_desc *L, double *const *u, const nrgpu_z4_params *p);

#define NMAXRP 8

static void lagrange(int n, double x, double *c)
{
  for (int i = 0; i < n; i++) {
    double d = 1;
    for (int j = 0; j < n; j++)
      if (j != i) d *= (x - 0.0 - j * 1.0) / ((i - j) * 1.0);
    c[i] = d;
  }
}

/* index helpers of box.c:284-307 */
static int parent_index(double cx0, double cdx, double fx0, double fdx, int fi)
{
  return (int)(0.5 + (fx0 + fi * fdx - cx0) / cdx);
}
static int point_index(double X0, double dX, double x0, double dx, int i)
{
  return (int)((x0 + i * dx - X0) / dX);
}

typedef struct { int n[3]; double x0[3], dx[3]; long off; } box_t;

static box_t box_of(const nrgpu_level_desc *L, int ib)
{
  box_t b;
  b.n[0] = L->box[ib].m; b.n[1] = L->box[ib].n; b.n[2] = L->box[ib].o;
  b.x0[0] = L->box[ib].x0; b.x0[1] = L->box[ib].y0; b.x0[2] = L->box[ib].z0;
  b.dx[0] = L->dx; b.dx[1] = L->dy; b.dx[2] = L->dz;
  b.off = L->box[ib].noffset;
  return b;
}

static long at(const box_t *b, int i, int j, int k) { return b->off + i + (long)b->n[0] * (j + (long)b->n[1] * k); }

/* the coarse box holding every parent point of the fine box (box->pr) */
static int parent_box(const nrgpu_level_desc *C, const box_t *f)
{
  for (int ib = 0; ib < C->nboxes; ib++) {
    box_t c = box_of(C, ib);
    int ok = 1;
    for (int d = 0; d < 3; d++) {
      int lo = parent_index(c.x0[d], c.dx[d], f->x0[d], f->dx[d], 0);
      int hi = parent_index(c.x0[d], c.dx[d], f->x0[d], f->dx[d], f->n[d] - 1);
      if (lo < 0 || hi >= c.n[d]) ok = 0;
    }
    if (ok) return ib;
  }
  return -1;
}

/* setRPflags (flag.c:122-255) of one fine box and its parent box, no
 * symmetry: flagprolong over the fine box, flagrestrict on the parent box
 * (the caller clears cr) */
static int pair_flags(const box_t *cp, const box_t *fp_box, int nbuffer, double *fp, double *cr)
{
  box_t f = *fp_box, c = *cp;
  int np = f.n[0] * f.n[1] * f.n[2];
  for (int k = 0; k < f.n[2]; k++)
    for (int j = 0; j < f.n[1]; j++)
      for (int i = 0; i < f.n[0]; i++) {
        const int idx[3] = {i, j, k};
        int m[3];
        for (int d = 0; d < 3; d++) {
          double lo = f.x0[d], hi = f.x0[d] + (f.n[d] - 1) * f.dx[d];
          double x = f.x0[d] + idx[d] * f.dx[d];
          int n;
          m[d] = np;
          n = (int)(1.5 + (x - lo) / f.dx[d]);
          if (n <= nbuffer) m[d] = n;
          n = (int)(1.5 - (x - hi) / f.dx[d]);
          if (n <= nbuffer) m[d] = n;
        }
        int ii = m[0];
        if (ii > m[1]) ii = m[1];
        if (ii > m[2]) ii = m[2];
        fp[at(&f, i, j, k)] = ii < np ? ii : 0;
      }
  for (int pass = 0; pass < 2; pass++)
    for (int k = 0; k < f.n[2]; k++)
      for (int j = 0; j < f.n[1]; j++)
        for (int i = 0; i < f.n[0]; i++) {
          double p = fp[at(&f, i, j, k)];
          int pi = parent_index(c.x0[0], c.dx[0], f.x0[0], f.dx[0], i);
          int pj = parent_index(c.x0[1], c.dx[1], f.x0[1], f.dx[1], j);
          int pk = parent_index(c.x0[2], c.dx[2], f.x0[2], f.dx[2], k);
          if (pi < 0 || pj < 0 || pk < 0 || pi >= c.n[0] || pj >= c.n[1] || pk >= c.n[2]) return -1;
          long q = at(&c, pi, pj, pk);
          if (pass == 0 && p == 0) cr[q] = 3;
          if (pass == 1) {
            if (p >= 3) cr[q] = 2;
            else if (p == 2) cr[q] = 1;
          }
        }
  return 0;
}

/* setRPflags of every fine box: fp over the fine level, cr over the coarse
 * level (with several fine boxes, the union of the pairs' flags) */
int oracle_fmr_flags(const nrgpu_level_desc *C, const nrgpu_level_desc *F, int nbuffer, double *fp, double *cr)
{
  for (long q = 0; q < C->npoints; q++) cr[q] = 0;
  for (int ib = 0; ib < F->nboxes; ib++) {
    box_t f = box_of(F, ib);
    int pb = parent_box(C, &f);
    if (pb < 0) return -1;
    box_t c = box_of(C, pb);
    if (pair_flags(&c, &f, nbuffer, fp, cr)) return -1;
  }
  return 0;
}

/* restriction of nv variables from the fine box f into its parent box c
 * (restrict_varlist_boxtobox_N with nbuffer >= 3, i.e. flagrestrict >= 3) */
static int restrict_pair(const box_t *cp, const box_t *fp_box, const double *cr, int nv, double *const *uc,
                         double *const *uf, int order)
{
  box_t f = *fp_box, c = *cp;
  const int b = order / 2;
  int ic[6] = {1 << 30, -(1 << 30), 1 << 30, -(1 << 30), 1 << 30, -(1 << 30)};
  long n = 0;
  for (int k = 0; k < c.n[2]; k++)
    for (int j = 0; j < c.n[1]; j++)
      for (int i = 0; i < c.n[0]; i++)
        if (cr[at(&c, i, j, k)] >= 3) {
          const int idx[3] = {i, j, k};
          for (int d = 0; d < 3; d++) {
            if (idx[d] < ic[2 * d]) ic[2 * d] = idx[d];
            if (idx[d] > ic[2 * d + 1]) ic[2 * d + 1] = idx[d];
          }
          n++;
        }
  if (!n) return 0;
  int ifb[6];
  for (int d = 0; d < 3; d++) {
    ifb[2 * d] = point_index(f.x0[d], f.dx[d], c.x0[d], c.dx[d], ic[2 * d]) - b + 1;
    ifb[2 * d + 1] = point_index(f.x0[d], f.dx[d], c.x0[d], c.dx[d], ic[2 * d + 1]) + b;
    if (ifb[2 * d] < 0 || ifb[2 * d + 1] >= f.n[d]) return -2;  /* boxes too small */
  }
  double w[NMAXRP];
  lagrange(order, order / 2.0 - 0.5, w);
  for (int v = 0; v < nv; v++) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int K = ic[4]; K <= ic[5]; K++)
      for (int J = ic[2]; J <= ic[3]; J++)
        for (int I = ic[0]; I <= ic[1]; I++) {
          int fx = ifb[0] + 2 * (I - ic[0]), fy = ifb[2] + 2 * (J - ic[2]), fz = ifb[4] + 2 * (K - ic[4]);
          double sx = 0;
          for (int px = 0; px < order; px++) {
            double sy = 0;
            for (int py = 0; py < order; py++) {
              double sz = 0;
              for (int pz = 0; pz < order; pz++) sz += w[pz] * uf[v][at(&f, fx + px, fy + py, fz + pz)];
              sy += w[py] * sz;
            }
            sx += w[px] * sy;
          }
          uc[v][at(&c, I, J, K)] = sx;
        }
  }
  return 0;
}

/* prolongation of nv variables from the parent box c into the fine box f
 * (prolong_varlist_boxtobox_N with nbuffer >= 3) */
static int prolong_pair(const box_t *cp, const box_t *fp_box, const double *fp, int nv, double *const *uc,
                        double *const *uf, int order, int amr_nbuffer)
{
  box_t f = *fp_box, c = *cp;
  const int b = order / 2;
  int ifb[6] = {1 << 30, -(1 << 30), 1 << 30, -(1 << 30), 1 << 30, -(1 << 30)};
  int if0[6] = {1 << 30, -(1 << 30), 1 << 30, -(1 << 30), 1 << 30, -(1 << 30)};
  long n = 0;
  for (int k = 0; k < f.n[2]; k++)
    for (int j = 0; j < f.n[1]; j++)
      for (int i = 0; i < f.n[0]; i++) {
        const int idx[3] = {i, j, k};
        double p = fp[at(&f, i, j, k)];
        int *bb = (p > 0 && amr_nbuffer >= p) ? ifb : if0;
        if (bb == ifb) n++;
        for (int d = 0; d < 3; d++) {
          if (idx[d] < bb[2 * d]) bb[2 * d] = idx[d];
          if (idx[d] > bb[2 * d + 1]) bb[2 * d + 1] = idx[d];
        }
      }
  if (!n) return 0;
  int ic[6];
  for (int d = 0; d < 3; d++) {
    ic[2 * d] = point_index(c.x0[d], c.dx[d], f.x0[d], f.dx[d], ifb[2 * d]) - b + 1;
    ic[2 * d + 1] = point_index(c.x0[d], c.dx[d], f.x0[d], f.dx[d], ifb[2 * d + 1]) + b;
    if (ic[2 * d] < 0 || ic[2 * d + 1] >= c.n[d]) return -2;  /* boxes too small */
    if ((ifb[2 * d + 1] - ifb[2 * d] + 1) % 2) return -3;      /* pairs of children only */
  }
  double c1[NMAXRP], c2[NMAXRP];
  lagrange(order, order / 2.0 - 0.25, c1);
  lagrange(order, order / 2.0 - 0.75, c2);
  for (int v = 0; v < nv; v++) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int k = ifb[4]; k <= ifb[5]; k++)
      for (int j = ifb[2]; j <= ifb[3]; j++)
        for (int i = ifb[0]; i <= ifb[1]; i++) {
          int i0 = ifb[0] + 2 * ((i - ifb[0]) / 2);
          if (i0 >= if0[0] && i0 <= if0[1] && j >= if0[2] && j <= if0[3] && k >= if0[4] && k <= if0[5]) continue;
          const int t[3] = {i - ifb[0], j - ifb[2], k - ifb[4]};
          int s[3];
          const double *w[3];
          for (int d = 0; d < 3; d++) {
            s[d] = ic[2 * d] + t[d] / 2 + t[d] % 2;
            w[d] = t[d] % 2 ? c2 : c1;
          }
          double sx = 0;
          for (int px = 0; px < order; px++) {
            double sy = 0;
            for (int py = 0; py < order; py++) {
              double sz = 0;
              for (int pz = 0; pz < order; pz++) sz += w[2][pz] * uc[v][at(&c, s[0] + px, s[1] + py, s[2] + pz)];
              sy += w[1][py] * sz;
            }
            sx += w[0][px] * sy;
          }
          uf[v][at(&f, i, j, k)] = sx;
        }
  }
  return 0;
}

/* restrict_prolong_varlist (inject.c:63-100) with nbuffer = 3: restrict
 * the child into uc, then prolong uc into the child's buffer zone */
int oracle_fmr_restrict_prolong(const nrgpu_level_desc *C, const nrgpu_level_desc *F, int nv, double *const *uc,
                                double *const *uf, int order, int amr_nbuffer)
{
  double *fp = malloc(sizeof(double) * F->npoints), *cr = malloc(sizeof(double) * C->npoints);
  int e = 0;
  /* every pair is restricted, with its own flags, before any is prolonged */
  for (int ib = 0; ib < F->nboxes && !e; ib++) {
    box_t f = box_of(F, ib);
    int pb = parent_box(C, &f);
    if (pb < 0) {
      e = -1;
      break;
    }
    box_t c = box_of(C, pb);
    for (long q = 0; q < C->npoints; q++) cr[q] = 0;
    e = pair_flags(&c, &f, amr_nbuffer, fp, cr);
    if (!e) e = restrict_pair(&c, &f, cr, nv, uc, uf, order);
  }
  for (int ib = 0; ib < F->nboxes && !e; ib++) {
    box_t f = box_of(F, ib), c = box_of(C, parent_box(C, &f));
    e = prolong_pair(&c, &f, fp, nv, uc, uf, order, amr_nbuffer);
  }
  free(fp);
  free(cr);
  return e;
}

/* r = ca a + cb b with vladd's special cases (variables.c:575-650) */
static void vl_add(long np, int nv, double *const *r, double ca, double *const *a, double cb, double *const *b)
{
  for (int v = 0; v < nv; v++)
#pragma omp parallel for schedule(static)
    for (long i = 0; i < np; i++) {
      if (ca == 0 && cb == 0) r[v][i] = 0;
      else if (ca == 0) r[v][i] = cb * b[v][i];
      else if (cb == 0) r[v][i] = ca * a[v][i];
      else r[v][i] = ca * a[v][i] + cb * b[v][i];
    }
}

/* one step of a level: evolve() with the time interpolation of a level that
 * has a child around the RK4 stages (evolve.c:292-340, 371-380), then the
 * algebraic constraints (the EVOLVE functions after evolve).  system 0:
 * BSSN with nrgpu_bssn_params, 1: Z4c with nrgpu_z4_params.  iteration is
 * the level's iteration before the step; with_child = 0 skips the
 * interpolant (uprev, upp unused).  order_ti 2..6; for orders 4-6, hist
 * holds the older time levels u(n-2), u(n-3), u(n-4) (u_p2, u_p3, u_p4 of
 * evolve.c:289-294), shifted back as the reference does (:336-338). */
int oracle_fmr_evolve_level_h(const nrgpu_level_desc *L, int system, const void *params, int nv, double *const *u,
                              double *const *uprev, double *const *upp, double *const *p2, double *const *p3,
                              double *const *p4, double dt, int iteration, int with_child, int order_ti)
{
  const long np = L->npoints;
  int o = 0, err = 0;
  if (with_child) {
    if (order_ti < 2 || order_ti > 6) return -5;
    if ((order_ti >= 4 && !p2) || (order_ti >= 5 && !p3) || (order_ti >= 6 && !p4)) return -1;
    o = iteration + 2 > order_ti ? order_ti : iteration + 2;
    if (o == 2) vl_add(np, nv, upp, 0.5, u, 0.0, u);
    if (o == 3) vl_add(np, nv, upp, 0.75, u, -0.125, uprev);
    if (o == 4) {
      vl_add(np, nv, upp, 15.0 / 16, u, -5.0 / 16, uprev);
      vl_add(np, nv, upp, 1.0, upp, 1.0 / 16, p2);
    }
    if (o == 5) {
      vl_add(np, nv, upp, 140.0 / 128, u, -70.0 / 128, uprev);
      vl_add(np, nv, upp, 1.0, upp, 28.0 / 128, p2);
      vl_add(np, nv, upp, 1.0, upp, -5.0 / 128, p3);
    }
    if (o == 6) {
      vl_add(np, nv, upp, 315.0 / 256, u, -210.0 / 256, uprev);
      vl_add(np, nv, upp, 1.0, upp, 126.0 / 256, p2);
      vl_add(np, nv, upp, 1.0, upp, -45.0 / 256, p3);
      vl_add(np, nv, upp, 1.0, upp, 7.0 / 256, p4);
    }
    for (int v = 0; v < nv; v++) {
      if (o >= 6) memcpy(p4[v], p3[v], sizeof(double) * np);
      if (o >= 5) memcpy(p3[v], p2[v], sizeof(double) * np);
      if (o >= 4) memcpy(p2[v], uprev[v], sizeof(double) * np);
      /* the RK4 step's u_p copy, kept as u(n-1) for the next step */
      memcpy(uprev[v], u[v], sizeof(double) * np);
    }
  }
  if (system == 0) err |= oracle_bssn_rk4_stages(L, u, dt, (const nrgpu_bssn_params *)params);
  else err |= oracle_z4_rk4_stages(L, u, dt, (const nrgpu_z4_params *)params);
  if (with_child) {
    static const double c[7] = {0, 0, 1.0 / 2, 3. / 8, 5. / 16, 35. / 128, 63. / 256};
    vl_add(np, nv, upp, 1.0, upp, c[o], u);
  }
  if (system == 0) oracle_bssn_algcon(L, u, (const nrgpu_bssn_params *)params);
  else oracle_z4_algcon(L, u, (const nrgpu_z4_params *)params);
  return err;
}

int oracle_fmr_evolve_level(const nrgpu_level_desc *L, int system, const void *params, int nv, double *const *u,
                            double *const *uprev, double *const *upp, double dt, int iteration, int with_child,
                            int order_ti)
{
  if (with_child && (order_ti < 2 || order_ti > 3)) return -5;
  return oracle_fmr_evolve_level_h(L, system, params, nv, u, uprev, upp, 0, 0, 0, dt, iteration, with_child,
                                   order_ti);
}
