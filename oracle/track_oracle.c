/* track_oracle.c -- CPU restatement of the reference's shift-integration
 * puncture tracker.  TEST INFRASTRUCTURE ONLY: the checker of the tracker
 * kernel (baum_b200/csrc/nrgpu_track.cu), pinned to the reference's own
 * results in tests/golden/track_*.npz; never product code.
 *
 * Followed, step by step:
 *   interpolate_xyz_scalar   utility/interpolate/interpolate.c:419-470
 *     cube origin from the level's lower corner, first node that matches it
 *     (dequal), the cube must fit in that node's box
 *     (interpolate_fillindexcube, interpolate.c:53-92), else the value is 0
 *   interpolate_TriN         interpolate.c:121-160 (LAGRANGE: z, then y, then x)
 *   coefficients_lagrange_N  interpolate/lagrange.c:13-27
 *   interpolate_lagrange_N   lagrange.c:30-39
 *   track_moving_puncture_integrate  Gauge/moving_punctures_integrate.c:29-100
 *     (half-grid test, shift one step earlier at the old position, three
 *     averaged corrector passes, z pinned for moving_puncture_fixz BH/BHNS)
 *   the position test of track_puncture  Gauge/moving_punctures.c:189-191
 *     (xyzinsidelevel, main/amr/points.c:100-133)
 *   findextremum, track_moving_puncture_extremum
 *                            moving_punctures_integrate.c:105-235
 *     (a parabola through three interpolated values per axis, the step
 *     clamped to one grid spacing, taken only if the value improves and the
 *     step is at least minmove)
 */
#include <math.h>

#include "../include/nrgpu.h"

#define EPS 1e-10 /* dequaleps, main/main/bam_main.h:19 */

static int dless(double a, double b) { return a < b - EPS; }
static int dequal(double a, double b) { return !(dless(a, b) || dless(b, a)); }

static void lagrange(int n, double x, double xmin, double h, double *c)
{
  for (int i = 0; i < n; i++) {
    double d = 1;
    for (int j = 0; j < n; j++)
      if (j != i) d *= (x - xmin - j * h) / ((i - j) * h);
    c[i] = d;
  }
}

static double dot(int n, const double *c, const double *u)
{
  double s = 0;
  for (int i = 0; i < n; i++) s += c[i] * u[i];
  return s;
}

/* the level's lower corner (the lattice origin of the cube search) */
static void level_origin(const nrgpu_level_desc *L, double *o)
{
  o[0] = L->box[0].x0;
  o[1] = L->box[0].y0;
  o[2] = L->box[0].z0;
  for (int b = 1; b < L->nboxes; b++) {
    if (L->box[b].x0 < o[0]) o[0] = L->box[b].x0;
    if (L->box[b].y0 < o[1]) o[1] = L->box[b].y0;
    if (L->box[b].z0 < o[2]) o[2] = L->box[b].z0;
  }
}

/* node index of coordinate c on a box axis from x0, or -1 */
static int node_of(double c, double x0, double h, int n)
{
  int i = (int)floor((c - x0) / h + 0.5);
  if (i < 0 || i >= n || !dequal(c, x0 + i * h)) return -1;
  return i;
}

double oracle_interpolate(const nrgpu_level_desc *L, const double *v, double x, double y, double z, int order)
{
  const double h[3] = {L->dx, L->dy, L->dz};
  const int a = order, n = (order - 1) / 2;
  double o[3], xc[3];
  const double p[3] = {x, y, z};
  level_origin(L, o);
  for (int d = 0; d < 3; d++) xc[d] = o[d] + h[d] * (floor((p[d] - o[d] + EPS) / h[d]) - n);
  for (int b = 0; b < L->nboxes; b++) {
    const nrgpu_box *B = &L->box[b];
    int i = node_of(xc[0], B->x0, h[0], B->m);
    int j = node_of(xc[1], B->y0, h[1], B->n);
    int k = node_of(xc[2], B->z0, h[2], B->o);
    if (i < 0 || j < 0 || k < 0) continue;
    /* the first node that matches decides: the cube must fit in its box */
    if (i + a > B->m || j + a > B->n || k + a > B->o) return 0.0;
    double c[8], w[8], vv[8][8];
    lagrange(a, z, xc[2], h[2], c);
    for (int ii = 0; ii < a; ii++)
      for (int jj = 0; jj < a; jj++) {
        double line[8];
        for (int kk = 0; kk < a; kk++)
          line[kk] = v[B->noffset + (i + ii) + B->m * (j + jj) + B->m * B->n * (k + kk)];
        vv[ii][jj] = dot(a, c, line);
      }
    lagrange(a, y, xc[1], h[1], c);
    for (int ii = 0; ii < a; ii++) w[ii] = dot(a, c, vv[ii]);
    lagrange(a, x, xc[0], h[0], c);
    return dot(a, c, w);
  }
  return 0.0;
}

static int inside_level(const nrgpu_level_desc *L, const double *p)
{
  const double h[3] = {L->dx, L->dy, L->dz};
  int inside = 0;
  for (int b = 0; b < L->nboxes; b++) {
    const nrgpu_box *B = &L->box[b];
    const double lo[3] = {B->x0, B->y0, B->z0};
    const int n[3] = {B->m, B->n, B->o};
    int in = 1;
    for (int d = 0; d < 3; d++)
      if (dless(p[d], lo[d]) || dless(lo[d] + (n[d] - 1) * h[d], p[d])) in = 0;
    inside += in;
  }
  return inside;
}

/* n punctures: pold[3n] -> pnew[3n]; moved[n] is the integrator's return
 * value, inside[n] the position test of the new location */
int oracle_track_punctures(const nrgpu_level_desc *L, const double *const *beta, const double *const *beta_p,
                           double dt, int order, int fixz, int np, const double *pold, double *pnew, int *moved,
                           int *inside)
{
  if (order < 2 || order > 8) return NRGPU_ERR_UNSUPPORTED;
  for (int q = 0; q < np; q++) {
    const double *p1 = pold + 3 * q;
    double *p0 = pnew + 3 * q;
    double b1[3], b0[3];
    int skip = 0;
    for (int d = 0; d < 3; d++) {
      p0[d] = p1[d];
      if ((L->symmetry >> d & 1) && dless(p1[d], 0)) skip = 1;
    }
    moved[q] = !skip;
    if (!skip) {
      for (int d = 0; d < 3; d++) b1[d] = oracle_interpolate(L, beta_p[d], p1[0], p1[1], p1[2], order);
      for (int it = 0; it < 3; it++) {
        for (int d = 0; d < 3; d++) b0[d] = oracle_interpolate(L, beta[d], p0[0], p0[1], p0[2], order);
        for (int d = 0; d < 3; d++) p0[d] = p1[d] - dt * 0.5 * (b0[d] + b1[d]);
      }
      if (fixz) p0[2] = p1[2];
    }
    inside[q] = inside_level(L, p0);
  }
  return 0;
}

/* the vertex of the parabola through (-1, vm), (0, v0), (1, vp), clamped to
 * [-1, 1]; toward the larger neighbour when the curvature vanishes */
static double findextremum(double vm, double v0, double vp, int max)
{
  double v;
  if (!isfinite(vm) || !isfinite(v0) || !isfinite(vp)) return 0.;
  if (fabs(0.5 * (vp + vm) - v0) <= 1e-10) {
    if ((vp > v0) && (vp > vm)) v = 1.;
    else if ((vm > v0) && (vm > vp)) v = -1.;
    else v = 0.;
    v *= max ? 1. : -1.;
  } else {
    v = (vm - vp) / (4. * (0.5 * (vp + vm) - v0));
    v = v > 1. ? 1. : v;
    v = v < -1. ? -1. : v;
  }
  return v;
}

/* extremum search of var around each old position: pnew, and the position
 * test of the new location (the integrator's return value is always 1) */
int oracle_track_extremum(const nrgpu_level_desc *L, const double *var, int find_max, double minmove, int order,
                          int fixz, int np, const double *pold, double *pnew, int *inside)
{
  if (order < 2 || order > 8) return NRGPU_ERR_UNSUPPORTED;
  const double h[3] = {L->dx, L->dy, L->dz};
  const double minimal_move = minmove * L->dx;
  for (int q = 0; q < np; q++) {
    const double *p0 = pold + 3 * q;
    double *p1 = pnew + 3 * q;
    double d[3];
    const double v0 = oracle_interpolate(L, var, p0[0], p0[1], p0[2], order);
    for (int a = 0; a < 3; a++) {
      double pm[3] = {p0[0], p0[1], p0[2]}, pp[3] = {p0[0], p0[1], p0[2]};
      pm[a] = p0[a] - h[a];
      pp[a] = p0[a] + h[a];
      const double vm = oracle_interpolate(L, var, pm[0], pm[1], pm[2], order);
      const double vp = oracle_interpolate(L, var, pp[0], pp[1], pp[2], order);
      d[a] = findextremum(vm, v0, vp, find_max) * h[a];
    }
    const double v = oracle_interpolate(L, var, p0[0] + d[0], p0[1] + d[1], p0[2] + d[2], order);
    if (!isfinite(v) || !isfinite(v0) || (find_max && v <= v0) || (!find_max && v >= v0) ||
        sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) < minimal_move)
      d[0] = d[1] = d[2] = 0.;
    for (int a = 0; a < 3; a++) p1[a] = p0[a] + d[a];
    if (fixz) p1[2] = p0[2];
    inside[q] = inside_level(L, p1);
  }
  return 0;
}
