/* mg_oracle.c -- CPU restatement of the reference's puncture multigrid.
 *
 * TEST INFRASTRUCTURE ONLY (the checker of the CUDA multigrid; loaded by
 * tests/ and bench.py's cpu_baseline leg through oracle/oracle.py).
 *
 * Restates, for the single-box puncture grid with a Robin outer boundary:
 *   puncture coefficients  SetMWBL / mwblpsiofxyz (ConformalFactor.c:81-134),
 *                          BY_Kofxyz (ExtrinsicCurvature.c:61-113),
 *                          SetPunctureCoefficients (Punctures.c:320-362)
 *   the stack              coarsegridsize / makestack (makestack.c:36-127),
 *                          initializestack (makestack.c:139-170)
 *   Robin normals / BC     find_robin_normal (robin.c:29-143),
 *                          set_boundary_robin (robin.c:146-223)
 *   operator / smoother    Lpuncture_nonlin, Lpuncture_GS (PunctureSolve.c:21-138)
 *                          through uni_gauss_seidel (relax.c:174-190)
 *   FAS transfer           finetocoarse, coarsetofine (fasmg.c:41-122),
 *                          mg_restrict_var, mg_prolong_var (restrictprolong.c:21-122)
 *   cycles                 fullVdriver, solve (solve.c:20-161), exactsolve
 *                          (exactsolve.c:18-77), restau (residual.c:42-75)
 *   norms                  l2norm = RMS over flag-0 points (reduce.c:209-246)
 * Level 0 of the stack is the coarsest; every stack level is one box with
 * its outer layer flagged PHYBOUND.  In this configuration the reference's
 * order -4 prolongation of the full-V driver and the refinement-boundary
 * prolongation are never reached (restrictprolong.c:184-209: all levels are
 * at or below ltop), so trilinear prolongation is used throughout.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  int m;          /* points per direction (cube) */
  double dx, x0;  /* spacing, coordinate of point 0 */
  long np;
  int *flag;      /* 0 inner, 1 PHYBOUND */
  long *normal;   /* Robin normal neighbour of boundary points */
  double *u, *v, *w, *f, *a, *b;
} mglevel;

typedef struct {
  int npre, npost, exact_nmin, exact_nmax, vnmin, vnmax, fullV, size_nmin, levels_nmax;
  double tol, falloff;
} mgpar;

#define IJK(L, i, j, k) ((long)(i) + (long)(L)->m * ((long)(j) + (long)(L)->m * (long)(k)))

static double xof(const mglevel *L, int i) { return L->x0 + i * L->dx; }

static void level_init(mglevel *L, int m, double dx)
{
  long q;
  L->m = m;
  L->dx = dx;
  L->x0 = -(m - 1) * dx / 2;
  L->np = (long)m * m * m;
  L->flag = calloc(L->np, sizeof(int));
  L->normal = calloc(L->np, sizeof(long));
  L->u = calloc(L->np, sizeof(double));
  L->v = calloc(L->np, sizeof(double));
  L->w = calloc(L->np, sizeof(double));
  L->f = calloc(L->np, sizeof(double));
  L->a = calloc(L->np, sizeof(double));
  L->b = calloc(L->np, sizeof(double));
  for (q = 0; q < L->np; q++) {
    int i = q % m, j = (q / m) % m, k = q / ((long)m * m);
    L->flag[q] = (i == 0 || j == 0 || k == 0 || i == m - 1 || j == m - 1 || k == m - 1);
  }
}

static void level_free(mglevel *L)
{
  free(L->flag); free(L->normal); free(L->u); free(L->v); free(L->w); free(L->f); free(L->a); free(L->b);
}

/* find_robin_normal: average of unit directions to the non-boundary members
 * of the 27-point neighbourhood (missing neighbours count as the point
 * itself, which is a boundary point), then the direction with the largest
 * projection, first maximum in (i,j,k) loop order */
static void robin_normals(mglevel *L)
{
  int m = L->m;
  long q;
  for (q = 0; q < L->np; q++) {
    int i = q % m, j = (q / m) % m, k = q / ((long)m * m);
    int a, b, c;
    double vx = 0, vy = 0, vz = 0, max = 0;
    long best = q;
    if (!L->flag[q]) continue;
    for (a = 0; a < 3; a++)
      for (b = 0; b < 3; b++)
        for (c = 0; c < 3; c++) {
          int ii = i + a - 1, jj = j + b - 1, kk = k + c - 1;
          long n;
          double s;
          if (ii < 0 || jj < 0 || kk < 0 || ii >= m || jj >= m || kk >= m) continue;
          n = IJK(L, ii, jj, kk);
          if (L->flag[n]) continue;
          s = sqrt((double)((a - 1) * (a - 1) + (b - 1) * (b - 1) + (c - 1) * (c - 1)));
          vx += (a - 1) / s; vy += (b - 1) / s; vz += (c - 1) / s;
        }
    for (a = 0; a < 3; a++)
      for (b = 0; b < 3; b++)
        for (c = 0; c < 3; c++) {
          int ii = i + a - 1, jj = j + b - 1, kk = k + c - 1;
          long n;
          double s, dot;
          if (ii < 0 || jj < 0 || kk < 0 || ii >= m || jj >= m || kk >= m) continue;
          n = IJK(L, ii, jj, kk);
          if (L->flag[n]) continue;
          s = sqrt((double)((a - 1) * (a - 1) + (b - 1) * (b - 1) + (c - 1) * (c - 1)));
          dot = (vx * (a - 1) + vy * (b - 1) + vz * (c - 1)) / s;
          if (dot > max) { max = dot; best = n; }
        }
    L->normal[q] = best;
  }
}

/* set_boundary_robin for one scalar with far limit 0 */
static void robin(const mglevel *L, double *u, double falloff)
{
  int m = L->m;
  long q;
#pragma omp parallel for schedule(static)
  for (q = 0; q < L->np; q++) {
    long n;
    int i, j, k, ni, nj, nk;
    double x1, y1, z1, x0, y0, z0, x, y, z;
    if (!L->flag[q]) continue;
    n = L->normal[q];
    i = q % m; j = (q / m) % m; k = q / ((long)m * m);
    ni = n % m; nj = (n / m) % m; nk = n / ((long)m * m);
    x1 = xof(L, i); y1 = xof(L, j); z1 = xof(L, k);
    x0 = xof(L, ni); y0 = xof(L, nj); z0 = xof(L, nk);
    x = 0.5 * (x1 + x0); y = 0.5 * (y1 + y0); z = 0.5 * (z1 + z0);
    if (falloff == 0) {
      /* Dirichlet variant with robin_1oR_constant = 0 */
      u[q] = -u[n];
    } else {
      double vx = x1 - x0, vy = y1 - y0, vz = z1 - z0;
      double c = 0.5 * falloff * (vx * x + vy * y + vz * z) / (x * x + y * y + z * z);
      u[q] = 2 * c * 0.0 + u[n] * (1 - c) / (1 + c);
    }
  }
}

#define FALLOFF_U 1.0  /* punctures_robin_falloff, set for u and its duplicates */
#define FALLOFF_RF 0.0 /* punctures_r, punctures_f: no boundary info set */

/* Lpuncture_nonlin: Robin on u first, then L u on inner points */
static void lop(const mglevel *L, double *u, double *lu)
{
  int m = L->m;
  double cx = 1 / (L->dx * L->dx), cc = -2 * (cx + cx + cx);
  long q;
  robin(L, u, FALLOFF_U);
#pragma omp parallel for schedule(static)
  for (q = 0; q < L->np; q++) {
    if (L->flag[q]) continue;
    lu[q] = cc * u[q] + cx * (u[q - 1] + u[q + 1]) + cx * (u[q - m] + u[q + m]) +
            cx * (u[q - (long)m * m] + u[q + (long)m * m]) + L->b[q] * pow(1 + L->a[q] * (1 + u[q]), -7.0);
  }
}

/* Lpuncture_GS: Jacobi update of un from uo, then Robin on un */
static void lgs(const mglevel *L, const double *uo, double *un)
{
  int m = L->m;
  double cx = 1 / (L->dx * L->dx), cc = -2 * (cx + cx + cx);
  long q;
#pragma omp parallel for schedule(static)
  for (q = 0; q < L->np; q++) {
    double lu, lii;
    if (L->flag[q]) continue;
    lu = cc * uo[q] + cx * (uo[q - 1] + uo[q + 1]) + cx * (uo[q - m] + uo[q + m]) +
         cx * (uo[q - (long)m * m] + uo[q + (long)m * m]) + L->b[q] * pow(1 + L->a[q] * (1 + uo[q]), -7.0);
    lii = cc - 7 * L->b[q] * L->a[q] * pow(1 + L->a[q] * (1 + uo[q]), -8.0);
    un[q] = uo[q] + (L->f[q] - lu) / lii;
  }
  robin(L, un, FALLOFF_U);
}

/* one uni_gauss_seidel sweep: v = u, u = GS(v), v = 0 */
static void sweep(mglevel *L)
{
  memcpy(L->v, L->u, L->np * sizeof(double));
  lgs(L, L->v, L->u);
  memset(L->v, 0, L->np * sizeof(double));
}

static double l2inner(const mglevel *L, const double *r)
{
  long q, n = 0;
  double s = 0;
  for (q = 0; q < L->np; q++)
    if (!L->flag[q]) { s += r[q] * r[q]; n++; }
  return n ? sqrt(s / n) : -1;
}

/* residual norm: v = L u - f (inner), boundary of v by its own condition */
static double findres(mglevel *L)
{
  long q;
  lop(L, L->u, L->v);
  for (q = 0; q < L->np; q++)
    if (!L->flag[q]) L->v[q] = L->v[q] - L->f[q];
  robin(L, L->v, FALLOFF_RF);
  return l2inner(L, L->v);
}

/* 8-point average of the fine children of every inner coarse point */
static void restrict8(const mglevel *F, const double *fv, const mglevel *Cl, double *cv)
{
  int mc = Cl->m, mf = F->m;
  long q;
#pragma omp parallel for schedule(static)
  for (q = 0; q < Cl->np; q++) {
    int I, J, K, i, j, k;
    long f0;
    if (Cl->flag[q]) continue;
    I = q % mc; J = (q / mc) % mc; K = q / ((long)mc * mc);
    /* box_child_index: (cx0 + I cdx - fx0)/fdx truncated */
    i = (int)((xof(Cl, I) - F->x0) / F->dx);
    j = (int)((xof(Cl, J) - F->x0) / F->dx);
    k = (int)((xof(Cl, K) - F->x0) / F->dx);
    f0 = IJK(F, i, j, k);
    cv[q] = 0.125 * (fv[f0] + fv[f0 + 1 + mf + (long)mf * mf] + fv[f0 + 1] + fv[f0 + mf] +
                     fv[f0 + (long)mf * mf] + fv[f0 + 1 + mf] + fv[f0 + 1 + (long)mf * mf] +
                     fv[f0 + mf + (long)mf * mf]);
  }
  (void)mf;
}

/* trilinear prolongation onto the inner fine points (mg_prolong_var) */
static void prolong2(const mglevel *Cl, const double *cv, const mglevel *F, double *fv)
{
  int mc = Cl->m, mf = F->m;
  long q;
#pragma omp parallel for schedule(static)
  for (q = 0; q < F->np; q++) {
    int i, j, k, ci, cj, ck;
    long c0;
    double kx1, ky1, kz1, kx0, ky0, kz0;
    if (F->flag[q]) continue;
    i = q % mf; j = (q / mf) % mf; k = q / ((long)mf * mf);
    ci = (int)((xof(F, i) - Cl->x0) / Cl->dx);
    cj = (int)((xof(F, j) - Cl->x0) / Cl->dx);
    ck = (int)((xof(F, k) - Cl->x0) / Cl->dx);
    c0 = IJK(Cl, ci, cj, ck);
    kx1 = (xof(F, i) - xof(Cl, ci)) / Cl->dx;
    ky1 = (xof(F, j) - xof(Cl, cj)) / Cl->dx;
    kz1 = (xof(F, k) - xof(Cl, ck)) / Cl->dx;
    kx0 = 1 - kx1; ky0 = 1 - ky1; kz0 = 1 - kz1;
    fv[q] = kx0 * ky0 * kz0 * cv[c0] + kx1 * ky0 * kz0 * cv[c0 + 1] + kx0 * ky1 * kz0 * cv[c0 + mc] +
            kx1 * ky1 * kz0 * cv[c0 + 1 + mc] + kx0 * ky0 * kz1 * cv[c0 + (long)mc * mc] +
            kx1 * ky0 * kz1 * cv[c0 + 1 + (long)mc * mc] + kx0 * ky1 * kz1 * cv[c0 + mc + (long)mc * mc] +
            kx1 * ky1 * kz1 * cv[c0 + 1 + mc + (long)mc * mc];
  }
}

/* finetocoarse (fasmg.c:41-92) */
static void finetocoarse(mglevel *h, mglevel *H)
{
  long q;
  lop(h, h->u, h->v);                   /* vh = L uh */
  restrict8(h, h->v, H, H->v);          /* vH = R vh */
  for (q = 0; q < h->np; q++)           /* vh = vh - fh */
    if (!h->flag[q]) h->v[q] -= h->f[q];
  robin(h, h->v, FALLOFF_RF);
  restrict8(h, h->u, H, H->u);          /* uH = R uh */
  robin(H, H->u, FALLOFF_U);
  lop(H, H->u, H->f);                   /* fH = L uH */
  for (q = 0; q < H->np; q++)           /* fH = fH - vH */
    if (!H->flag[q]) H->f[q] -= H->v[q];
  robin(H, H->f, FALLOFF_RF);
  restrict8(h, h->f, H, H->v);          /* vH = R fh */
  for (q = 0; q < H->np; q++)           /* fH = vH + fH */
    if (!H->flag[q]) H->f[q] = H->v[q] + H->f[q];
  robin(H, H->f, FALLOFF_RF);
  memcpy(H->w, H->u, H->np * sizeof(double));  /* wH = uH */
}

/* coarsetofine (fasmg.c:98-122) */
static void coarsetofine(mglevel *H, mglevel *h)
{
  long q;
  for (q = 0; q < H->np; q++)           /* vH = uH - wH */
    if (!H->flag[q]) H->v[q] = H->u[q] - H->w[q];
  robin(H, H->v, FALLOFF_RF);
  prolong2(H, H->v, h, h->v);           /* vh = P vH */
  for (q = 0; q < h->np; q++)           /* uh = uh + vh */
    if (!h->flag[q]) h->u[q] += h->v[q];
  robin(h, h->u, FALLOFF_U);
}

static int exactsolve(mglevel *L, const mgpar *p)
{
  int i;
  double normres;
  findres(L);
  for (i = 1; i <= p->exact_nmax; i++) {
    sweep(L);
    if (i >= p->exact_nmin) {
      normres = findres(L);
      if (normres < p->tol / 10) break;
    }
  }
  findres(L);
  return i;
}

static void solve(mglevel *lv, int l, const mgpar *p)
{
  int i;
  if (l == 0) {
    exactsolve(&lv[0], p);
    return;
  }
  for (i = 0; i < p->npre; i++) sweep(&lv[l]);
  finetocoarse(&lv[l], &lv[l - 1]);
  solve(lv, l - 1, p);
  coarsetofine(&lv[l - 1], &lv[l]);
  for (i = 0; i < p->npost; i++) sweep(&lv[l]);
}

/* stack sizes: coarsegridsize (makestack.c:36-79) for one rank */
int oracle_mg_stack_sizes(int m, int size_nmin, int levels_nmax, int *sizes, int maxlevels)
{
  int n = 0, l = 1;
  sizes[n++] = m;
  while (n < maxlevels) {
    int mnew;
    if (levels_nmax != -1 && l > levels_nmax) break;
    if ((m - 2) % 4) break;
    mnew = m / 2 + 1;
    if (mnew < size_nmin) break;
    if (mnew < 4) break;  /* mg_size_nmin_local = 4 on one rank */
    sizes[n++] = m = mnew;
    l++;
  }
  return n;
}

/* Brill-Lindquist + Bowen-York coefficients a, b on a cube of m points */
void oracle_puncture_coefficients(int m, double dx, int npunc, const double *mass, const double *pos,
                                  const double *mom, const double *spin, double *a, double *b)
{
  double x0 = -(m - 1) * dx / 2;
  long q, np = (long)m * m * m;
#pragma omp parallel for
  for (q = 0; q < np; q++) {
    int i = q % m, j = (q / m) % m, k = q / ((long)m * m), n, s, t;
    double x = x0 + i * dx, y = x0 + j * dx, z = x0 + k * dx;
    double p = 0, K[3][3] = {{0}}, K2, psi;
    for (n = 0; n < npunc; n++) {
      double xi = x - pos[3 * n], yi = y - pos[3 * n + 1], zi = z - pos[3 * n + 2];
      double r = sqrt(xi * xi + yi * yi + zi * zi), N[3], NP, eNS[3];
      const double *P = mom + 3 * n, *S = spin + 3 * n;
      if (!(r < 0.0 - 1e-10 || 0.0 < r - 1e-10)) r = 1e-15; /* dequal(r,0) -> EPSZERO */
      p += mass[n] * (1 / r) * (0.5);
      N[0] = xi / r; N[1] = yi / r; N[2] = zi / r;
      NP = N[0] * P[0] + N[1] * P[1] + N[2] * P[2];
      eNS[0] = N[1] * S[2] - N[2] * S[1];
      eNS[1] = N[2] * S[0] - N[0] * S[2];
      eNS[2] = N[0] * S[1] - N[1] * S[0];
      for (s = 0; s < 3; s++)
        for (t = s; t < 3; t++)
          K[s][t] += 1.5 / (r * r) * (N[s] * P[t] + N[t] * P[s] - ((s == t) - N[s] * N[t]) * NP) -
                     3.0 / (r * r * r) * (eNS[s] * N[t] + eNS[t] * N[s]);
    }
    psi = p + 1.0;
    a[q] = 1 / (psi - 1);
    K2 = K[0][0] * K[0][0] + K[1][1] * K[1][1] + K[2][2] * K[2][2] + 2 * K[0][1] * K[0][1] +
         2 * K[0][2] * K[0][2] + 2 * K[1][2] * K[1][2];
    b[q] = 0.125 * pow(a[q], 7.0) * K2;
  }
}

/* multigrid (multigrid.c:35-123) on one cube: u in/out (initial guess,
 * boundary included), a, b coefficients; returns the number of V cycles
 * on the finest level; res_hist[n] = residual before cycle n (finest) */
int oracle_mg_solve(int m, double dx, const double *a, const double *b, double *u, int npre, int npost,
                    int exact_nmin, int exact_nmax, int vnmin, int vnmax, int fullV, int size_nmin,
                    int levels_nmax, double tol, double *res_hist, int *nlevels_out)
{
  int sizes[32], nl, l, n = 0, top;
  mglevel lv[32];
  mgpar p;
  p.npre = npre; p.npost = npost; p.exact_nmin = exact_nmin; p.exact_nmax = exact_nmax;
  p.vnmin = vnmin; p.vnmax = vnmax; p.fullV = fullV; p.size_nmin = size_nmin;
  p.levels_nmax = levels_nmax; p.tol = tol; p.falloff = 1;
  nl = oracle_mg_stack_sizes(m, size_nmin, levels_nmax, sizes, 32);
  top = nl - 1;
  /* level index 0 = coarsest */
  for (l = 0; l < nl; l++) {
    int s = sizes[nl - 1 - l];
    level_init(&lv[l], s, dx * (double)(1 << (nl - 1 - l)));
  }
  memcpy(lv[top].u, u, lv[top].np * sizeof(double));
  memcpy(lv[top].a, a, lv[top].np * sizeof(double));
  memcpy(lv[top].b, b, lv[top].np * sizeof(double));
  for (l = 0; l <= top; l++) robin_normals(&lv[l]);
  /* initializestack: restrict coefficients and fields down the stack */
  for (l = top; l > 0; l--) {
    restrict8(&lv[l], lv[l].a, &lv[l - 1], lv[l - 1].a);
    restrict8(&lv[l], lv[l].b, &lv[l - 1], lv[l - 1].b);
    restrict8(&lv[l], lv[l].u, &lv[l - 1], lv[l - 1].u);
  }
  /* v, w, f start at zero on every level (multigrid.c:91-98) */
  for (l = fullV ? 0 : top; l <= top; l++) {
    for (n = 0; n < vnmax; n++) {
      if (n >= vnmin) {
        double r2 = findres(&lv[l]);
        if (l == top && res_hist) res_hist[n] = r2;
        if (r2 <= tol) break;
      }
      solve(lv, l, &p);
      if (l == 0) break;
    }
    if (l < top) {
      prolong2(&lv[l], lv[l].u, &lv[l + 1], lv[l + 1].u);
      robin(&lv[l + 1], lv[l + 1].u, FALLOFF_U);
    }
  }
  memcpy(u, lv[top].u, lv[top].np * sizeof(double));
  if (nlevels_out) *nlevels_out = nl;
  for (l = 0; l < nl; l++) level_free(&lv[l]);
  return n;
}
