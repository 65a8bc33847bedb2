/* nrharness.c -- a BAM project compiled only into the oracle binary
 * oracle/_ref/bam.  Test infrastructure, never product code.
 *
 * It does three things to make the reference's own CPU evolution and
 * multigrid comparable with the GPU path, bit for bit in layout:
 *   1. nrharness_data = fourier: after the evolution system's startup
 *      (POST_INITIALDATA, bssn.c:260 / z4.c:176 run before this module),
 *      overwrite every evolved variable with a flat background plus a sum of
 *      seeded Fourier modes (the synthetic data of the batched FMR workload).
 *      The generator (splitmix64 draws, mode layout) is restated in
 *      baum_b200/synthetic.py so the GPU side can rebuild the same state.
 *   2. nrharness_rhs = yes: evaluate the registered RHS once on the initial
 *      state through the reference's evolve_rhs (evolve.c:37), including the
 *      boundary callback, and dump it.
 *   3. nrharness_dump = "i0 i1 ...": dump the evolved variables of every
 *      level after those level iterations (POST_EVOLVE), and after the
 *      initial data when 0 is listed.
 *   6. nrharness_admmass = yes: with the reference's ADM_mass project, dump
 *      its integrands and their inputs and write its sphere integrals with
 *      all digits (admmass_itN_lL.bin/.txt).
 *   5. nrharness_dump_moved = yes: dump every level that move_box moved,
 *      after the move (POST_MOVEBOX), as moved_itN_lL.bin.
 *   4. nrharness_track = yes: with each of those dumps, run the reference's
 *      shift-integration puncture tracker (track_moving_puncture_integrate,
 *      Gauge/moving_punctures_integrate.c:29-100) from every start position
 *      of nrharness_track_points on that level, with the z coordinate free
 *      and pinned (moving_puncture_fixz), and write the results as text
 *      (track_itN_lL.txt) beside a dump of the current and previous shift.
 * Dump format (little endian), one file per (tag, level):
 *   int64 magic 0x3147524e ("NRG1"), l, nboxes, nvars, npoints, iteration
 *   double time, dx, dy, dz, dt
 *   per box: int64 m, n, o, noffset; double x0, y0, z0
 *   per var: char name[32]
 *   int32 boundary[npoints]
 *   double data[nvars][npoints]
 */
#include "bam.h"
#include "bam_nrharness.h"

static unsigned long long sm_state;
static unsigned long long splitmix64(void)
{
  unsigned long long z = (sm_state += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static double uniform01(void) { return (splitmix64() >> 11) * (1.0 / 9007199254740992.0); }

static int is_unit_background(const char *name)
{
  const char *unit[] = {"bssn_gxx", "bssn_gyy", "bssn_gzz", "bssn_chi",
                        "z4_gxx", "z4_gyy", "z4_gzz", "z4_chi", "alpha", 0};
  int i;
  for (i = 0; unit[i]; i++) if (!strcmp(name, unit[i])) return 1;
  return 0;
}

static void dump_varlist(tL *level, tVarList *vl, const char *tag)
{
  char fn[1024];
  FILE *f;
  long long hdr[6];
  double dh[5];
  int b, v;
  snprintf(fn, sizeof fn, "%s/%s_l%d.bin", Gets("nrharness_dir"), tag, level->l);
  f = fopen(fn, "wb");
  if (!f) errorexits("nrharness: cannot open %s", fn);
  hdr[0] = 0x3147524e; hdr[1] = level->l; hdr[2] = level->nboxes; hdr[3] = vl->n;
  hdr[4] = level->npoints; hdr[5] = level->iteration;  /* before the step */
  fwrite(hdr, sizeof(long long), 6, f);
  dh[0] = level->time; dh[1] = level->dx; dh[2] = level->dy; dh[3] = level->dz; dh[4] = level->dt;
  fwrite(dh, sizeof(double), 5, f);
  for (b = 0; b < level->nboxes; b++) {
    tB *box = level->box[b];
    long long bi[4] = {box->m, box->n, box->o, box->noffset};
    double bx[3] = {box->x0, box->y0, box->z0};
    fwrite(bi, sizeof(long long), 4, f);
    fwrite(bx, sizeof(double), 3, f);
  }
  for (v = 0; v < vl->n; v++) {
    char name[32];
    memset(name, 0, sizeof name);
    strncpy(name, VarName(vl->index[v]), 31);
    fwrite(name, 1, 32, f);
  }
  fwrite(level->boundary, sizeof(int), level->npoints, f);
  for (v = 0; v < vl->n; v++) {
    double *p = level->v[vl->index[v]];
    if (!p) errorexits("nrharness: variable %s not enabled", VarName(vl->index[v]));
    fwrite(p, sizeof(double), level->npoints, f);
  }
  fclose(f);
  printf("nrharness: wrote %s\n", fn);
}

/* ADM variables (bssn_to_adm / z4_to_adm have run at POST_EVOLVE, before
 * this module) and the constraints of adm_constraints_N (adm.c:14-74),
 * dumped together */
void adm_constraints_N(tVarList *ucon, tVarList *uadm);
static void dump_constraints(tL *level, const char *tag)
{
  tVarList *con = vlalloc(level), *adm = vlalloc(level), *all = vlalloc(level);
  vlpush(con, Ind("ham"));
  vlpush(con, Ind("momx"));
  if (Getv("adm_normalizedConstraints", "yes")) {
    vlpush(con, Ind("normham"));
    vlpush(con, Ind("normmomx"));
  }
  enablevarlist(con);
  vlpush(adm, Ind("adm_gxx"));
  vlpush(adm, Ind("adm_Kxx"));
  vlpush(adm, Ind("adm_psi"));
  vlpush(adm, Ind("adm_dpsiopsix"));
  vlpush(adm, Ind("adm_ddpsiopsixx"));
  adm_constraints_N(con, adm);
  vlpush(all, Ind("adm_gxx"));
  vlpush(all, Ind("adm_Kxx"));
  vlpush(all, Ind("ham"));
  vlpush(all, Ind("momx"));
  if (Getv("adm_normalizedConstraints", "yes")) {
    vlpush(all, Ind("normham"));
    vlpush(all, Ind("normmomx"));
  }
  dump_varlist(level, all, tag);
  vlfree(con);
  vlfree(adm);
  vlfree(all);
}

static int dump_requested(int iteration)
{
  char s[32];
  snprintf(s, sizeof s, "%d", iteration);
  return Getv("nrharness_dump", s);
}

static void set_fourier(tL *level, tVarList *u)
{
  const int nmodes = Geti("nrharness_nmodes");
  const double amp = Getd("nrharness_amp");
  const double L = Getd("nrharness_length");
  double k[64][3], cf, ph;
  double *x = level->v[Ind("x")], *y = level->v[Ind("y")], *z = level->v[Ind("z")];
  int m, v, i;
  if (nmodes > 64) errorexit("nrharness: at most 64 modes");
  sm_state = (unsigned long long)Geti("nrharness_seed");
  for (m = 0; m < nmodes; m++)
    for (i = 0; i < 3; i++) {
      /* integer wave numbers in [-2, 2] per axis on the box length L */
      int n = (int)(splitmix64() % 5ULL) - 2;
      k[m][i] = 2.0 * PI * n / L;
    }
  for (v = 0; v < u->n; v++) {
    double *p = level->v[u->index[v]];
    double base = is_unit_background(VarName(u->index[v])) ? 1.0 : 0.0;
    double c[64], phase[64];
    for (m = 0; m < nmodes; m++) {
      c[m] = 2.0 * uniform01() - 1.0;
      phase[m] = 2.0 * PI * uniform01();
    }
    for (i = 0; i < level->npoints; i++) {
      double s = 0;
      for (m = 0; m < nmodes; m++)
        s += c[m] * sin(k[m][0] * x[i] + k[m][1] * y[i] + k[m][2] * z[i] + phase[m]);
      p[i] = base + amp * s;
    }
  }
  (void)cf; (void)ph;
}

int nrharness_post_initialdata(tL *level)
{
  tVarList *u = 0;
  evolve_vlretrieve(&u, 0, 0);
  if (u) u->level = level;
  if (Getv("nrharness_data", "fourier")) {
    if (!u) errorexit("nrharness: no evolved variables");
    set_fourier(level, u);
  }
  if (Getv("nrharness_mg", "yes")) {
    tVarList *vl = vlalloc(level);
    vlpush(vl, Ind("punctures_u"));
    if (level->v[Ind("punctures_u")]) dump_varlist(level, vl, "mg_u");
    vlfree(vl);
  }
  if (Getv("nrharness_flags", "yes")) {
    /* refinement flags of setRPflags (flag.c:122-255): flagprolong on levels
       with a parent, flagrestrict on levels with a child */
    tVarList *vl = vlalloc(level);
    if (level->v[Ind("flagprolong")]) vlpush(vl, Ind("flagprolong"));
    if (level->v[Ind("flagrestrict")]) vlpush(vl, Ind("flagrestrict"));
    if (vl->n) dump_varlist(level, vl, "flags");
    vlfree(vl);
  }
  if (u && dump_requested(0)) dump_varlist(level, u, "state_it0");
  if (u && Getv("nrharness_rhs", "yes")) {
    tVarList *r = AddDuplicateEnable(u, "_nrh");
    evolve_rhs(r, u, 0.0, u, 0);
    dump_varlist(level, r, "rhs_it0");
  }
  return 0;
}

static void dump_track(tL *level, const char *tag);
static void dump_0d(tL *level, tVarList *u, const char *tag);

int nrharness_post_evolve(tL *level)
{
  tVarList *u = 0;
  char tag[64];
  evolve_vlretrieve(&u, 0, 0);
  if (!u) return 0;
  u->level = level;
  /* POST_EVOLVE runs before the level's iteration counter is advanced
     (main.c:466-474): this is the state after iteration+1 steps */
  if (dump_requested(level->iteration + 1)) {
    snprintf(tag, sizeof tag, "state_it%d", level->iteration + 1);
    dump_varlist(level, u, tag);
    if (Getv("nrharness_constraints", "yes")) {
      snprintf(tag, sizeof tag, "con_it%d", level->iteration + 1);
      dump_constraints(level, tag);
    }
    if (Getv("nrharness_0d", "yes")) {
      snprintf(tag, sizeof tag, "red0d_it%d", level->iteration + 1);
      dump_0d(level, u, tag);
    }
    if (Getv("nrharness_track", "yes")) {
      snprintf(tag, sizeof tag, "track_it%d", level->iteration + 1);
      dump_track(level, tag);
    }
  }
  return 0;
}

/* after move_box (main.c:428-435, POST_MOVEBOX on every moved level): the
   moved level's state, the state at the end of the coarse step for a level
   that moved after its last POST_EVOLVE */
int nrharness_post_movebox(tL *level)
{
  tVarList *u = 0;
  char tag[64];
  if (!Getv("nrharness_dump_moved", "yes")) return 0;
  evolve_vlretrieve(&u, 0, 0);
  if (!u) return 0;
  u->level = level;
  snprintf(tag, sizeof tag, "moved_it%d", level->iteration);
  dump_varlist(level, u, tag);
  return 0;
}

/* ANALYZE after ADM_mass (projects/ADM_mass/ADM_mass.c:11-225, run with
   ADM_mass_persist = yes so its integrands stay): on the coarsest level of
   a time-aligned stack, at a dump iteration, every level of the stack is
   dumped with the integrands and their inputs (admmass_itN_lL.bin), and the
   reference's integral_over_sphere of each integrand at each radius of
   ADM_mass_r that lies safely inside the level is written with all digits
   (admmass_itN_lL.txt: radius, then the 8 integrals) */
double integral_over_sphere(tL *level, double x0, double y0, double z0, int ntheta, int nphi, double r,
                            int index, int order);
/* after Invariants (projects/Invariants/Invariants.c:48-252, run with
   invariants_persist = yes): rpsi4, ipsi4 (restricted, prolonged and
   rescaled by r) and Csqr with their inputs on every level of the stack */
static void dump_psi4(tL *level)
{
  tG *g = level->grid;
  char tag[64];
  int l;
  for (l = level->l; l <= g->lmax; l++) {
    tL *lv = g->level[l];
    tVarList *vl = vlalloc(lv);
    vlpush(vl, Ind("rpsi4"));
    vlpush(vl, Ind("ipsi4"));
    vlpush(vl, Ind("Csqr"));
    vlpush(vl, Ind("adm_gxx"));
    vlpush(vl, Ind("adm_Kxx"));
    vlpush(vl, Ind("alpha"));
    vlpush(vl, Ind("betax"));
    snprintf(tag, sizeof tag, "psi4_it%d", lv->iteration);
    dump_varlist(lv, vl, tag);
    vlfree(vl);
  }
}

int nrharness_analyze(tL *level)
{
  if (Getv("nrharness_psi4", "yes") && dump_requested(level->iteration) && !parentaligned(level))
    dump_psi4(level);
  static const char *names[8] = {"ADM_mass_integrand", "ADM_mass_integrand_chi", "ADM_mass_Pxint",
                                 "ADM_mass_Pyint", "ADM_mass_Pzint", "ADM_mass_Jxint", "ADM_mass_Jyint",
                                 "ADM_mass_Jzint"};
  tG *g = level->grid;
  char tag[64], fn[1024];
  int l, v;
  if (!Getv("nrharness_admmass", "yes") || !dump_requested(level->iteration) || parentaligned(level)) return 0;
  for (l = level->l; l <= g->lmax; l++) {
    tL *lv = g->level[l];
    tVarList *vl = vlalloc(lv);
    char *rs, *r1;
    FILE *f;
    for (v = 0; v < 8; v++) vlpush(vl, Ind(names[v]));
    vlpush(vl, Ind("adm_gxx"));
    vlpush(vl, Ind("adm_Kxx"));
    vlpush(vl, Ind("bssn_K"));
    vlpush(vl, Ind("bssn_chi"));
    snprintf(tag, sizeof tag, "admmass_it%d", lv->iteration);
    dump_varlist(lv, vl, tag);
    vlfree(vl);
    snprintf(fn, sizeof fn, "%s/%s_l%d.txt", Gets("nrharness_dir"), tag, l);
    f = fopen(fn, "w");
    if (!f) errorexits("nrharness: cannot open %s", fn);
    rs = Gets("ADM_mass_r");
    while ((r1 = NextEntry(rs))) {
      double r = atof(r1);
      if (!centered_sphere_safely_inside_level(lv, r)) continue;
      fprintf(f, "%.17e", r);
      for (v = 0; v < 8; v++)
        fprintf(f, " %.17e", integral_over_sphere(lv, 0, 0, 0, Geti("ADM_mass_ncircles"), Geti("ADM_mass_npoints"),
                                                  r, Ind(names[v]), Geti("order_centered")));
      fprintf(f, "\n");
    }
    fclose(f);
  }
  return 0;
}

/* the reference's trackers and the globals of moving_punctures.c:13-14 */
int track_moving_puncture_integrate(tL *level, int np, double *pold, double *pnew);
int track_moving_puncture_extremum(tL *level, int np, double *pold, double *pnew);
int xyzinsidelevel(tL *level, double x, double y, double z);
extern int pintoxyplane;

static void dump_track(tL *level, const char *tag)
{
  tVarList *vl = vlalloc(level);
  char fn[1024];
  const char *s = Gets("nrharness_track_points");
  char *end;
  double p[3], pnew[3];
  int i, fix, moved, save;
  FILE *f;
  /* a vector is pushed by its first component: betax..z, betax_p..z_p */
  vlpush(vl, Ind("betax"));
  vlpush(vl, Ind("betax_p"));
  vlpush(vl, Ind("alpha"));
  dump_varlist(level, vl, tag);
  vlfree(vl);
  snprintf(fn, sizeof fn, "%s/%s_l%d.txt", Gets("nrharness_dir"), tag, level->l);
  f = fopen(fn, "w");
  if (!f) errorexits("nrharness: cannot open %s", fn);
  /* the tracker runs on the level lmaxpunc names (grid.c:287-294) */
  save = level->grid->lmaxpunc[0];
  level->grid->lmaxpunc[0] = level->l;
  for (;;) {
    for (i = 0; i < 3; i++) {
      p[i] = strtod(s, &end);
      if (end == s) break;
      s = end;
    }
    if (i < 3) break;
    for (fix = 0; fix <= 2; fix += 2) {
      pintoxyplane = fix;
      moved = track_moving_puncture_integrate(level, 0, p, pnew);
      fprintf(f, "%d %d %.17g %.17g %.17g %.17g %.17g %.17g %d\n", fix, moved, p[0], p[1], p[2],
              pnew[0], pnew[1], pnew[2], xyzinsidelevel(level, pnew[0], pnew[1], pnew[2]));
    }
    /* the extremum search (moving_puncture_track_method = ext) on
       moving_puncture_track_var, rows 10 (z free) and 11 (z pinned) */
    if (Getv("physics", "Gauge"))
      for (fix = 0; fix <= 1; fix++) {
        pintoxyplane = fix;
        moved = track_moving_puncture_extremum(level, 0, p, pnew);
        fprintf(f, "%d %d %.17g %.17g %.17g %.17g %.17g %.17g %d\n", 10 + fix, moved, p[0], p[1], p[2],
                pnew[0], pnew[1], pnew[2], xyzinsidelevel(level, pnew[0], pnew[1], pnew[2]));
      }
  }
  pintoxyplane = 0;
  level->grid->lmaxpunc[0] = save;
  fclose(f);
  printf("nrharness: wrote %s\n", fn);
}

/* the reductions of write_level_0d (utility/output/output0d.c:28-116) on
 * the evolved list, one line per type 0..4 (max, min, norm, normInf,
 * integral) with the same corrections (norm times sqrt(nvars), integral
 * times dx^3) */
static void dump_0d(tL *level, tVarList *u, const char *tag)
{
  char fn[1024];
  double *r;
  int t, j;
  FILE *f;
  snprintf(fn, sizeof fn, "%s/%s_l%d.txt", Gets("nrharness_dir"), tag, level->l);
  f = fopen(fn, "w");
  if (!f) errorexits("nrharness: cannot open %s", fn);
  for (t = 0; t <= 4; t++) {
    if (t == 0) bampi_allreduce_max(u, &r);
    if (t == 1) bampi_allreduce_min(u, &r);
    if (t == 2) bampi_allreduce_norm(u, &r);
    if (t == 3) bampi_allreduce_normInf(u, &r);
    if (t == 4) bampi_allreduce_sum(u, &r);
    for (j = 0; j < u->n; j++) {
      double v = r[j];
      if (t == 2) v *= sqrt(u->n);
      if (t == 4) v *= pow(level->dx, 3);
      fprintf(f, "%.17g ", v);
    }
    fprintf(f, "\n");
    free(r);
  }
  fclose(f);
  printf("nrharness: wrote %s\n", fn);
}

void bam_nrharness(void)
{
  if (!Getv("physics", "nrharness")) return;
  printf("Adding nrharness (oracle dump harness)\n");
  AddPar("nrharness_dir", ".", "directory for raw FP64 dumps");
  AddPar("nrharness_dump", "none", "level iterations after which to dump the evolved variables");
  AddPar("nrharness_rhs", "no", "dump one RHS evaluation of the initial state [no,yes]");
  AddPar("nrharness_mg", "no", "dump punctures_u after the initial data solve [no,yes]");
  AddPar("nrharness_flags", "no", "dump the refinement flags of every level after the initial data [no,yes]");
  AddPar("nrharness_constraints", "no", "with each state dump also dump ADM variables and constraints [no,yes]");
  AddPar("nrharness_0d", "no", "with each state dump write the 0d reductions of the evolved list [no,yes]");
  AddPar("nrharness_track", "no", "with each state dump run the shift-integration tracker [no,yes]");
  AddPar("nrharness_track_points", "", "start positions of the tracker, x y z per position");
  AddPar("nrharness_data", "none", "synthetic data over the evolved variables [none,fourier]");
  AddPar("nrharness_amp", "1e-3", "amplitude of the Fourier perturbation");
  AddPar("nrharness_nmodes", "8", "number of Fourier modes");
  AddPar("nrharness_seed", "1", "seed of the mode generator");
  AddPar("nrharness_length", "16", "box length that sets the wave numbers");
  AddFun(POST_INITIALDATA, nrharness_post_initialdata, "oracle harness: synthetic data and dumps");
  AddFun(POST_EVOLVE, nrharness_post_evolve, "oracle harness: dumps");
  AddPar("nrharness_dump_moved", "no", "dump every level that move_box moved, after the move [no,yes]");
  AddPar("nrharness_admmass", "no", "with ADM_mass: dump its integrands and full-precision integrals [no,yes]");
  AddPar("nrharness_psi4", "no", "with Invariants: dump rpsi4, ipsi4, Csqr and their inputs [no,yes]");
  AddFun(ANALYZE, nrharness_analyze, "oracle harness: ADM mass integrands and integrals");
  AddFun(POST_MOVEBOX, nrharness_post_movebox, "oracle harness: dumps of moved levels");
}
