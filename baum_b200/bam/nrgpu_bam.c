/* nrgpu_bam.c -- BAM project module that plugs the B200 path (libnrgpu.so,
 * include/nrgpu.h) into the reference's evolution as a drop-in.
 *
 * Add to a BAM tree as src/projects/nrgpu (projects += src/projects/nrgpu in
 * MyConfig, after bssn) and link -lnrgpu -lcudart.  A parfile switches it on:
 *
 *   physics    = adm bssn ... nrgpu
 *   nrgpu_mode = callback   the reference's "geometry" and "geometry_bound"
 *                           callbacks (evolve.c:185) are replaced; every call
 *                           mirrors its var lists to the GPU and back, so the
 *                           reference's RK4, vladd and algcon run unchanged
 *   nrgpu_mode = resident   the whole RK4 step plus algcon runs on the GPU at
 *                           the EVOLVE hook; the reference's evolve() is
 *                           switched off by registering a null "geometry"
 *                           (evolve.c:231-235) and the host state is refreshed
 *                           after every step for ANALYZE/OUTPUT/checkpoint.
 *                           Set bssn_register_algcon = no with this mode.
 *   nrgpu_mode = fmr        the whole Berger-Oliger step of all levels (one
 *                           or several boxes each) runs on the GPU at level
 *                           0's EVOLVE hook; set bssn/z4_register_algcon = no.
 *                           With Gauge = moving_puncture the punctures are
 *                           tracked on the device (nrgpu_fmr_track).
 * physics with z4 selects the Z4c system (all three modes).
 *
 *   nrgpu_multigrid = yes   the puncture initial-data solve (punctures_solver
 *                           = multigrid, PunctureSolve.c:282) runs on the
 *                           GPU (nrgpu_mg_solve) when the grid is one cubic
 *                           box centred on the origin with the second-order
 *                           puncture operator, a Robin boundary and V cycles;
 *                           otherwise BAM's own multigrid runs.  The solver is
 *                           reached through PickEllipticSolver's function
 *                           pointer (Punctures.c:283-311): a tree carrying
 *                           this module adds the keyword there
 *                           (punctures_solver = multigrid -> nrgpu_multigrid),
 *                           or links with -Wl,--wrap=multigrid, which sends
 *                           the pointer to __wrap_multigrid below.
 *
 * Parameters are read exactly where bssn_rhs_movpunc_N reads them
 * (bssn_rhs_movpunc_N.c:107-145), the boundary speeds and far limits from the
 * variable database (VarFarLimit/VarPropSpeed, variables.c:246-248), and the
 * dissipation factor from get_dissipation_factor (evolve.c:489).  A negative
 * status from the library becomes errorexit(), as in the reference.
 */
#include "bam.h"
#include "bssn.h"
#include "../../../include/nrgpu.h"

#define NV NRGPU_BSSN_NVARS
#define ZNV NRGPU_Z4_NVARS

/* defined by the z4 project (z4.c:8) when it is linked; the weak reference
 * lets a BSSN-only tree link this module too */
extern int METRIC_z4_INDX_VAR __attribute__((weak));

static int nrgpu_mode_resident = 0;
static int nrgpu_mode_fmr = 0;
static int nrgpu_system_z4 = 0;

typedef struct {
  tL *bamlevel;
  nrgpu_level *lev;
  int npoints;
  double *d_state;  /* [NV][npoints] resident state (resident mode) */
  double *d_a, *d_b, *d_c;
  int uploaded;
  int tuned;        /* rhs block shape picked by nrgpu_level_autotune */
} nrgpu_slot;

static nrgpu_slot slots[64];

/* cudart entry points used by this module (declared here so no CUDA header
 * is needed to compile a BAM project) */
extern int cudaMalloc(void **p, size_t n);
extern int cudaFree(void *p);
extern int cudaMemcpy(void *d, const void *s, size_t n, int kind);
extern int cudaDeviceSynchronize(void);

static void check(int status, const char *what)
{
  if (status != NRGPU_OK) errorexits("nrgpu: %s", (char *)nrgpu_last_error());
  (void)what;
}

static void read_params(tL *level, tVarList *u, nrgpu_bssn_params *p)
{
  int j;
  nrgpu_bssn_params_default(p);
  p->order_centered = Geti("order_centered");
  p->order_advection = Geti("order_advection");
  p->advection_lopsided = Geti("advection_lopsided");
  p->advection_lopsided6 = Geti("advection_lopsided6");
  p->order_dissipation = Geti("order_dissipation");
  p->dissfactor = get_dissipation_factor(level);
  p->forceKzerofactor = Getv("bssn_forceKzero", "no");
  p->subtractA = Getv("bssn_subtractA", "yes");
  p->normalizedetg = Getv("bssn_normalizedetg", "yes");
  p->oploglapse = Getv("bssn_lapse", "1+log");
  p->oploglapse2 = Getv("bssn_lapse", "1+log2");
  p->oplogwithshift = Getv("bssn_lapse", "withshift");
  p->harmoniclapse = Getv("bssn_lapse", "harmonic");
  p->gamma0factor = Getv("bssn_shift", "gamma0");
  p->gamma2factor = Getv("bssn_shift", "gamma2");
  p->withGadv = Getv("bssn_shift", "withGadv");
  p->withShiftadv = Getv("bssn_shift", "withShiftadv");
  p->withBadv = Getv("bssn_shift", "withBadv");
  p->withB = !Getv("bssn_shift", "withoutB");
  p->lapseharmonicf = Getd("bssn_lapseharmonicf");
  p->shiftalphapower = Getd("bssn_shiftalphapower");
  p->shiftgammacoeff = Getd("bssn_shiftgammacoeff");
  p->shiftGalphapower = Getd("bssn_shiftgammaalphapower");
  p->shiftdriver = Getd("bssn_shiftdriver");
  p->chiDivFloor = Getd("bssn_chi_div_floor");
  p->chipsipower = Getd("bssn_chi_psipower");
  if (Getv("bssn_use_eta", "yes")) errorexit("nrgpu: bssn_use_eta is not supported");
  if (level->shells) errorexit("nrgpu: shells are not supported");
  for (j = 0; j < NV; j++) {
    int i = u->index[METRIC_bssn_INDX_VAR + j];
    p->bc_var0[j] = VarFarLimit(i);
    p->bc_speed[j] = Getv("boundary_radconstant", VarName(i)) ? 0.0 : VarPropSpeed(i);
  }
}

/* the parameters z4_rhs_movpunc_N reads (z4_rhs_movpunc_N.c:109-138) */
static void read_params_z4(tL *level, tVarList *u, nrgpu_z4_params *p)
{
  int j;
  memset(p, 0, sizeof *p);
  p->order_centered = Geti("order_centered");
  p->order_advection = Geti("order_advection");
  p->advection_lopsided = Geti("advection_lopsided");
  p->advection_lopsided6 = Geti("advection_lopsided6");
  p->order_dissipation = Geti("order_dissipation");
  p->dissfactor = get_dissipation_factor(level);
  p->kappa1 = Getd("z4_kappa1");
  p->kappa2 = Getd("z4_kappa2");
  p->zeroThetaRHS = Getv("z4_zeroThetaRHS", "no");
  p->useNPTs = Getv("z4_useNPTs", "yes");
  p->subtractA = Getv("z4_subtractA", "yes");
  p->normalizedetg = Getv("z4_normalizedetg", "yes");
  p->oploglapse = Getv("z4_lapse", "1+log");
  p->oploglapse2 = Getv("z4_lapse", "1+log2");
  p->oplogwithshift = Getv("z4_lapse", "withshift");
  p->harmoniclapse = Getv("z4_lapse", "harmonic");
  p->gamma0factor = Getv("z4_shift", "gamma0");
  p->gamma2factor = Getv("z4_shift", "gamma2");
  p->withGadv = Getv("z4_shift", "withGadv");
  p->withShiftadv = Getv("z4_shift", "withShiftadv");
  p->withBadv = Getv("z4_shift", "withBadv");
  p->withB = Getv("z4_shift", "withB");
  p->lapseharmonicf = Getd("z4_lapseharmonicf");
  p->shiftalphapower = Getd("z4_shiftalphapower");
  p->shiftgammacoeff = Getd("z4_shiftgammacoeff");
  p->shiftdriver = Getd("z4_shiftdriver");
  p->chiDivFloor = Getd("z4_chi_div_floor");
  p->chipsipower = Getd("z4_chi_psipower");
  if (Getv("z4_forceKzero", "yes")) errorexit("nrgpu: z4_forceKzero is not supported");
  if (level->shells) errorexit("nrgpu: shells are not supported");
  /* set_boundary's background branch on level 0 (boundary.c:190-210, z4.c:
     251-271): radcentered or CPBC2 */
  if (Getv("boundary", "background") && level->l == 0) {
    if (Getv("boundary", "radiative")) errorexit("nrgpu: boundary = radiative and background together");
    p->boundary = Getv("boundary", "radcentered") ? 1 : 2;
  }
  /* the radiative condition's far limits and speeds (boundary_radconstant
     exists only where the radiative boundary is registered) */
  for (j = 0; j < ZNV; j++) {
    int i = u->index[METRIC_z4_INDX_VAR + j];
    p->bc_var0[j] = VarFarLimit(i);
    p->bc_speed[j] = GetvLax("boundary_radconstant", VarName(i)) ? 0.0 : VarPropSpeed(i);
  }
}

/* the reflection axes of set_boundary_symmetry (symmetry.c:93-140) */
static int grid_symmetry(void)
{
  if (Getv("grid", "quadrant") || Getv("grid", "rotant"))
    errorexit("nrgpu: the inversion symmetry of grid = quadrant/rotant is not supported");
  if (Getv("grid", "octant")) return 7;
  if (Getv("grid", "qreflect")) return 6;
  if (Getv("grid", "bitant")) return 4;
  return 0;
}

static nrgpu_slot *slot_of(tL *level)
{
  nrgpu_slot *s = &slots[level->l];
  if (level->l >= 64) errorexit("nrgpu: too many levels");
  if (s->bamlevel != level || s->npoints != level->npoints) {
    nrgpu_box box[256];
    nrgpu_level_desc d;
    int b;
    if (level->nboxes > 256) errorexit("nrgpu: too many boxes");
    for (b = 0; b < level->nboxes; b++) {
      tB *bx = level->box[b];
      box[b].m = bx->m; box[b].n = bx->n; box[b].o = bx->o;
      box[b].noffset = bx->noffset;
      box[b].x0 = bx->x0; box[b].y0 = bx->y0; box[b].z0 = bx->z0;
    }
    d.nboxes = level->nboxes; d.box = box; d.npoints = level->npoints;
    d.dx = level->dx; d.dy = level->dy; d.dz = level->dz;
    d.boundary = level->boundary;
    d.symmetry = grid_symmetry();
    if (s->lev) nrgpu_level_destroy(s->lev);
    check(nrgpu_level_create(&d, &s->lev), "level");
    s->bamlevel = level;
    s->npoints = level->npoints;
    s->uploaded = 0;
    s->tuned = 0;
    if (cudaMalloc((void **)&s->d_state, sizeof(double) * ZNV * level->npoints) ||
        cudaMalloc((void **)&s->d_a, sizeof(double) * ZNV * level->npoints) ||
        cudaMalloc((void **)&s->d_b, sizeof(double) * ZNV * level->npoints) ||
        cudaMalloc((void **)&s->d_c, sizeof(double) * ZNV * level->npoints))
      errorexit("nrgpu: device allocation failed");
  }
  return s;
}

static int nvars(void) { return nrgpu_system_z4 ? ZNV : NV; }
static int first_var(void) { return nrgpu_system_z4 ? METRIC_z4_INDX_VAR : METRIC_bssn_INDX_VAR; }

static void lists(double *base, int npoints, double **ptr)
{
  int j;
  for (j = 0; j < nvars(); j++) ptr[j] = base + (size_t)j * npoints;
}

static void copy_vl(tL *level, tVarList *vl, double *dev, int to_device)
{
  int j;
  for (j = 0; j < nvars(); j++) {
    double *h = level->v[vl->index[first_var() + j]];
    double *d = dev + (size_t)j * level->npoints;
    if (cudaMemcpy(to_device ? (void *)d : (void *)h, to_device ? (void *)h : (void *)d,
                   sizeof(double) * level->npoints, to_device ? 1 : 2))
      errorexit("nrgpu: copy failed");
  }
}

/* "geometry" callback: replaces bssn_evolve/bssn_rhs_movpunc_N (bssn.c:17) */
void nrgpu_bssn_evolve_cb(tVarList *unew, tVarList *upre, double c, tVarList *ucur)
{
  tL *level = ucur->level;
  nrgpu_slot *s = slot_of(level);
  nrgpu_bssn_params p;
  double *n[NV], *pr[NV], *cu[NV];
  timer_start(level, "bssn_rhs");
  read_params(level, ucur, &p);
  lists(s->d_a, level->npoints, n);
  lists(s->d_b, level->npoints, pr);
  lists(s->d_c, level->npoints, cu);
  copy_vl(level, ucur, s->d_c, 1);
  copy_vl(level, unew, s->d_a, 1);  /* points the rhs does not touch keep their values */
  if (c != 0.0) copy_vl(level, upre, s->d_b, 1);
  check(nrgpu_bssn_rhs(s->lev, n, c != 0.0 ? pr : cu, c, cu, &p, 0), "rhs");
  copy_vl(level, unew, s->d_a, 0);
  timer_stop(level, "bssn_rhs");
}

/* "geometry_bound" callback: replaces bssn_rhs_boundary (bssn.c:28) */
void nrgpu_bssn_boundary_cb(tVarList *unew, tVarList *upre, double c, tVarList *ucur)
{
  tL *level = ucur->level;
  nrgpu_slot *s = slot_of(level);
  nrgpu_bssn_params p;
  double *n[NV], *pr[NV], *cu[NV];
  read_params(level, ucur, &p);
  lists(s->d_a, level->npoints, n);
  lists(s->d_b, level->npoints, pr);
  lists(s->d_c, level->npoints, cu);
  copy_vl(level, ucur, s->d_c, 1);
  copy_vl(level, unew, s->d_a, 1);
  if (c != 0.0) copy_vl(level, upre, s->d_b, 1);
  check(nrgpu_bssn_boundary(s->lev, n, c != 0.0 ? pr : cu, c, cu, &p, 0), "boundary");
  copy_vl(level, unew, s->d_a, 0);
}

/* "geometry" callback of the Z4c system: replaces z4_evolve /
 * z4_rhs_movpunc_N (z4.c:17-19, registered at z4.c:245) */
void nrgpu_z4_evolve_cb(tVarList *unew, tVarList *upre, double c, tVarList *ucur)
{
  tL *level = ucur->level;
  nrgpu_slot *s = slot_of(level);
  nrgpu_z4_params p;
  double *n[ZNV], *pr[ZNV], *cu[ZNV];
  timer_start(level, "z4_rhs");
  read_params_z4(level, ucur, &p);
  lists(s->d_a, level->npoints, n);
  lists(s->d_b, level->npoints, pr);
  lists(s->d_c, level->npoints, cu);
  copy_vl(level, ucur, s->d_c, 1);
  copy_vl(level, unew, s->d_a, 1);
  if (c != 0.0) copy_vl(level, upre, s->d_b, 1);
  check(nrgpu_z4_rhs(s->lev, n, c != 0.0 ? pr : cu, c, cu, &p, 0), "rhs");
  copy_vl(level, unew, s->d_a, 0);
  /* the background boundary extrapolates the state itself onto the
     boundary (z4_rhs_movpunc_N.c:148-152); BAM's RK4 keeps those values */
  if (p.boundary) copy_vl(level, ucur, s->d_c, 0);
  timer_stop(level, "z4_rhs");
}

/* "geometry_bound" callback of the Z4c system: replaces set_boundary
 * (z4.c:248) with the radiative condition and the symmetry reflections, or
 * on level 0 with its background branch (radcentered or CPBC2) */
void nrgpu_z4_boundary_cb(tVarList *unew, tVarList *upre, double c, tVarList *ucur)
{
  tL *level = ucur->level;
  nrgpu_slot *s = slot_of(level);
  nrgpu_z4_params p;
  double *n[ZNV], *pr[ZNV], *cu[ZNV];
  read_params_z4(level, ucur, &p);
  lists(s->d_a, level->npoints, n);
  lists(s->d_b, level->npoints, pr);
  lists(s->d_c, level->npoints, cu);
  copy_vl(level, ucur, s->d_c, 1);
  copy_vl(level, unew, s->d_a, 1);
  if (c != 0.0) copy_vl(level, upre, s->d_b, 1);
  check(nrgpu_z4_boundary(s->lev, n, c != 0.0 ? pr : cu, c, cu, &p, 0), "boundary");
  copy_vl(level, unew, s->d_a, 0);
  if (p.boundary) copy_vl(level, ucur, s->d_c, 0);
}

/* EVOLVE hook of the resident mode: evolve_rk_rk4 + algcon on the device */
int nrgpu_evolve_resident(tL *level)
{
  tVarList *u = 0;
  nrgpu_slot *s;
  double *st[ZNV];
  if (!nrgpu_mode_resident) return 0;
  evolve_vlretrieve(&u, 0, 0);
  if (!u) errorexit("nrgpu: no evolution list");
  u->level = level;
  timer_start(level, "evolve");
  s = slot_of(level);
  lists(s->d_state, level->npoints, st);
  if (!s->uploaded) {
    copy_vl(level, u, s->d_state, 1);
    s->uploaded = 1;
  }
  if (nrgpu_system_z4) {
    nrgpu_z4_params p;
    read_params_z4(level, u, &p);
    if (!s->tuned) check(nrgpu_level_autotune(s->lev, NRGPU_SYSTEM_Z4C, &p, 0, 0), "autotune");
    s->tuned = 1;
    check(nrgpu_z4_rk4_step(s->lev, st, level->dt, &p, 0), "rk4");
  } else {
    nrgpu_bssn_params p;
    read_params(level, u, &p);
    if (!s->tuned) check(nrgpu_level_autotune(s->lev, NRGPU_SYSTEM_BSSN, &p, 0, 0), "autotune");
    s->tuned = 1;
    check(nrgpu_bssn_rk4_step(s->lev, st, level->dt, &p, 0), "rk4");
  }
  copy_vl(level, u, s->d_state, 0);
  timer_stop(level, "evolve");
  return 0;
}

/* EVOLVE hook of the mesh-refinement mode, on level 0: one coarse step of
 * every level (advance_levelandsublevels, main.c:397-418, with the time
 * interpolation and restrict_prolong_evolve) on the device, then every
 * level's state back to the host arrays.  BAM still walks the finer levels:
 * their EVOLVE is a no-op here and in evolve() (null "geometry"), so BAM
 * never allocates the time interpolant; its restrict_prolong_evolve then
 * does nothing at unaligned times (restrict_varlist/prolong_varlist return
 * on a null list) and, at aligned times, recomputes from the host arrays
 * exactly what the device already did.  POST_EVOLVE, ANALYZE and OUTPUT see
 * every level at the end of the coarse step. */
static nrgpu_fmr *fmr_h = 0;
static double *fmr_state[64];
/* puncture tracking in this mode (Gauge = moving_puncture): the device
 * tracks on the finest level after each of its steps.  BAM's own
 * track_puncture cannot run here: the host arrays already hold the end of
 * the coarse step and the previous time level (betax_p) is never allocated,
 * since BAM's evolve does not run.  So the set-up takes it out of the loop
 * (lmaxpunc = -1: track_puncture skips every level,
 * Gauge/moving_punctures.c:142) and nrgpu_track_fmr, an ANALYZE function,
 * puts the device's positions in its place (grid->puncpos and the
 * moving_punctureN_x/y/z parameters that BAM's checkpoint writes) */
static int fmr_ntrack = 0;
static double fmr_tpos[3 * NRGPU_MAX_PUNCTURES];

static void fmr_track_setup(tG *g, tVarList *u)
{
  int np, i, n, method, var = -1, fixz;
  if (!Getv("physics", "Gauge") || !Getv("Gauge", "moving_puncture") || !Getv("moving_puncture_track", "yes"))
    return;
  /* track_puncture's choices (Gauge/moving_punctures.c:123-134) */
  if (Getv("moving_puncture_track_method", "ext")) method = 0;
  else if (Getv("moving_puncture_track_method", "int")) method = 1;
  else if (Getv("moving_puncture_track_method", "extint")) method = 2;
  else errorexit("nrgpu: moving_puncture_track_method is not ext, int or extint");
  if (Getv("moving_puncture_fixz", "NS")) fixz = 1;
  else if (Getv("moving_puncture_fixz", "BH")) fixz = 2;
  else if (Getv("moving_puncture_fixz", "BHNS")) fixz = 3;
  else if (Getv("moving_puncture_fixz", "none")) fixz = 0;
  else errorexit("nrgpu: moving_puncture_fixz is not NS, BH, BHNS or none");
  if (method != 1) {
    /* the searched variable must be one the device evolves */
    int k = Ind(Gets("moving_puncture_track_var"));
    for (i = 0; i < nvars(); i++)
      if (u->index[first_var() + i] == k) var = i;
    if (var < 0) errorexit("nrgpu: moving_puncture_track_var is not in the evolved list");
  }
  n = Geti("nobjects");
  if (n < 1 || n > NRGPU_MAX_PUNCTURES) errorexit("nrgpu: nobjects out of range for tracking");
  for (np = 0; np < n; np++) {
    if (g->lmaxpunc[np] != g->lmax) errorexit("nrgpu: the fmr mode tracks punctures on the finest level only");
    for (i = 0; i < 3; i++) fmr_tpos[3 * np + i] = g->puncpos[np][i];
    g->lmaxpunc[np] = -1;
  }
  check(nrgpu_fmr_track(fmr_h, n, fmr_tpos, fixz == 2 || fixz == 3), "track");
  check(nrgpu_fmr_track_method(fmr_h, method, var < 0 ? 0 : var, Getv("moving_puncture_track_mode", "max"),
                               Getd("moving_puncture_track_minmove"), fixz == 1 || fixz == 3), "track method");
  fmr_ntrack = n;
}

int nrgpu_track_fmr(tL *level)
{
  tG *g = level->grid;
  char str[100];
  int np, i;
  if (!nrgpu_mode_fmr || !fmr_ntrack || level->l != g->lmax) return 0;
  for (np = 0; np < fmr_ntrack; np++)
    for (i = 0; i < 3; i++) {
      g->puncpos[np][i] = fmr_tpos[3 * np + i];
      sprintf(str, "moving_puncture%d_%c", np + 1, 'x' + i);
      if (ExistPar(str)) Setd(str, fmr_tpos[3 * np + i]);
    }
  return 0;
}

/* Moving boxes in this mode (amr = ... move): BAM's own move_box
 * (main/amr/move.c:808-986) moves the host levels and their host data; here
 * the data live on the device.  So BAM's call (main.c:428) is sent to
 * __wrap_move_box, which does nothing in this mode, and the device
 * hierarchy calls fmr_move at the same points of its recursion
 * (nrgpu_fmr_set_move).  fmr_move replays move_box's decisions with BAM's
 * own functions: find_nested_bboxes on each parent, at the parent's time on
 * the device and with the device's tracked positions, and make_level_bboxes
 * for every level whose boxes change; then one nrgpu_fmr_regrid moves the
 * device data of those levels (the copy and prolongation of move_overlap)
 * and the old host levels are freed as move_box frees them. */
void find_nested_bboxes(tL *level, int *pnboxes, tSBox *box);
tL *make_level_bboxes(tL *level, int nboxes, tSBox *box, int pr);

static double *fmr_ptrs[64 * ZNV]; /* the state pointers given to nrgpu_fmr_advance */

/* box_equal (move.c:20-27) */
static int sbox_equal(const double *a, const double *b)
{
  int i;
  for (i = 0; i < 6; i++)
    if (!dequal(a[i], b[i])) return 0;
  return 1;
}

static int fmr_move(void *user, nrgpu_fmr *F, int l, void *stream)
{
  tG *g = (tG *)user;
  nrgpu_level_desc d[16];
  nrgpu_box box[16][8];
  double *unew[16 * ZNV];
  double *fresh[16];
  tL *old[16];
  int lv, b, j, np, nv = nvars(), nmove = 0, nlev = g->lmax - l + 1;
  if (nlev < 1) return 0;
  if (fmr_ntrack) {
    check(nrgpu_fmr_punctures(F, fmr_tpos, 0), "punctures");
    for (np = 0; np < fmr_ntrack; np++)
      for (j = 0; j < 3; j++) g->puncpos[np][j] = fmr_tpos[3 * np + j];
  }
  memset(unew, 0, sizeof unew);
  for (lv = l; lv <= g->lmax; lv++) {
    tL *lc = g->level[lv - 1], *lold = g->level[lv], *lnew;
    tSBox *sb = bcalloc(3 * sizeof(tSBox));
    double tsave = lc->time;
    int itsave = lc->iteration, nboxes;
    int i = lv - l;
    d[i].nboxes = 0;
    fresh[i] = 0;
    old[i] = 0;
    /* the parent's time on the device (main.c:482-483) */
    lc->iteration = nrgpu_fmr_iteration(F, lv - 1);
    lc->time = lc->iteration * lc->dt;
    find_nested_bboxes(lc, &nboxes, sb);
    lc->time = tsave;
    lc->iteration = itsave;
    if (lc->sbox && lc->nsboxes == nboxes) {
      for (j = 0; j < nboxes; j++)
        if (!sbox_equal(lc->sbox[j].bbox, sb[j].bbox)) break;
      if (j == nboxes) {
        free(sb);
        continue;
      }
    }
    free(lc->sbox);
    lc->sbox = sb;
    lc->nsboxes = nboxes;
    if (lold->prlocal) {
      if (lold->nboxes > 1) free_level(lold->prlocal);
      lold->prlocal = 0;
    }
    lnew = make_level_bboxes(lc, nboxes, sb, 0);
    lnew->time = lold->time;
    lnew->iteration = lold->iteration;
    lnew->dt = lold->dt;
    test_box_consistency_level(lc, lnew);
    if (lnew->nboxes < 1 || lnew->nboxes > 8) errorexit("nrgpu: the refinement mode takes 1 to 8 boxes per level");
    for (b = 0; b < lnew->nboxes; b++) {
      tB *bx = lnew->box[b];
      box[i][b].m = bx->m; box[i][b].n = bx->n; box[i][b].o = bx->o; box[i][b].noffset = bx->noffset;
      box[i][b].x0 = bx->x0; box[i][b].y0 = bx->y0; box[i][b].z0 = bx->z0;
    }
    d[i].nboxes = lnew->nboxes; d[i].box = box[i]; d[i].npoints = lnew->npoints;
    d[i].dx = lnew->dx; d[i].dy = lnew->dy; d[i].dz = lnew->dz; d[i].boundary = lnew->boundary;
    d[i].symmetry = grid_symmetry();
    if (cudaMalloc((void **)&fresh[i], sizeof(double) * nv * lnew->npoints))
      errorexit("nrgpu: device allocation failed");
    lists(fresh[i], lnew->npoints, unew + i * nv);
    old[i] = lold;
    nmove++;
  }
  if (!nmove) return 0;
  check(nrgpu_fmr_regrid(F, l, nlev, d, fmr_ptrs, unew, stream), "regrid");
  for (lv = l; lv <= g->lmax; lv++) {
    int i = lv - l;
    if (!fresh[i]) continue;
    cudaFree(fmr_state[lv]);
    fmr_state[lv] = fresh[i];
    lists(fresh[i], g->level[lv]->npoints, fmr_ptrs + lv * nv);
    free_level(old[i]);
  }
  if (Getv("amr_verbose", "move") || Getv("amr_verbose", "all"))
    printf("nrgpu: moved %d level(s) from level %d on\n", nmove, l);
  return 0;
}

#ifdef NRGPU_WRAP_MOVE_BOX
/* the wrapped move_box of a build linked with -Wl,--wrap=move_box */
int __real_move_box(tG *g, int l);
int __wrap_move_box(tG *g, int l)
{
  if (nrgpu_mode_fmr) return 0;  /* moved inside the device's coarse step */
  return __real_move_box(g, l);
}
#endif

int nrgpu_evolve_fmr(tL *level)
{
  tG *g = level->grid;
  tVarList *u = 0;
  int l, nl, nv = nvars();
  double **ptrs = fmr_ptrs;
  if (!nrgpu_mode_fmr || level->l != 0) return 0;
  nl = g->lmax + 1;
  if (g->lmin != 0 || nl > 16) errorexit("nrgpu: levels 0..lmax with lmax < 16");
  evolve_vlretrieve(&u, 0, 0);
  if (!u) errorexit("nrgpu: no evolution list");
  timer_start(level, "evolve");
  if (!fmr_h) {
    nrgpu_level_desc d[16];
    nrgpu_box box[16][8];
    double dt[16];
    nrgpu_bssn_params bp[16];
    nrgpu_z4_params zp[16];
    nrgpu_fmr_params fp;
    for (l = 0; l < nl; l++) {
      tL *lv = g->level[l];
      int b;
      if (lv->nboxes < 1 || lv->nboxes > 8) errorexit("nrgpu: the refinement mode takes 1 to 8 boxes per level");
      for (b = 0; b < lv->nboxes; b++) {
        tB *bx = lv->box[b];
        box[l][b].m = bx->m; box[l][b].n = bx->n; box[l][b].o = bx->o; box[l][b].noffset = bx->noffset;
        box[l][b].x0 = bx->x0; box[l][b].y0 = bx->y0; box[l][b].z0 = bx->z0;
      }
      d[l].nboxes = lv->nboxes; d[l].box = box[l]; d[l].npoints = lv->npoints;
      d[l].dx = lv->dx; d[l].dy = lv->dy; d[l].dz = lv->dz; d[l].boundary = lv->boundary;
      d[l].symmetry = grid_symmetry();
      dt[l] = lv->dt;
      u->level = lv;
      if (nrgpu_system_z4) read_params_z4(lv, u, &zp[l]);
      else read_params(lv, u, &bp[l]);
      if (cudaMalloc((void **)&fmr_state[l], sizeof(double) * nv * lv->npoints))
        errorexit("nrgpu: device allocation failed");
      copy_vl(lv, u, fmr_state[l], 1);
    }
    nrgpu_fmr_params_default(&fp);
    fp.system = nrgpu_system_z4 ? NRGPU_SYSTEM_Z4C : NRGPU_SYSTEM_BSSN;
    fp.lbo = g->lbo;
    fp.order_timeinterpolation = Geti("order_timeinterpolation");
    fp.order_RP = Geti("order_RP");
    fp.nbuffer = Geti("amr_nbuffer");
    check(nrgpu_fmr_create(nl, d, dt, nrgpu_system_z4 ? (void *)zp : (void *)bp, &fp, &fmr_h), "fmr");
    fmr_track_setup(g, u);
    if (Getv("amr", "move")) {
#ifndef NRGPU_WRAP_MOVE_BOX
      errorexit("nrgpu: moving boxes in the fmr mode need a build linked with -Wl,--wrap=move_box");
#endif
      check(nrgpu_fmr_set_move(fmr_h, fmr_move, g), "move");
    }
  }
  for (l = 0; l < nl; l++) lists(fmr_state[l], g->level[l]->npoints, ptrs + l * nv);
  check(nrgpu_fmr_advance(fmr_h, ptrs, 1, 0), "fmr advance");
  if (fmr_ntrack) {
    check(nrgpu_fmr_punctures(fmr_h, fmr_tpos, 0), "punctures");
    for (l = 0; l < fmr_ntrack; l++)
      printf("nrgpu: puncture %d at %.17g %.17g %.17g\n", l + 1, fmr_tpos[3 * l], fmr_tpos[3 * l + 1],
             fmr_tpos[3 * l + 2]);
  }
  for (l = 0; l < nl; l++) {
    u->level = g->level[l];
    copy_vl(g->level[l], u, fmr_state[l], 0);
  }
  u->level = level;
  timer_stop(level, "evolve");
  return 0;
}

/* ---- puncture initial data: the multigrid on the device --------------------- */

typedef void (*mg_operator)(tL *, tVarList *, tVarList *);
/* the second-order puncture operator and its relaxation (PunctureSolve.c:21,108) */
void Lpuncture_nonlin(tL *level, tVarList *vllu, tVarList *vlu);
void Lpuncture_GS(tL *level, tVarList *vlv, tVarList *vlu);
/* BAM's own multigrid (multigrid.c:35).  A build linked with
 * -Wl,--wrap=multigrid compiles this module with NRGPU_WRAP_MULTIGRID: every
 * reference to multigrid then lands on __wrap_multigrid, and BAM's solver is
 * __real_multigrid. */
#ifdef NRGPU_WRAP_MULTIGRID
int __real_multigrid(tL *level, tVarList *u, tVarList *f, tVarList *v, tVarList *c, int itmax, double tol,
                     double *normres, mg_operator lop, mg_operator lgs);
#define HOST_MULTIGRID __real_multigrid
#else
int multigrid(tL *level, tVarList *u, tVarList *f, tVarList *v, tVarList *c, int itmax, double tol,
              double *normres, mg_operator lop, mg_operator lgs);
#define HOST_MULTIGRID multigrid
#endif

/* multigrid(level, u, f, v, c, itmax, tol, &normres, lop, lgs) of the puncture
 * solve: c = (punctures_a, punctures_b), u = punctures_u holds the initial
 * guess and receives the solution; f and v are the reference's work lists
 * (f = 0 on every level, multigrid.c:97-104), not needed on the device */
int nrgpu_multigrid(tL *level, tVarList *u, tVarList *f, tVarList *v, tVarList *c, int itmax, double tol,
                    double *normres, mg_operator lop, mg_operator lgs)
{
  const char *why = 0;
  tG *g = level->grid;
  tB *box = level->nboxes == 1 ? level->box[0] : 0;
  nrgpu_mg_params mp;
  nrgpu_mg *mg = 0;
  double *d = 0, res = 0.0;
  int ncyc = 0, m = 0, i;
  size_t n, bytes;

  if (!Getv("nrgpu_multigrid", "yes")) why = "nrgpu_multigrid = no";
  else if (lop != Lpuncture_nonlin || lgs != Lpuncture_GS) why = "not the second-order puncture operator";
  else if (g->lmin != g->lmax || !box || !c || c->n < 2) why = "more than one level or box";
  else if (!Getv("punctures_boundary", "robin")) why = "punctures_boundary is not robin";
  else if (!Getv("mg_setbound", "set_boundary_elliptic")) why = "mg_setbound";
  else if (Geti("mg_wcycle_nmax") > 0 || Geti("mg_vcycle_nmin") != 0) why = "W cycles or mg_vcycle_nmin";
  else if (box->m != box->n || box->m != box->o || level->dx != level->dy || level->dx != level->dz)
    why = "not a cube";
  else if (fabs(box->x0 + 0.5 * (box->m - 1) * level->dx) > 1e-12 * level->dx ||
           fabs(box->y0 + 0.5 * (box->n - 1) * level->dy) > 1e-12 * level->dy ||
           fabs(box->z0 + 0.5 * (box->o - 1) * level->dz) > 1e-12 * level->dz)
    why = "box not centred on the origin";
  if (!why) {
    m = box->m;
    nrgpu_mg_params_default(&mp);
    mp.npre = Geti("mg_relax_npre");
    mp.npost = Geti("mg_relax_npost");
    mp.exact_nmin = Geti("mg_exact_nmin");
    mp.exact_nmax = Geti("mg_exact_nmax");
    mp.vcycle_nmin = Geti("mg_vcycle_nmin");
    mp.vcycle_nmax = Geti("mg_vcycle_nmax");
    mp.fullV = Getv("mg_typeofcycles", "fullV");
    mp.size_nmin = Geti("mg_size_nmin");
    mp.levels_nmax = Geti("mg_levels_nmax");
    mp.tol = tol;
    mp.falloff = Getd("punctures_robin_falloff");
    if (nrgpu_mg_create(m, level->dx, &mp, &mg) != NRGPU_OK) why = (const char *)nrgpu_last_error();
  }
  if (why) {
    printf("nrgpu: multigrid on the host (%s)\n", why);
    return HOST_MULTIGRID(level, u, f, v, c, itmax, tol, normres, lop, lgs);
  }
  n = (size_t)m * m * m;
  bytes = sizeof(double) * n;
  if (cudaMalloc((void **)&d, 3 * bytes)) errorexit("nrgpu: device allocation failed");
  for (i = 0; i < 2; i++)
    if (cudaMemcpy(d + i * n, level->v[c->index[i]], bytes, 1)) errorexit("nrgpu: copy failed");
  if (cudaMemcpy(d + 2 * n, level->v[u->index[0]], bytes, 1)) errorexit("nrgpu: copy failed");
  check(nrgpu_mg_solve(mg, d, d + n, d + 2 * n, &ncyc, &res, 0), "multigrid");
  if (cudaMemcpy(level->v[u->index[0]], d + 2 * n, bytes, 2)) errorexit("nrgpu: copy failed");
  cudaFree(d);
  nrgpu_mg_destroy(mg);
  if (normres) *normres = res;
  printf("nrgpu_multigrid: %d V-cycles on the GPU, residual %.3e\n", ncyc, res);
  return 0;
}

#ifdef NRGPU_WRAP_MULTIGRID
/* the wrapped entry of a build linked with -Wl,--wrap=multigrid */
int __wrap_multigrid(tL *level, tVarList *u, tVarList *f, tVarList *v, tVarList *c, int itmax, double tol,
                     double *normres, mg_operator lop, mg_operator lgs)
{
  return nrgpu_multigrid(level, u, f, v, c, itmax, tol, normres, lop, lgs);
}
#endif

int nrgpu_startup(tL *level)
{
  if (level->l != 0) return 0;
  check(nrgpu_init(Geti("nrgpu_device")), "init");
  nrgpu_system_z4 = Getv("physics", "z4");
  if (nrgpu_system_z4 && !&METRIC_z4_INDX_VAR) errorexit("nrgpu: physics z4 without the z4 project");
  if (Getv("nrgpu_mode", "resident") || Getv("nrgpu_mode", "fmr")) {
    nrgpu_mode_resident = Getv("nrgpu_mode", "resident");
    nrgpu_mode_fmr = Getv("nrgpu_mode", "fmr");
    set_rhs_func_register("geometry", 0);  /* evolve() returns at once */
    if (Getv(nrgpu_system_z4 ? "z4_register_algcon" : "bssn_register_algcon", "yes"))
      errorexit("nrgpu: the GPU runs the algebraic constraints in this mode, set bssn/z4_register_algcon = no");
  } else if (nrgpu_system_z4) {
    set_rhs_func_register("geometry", nrgpu_z4_evolve_cb);
    set_rhs_func_register("geometry_bound", nrgpu_z4_boundary_cb);
  } else {
    set_rhs_func_register("geometry", nrgpu_bssn_evolve_cb);
    set_rhs_func_register("geometry_bound", nrgpu_bssn_boundary_cb);
  }
  printf("nrgpu: %s mode on device %d\n",
         nrgpu_mode_fmr ? "fmr" : (nrgpu_mode_resident ? "resident" : "callback"), Geti("nrgpu_device"));
  return 0;
}

void bam_nrgpu(void)
{
  if (!Getv("physics", "nrgpu")) return;
  printf("Adding nrgpu (B200 evolution path)\n");
  AddPar("nrgpu_mode", "callback", "how the GPU path plugs in [callback,resident,fmr]");
  AddPar("nrgpu_device", "0", "CUDA device");
  AddPar("nrgpu_multigrid", "no", "puncture initial-data multigrid on the GPU [no,yes]");
  AddFun(POST_INITIALDATA, nrgpu_startup, "nrgpu: register the GPU evolution");
  AddFun(EVOLVE, nrgpu_evolve_resident, "nrgpu: resident RK4 step");
  AddFun(EVOLVE, nrgpu_evolve_fmr, "nrgpu: one coarse step of all levels");
  AddFun(ANALYZE, nrgpu_track_fmr, "nrgpu: puncture positions tracked on the device");
}
