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

static int nrgpu_mode_resident = 0;

typedef struct {
  tL *bamlevel;
  nrgpu_level *lev;
  int npoints;
  double *d_state;  /* [NV][npoints] resident state (resident mode) */
  double *d_a, *d_b, *d_c;
  int uploaded;
} nrgpu_slot;

static nrgpu_slot slots[64];

/* cudart entry points used by this module (declared here so no CUDA header
 * is needed to compile a BAM project) */
extern int cudaMalloc(void **p, size_t n);
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
    if (s->lev) nrgpu_level_destroy(s->lev);
    check(nrgpu_level_create(&d, &s->lev), "level");
    s->bamlevel = level;
    s->npoints = level->npoints;
    s->uploaded = 0;
    if (cudaMalloc((void **)&s->d_state, sizeof(double) * NV * level->npoints) ||
        cudaMalloc((void **)&s->d_a, sizeof(double) * NV * level->npoints) ||
        cudaMalloc((void **)&s->d_b, sizeof(double) * NV * level->npoints) ||
        cudaMalloc((void **)&s->d_c, sizeof(double) * NV * level->npoints))
      errorexit("nrgpu: device allocation failed");
  }
  return s;
}

static void lists(double *base, int npoints, double **ptr)
{
  int j;
  for (j = 0; j < NV; j++) ptr[j] = base + (size_t)j * npoints;
}

static void copy_vl(tL *level, tVarList *vl, double *dev, int to_device)
{
  int j;
  for (j = 0; j < NV; j++) {
    double *h = level->v[vl->index[METRIC_bssn_INDX_VAR + j]];
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

/* EVOLVE hook of the resident mode: evolve_rk_rk4 + algcon on the device */
int nrgpu_evolve_resident(tL *level)
{
  tVarList *u = 0;
  nrgpu_slot *s;
  nrgpu_bssn_params p;
  double *st[NV];
  if (!nrgpu_mode_resident) return 0;
  evolve_vlretrieve(&u, 0, 0);
  if (!u) errorexit("nrgpu: no evolution list");
  u->level = level;
  timer_start(level, "evolve");
  s = slot_of(level);
  read_params(level, u, &p);
  lists(s->d_state, level->npoints, st);
  if (!s->uploaded) {
    copy_vl(level, u, s->d_state, 1);
    s->uploaded = 1;
  }
  check(nrgpu_bssn_rk4_step(s->lev, st, level->dt, &p, 0), "rk4");
  copy_vl(level, u, s->d_state, 0);
  timer_stop(level, "evolve");
  return 0;
}

int nrgpu_startup(tL *level)
{
  if (level->l != 0) return 0;
  check(nrgpu_init(Geti("nrgpu_device")), "init");
  if (Getv("nrgpu_mode", "resident")) {
    nrgpu_mode_resident = 1;
    set_rhs_func_register("geometry", 0);  /* evolve() returns at once */
    if (Getv("bssn_register_algcon", "yes"))
      errorexit("nrgpu: resident mode runs algcon on the GPU, set bssn_register_algcon = no");
  } else {
    set_rhs_func_register("geometry", nrgpu_bssn_evolve_cb);
    set_rhs_func_register("geometry_bound", nrgpu_bssn_boundary_cb);
  }
  printf("nrgpu: %s mode on device %d\n", nrgpu_mode_resident ? "resident" : "callback",
         Geti("nrgpu_device"));
  return 0;
}

void bam_nrgpu(void)
{
  if (!Getv("physics", "nrgpu")) return;
  printf("Adding nrgpu (B200 evolution path)\n");
  AddPar("nrgpu_mode", "callback", "how the GPU path plugs in [callback,resident]");
  AddPar("nrgpu_device", "0", "CUDA device");
  AddFun(POST_INITIALDATA, nrgpu_startup, "nrgpu: register the GPU evolution");
  AddFun(EVOLVE, nrgpu_evolve_resident, "nrgpu: resident RK4 step");
}
