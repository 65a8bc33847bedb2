/* nrgpu.h -- C ABI of the B200 (sm_100a) hot path of BAM's Einstein
 * evolution: the BSSN right-hand side over tVarList boxes, its radiative
 * boundary, the RK4 substep update and the algebraic constraints.
 *
 * Everything here is plain C: pointers, sizes and POD structs.  A BAM
 * project module (baum_b200/bam/nrgpu_bam.c) binds these entry points to the
 * reference's callback registry; Python tests bind them with ctypes.
 *
 * Data contract (mirrors the reference's storage, bam_amr.h:10-131 and
 * bam_amr_loops_box.h:54-68): one FP64 array per variable per level, all
 * boxes of the level concatenated at box->noffset, x fastest inside a box
 * (di = 1, dj = m, dk = m*n).  Variable lists are arrays of pointers in the
 * reference's evolve-list order, e.g. for BSSN (bssn.c:315-322):
 *   g11 g12 g13 g22 g23 g33 chi A11 A12 A13 A22 A23 A33 K G1 G2 G3
 *   alpha beta1 beta2 beta3 B1 B2 B3                      (24 variables)
 * "Device" pointers are CUDA global memory on the level's device; "host"
 * pointers are ordinary (preferably pinned) host memory.
 *
 * Errors: every entry point returns an int status (NRGPU_OK = 0, negative on
 * error) and never aborts; nrgpu_last_error() gives the message.  The BAM
 * binding turns a negative status into errorexit(), which is what the
 * reference does on failure (bam_main.h:112-117).
 */
#ifndef NRGPU_H
#define NRGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NRGPU_ABI_VERSION 1

enum {
  NRGPU_OK = 0,
  NRGPU_ERR_ARG = -1,         /* bad argument (null pointer, size, order) */
  NRGPU_ERR_CUDA = -2,        /* a CUDA runtime call failed */
  NRGPU_ERR_NAN = -3,         /* a NaN/Inf appeared in a right-hand side */
  NRGPU_ERR_NOMEM = -4,       /* device allocation failed */
  NRGPU_ERR_UNSUPPORTED = -5, /* feature outside the implemented set */
  NRGPU_ERR_TIMEOUT = -6      /* a bounded device wait gave up */
};

/* boundary flag values (bam_amr.h:117-126) */
enum {
  NRGPU_REFBOUND = -1, NRGPU_NOTBOUND = 0, NRGPU_PHYBOUND = 1, NRGPU_GHOBOUND = 2,
  NRGPU_SYMBOUND = 3
};

#define NRGPU_BSSN_NVARS 24

/* one box of a level (tB, bam_amr.h:10-30) */
typedef struct {
  int m, n, o;        /* points per direction, outer boundary layer included */
  int noffset;        /* offset of point (0,0,0) in the level arrays */
  double x0, y0, z0;  /* coordinates of point (0,0,0) */
} nrgpu_box;

/* a level (tL, bam_amr.h:46-74): geometry plus the boundary flag of every
 * point.  The flags are copied; the caller keeps ownership of its arrays. */
typedef struct {
  int nboxes;
  const nrgpu_box *box;
  int npoints;            /* sum over boxes of m*n*o */
  double dx, dy, dz;
  const int *boundary;    /* host array [npoints], tL.boundary */
  int symmetry;           /* reflections about x = 0 (bit 0), y = 0 (bit 1) and
                             z = 0 (bit 2): grid = octant 7, bitant 4,
                             qreflect 6 (set_boundary_symmetry, symmetry.c:93-140);
                             the points below zero on those axes are the
                             SYMBOUND ghosts.  0: none */
} nrgpu_level_desc;

typedef struct nrgpu_level nrgpu_level;  /* opaque device mirror of a level */

/* Parameters that bssn_rhs_movpunc_N reads from the parameter database at
 * every call (bssn_rhs_movpunc_N.c:107-145).  The 0/1 "factors" are the
 * values of the reference's Getv() token tests, as doubles where the
 * reference multiplies with them. */
typedef struct {
  int order_centered;       /* 2, 4 or 6 */
  int order_advection;      /* 2, 4 or 6 */
  int advection_lopsided;   /* 4th-order stencil shift, bam_amr.c:50-57 */
  int advection_lopsided6;  /* 6th-order stencil shift */
  int order_dissipation;    /* 0 (off), 4 or 6 */
  double dissfactor;        /* get_dissipation_factor(level), evolve.c:489 */
  double forceKzerofactor;  /* Getv("bssn_forceKzero","no") */
  int subtractA;            /* Getv("bssn_subtractA","yes") */
  int normalizedetg;        /* Getv("bssn_normalizedetg","yes") */
  int oploglapse, oploglapse2, oplogwithshift, harmoniclapse;
  double gamma0factor, gamma2factor, withGadv, withShiftadv, withBadv, withB;
  double lapseharmonicf, shiftalphapower, shiftgammacoeff, shiftGalphapower,
         shiftdriver;
  double chiDivFloor, chipsipower;
  /* radiative boundary (set_boundary_rot_rad, radiative.c:105) per variable:
   * far limit var0 and propagation speed v, VarNameSetBoundaryInfo
   * (bssn.c:288-311) */
  double bc_var0[NRGPU_BSSN_NVARS];
  double bc_speed[NRGPU_BSSN_NVARS];
} nrgpu_bssn_params;

#define NRGPU_Z4_NVARS 25

/* Parameters that z4_rhs_movpunc_N reads (z4_rhs_movpunc_N.m:600-640).
 * Z4c evolve list (z4.c:234-242): g11..g33 chi A11..A33 Khat G1..G3 Theta
 * alpha beta1..3 B1..3 (25 variables). */
typedef struct {
  int order_centered, order_advection, advection_lopsided, advection_lopsided6;
  int order_dissipation;    /* 0, 4 or 6; applied to all 25 variables */
  double dissfactor;
  double kappa1, kappa2;    /* z4_kappa1, z4_kappa2 */
  double zeroThetaRHS;      /* Getv("z4_zeroThetaRHS","no"): 1 for the default */
  int useNPTs;              /* Getv("z4_useNPTs","yes"): must be 0 */
  int subtractA, normalizedetg;
  int oploglapse, oploglapse2, oplogwithshift, harmoniclapse;
  double gamma0factor, gamma2factor, withGadv, withShiftadv, withBadv, withB;
  double lapseharmonicf, shiftalphapower, shiftgammacoeff, shiftdriver;
  double chiDivFloor, chipsipower;
  double bc_var0[NRGPU_Z4_NVARS];
  double bc_speed[NRGPU_Z4_NVARS];
  /* arithmetic of the finite differences (no counterpart in the reference):
   * 0 FP64 throughout; 1 Kreiss-Oliger sums in FP32; 2 Kreiss-Oliger and
   * the centred first/second derivative sums in FP32.  The taps enter as
   * FP64 differences to the centre value rounded to FP32; state, algebra,
   * advection and RK4 stay FP64. */
  int precision;
  /* the box boundary on PHYBOUND points: 0 radiative (set_boundary's
   * radiative branch with bc_var0/bc_speed); 1 "background radcentered"
   * (z4_boundary_box_rad.c) and 2 "background" (CPBC2, z4_boundary_box.c):
   * set_boundary's background branch (utility/boundary/boundary.c:190-210),
   * which extrapolates the state on the boundary, sets the rhs of A, G,
   * Khat and Theta one point inside from the boundary conditions and
   * extrapolates the rhs onto the boundary (no symmetry grids) */
  int boundary;
} nrgpu_z4_params;

/* ---- library ---------------------------------------------------------- */

int nrgpu_abi_version(void);
const char *nrgpu_last_error(void);
/* select and initialise the CUDA device used by later calls */
int nrgpu_init(int device);

/* Fill p with the values a BAM parfile of the C1 kind produces; the caller
 * overrides fields.  Pure host code, usable without a GPU. */
void nrgpu_bssn_params_default(nrgpu_bssn_params *p);

/* ---- levels ----------------------------------------------------------- */

/* Device mirror of a level: geometry, flags and per-point masks; allocates
 * RK4 scratch lazily.  Replaces nothing in the reference (BAM keeps levels
 * in host memory only). */
int nrgpu_level_create(const nrgpu_level_desc *desc, nrgpu_level **out);
int nrgpu_level_destroy(nrgpu_level *lev);

/* ---- the hot path (device pointers) ------------------------------------- */

/* BSSN right-hand side on the inner points (boundary flag 0).
 * Replaces bssn_rhs_movpunc_N(unew, upre, c, ucur)
 * (bssn_rhs_movpunc_N.c:27, registered as "geometry", bssn.c:17,325).
 * c == 0: unew = rhs(ucur).  c != 0: unew = upre + c*rhs(ucur) followed by
 * the trace/determinant fixes of the reference (:15151-15380).
 * unew, upre, ucur: 24 device pointers each.  stream: a cudaStream_t or 0. */
int nrgpu_bssn_rhs(nrgpu_level *lev, double *const *unew, double *const *upre,
                   double c, double *const *ucur, const nrgpu_bssn_params *p,
                   void *stream);

/* Radiative boundary on the physical boundary points (flag PHYBOUND).
 * Replaces set_boundary(unew, upre, c, ucur) (boundary.c:25) for
 * boundary = radiative without rotation terms, i.e.
 * set_boundary_rot_rad (radiative.c:105) with rot = 0 for every variable. */
int nrgpu_bssn_boundary(nrgpu_level *lev, double *const *unew, double *const *upre,
                        double c, double *const *ucur, const nrgpu_bssn_params *p,
                        void *stream);

/* det(g) = 1 and tr(A) = 0 on all points.  Replaces bssn_algcon
 * (bssn_algcon.c:25) via bssn_algcon_wrapper (bssn.c:86). u: the 24-var list. */
int nrgpu_bssn_algcon(nrgpu_level *lev, double *const *u, const nrgpu_bssn_params *p,
                      void *stream);

/* r = a*x + b*y over all points of n variables.  Replaces vladd
 * (variables.c:650); with r == x and a == 1 it is vladdto (variables.c:721). */
int nrgpu_vladd(nrgpu_level *lev, int nvars, double *const *r, double a,
                double *const *x, double b, double *const *y, void *stream);

/* One full RK4 step of the level in place: evolve_rk_rk4 (rk.c:220) with
 * evolve_rhs (evolve.c:37) = RHS + radiative boundary in each stage, then the
 * algebraic constraints (bssn_algcon_wrapper, bssn.c:86).  The four stages
 * are fused kernels that also do the vladd/vladdto updates.  u: 24 device
 * pointers.  Uses scratch owned by the level (allocated on first call). */
int nrgpu_bssn_rk4_step(nrgpu_level *lev, double *const *u, double dt,
                        const nrgpu_bssn_params *p, void *stream);

/* nsteps RK4 steps starting from and returning to HOST arrays: uploads
 * host_u (24 host pointers), steps on the device, downloads the result into
 * host_u.  The end-to-end call of a host code that keeps its state in host
 * memory.  When the 24 arrays lie at one pitch (rows of one array) and the
 * level is one box of at least 16 planes, the box is copied as z slabs
 * (one 2D copy per slab) and the copies overlap the first stage of the
 * first step and the last stage of the last step; results are identical
 * either way.  Pinned host memory gives full PCIe bandwidth. */
int nrgpu_bssn_evolve_host(nrgpu_level *lev, double *const *host_u, int nsteps,
                           double dt, const nrgpu_bssn_params *p);

/* Device NaN/Inf flag of the level: set by the RHS kernels when any rhs is
 * not finite (the reference prints per point, check.c:235).  Reads and
 * clears it; *flag = 1 if set.  Returns NRGPU_ERR_TIMEOUT if a wait of the
 * staged-tile kernel for its shared-memory tiles ran out of time (the
 * kernel then stops computing and returns). */
int nrgpu_level_nan_flag(nrgpu_level *lev, int *flag);

/* One RK4 step of a single box (outer layer = physical boundary, inner
 * points elsewhere), exactly as nrgpu_bssn_rk4_step, for callers that cannot
 * allocate device memory: embedded hosts whose device memory is owned by
 * another runtime's pool, or a code that allocates nothing after start-up.
 * The library neither allocates nor frees anything in this call; its three
 * scratch lists live in a fixed device array of the library image, so the
 * box may hold at most 16384 points (m*n*o; larger boxes are rejected with
 * NRGPU_ERR_ARG) and every GPU that loads the library holds 9 MiB for it
 * until exit.  The first call on a device looks up that array's address;
 * make it before any stream capture.  All calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller.  The caller
 * passes u (24 device pointers, box->noffset == 0), updated in place.
 * A non-finite rhs is recorded in a status word of the library image, kept
 * over calls until nrgpu_bssn_noalloc_status reads it.  A cudaDeviceReset
 * between calls is not supported (the array's address is looked up once).
 * No counterpart in the reference. */
int nrgpu_bssn_rk4_step_noalloc(const nrgpu_box *box, double dx, double dy, double dz,
                                double *const *u, double dt, const nrgpu_bssn_params *p,
                                void *stream);
/* Status of nrgpu_bssn_rk4_step_noalloc since the last read, allocating
 * nothing: waits for `stream`, sets *flag = 1 if any rhs value was not
 * finite, and clears the word; returns NRGPU_ERR_ARG if an inner point had
 * no room for its stencil.  The companion of nrgpu_level_nan_flag for that
 * entry point.  No counterpart in the reference. */
int nrgpu_bssn_noalloc_status(int *flag, void *stream);

/* ---- Z4c (device pointers, 25-variable lists) -------------------------------- */

/* Replaces z4_rhs_movpunc_N(unew, upre, c, ucur) (z4_rhs_movpunc_N.c:23,
 * registered as "geometry" by z4_startup, z4.c:246); same semantics as
 * nrgpu_bssn_rhs.  z4_useNPTs must be off. */
int nrgpu_z4_rhs(nrgpu_level *lev, double *const *unew, double *const *upre, double c,
                 double *const *ucur, const nrgpu_z4_params *p, void *stream);
/* Replaces set_boundary for the Z4c list ("geometry_bound", z4.c:248). */
int nrgpu_z4_boundary(nrgpu_level *lev, double *const *unew, double *const *upre, double c,
                      double *const *ucur, const nrgpu_z4_params *p, void *stream);
/* evolve_rk_rk4 (rk.c:220) of the Z4c list + z4_algcon_wrapper (z4.c:49). */
int nrgpu_z4_rk4_step(nrgpu_level *lev, double *const *u, double dt, const nrgpu_z4_params *p,
                      void *stream);

/* ---- puncture initial data: the multigrid ---------------------------------- */

/* Parameters of the reference's multigrid (bam_multigrid.c:33-49) and of
 * the puncture solve (bam_punctures.c:110-178). */
typedef struct {
  int npre, npost;             /* mg_relax_npre / mg_relax_npost */
  int exact_nmin, exact_nmax;  /* mg_exact_nmin / mg_exact_nmax */
  int vcycle_nmin, vcycle_nmax;/* mg_vcycle_nmin (must be 0) / mg_vcycle_nmax */
  int fullV;                   /* mg_typeofcycles = fullV (1) or finest only (0) */
  int size_nmin, levels_nmax;  /* mg_size_nmin / mg_levels_nmax */
  double tol;                  /* punctures_tolerance, RMS residual */
  double falloff;              /* punctures_robin_falloff of u */
  int batch;                   /* V cycles per CUDA-graph launch (no counterpart) */
} nrgpu_mg_params;

typedef struct nrgpu_mg nrgpu_mg;  /* the multigrid stack on the device */

void nrgpu_mg_params_default(nrgpu_mg_params *p);

/* Build the stack for one cube of m^3 points (m - 2 divisible by 4 for each
 * coarsening), spacing dx, centred on the origin: makestack
 * (makestack.c:85-127) plus find_robin_normal on every level. */
int nrgpu_mg_create(int m, double dx, const nrgpu_mg_params *p, nrgpu_mg **out);
int nrgpu_mg_destroy(nrgpu_mg *mg);

/* Solve L(u) = Laplace u + b (1 + a (1+u))^-7 = 0 with a Robin boundary for
 * u by FAS multigrid.  Replaces multigrid(level, u, f, v, c, itmax, tol,
 * &normres, Lpuncture_nonlin, Lpuncture_GS) (multigrid.c:35, called from
 * PunctureSolve.c:282).  a, b, u: device arrays of m^3 doubles; u holds the
 * initial guess and receives the solution.  *ncycles = finest-level V
 * cycles, *normres = the final RMS residual. */
int nrgpu_mg_solve(nrgpu_mg *mg, const double *a, const double *b, double *u, int *ncycles,
                   double *normres, void *stream);
/* nsweeps damped Jacobi sweeps u <- u + omega (0 - L u) / L_ii of the
 * puncture equation on the finest level, each followed by the Robin
 * condition: smooths the grid-scale error of an initial guess (the learned
 * warm start) before nrgpu_mg_solve.  0 < omega <= 1.  No counterpart in the
 * reference (its smoother is undamped and runs only inside the V cycles). */
int nrgpu_mg_smooth(nrgpu_mg *mg, const double *a, const double *b, double *u, int nsweeps, double omega,
                    void *stream);

/* Brill-Lindquist + Bowen-York coefficients a = 1/(psi_BL - 1) and
 * b = a^7 K_ij K^ij / 8 on the m^3 cube (SetMWBL, SetBYK,
 * SetPunctureCoefficients: ConformalFactor.c:147, ExtrinsicCurvature.c:142,
 * Punctures.c:320).  Host arrays mass[n], pos/mom/spin[3n]; a, b device. */
int nrgpu_puncture_coefficients(int m, double dx, int npunc, const double *mass,
                                const double *pos, const double *mom, const double *spin,
                                double *a, double *b, void *stream);

/* ---- fixed mesh refinement -----------------------------------------------
 * Nested boxes, one or several boxes per level (separate boxes, such as a
 * binary's two punctures on the finer levels), each box made of whole cells
 * of the coarser box that holds it (the single-rank grid of amr = bo
 * newfmr, amr_fmr = nestedboxes).  The library derives the refinement flags
 * (setRPflags, main/amr/flag.c:122-255) per fine box and its parent box
 * from the boxes, and advances the whole hierarchy
 * by coarse steps: advance_levelandsublevels (main/main/main.c:397-418) with
 * the time interpolation of evolve (utility/evolve/evolve.c:292-340,
 * 371-380) and restrict_prolong_evolve (main/amr/inject.c:116-132) through
 * restrict_boxtobox_N / prolong_boxtobox_N
 * (utility/interpolate/interpolate_boxtobox_N.c:585-1223). */
typedef struct {
  int system;                   /* NRGPU_SYSTEM_BSSN or NRGPU_SYSTEM_Z4C */
  int lbo;                      /* levels l >= lbo subcycle (regrid.c:51-78) */
  int order_timeinterpolation;  /* 2 to 6 (bam_main.c:62, default 3) */
  int order_RP;                 /* 2, 4 or 6 (bam_main.c:58, default 4) */
  int nbuffer;                  /* amr_nbuffer (bam_amr.c) */
  int use_graph;                /* capture the coarse steps after the first
                                   in a CUDA graph and replay it */
  int autotune;                 /* 1: pick each level's rhs launch shape with
                                   nrgpu_level_autotune at creation; 2: the
                                   staged-tile rhs (nrgpu_level_tile) on every
                                   level it covers; 0: the default shape */
} nrgpu_fmr_params;

typedef struct nrgpu_fmr nrgpu_fmr;

/* levels[0] is the coarsest; dt[l] the level's time step (tL.dt);
 * sysparams: nlevels nrgpu_bssn_params or nrgpu_z4_params, one per level
 * (the dissipation factor differs between levels, evolve.c:486-530). */
int nrgpu_fmr_params_default(nrgpu_fmr_params *p);
int nrgpu_fmr_create(int nlevels, const nrgpu_level_desc *levels, const double *dt, const void *sysparams,
                     const nrgpu_fmr_params *p, nrgpu_fmr **out);
int nrgpu_fmr_destroy(nrgpu_fmr *fmr);
/* the refinement flags of level l (host arrays of the level's npoints, NULL
 * to skip): flagprolong (levels with a parent), flagrestrict (with a child;
 * with several child boxes the union of their pairs' flags, which the
 * reference keeps on a ghost parent of each child box instead) */
int nrgpu_fmr_flags(nrgpu_fmr *fmr, int l, double *flagprolong, double *flagrestrict);
/* restrict_prolong_varlist (inject.c:63-100) with nbuffer 3 between level
 * lfine and its parent: restrict lfine's uf into uc, then prolong uc into
 * lfine's buffer zone (nvars device pointers each) */
int nrgpu_fmr_restrict_prolong(nrgpu_fmr *fmr, int lfine, double *const *uc, double *const *uf, void *stream);
/* the same for a list of nvars (<= 25) other variables, as
 * set_boundary_refinement_cf (main/amr/inject.c:179-189) applies it to
 * analysis fields (the ADM mass integrands, ADM_mass.c:103-104) */
int nrgpu_fmr_restrict_prolong_vars(nrgpu_fmr *fmr, int lfine, int nvars, double *const *uc, double *const *uf,
                                    void *stream);
/* nsteps coarse steps of the hierarchy; u holds nlevels * nvars device
 * pointers, level-major.  The caller keeps the same u for a run. */
int nrgpu_fmr_advance(nrgpu_fmr *fmr, double *const *u, int nsteps, void *stream);
/* level iterations done so far (tL.iteration) */
int nrgpu_fmr_iteration(nrgpu_fmr *fmr, int l);
/* the rhs block shape (x, y, z) level l runs with, into block[3] */
int nrgpu_fmr_block(nrgpu_fmr *fmr, int l, int *block);

/* Checkpoint of the hierarchy's own state (no counterpart: the reference's
 * checkpoint, main/main/checkpoint.c:14-165, writes the level variables,
 * which stay with the caller here): the level iteration counters and, for
 * every level with a child, the previous step's copy and the time
 * interpolant, and the tracked puncture positions.  nrgpu_fmr_state_size
 * gives the bytes; nrgpu_fmr_save writes them to a host buffer and
 * nrgpu_fmr_load restores them into a hierarchy created with the same
 * levels and parameters and tracking as many punctures (refused otherwise).  Both
 * wait for the device.  With the caller's level states this resumes a run
 * bit for bit. */
int nrgpu_fmr_state_size(nrgpu_fmr *fmr, size_t *bytes);
int nrgpu_fmr_save(nrgpu_fmr *fmr, void *host, size_t bytes);
int nrgpu_fmr_load(nrgpu_fmr *fmr, const void *host, size_t bytes);

/* Puncture tracking inside the hierarchy's steps: track_puncture
 * (projects/Gauge/moving_punctures.c:135-200) with the shift integrator
 * (nrgpu_track_punctures) on the finest level, the reference's default
 * lmaxpunc = amr_lmax (main/amr/grid.c:287-294), after each of its steps
 * and its restriction/prolongation, where the reference's ANALYZE runs
 * (main/main/main.c:397-423); interpolation order = order_RP.  The shift
 * one step earlier is interpolated before the step, so no copy of it is
 * kept.  nrgpu_fmr_track sets n <= NRGPU_MAX_PUNCTURES start positions
 * (host [3n], the moving_punctureN_x/y/z of init_moving_puncture) and
 * fixz; n = 0 stops tracking.  nrgpu_fmr_punctures waits for the device
 * and returns the positions (host [3n]) and, if status is not NULL, the
 * last step's status per puncture (nrgpu_track_punctures). */
#define NRGPU_MAX_PUNCTURES 16
int nrgpu_fmr_track(nrgpu_fmr *fmr, int n, const double *pos, int fixz);
int nrgpu_fmr_punctures(nrgpu_fmr *fmr, double *pos, int *status);
/* The tracker per puncture, moving_puncture_track_method
 * (projects/Gauge/moving_punctures.c:123-180): method 1 "int" (the default:
 * the shift integrator for every puncture), 0 "ext" (the extremum search,
 * nrgpu_track_punctures_extremum, for every puncture), 2 "extint" (the
 * extremum search for the first puncture, the integrator for the rest).
 * The search runs on variable var of the system's list
 * (moving_puncture_track_var), a maximum if find_max
 * (moving_puncture_track_mode = max), with minmove
 * (moving_puncture_track_minmove) and fixz_ext (moving_puncture_fixz = NS
 * or BHNS); the integrator keeps the fixz of nrgpu_fmr_track. */
int nrgpu_fmr_track_method(nrgpu_fmr *fmr, int method, int var, int find_max, double minmove, int fixz_ext);

/* Moving boxes (move_box, main/amr/move.c:808-986).  A level moves by a
 * regrid: the caller gives the level's new boxes (same spacing, each made of
 * whole cells of a box of the parent, as make_level_bboxes builds them,
 * box.c:465-560) and new state buffers; the library moves every time level
 * of the level (the state u, and on a level with a child the previous step,
 * the time interpolant and the older time levels of order_timeinterpolation
 * 4-6) as move_overlap does (move.c:712-800): the points that an old box of
 * the level also holds are copied from it, all others are prolonged from
 * the parent at order_RP (prolong_varlist, interpolate_boxtobox_N.c:
 * 870-1010, into the points that no old box holds).  The refinement flags
 * and pairs with the parent, and with the child, are set up again.
 *
 * nrgpu_fmr_regrid moves levels lmin .. lmin + nlev - 1 (lmin >= 1),
 * coarsest first so that each prolongs from its parent's new state:
 * desc[i] holds level lmin + i's new boxes, or nboxes = 0 to keep the level
 * (its pairs are still set up again when its parent moved); u is the
 * caller's table of all levels' current state pointers (nlevels * nvars),
 * unew[i * nvars + v] the new buffers of level lmin + i (desc[i].npoints
 * points each; ignored for kept levels).  It waits for the stream; the
 * caller then puts unew into its table and frees the old buffers.
 *
 * nrgpu_fmr_set_move installs a hook that nrgpu_fmr_advance calls where the
 * reference calls move_box(g, l) (main/main/main.c:428): after level l - 1,
 * its sublevels, their restriction and prolongation and the puncture
 * tracking are done, when level l - 1 is not aligned in time with its own
 * parent (or l = 1).  The hook decides which of the levels l .. nlevels-1
 * move (find_nested_bboxes, move.c:121-463, is the reference's rule; the
 * tracked positions come from nrgpu_fmr_punctures), calls nrgpu_fmr_regrid
 * on `stream`, updates the pointer table that it gave to nrgpu_fmr_advance
 * (the advance reads the table after the hook returns) and returns 0, or
 * an error code that ends the advance.  With a hook, coarse steps run
 * without the CUDA graph.  fn = NULL removes the hook. */
typedef int (*nrgpu_fmr_move_fn)(void *user, nrgpu_fmr *fmr, int l, void *stream);
int nrgpu_fmr_set_move(nrgpu_fmr *fmr, nrgpu_fmr_move_fn fn, void *user);
int nrgpu_fmr_regrid(nrgpu_fmr *fmr, int lmin, int nlev, const nrgpu_level_desc *desc, double *const *u,
                     double *const *unew, void *stream);

/* ---- analysis: ADM mass, momentum and angular momentum ---------------------
 * ADM_mass (projects/ADM_mass/ADM_mass.c:11-225).  nrgpu_adm_mass_integrands
 * writes its eight integrands at the flag-0 points of a level (the other
 * points are left as they are): out[0] the ADM mass (adm_mass_integrand.c),
 * out[1] the mass from chi alone (adm_mass_integrand_chi.c), out[2..4] Px,
 * Py, Pz and out[5..7] Jx, Jy, Jz (adm_pj_integrand.c).  gK holds 12 device
 * arrays, the ADM metric gxx..gzz and curvature Kxx..Kzz (nrgpu_to_adm);
 * trK is the evolved trace K, chi the conformal factor (bssn_K, bssn_chi).
 * First derivatives by the 2nd-order centred stencil, as the reference's
 * integrands take them.  On a hierarchy the reference then fills every
 * level's boundary from its parent and its covered interior from its child,
 * finest first (nrgpu_fmr_restrict_prolong_vars with nvars = 8).
 *
 * nrgpu_sphere_integral: integral_over_sphere with Simpson weights
 * (utility/NumericUtils/Integral_over_sphere.c:197-357) of the device array
 * f of a level over the sphere of radius r about (x0, y0, z0): ntheta
 * circles (odd) of nphi + 1 points (nphi even), values by Lagrange
 * interpolation of the given order (order_centered in ADM_mass); on
 * bitant, qreflect and octant grids the covered part times the symmetry
 * factor.  *result is 0 when a sphere point's interpolation cube is not on
 * the level, as in the reference.  Synchronises the stream. */
int nrgpu_adm_mass_integrands(nrgpu_level *L, const double *const *gK, const double *trK, const double *chi,
                              double *const *out, void *stream);
int nrgpu_sphere_integral(nrgpu_level *L, const double *f, double x0, double y0, double z0, double r, int ntheta,
                          int nphi, int order, double *result, void *stream);

/* ---- analysis: Psi4 and its modes -----------------------------------------
 * compute_curvature_invariants (projects/Invariants/Invariants.c:48-252).
 * nrgpu_psi4: rpsi4, ipsi4 (and Csqr, the square of the Weyl tensor, when
 * csqr is not NULL) of curvature_invariants_N (curvature_invariants_N.m:
 * 14-208) at the flag-0 points, from the ADM metric and curvature gK (12
 * device arrays), the lapse and the shift (3); derivatives at
 * order_centered (2, 4, 6) with the order ladder near box faces; tetrad
 * kinnersley = 0 (Gram-Schmidt, invariants_tetrad = GS) or 1; flat = 1 for
 * gauss_codacci_mainardi = flat; origin (NULL: 0) is the sphere origin
 * (sphere_x0..z0).  On a hierarchy the reference then restricts and
 * prolongs rpsi4, ipsi4 and Csqr finest first
 * (nrgpu_fmr_restrict_prolong_vars) and multiplies psi4 by the distance to
 * invariants_x0..z0 (nrgpu_psi4_rescale, rescale_psi4, Invariants.c:
 * 263-284).
 * nrgpu_psi4_modes: compute_modes (Invariants.c:367-540): for l = lmin..lmax
 * (2 <= lmin, lmax <= 12) and every m, the spin-weight -2 harmonic
 * projection conj(Y_lm) psi4 formed at every point and integrated over the
 * sphere of each radius (nrgpu_sphere_integral with ntheta, nphi, order =
 * invariants_ntheta, _nphi, _order); out[((n * (lmax-lmin+1) + l-lmin) *
 * (2 lmax + 1) + m + l) * 2 + {0, 1}] = (real, imaginary) part.  No
 * symmetry grids.  Synchronises the stream. */
int nrgpu_psi4(nrgpu_level *L, const double *const *gK, const double *alpha, const double *const *beta,
               int order_centered, int kinnersley, int flat, const double *origin, double *rpsi4, double *ipsi4,
               double *csqr, void *stream);
int nrgpu_psi4_rescale(nrgpu_level *L, double *rpsi4, double *ipsi4, const double *origin, void *stream);
int nrgpu_psi4_modes(nrgpu_level *L, const double *rpsi4, const double *ipsi4, const double *origin, int lmin,
                     int lmax, const double *radii, int nr, int ntheta, int nphi, int order, double *out,
                     void *stream);

/* the evolution systems */
enum { NRGPU_SYSTEM_BSSN = 0, NRGPU_SYSTEM_Z4C = 1 };

/* ---- launch-shape autotuner (no counterpart in the reference) -------------
 * The rhs kernels compute one point per thread in blocks of 128 or 256
 * threads.  nrgpu_level_autotune times twenty block shapes (x, y, z
 * extents, from 32 x 4 x 1 and 8 x 16 x 1 to 8 x 4 x 4, 16 x 8 x 2 and
 * 8 x 8 x 4) for the level's boxes
 * and the given system (NRGPU_SYSTEM_BSSN / _Z4C) and parameters, on a flat
 * state in the level's RK4 scratch (the user's arrays are not touched),
 * keeps the fastest for the level and returns it in best_block[3] (may be
 * NULL).  For BSSN it also times the staged-tile kernel (16 x 4 x 4 tiles
 * whose fields are brought into shared memory by TMA loads) where the level
 * and parameters allow it, and keeps it when faster; best_block is then
 * {0, 0, 0}.  Waits for the stream.  nrgpu_level_block sets a shape
 * directly (powers of two, bx by bz = 128 or 256; default 32 x 4 x 1) and
 * turns the staged-tile kernel off.  Results do not depend on the shape;
 * the staged-tile kernel adds the same terms in another order (rounding
 * differences only). */
int nrgpu_level_autotune(nrgpu_level *L, int system, const void *params, void *stream, int *best_block);
int nrgpu_level_block(nrgpu_level *L, int bx, int by, int bz);
int nrgpu_level_get_block(nrgpu_level *L, int *block);
/* The BSSN interior rhs over TMA-staged tiles on every box it covers (runs
 * of order 4 or 6, even row length, 16-byte aligned fields, advection shift
 * 1 or 2 at 4th order, the centred 6th-order advection), the per-point
 * kernel elsewhere: on = 1 one block per tile, 2 the persistent form (one
 * block per SM walking the tiles, the next tile's fields loaded during the
 * current one), 0 off, -1 only queries.  Returns the setting. */
int nrgpu_level_tile(nrgpu_level *L, int on);
/* The Z4c interior rhs of all boxes of a level in one persistent launch:
 * the blocks take tiles from a queue over the boxes (an atomic counter)
 * until it is empty, each point computed as by the per-box kernel, so the
 * results are identical.  For levels of two or more boxes of one size that
 * has a compile-time-stride kernel (66, 72, 104, 136, 162, 168, 194 points
 * in x and y), 4th or 6th order, FP64; one launch per box otherwise.
 * on = 1 on, 0 off, -1 only queries; returns the setting.
 * nrgpu_level_autotune turns it on where it measures faster.  No
 * counterpart in the reference (advance_levelandsublevels, main.c:397-418,
 * steps the boxes of a level one after another). */
int nrgpu_level_queue(nrgpu_level *L, int on);

/* ---- ADM diagnostics ------------------------------------------------------
 * ADM metric and extrinsic curvature from the conformal variables:
 * bssn_to_adm_vl (projects/bssn/bssn.c:132-197) and z4_to_adm_vl
 * (projects/z4/z4.c:93-124), psi = chi^(1/chipsipower),
 * g_ij = psi^4 g~_ij, K_ij = psi^4 A~_ij + K g_ij / 3, on every point.
 * u: the first 14 evolved variables of either system (g~ 6, chi, A~ 6, K;
 * for Z4c the K slot is Khat, as in the reference); adm: g 6 then K 6. */
int nrgpu_to_adm(nrgpu_level *L, const double *const *u, double *const *adm, double chipsipower, void *stream);

/* adm_normalizedConstraints (projects/adm/bam_adm.c:40): no, yes,
 * "yes TermByTerm" */
enum { NRGPU_CON_PLAIN = 0, NRGPU_CON_NORMALIZED = 1, NRGPU_CON_TERMBYTERM = 2 };

/* Hamiltonian and momentum constraints of the ADM variables:
 * adm_constraints_N (projects/adm/adm_constraints_N.c:22, called by
 * computeadmconstraints, adm.c:14-74) without matter and with usepsi = 0,
 * on the points with boundary flag 0, centred order_centered with the
 * order ladder at box edges.  con: ham, mom1, mom2, mom3 and, for
 * mode != NRGPU_CON_PLAIN, normham, normmom1..3.  Flagged points of con are
 * not written. */
int nrgpu_adm_constraints(nrgpu_level *L, const double *const *adm, double *const *con, int order_centered,
                          int mode, void *stream);

/* norm2 (RMS) and normInf (max |u|) of nvars (<= 32) variables over the
 * points with boundary flag 0: bampi_allreduce_norm2 / bampi_allreduce_normInf
 * (main/bampi/reduce.c:209-266) on one rank.  Waits for the stream; the
 * results are in norm2[nvars], norminf[nvars] on return. */
int nrgpu_norms(nrgpu_level *L, const double *const *vars, int nvars, double *norm2, double *norminf,
                void *stream);

/* The scalars of the 0d output, write_level_0d (utility/output/output0d.c:
 * 28-116) with bampi_allreduce (main/bampi/reduce.c:37-135) on one rank,
 * for nvars (<= 32) variables over the points with boundary flag 0:
 * out[5 * v + t] for the output types t = 0 max, 1 min, 2 norm (RMS),
 * 3 normInf (max |u|), 4 integral (sum times dx^3).  Without such points:
 * -DBL_MAX, DBL_MAX, -1, -DBL_MAX, 0, as the reference.  Waits for the
 * stream. */
int nrgpu_output0d(nrgpu_level *L, const double *const *vars, int nvars, double *out, void *stream);

/* ---- puncture tracking ----------------------------------------------------
 * The shift-integration tracker, track_moving_puncture_integrate
 * (projects/Gauge/moving_punctures_integrate.c:29-100) with the position
 * test of track_puncture (projects/Gauge/moving_punctures.c:189-191), for n
 * punctures on level L: x_new solves x' = -beta(x) by three corrector
 * passes x0 = x1 - dt/2 (beta(x0) + beta_p(x1)); the shift is interpolated
 * with Lagrange cubes of order^3 points (interpolate_xyz_scalar,
 * utility/interpolate/interpolate.c:419-470; 2 <= order <= 8, the
 * reference's order_RP), 0 where the cube does not fit in the box of its
 * corner node.  A position below a symmetry plane of the level stays
 * (grid->half); fixz keeps z (moving_puncture_fixz = BH or BHNS); a new
 * position off the level is not taken.  beta, beta_p: 3 device pointers
 * each (the level's shift now and one step earlier); pos: device [3n],
 * updated in place; status: device [n] or NULL, per puncture bit 0 = the
 * integration ran, bit 1 = the new position is on the level (taken).
 * Positions equal the reference's bit for bit. */
int nrgpu_track_punctures(nrgpu_level *L, const double *const *beta, const double *const *beta_p, double dt,
                          int order, int fixz, int n, double *pos, int *status, void *stream);
/* The extremum search, track_moving_puncture_extremum
 * (projects/Gauge/moving_punctures_integrate.c:160-235, with findextremum,
 * :105-140; moving_puncture_track_method = ext), on the level variable var
 * (device [npoints], moving_puncture_track_var, the lapse by default): per
 * axis a parabola through var at x - h, x, x + h, a step to its vertex
 * clamped to one spacing, kept only when var at the new point is larger
 * (find_max) or smaller than at the old one and the step is at least
 * minmove * dx (moving_puncture_track_minmove).  fixz keeps z
 * (moving_puncture_fixz = NS or BHNS).  pos, status and the position test
 * as for nrgpu_track_punctures (status bit 0 is always set).  Positions
 * equal the reference's bit for bit. */
int nrgpu_track_punctures_extremum(nrgpu_level *L, const double *var, int find_max, double minmove, int order,
                                   int fixz, int n, double *pos, int *status, void *stream);

/* ---- learned warm start of the puncture solve ----------------------------
 * No counterpart in the reference.  A coordinate MLP (NRGPU_MLP_IN features
 * -> 4 hidden layers of NRGPU_MLP_HIDDEN, SiLU -> 1) conditioned on the
 * binary's parameters predicts the correction u that PunctureData
 * (Punctures.c:439) otherwise solves for from u = 0.  BF16 products with
 * FP32 accumulation on the tensor cores; FP32 master weights and Adam.
 * A conditioning vector is 20 doubles: m1 m2, pos1 pos2, mom1 mom2,
 * spin1 spin2 (the parameters of ReadPunctureParameters, Punctures.c:221). */
#define NRGPU_MLP_IN 32
#define NRGPU_MLP_HIDDEN 128
typedef struct nrgpu_mlp nrgpu_mlp;
int nrgpu_mlp_nparams(void);
int nrgpu_mlp_create(int max_batch, nrgpu_mlp **out);
int nrgpu_mlp_destroy(nrgpu_mlp *mlp);
int nrgpu_mlp_set_params(nrgpu_mlp *mlp, const float *host_params, int n);
int nrgpu_mlp_get_params(nrgpu_mlp *mlp, float *host_params, int n);
/* the table of nsets conditioning vectors (host, copied) that feature rows
 * refer to */
int nrgpu_mlp_set_conditions(nrgpu_mlp *mlp, const double *host_cond, int nsets);
/* feature rows of n points: row r is grid point d_pt[r] (x fastest) of the
 * m^3 cube of spacing dx centred on the origin, for binary d_set[r] of the
 * conditioning table (d_set, d_pt: device int arrays) */
int nrgpu_mlp_features(nrgpu_mlp *mlp, const int *d_set, const int *d_pt, int n, int m, double dx, void *stream);
/* the last n feature rows as BF16 bit patterns (host [n][NRGPU_MLP_IN]) */
int nrgpu_mlp_copy_features(nrgpu_mlp *mlp, int n, uint16_t *host);
/* one step on the last feature rows against targets d_y[n] (device):
 * forward, MSE loss, backward, and with update != 0 an Adam step of rate
 * lr.  The loss is written to *loss (host) when loss != NULL. */
int nrgpu_mlp_train_step(nrgpu_mlp *mlp, const float *d_y, int n, float lr, int update, float *loss,
                         void *stream);
/* the gradients of the last train step, in the parameter layout */
int nrgpu_mlp_gradients(nrgpu_mlp *mlp, float *host_grad, int n);
/* network output of the last feature rows into d_out[n] (device) */
int nrgpu_mlp_forward(nrgpu_mlp *mlp, int n, float *d_out, void *stream);
/* the warm start: u[m^3] (device, FP64) = uscale * network output at every
 * point of the m^3 cube, for one binary (replaces the conditioning table) */
int nrgpu_mlp_predict_u(nrgpu_mlp *mlp, const double *host_cond, int m, double dx, double uscale, double *u,
                        void *stream);
/* The same prediction in FP32 on the CUDA cores from the FP32 master
 * weights (features rounded to FP32, not BF16): the evaluation path, whose
 * guess carries no BF16 grid-scale noise. */
int nrgpu_mlp_predict_u_fp32(nrgpu_mlp *mlp, const double *host_cond, int m, double dx, double uscale, double *u,
                             void *stream);
/* The same prediction on the tensor cores (tcgen05.mma, FP32 accumulators in
 * tensor memory): one persistent CTA per SM holds W1..W4 in shared memory as
 * BF16 and runs the four 128-wide layers of 128-point tiles back to back;
 * BF16 features and activations as in training.  Asynchronous on `stream`;
 * nrgpu_mlp_tc_status reports whether a bounded wait inside it ran out. */
int nrgpu_mlp_predict_u_tc(nrgpu_mlp *mlp, const double *host_cond, int m, double dx, double uscale, double *u,
                           void *stream);
/* synchronises the device; *timed_out = 1 (and NRGPU_ERR_TIMEOUT) when the
 * last tensor-core prediction gave up waiting for its MMAs (its output is
 * then incomplete), else 0 */
int nrgpu_mlp_tc_status(nrgpu_mlp *mlp, int *timed_out);

/* ---- diagnostics -------------------------------------------------------- */

/* Measured FP64 FMA throughput of the current device (FLOP/s, 2 per FMA),
 * the denominator of the FP64 roofline.  No counterpart in the reference. */
int nrgpu_probe_fp64_peak(int iters, double *flops_per_s, float *ms);

#ifdef __cplusplus
}
#endif
#endif /* NRGPU_H */
