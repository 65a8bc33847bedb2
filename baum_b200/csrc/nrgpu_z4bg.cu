// nrgpu_z4bg.cu -- the Z4c "background" box boundary (sm_100a, FP64).
//
// The rhs with this boundary first extrapolates its input state onto the
// PHYBOUND points (z4_rhs_movpunc_N.c:148-152, level 0, no shells), so the
// stencils of the points next to the boundary see those values;
// nrgpu_z4_background_extrapolate is that step.
// set_boundary's background branch (utility/boundary/boundary.c:190-210):
//   1. the state ucur extrapolated onto the PHYBOUND points
//      (set_boundary_extrapolate, utility/boundary/extrapolate.c:22-47:
//      per direction a linear extrapolation from the two inner neighbours
//      where the point is at a box face, the mean of those directions;
//      three passes, so that edges and corners see their faces' new values);
//   2. the rhs of A, G, Khat and Theta at the points one inside the box
//      (boundaryNaway(1)) from the boundary condition:
//        mode 1, "background radcentered" (z4_boundary_box_rad.m):
//          rTheta = -s.dTheta - Theta/r, rKhat = -sqrt2 (s.dKhat + Khat/r),
//          rG_a = -s^b d_b G_a - G_a/r, rA_ab = -s^c d_c A_ab - A_ab/r,
//          s = x/r, centred 2nd-order first derivatives;
//        mode 2, "background" (z4_boundary_box.m, CPBC2): the constraint-
//          preserving conditions, nrgpu_z4bg_cpbc.cu;
//      unew = rhs (c = 0) or upre + c rhs;
//   3. the rhs extrapolated onto the PHYBOUND points the same way.
// The RK4 step with this boundary is evolve_rk_rk4 (utility/evolve/rk.c:
// 220-260) written out: the state's copy u_p is kept apart, because the
// first stage extrapolates the state itself (its input is u_c), which the
// step then keeps, while the later stage inputs start from u_p.
#include "nrgpu_level.cuh"

namespace {

constexpr int NV = NRGPU_Z4_NVARS;

struct Vars {
  double *p[NV];
};

// one thread per (PHYBOUND point, variable): one pass of
// set_boundary_extrapolate
__global__ void extrapolate_kernel(Vars V, const FlagPoint *__restrict__ fp, int nfp, const BoxGeo *__restrict__ box) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nfp) return;
  const FlagPoint P = fp[q];
  if (P.flag != NRGPU_PHYBOUND) return;
  const BoxGeo B = box[P.box];
  double *f = V.p[blockIdx.y];
  const int idx[3] = {P.i, P.j, P.k}, n[3] = {B.m, B.n, B.o};
  const long st[3] = {1, B.m, (long)B.m * B.n};
  const long c = P.ijk;
  double val[3];
  int use[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const long m1 = idx[d] > 0 ? c - st[d] : c, p1 = idx[d] + 1 < n[d] ? c + st[d] : c;
    const long m2 = idx[d] > 1 ? m1 - st[d] : c, p2 = idx[d] + 2 < n[d] ? p1 + st[d] : c;
    if (p1 == c) {
      val[d] = 2.0 * f[m1] - f[m2];
      use[d] = 1;
    } else if (m1 == c) {
      val[d] = 2.0 * f[p1] - f[p2];
      use[d] = 1;
    } else {
      val[d] = 0.5 * (f[p1] + f[m1]);
      use[d] = 0;
    }
  }
  const int nu = use[0] + use[1] + use[2];
  f[c] = nu > 0 ? (use[0] * val[0] + use[1] * val[1] + use[2] * val[2]) / nu : (val[0] + val[1] + val[2]) / 3.0;
}

// z4_boundary_box_rad at one point one inside the box (variables 7..17 of
// the Z4c list: A (6), Khat, G (3), Theta)
__global__ void rad_kernel(Vars cur, Vars nw, Vars pre, double c, const FlagPoint *__restrict__ lad, int nlad,
                           const BoxGeo *__restrict__ box, double dx, double dy, double dz) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nlad) return;
  const FlagPoint P = lad[q];
  const BoxGeo B = box[P.box];
  const long x = P.ijk;
  const long st[3] = {1, B.m, (long)B.m * B.n};
  const double oo2h[3] = {1 / (2 * dx), 1 / (2 * dy), 1 / (2 * dz)};
  const double X = B.x0 + P.i * dx, Y = B.y0 + P.j * dy, Z = B.z0 + P.k * dz;
  const double r = sqrt(X * X + Y * Y + Z * Z);
  const double s[3] = {X / r, Y / r, Z / r};
  auto D = [&](int v, int d) { return oo2h[d] * (-cur.p[v][x - st[d]] + cur.p[v][x + st[d]]); };
  double rhs[11];
  // A_ab: variables 7..12
  for (int v = 0; v < 6; ++v)
    rhs[v] = -(s[0] * D(7 + v, 0) + s[1] * D(7 + v, 1) + s[2] * D(7 + v, 2)) - cur.p[7 + v][x] / r;
  // Khat: variable 13
  rhs[6] = -sqrt(2.0) * (s[0] * D(13, 0) + s[1] * D(13, 1) + s[2] * D(13, 2) + cur.p[13][x] / r);
  // G_a: variables 14..16
  for (int a = 0; a < 3; ++a)
    rhs[7 + a] = -(s[0] * D(14 + a, 0) + s[1] * D(14 + a, 1) + s[2] * D(14 + a, 2)) - cur.p[14 + a][x] / r;
  // Theta: variable 17
  rhs[10] = -(s[0] * D(17, 0) + s[1] * D(17, 1) + s[2] * D(17, 2)) - cur.p[17][x] / r;
  for (int v = 0; v < 11; ++v) nw.p[7 + v][x] = c != 0.0 ? pre.p[7 + v][x] + c * rhs[v] : rhs[v];
}

// r = a + c b, every product and sum rounded separately (vladd, vladdto)
__global__ void axpy_kernel(Vars r, Vars a, double c, Vars b, long np) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= np) return;
  const int v = blockIdx.y;
  r.p[v][i] = __dadd_rn(a.p[v][i], __dmul_rn(c, b.p[v][i]));
}

int fill(Vars *V, double *const *u, const char *what) {
  for (int v = 0; v < NV; ++v) {
    if (!u[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null %s pointer %d", what, v);
    V->p[v] = u[v];
  }
  return NRGPU_OK;
}

int extrapolate(nrgpu_level *L, const Vars &V, cudaStream_t st) {
  if (!L->nflagpts) return NRGPU_OK;
  for (int pass = 0; pass < 3; ++pass)
    extrapolate_kernel<<<dim3((L->nflagpts + 127) / 128, NV), 128, 0, st>>>(V, L->d_flagpts, L->nflagpts, L->d_box);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

}  // namespace

int nrgpu_z4_cpbc_launch(nrgpu_level *L, double *const *ucur, double *const *unew, double *const *upre, double c,
                         const nrgpu_z4_params *p, cudaStream_t st);

int nrgpu_z4_background_extrapolate(nrgpu_level *L, double *const *u, cudaStream_t st) {
  if (L->nsym) return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "the background boundary on a symmetry grid");
  Vars V;
  int e;
  if ((e = fill(&V, u, "u"))) return e;
  return extrapolate(L, V, st);
}

int nrgpu_z4_background_boundary(nrgpu_level *L, double *const *unew, double *const *upre, double c,
                                 double *const *ucur, const nrgpu_z4_params *p, cudaStream_t st) {
  if (L->nsym) return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "the background boundary on a symmetry grid");
  Vars n, cu, pr;
  int e;
  if ((e = fill(&n, unew, "unew")) || (e = fill(&cu, ucur, "ucur"))) return e;
  if (c != 0.0) {
    if ((e = fill(&pr, upre, "upre"))) return e;
  } else {
    pr = cu;
  }
  if ((e = extrapolate(L, cu, st))) return e;
  // the flag-0 points one inside a box face: the distance-1 segment of the
  // ladder (boundaryNaway(1) among the inner points, where every box face
  // carries a boundary flag)
  if (L->nladder[0]) return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "the background boundary with unflagged box faces");
  const int nlad = L->nladder[1] - L->nladder[0];
  if (nlad > 0) {
    if (p->boundary == 1) {
      rad_kernel<<<(nlad + 127) / 128, 128, 0, st>>>(cu, n, pr, c, L->d_ladder + L->nladder[0], nlad, L->d_box, L->dx,
                                                     L->dy, L->dz);
      NRGPU_CUDA_TRY(cudaGetLastError());
    } else if ((e = nrgpu_z4_cpbc_launch(L, ucur, unew, c != 0.0 ? upre : ucur, c, p, st))) {
      return e;
    }
  }
  return extrapolate(L, n, st);
}

int nrgpu_z4_rk4_background(nrgpu_level *L, double *const *u, double dt, const nrgpu_z4_params *p, cudaStream_t st) {
  if (L->nsym) return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "the background boundary on a symmetry grid");
  Vars U;
  int e;
  if ((e = fill(&U, u, "u"))) return e;
  double *scr = nullptr;
  if ((e = nrgpu_level_scratch(L, &scr))) return e;
  const long np = L->npoints;
  Vars UP, R, V;
  double *pu[NV], *pup[NV], *pr[NV], *pv[NV];
  for (int v = 0; v < NV; ++v) {
    pu[v] = u[v];
    pup[v] = UP.p[v] = scr + (0L * NV + v) * np;
    pr[v] = R.p[v] = scr + (1L * NV + v) * np;
    pv[v] = V.p[v] = scr + (2L * NV + v) * np;
  }
  for (int v = 0; v < NV; ++v)
    NRGPU_CUDA_TRY(cudaMemcpyAsync(UP.p[v], U.p[v], sizeof(double) * np, cudaMemcpyDeviceToDevice, st));
  const dim3 g((unsigned)((np + 255) / 256), NV);
  const double a[4] = {0.0, dt / 2, dt / 2, dt}, b[4] = {dt / 6, dt / 3, dt / 3, dt / 6};
  for (int s = 0; s < 4; ++s) {
    double *const *cur = pu;
    if (s) {
      axpy_kernel<<<g, 256, 0, st>>>(V, UP, a[s], R, np);  // v = u_p + a r
      NRGPU_CUDA_TRY(cudaGetLastError());
      cur = pv;
    }
    if ((e = nrgpu_z4_rhs(L, pr, pup, 0.0, cur, p, st))) return e;
    if ((e = nrgpu_z4_background_boundary(L, pr, pup, 0.0, cur, p, st))) return e;
    axpy_kernel<<<g, 256, 0, st>>>(U, U, b[s], R, np);  // u += b r
    NRGPU_CUDA_TRY(cudaGetLastError());
  }
  return NRGPU_OK;
}
