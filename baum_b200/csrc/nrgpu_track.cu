// nrgpu_track.cu -- the shift-integration puncture tracker on the device.
//
// track_moving_puncture_integrate (Gauge/moving_punctures_integrate.c:29-100):
// the new position of a puncture solves x' = -beta(x) over one step by three
// corrector passes, x0 = x1 - dt/2 (beta(x0) + beta_p(x1)), with the shift
// interpolated by interpolate_xyz_scalar (utility/interpolate/interpolate.c:
// 419-470): a Lagrange cube of order^3 points whose corner is the node at
// floor((x - xmin + dequaleps)/dx) - (order-1)/2 from the level's lower
// corner; the first box holding that node must hold the whole cube, else the
// value is 0; the sums run over z, then y, then x (interpolate_TriN,
// interpolate.c:121-160) with the products of coefficients_lagrange_N
// (lagrange.c:13-27).  track_puncture (Gauge/moving_punctures.c:135-200)
// keeps the old position when the new one is off the level.
//
// The extremum search (track_moving_puncture_extremum,
// moving_punctures_integrate.c:160-235, with findextremum, :105-140) fits a
// parabola through the tracked variable at x - dx, x, x + dx per axis,
// steps to its vertex (at most one spacing), and keeps the step only if the
// variable improves and the step is at least minmove * dx.
//
// One warp per puncture: the 32 lanes fetch each interpolation cube into
// shared memory together (one round trip instead of order^2 dependent
// ones), then every lane forms the same sums.  Every product, quotient and
// sum is rounded separately (no contraction into FMAs), in the reference's
// order, so the positions equal the reference's bit for bit.
#include <math.h>

#include "nrgpu_level.cuh"

namespace {

constexpr double kEps = 1e-10;  // dequaleps (main/main/bam_main.h:19)
constexpr int kMaxOrder = 8;

__device__ __forceinline__ bool dless(double a, double b) { return a < __dsub_rn(b, kEps); }
__device__ __forceinline__ bool dequal(double a, double b) { return !(dless(a, b) || dless(b, a)); }

struct TrackArgs {
  const BoxGeo *box;
  int nboxes, symmetry;
  double o[3], h[3];  // the level's lower corner and spacings
  const double *beta[3], *beta_p[3];
  double dt;
  int order, fixz, n;
  double *pos;   // [3n], in/out
  double *b1;    // [3n]: shift one step earlier at the old positions (phases 1, 2)
  int *status;   // [n] or null: bit 0 integrated, bit 1 new position on the level
};

__device__ void lagrange(int n, double x, double xmin, double h, double *c) {
  for (int i = 0; i < n; i++) {
    double d = 1.0;
    for (int j = 0; j < n; j++)
      if (j != i)
        d = __dmul_rn(d, __ddiv_rn(__dsub_rn(__dsub_rn(x, xmin), __dmul_rn((double)j, h)),
                                   __dmul_rn((double)(i - j), h)));
    c[i] = d;
  }
}

__device__ __forceinline__ double dot(int n, const double *c, const double *u) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s = __dadd_rn(s, __dmul_rn(c[i], u[i]));
  return s;
}

__device__ int node_of(double c, double x0, double h, int n) {
  const int i = (int)floor(__dadd_rn(__ddiv_rn(__dsub_rn(c, x0), h), 0.5));
  if (i < 0 || i >= n || !dequal(c, __dadd_rn(x0, __dmul_rn((double)i, h)))) return -1;
  return i;
}

// cube: the warp's shared buffer of kMaxOrder^3 values; all lanes call
// with the same arguments
__device__ double interpolate(const TrackArgs &A, const double *v, const double p[3], double *cube) {
  const int a = A.order, nh = (A.order - 1) / 2;
  double xc[3];
  for (int d = 0; d < 3; d++)
    xc[d] = __dadd_rn(A.o[d], __dmul_rn(A.h[d], floor(__ddiv_rn(__dadd_rn(__dsub_rn(p[d], A.o[d]), kEps), A.h[d])) -
                                                      (double)nh));
  for (int b = 0; b < A.nboxes; b++) {
    const BoxGeo B = A.box[b];
    const int i = node_of(xc[0], B.x0, A.h[0], B.m);
    const int j = node_of(xc[1], B.y0, A.h[1], B.n);
    const int k = node_of(xc[2], B.z0, A.h[2], B.o);
    if (i < 0 || j < 0 || k < 0) continue;
    if (i + a > B.m || j + a > B.n || k + a > B.o) return 0.0;
    const int lane = threadIdx.x & 31, a3 = a * a * a;
    for (int t = lane; t < a3; t += 32) {
      const int ii = t % a, jj = (t / a) % a, kk = t / (a * a);
      cube[t] = v[(long)B.noffset + (i + ii) + (long)B.m * (j + jj) + (long)B.m * B.n * (k + kk)];
    }
    __syncwarp();
    double c[kMaxOrder], w[kMaxOrder], vv[kMaxOrder][kMaxOrder], line[kMaxOrder];
    lagrange(a, p[2], xc[2], A.h[2], c);
    for (int ii = 0; ii < a; ii++)
      for (int jj = 0; jj < a; jj++) {
        for (int kk = 0; kk < a; kk++) line[kk] = cube[ii + a * jj + a * a * kk];
        vv[ii][jj] = dot(a, c, line);
      }
    __syncwarp();  // every lane has read the cube before the next fetch
    lagrange(a, p[1], xc[1], A.h[1], c);
    for (int ii = 0; ii < a; ii++) w[ii] = dot(a, c, vv[ii]);
    lagrange(a, p[0], xc[0], A.h[0], c);
    return dot(a, c, w);
  }
  return 0.0;
}

__device__ bool on_level(const TrackArgs &A, const double p[3]) {
  for (int b = 0; b < A.nboxes; b++) {
    const BoxGeo B = A.box[b];
    const double lo[3] = {B.x0, B.y0, B.z0};
    const int n[3] = {B.m, B.n, B.o};
    bool in = true;
    for (int d = 0; d < 3; d++)
      if (dless(p[d], lo[d]) || dless(__dadd_rn(lo[d], __dmul_rn((double)(n[d] - 1), A.h[d])), p[d])) in = false;
    if (in) return true;
  }
  return false;
}

__device__ bool below_half(const TrackArgs &A, const double p[3]) {
  for (int d = 0; d < 3; d++)
    if ((A.symmetry >> d & 1) && dless(p[d], 0.0)) return true;
  return false;
}

// phase 0: one call with beta and beta_p; phase 1: before the step, the
// shift at the old positions into b1; phase 2: after the step, from b1
__global__ void __launch_bounds__(32) track_kernel(TrackArgs A, int phase) {
  __shared__ double cube[kMaxOrder * kMaxOrder * kMaxOrder];
  const int q = blockIdx.x;
  if (q >= A.n) return;
  const bool lead = threadIdx.x == 0;
  double p1[3], p0[3], b1[3], b0[3];
  for (int d = 0; d < 3; d++) p1[d] = A.pos[3 * q + d];
  __syncwarp();  // every lane has read pos before lane 0 writes it
  const bool skip = below_half(A, p1);
  if (phase == 1) {
    if (!skip)
      for (int d = 0; d < 3; d++) {
        const double b = interpolate(A, A.beta[d], p1, cube);
        if (lead) A.b1[3 * q + d] = b;
      }
    return;
  }
  for (int d = 0; d < 3; d++) p0[d] = p1[d];
  if (!skip) {
    for (int d = 0; d < 3; d++) b1[d] = phase == 0 ? interpolate(A, A.beta_p[d], p1, cube) : A.b1[3 * q + d];
    for (int it = 0; it < 3; it++) {
      for (int d = 0; d < 3; d++) b0[d] = interpolate(A, A.beta[d], p0, cube);
      for (int d = 0; d < 3; d++) p0[d] = __dsub_rn(p1[d], __dmul_rn(__dmul_rn(A.dt, 0.5), __dadd_rn(b0[d], b1[d])));
    }
    if (A.fixz) p0[2] = p1[2];
  }
  const bool in = on_level(A, p0);
  if (!lead) return;
  if (in)
    for (int d = 0; d < 3; d++) A.pos[3 * q + d] = p0[d];
  if (A.status) A.status[q] = (skip ? 0 : 1) | (in ? 2 : 0);
}

__device__ double findextremum(double vm, double v0, double vp, bool max) {
  if (!isfinite(vm) || !isfinite(v0) || !isfinite(vp)) return 0.0;
  const double curv = __dsub_rn(__dmul_rn(0.5, __dadd_rn(vp, vm)), v0);
  double v;
  if (fabs(curv) <= 1e-10) {
    if ((vp > v0) && (vp > vm)) v = 1.0;
    else if ((vm > v0) && (vm > vp)) v = -1.0;
    else v = 0.0;
    v = __dmul_rn(v, max ? 1.0 : -1.0);
  } else {
    v = __ddiv_rn(__dsub_rn(vm, vp), __dmul_rn(4.0, curv));
    v = v > 1.0 ? 1.0 : v;
    v = v < -1.0 ? -1.0 : v;
  }
  return v;
}

// extremum search of the tracked variable (passed as A.beta[0]) for a
// maximum (find_max) or minimum; steps shorter than minimal_move are dropped;
// A.fixz keeps z (pintoxyplane 1 or 3 in the reference)
__global__ void __launch_bounds__(32) extremum_kernel(TrackArgs A, int find_max, double minimal_move) {
  __shared__ double cube[kMaxOrder * kMaxOrder * kMaxOrder];
  const int q = blockIdx.x;
  if (q >= A.n) return;
  const double *var = A.beta[0];
  double p0[3], p1[3], d[3];
  for (int a = 0; a < 3; a++) p0[a] = A.pos[3 * q + a];
  __syncwarp();
  const double v0 = interpolate(A, var, p0, cube);
  for (int a = 0; a < 3; a++) {
    double pm[3] = {p0[0], p0[1], p0[2]}, pp[3] = {p0[0], p0[1], p0[2]};
    pm[a] = __dsub_rn(p0[a], A.h[a]);
    pp[a] = __dadd_rn(p0[a], A.h[a]);
    const double vm = interpolate(A, var, pm, cube);
    const double vp = interpolate(A, var, pp, cube);
    d[a] = __dmul_rn(findextremum(vm, v0, vp, find_max), A.h[a]);
  }
  for (int a = 0; a < 3; a++) p1[a] = __dadd_rn(p0[a], d[a]);
  const double v = interpolate(A, var, p1, cube);
  const double len = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])), __dmul_rn(d[2], d[2])));
  if (!isfinite(v) || !isfinite(v0) || (find_max && v <= v0) || (!find_max && v >= v0) || len < minimal_move)
    for (int a = 0; a < 3; a++) p1[a] = p0[a];
  if (A.fixz) p1[2] = p0[2];
  const bool in = on_level(A, p1);
  if (threadIdx.x != 0) return;
  if (in)
    for (int a = 0; a < 3; a++) A.pos[3 * q + a] = p1[a];
  if (A.status) A.status[q] = 1 | (in ? 2 : 0);
}

int make_args(nrgpu_level *L, const double *const *beta, const double *const *beta_p, double dt, int order, int fixz,
              int n, double *pos, double *b1, int *status, TrackArgs *A) {
  if (!L || !beta || !pos || n < 1) return nrgpu_set_error(NRGPU_ERR_ARG, "bad arguments");
  if (order < 2 || order > kMaxOrder)
    return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "interpolation order %d (2..%d)", order, kMaxOrder);
  A->box = L->d_box;
  A->nboxes = L->nboxes;
  A->symmetry = L->symmetry;
  A->o[0] = L->hbox[0].x0;
  A->o[1] = L->hbox[0].y0;
  A->o[2] = L->hbox[0].z0;
  for (int b = 1; b < L->nboxes; b++) {
    A->o[0] = fmin(A->o[0], L->hbox[b].x0);
    A->o[1] = fmin(A->o[1], L->hbox[b].y0);
    A->o[2] = fmin(A->o[2], L->hbox[b].z0);
  }
  A->h[0] = L->dx;
  A->h[1] = L->dy;
  A->h[2] = L->dz;
  for (int d = 0; d < 3; d++) {
    if (!beta[d]) return nrgpu_set_error(NRGPU_ERR_ARG, "null beta[%d]", d);
    A->beta[d] = beta[d];
    A->beta_p[d] = beta_p ? beta_p[d] : nullptr;
  }
  A->dt = dt;
  A->order = order;
  A->fixz = fixz ? 1 : 0;
  A->n = n;
  A->pos = pos;
  A->b1 = b1;
  A->status = status;
  return NRGPU_OK;
}

}  // namespace

int nrgpu_track_before_step(nrgpu_level *L, const double *const *beta, int order, int n, const double *pos,
                            double *b1, cudaStream_t st) {
  TrackArgs A;
  int e = make_args(L, beta, nullptr, 0.0, order, 0, n, (double *)pos, b1, nullptr, &A);
  if (e) return e;
  track_kernel<<<n, 32, 0, st>>>(A, 1);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

int nrgpu_track_after_step(nrgpu_level *L, const double *const *beta, double dt, int order, int fixz, int n,
                           double *pos, const double *b1, int *status, cudaStream_t st) {
  TrackArgs A;
  int e = make_args(L, beta, nullptr, dt, order, fixz, n, pos, (double *)b1, status, &A);
  if (e) return e;
  track_kernel<<<n, 32, 0, st>>>(A, 2);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_track_punctures(nrgpu_level *L, const double *const *beta, const double *const *beta_p,
                                     double dt, int order, int fixz, int n, double *pos, int *status, void *stream) {
  if (!beta_p) return nrgpu_set_error(NRGPU_ERR_ARG, "null beta_p");
  for (int d = 0; d < 3; d++)
    if (!beta_p[d]) return nrgpu_set_error(NRGPU_ERR_ARG, "null beta_p[%d]", d);
  TrackArgs A;
  int e = make_args(L, beta, beta_p, dt, order, fixz, n, pos, nullptr, status, &A);
  if (e) return e;
  NRGPU_CUDA_TRY(cudaSetDevice(L->device));
  track_kernel<<<n, 32, 0, (cudaStream_t)stream>>>(A, 0);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

int nrgpu_track_extremum_on(nrgpu_level *L, const double *var, int find_max, double minmove, int order, int fixz,
                            int n, double *pos, int *status, cudaStream_t st) {
  if (!var) return nrgpu_set_error(NRGPU_ERR_ARG, "null var");
  const double *v3[3] = {var, var, var};
  TrackArgs A;
  int e = make_args(L, v3, nullptr, 0.0, order, fixz, n, pos, nullptr, status, &A);
  if (e) return e;
  extremum_kernel<<<n, 32, 0, st>>>(A, find_max ? 1 : 0, minmove * L->dx);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_track_punctures_extremum(nrgpu_level *L, const double *var, int find_max, double minmove,
                                              int order, int fixz, int n, double *pos, int *status, void *stream) {
  if (!L) return nrgpu_set_error(NRGPU_ERR_ARG, "null level");
  NRGPU_CUDA_TRY(cudaSetDevice(L->device));
  return nrgpu_track_extremum_on(L, var, find_max, minmove, order, fixz, n, pos, status, (cudaStream_t)stream);
}
