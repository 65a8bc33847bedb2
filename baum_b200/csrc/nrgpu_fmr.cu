// nrgpu_fmr.cu -- fixed mesh refinement around the evolution (sm_100a), FP64:
// the Berger-Oliger recursion of nested boxes with Lagrange restriction and
// prolongation and time interpolation of the parent to the child's half step.
//   flags            setRPflags (flag.c:122-255), host, once
//   restrict_kernel  restrict_boxtobox_N (interpolate_boxtobox_N.c:1055-1223)
//   prolong_kernel   prolong_boxtobox_N (interpolate_boxtobox_N.c:585-869)
//   ti_start/finish  evolve.c:292-340, 371-380 (orders 2 to 6)
//   nrgpu_fmr_advance advance_levelandsublevels (main.c:397-418) with
//                    restrict_prolong_evolve (inject.c:116-132)
// The reference does restriction and prolongation as three 1-D sweeps
// through temporary arrays (z, then y, then x).  Here one thread computes one
// output point of one variable as the same nested sums in the same order,
// with explicit round-to-nearest multiplies and adds (no contraction into
// FMA), so that restriction, prolongation and time interpolation give the
// reference's values bit for bit from the same inputs; nothing is staged
// through global temporaries.
#include <string.h>
#include <algorithm>
#include <vector>
#include "nrgpu_level.cuh"

namespace {

constexpr int kMaxLevels = 16;
constexpr int kMaxVars = NRGPU_Z4_NVARS;
constexpr int kMaxOrder = 8;

struct Ptrs {
  double *p[kMaxVars];
};

struct Box3 {
  int n[3];
  long off;
};

__device__ __forceinline__ long at3(const Box3 &b, int i, int j, int k) {
  return b.off + i + (long)b.n[0] * (j + (long)b.n[1] * k);
}

struct RGeom {  // restriction of one child into its parent
  int ic[6];    // coarse bounding box of flagrestrict >= 3
  int if0[3];   // fine point of the first stencil of ic[0], ic[2], ic[4]
  double w[kMaxOrder];
};

struct PGeom {  // prolongation of a parent into its child
  int fb[6];    // fine bounding box of 1 <= flagprolong <= nbuffer
  int f0[6];    // fine bounding box of the other points (skipped pairs)
  int cs[3];    // coarse start of the first output pair per direction
  double c1[kMaxOrder], c2[kMaxOrder];
};

template <int N>
__device__ __forceinline__ double dot_rn(const double *w, const double *u) {
  double s = 0.0;
#pragma unroll
  for (int p = 0; p < N; ++p) s = __dadd_rn(s, __dmul_rn(w[p], u[p]));
  return s;
}

// one thread per (coarse output point, variable)
template <int N>
__global__ void restrict_kernel(Ptrs uc, Ptrs uf, Box3 cb, Box3 fb, RGeom G, int npts) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= npts) return;
  const int v = blockIdx.y;
  const int nI = G.ic[1] - G.ic[0] + 1, nJ = G.ic[3] - G.ic[2] + 1;
  const int I = G.ic[0] + q % nI, J = G.ic[2] + (q / nI) % nJ, K = G.ic[4] + q / (nI * nJ);
  const int fx = G.if0[0] + 2 * (I - G.ic[0]), fy = G.if0[1] + 2 * (J - G.ic[2]), fz = G.if0[2] + 2 * (K - G.ic[4]);
  const double *f = uf.p[v];
  double sx[N], sy[N], sz[N];
#pragma unroll
  for (int px = 0; px < N; ++px) {
#pragma unroll
    for (int py = 0; py < N; ++py) {
#pragma unroll
      for (int pz = 0; pz < N; ++pz) sz[pz] = __ldg(f + at3(fb, fx + px, fy + py, fz + pz));
      sy[py] = dot_rn<N>(G.w, sz);
    }
    sx[px] = dot_rn<N>(G.w, sy);
  }
  uc.p[v][at3(cb, I, J, K)] = dot_rn<N>(G.w, sx);
}

// one thread per (fine point written by the prolongation, variable): the
// points of the prolongation box that prolong_boxtobox_N writes (it skips
// the pairs whose first point lies in the inner box), listed at set-up as
// offsets in the prolongation box
template <int N>
__global__ void prolong_kernel(Ptrs uc, Ptrs uf, Box3 cb, Box3 fb, PGeom G, const int *__restrict__ list,
                               int npts) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= npts) return;
  const int q = list[n];
  const int v = blockIdx.y;
  const int nI = G.fb[1] - G.fb[0] + 1, nJ = G.fb[3] - G.fb[2] + 1;
  const int t[3] = {q % nI, (q / nI) % nJ, q / (nI * nJ)};
  const int i = G.fb[0] + t[0], j = G.fb[2] + t[1], k = G.fb[4] + t[2];
  int s[3];
  const double *w[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    s[d] = G.cs[d] + t[d] / 2 + (t[d] & 1);
    w[d] = (t[d] & 1) ? G.c2 : G.c1;
  }
  const double *c = uc.p[v];
  double sx[N], sy[N], sz[N];
#pragma unroll
  for (int px = 0; px < N; ++px) {
#pragma unroll
    for (int py = 0; py < N; ++py) {
#pragma unroll
      for (int pz = 0; pz < N; ++pz) sz[pz] = __ldg(c + at3(cb, s[0] + px, s[1] + py, s[2] + pz));
      sy[py] = dot_rn<N>(w[2], sz);
    }
    sx[px] = dot_rn<N>(w[1], sy);
  }
  uf.p[v][at3(fb, i, j, k)] = dot_rn<N>(w[0], sx);
}

// vladd (variables.c:575-650) with its special cases, and the u_p copy of
// the RK4 step: upp = ca u + cb up; up = u
__global__ void ti_start_kernel(Ptrs u, double *up, double *upp, double ca, double cb, long np, int nv) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= np * nv) return;
  const int v = (int)(t / np);
  const long i = t - (long)v * np;
  const double a = u.p[v][i];
  const double b = up[t];
  double r;
  if (ca == 0.0 && cb == 0.0) r = 0.0;
  else if (ca == 0.0) r = __dmul_rn(cb, b);
  else if (cb == 0.0) r = __dmul_rn(ca, a);
  else r = __dadd_rn(__dmul_rn(ca, a), __dmul_rn(cb, b));
  upp[t] = r;
  up[t] = a;
}

// vladd (variables.c:650) of two terms with its special cases
__device__ __forceinline__ double vladd_rn(double ca, double a, double cb, double b) {
  if (ca == 0.0 && cb == 0.0) return 0.0;
  if (ca == 0.0) return __dmul_rn(cb, b);
  if (cb == 0.0) return __dmul_rn(ca, a);
  return __dadd_rn(__dmul_rn(ca, a), __dmul_rn(cb, b));
}

// the start of the time interpolation of order o = 4, 5, 6 (evolve.c:
// 316-333): the vladd chain onto upp, then the time levels shifted back
// (:336-338) and the RK4 step's u_p copy, element by element
__global__ void ti_start_hist_kernel(Ptrs u, double *up, double *upp, double *p2, double *p3, double *p4, int o,
                                     long np, int nv) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= np * nv) return;
  const int v = (int)(t / np);
  const long i = t - (long)v * np;
  const double a = u.p[v][i], b = up[t], h2 = p2[t];
  const double h3 = o >= 5 ? p3[t] : 0.0, h4 = o >= 6 ? p4[t] : 0.0;
  double r;
  if (o == 4) {
    r = vladd_rn(15.0 / 16, a, -5.0 / 16, b);
    r = vladd_rn(1.0, r, 1.0 / 16, h2);
  } else if (o == 5) {
    r = vladd_rn(140.0 / 128, a, -70.0 / 128, b);
    r = vladd_rn(1.0, r, 28.0 / 128, h2);
    r = vladd_rn(1.0, r, -5.0 / 128, h3);
  } else {
    r = vladd_rn(315.0 / 256, a, -210.0 / 256, b);
    r = vladd_rn(1.0, r, 126.0 / 256, h2);
    r = vladd_rn(1.0, r, -45.0 / 256, h3);
    r = vladd_rn(1.0, r, 7.0 / 256, h4);
  }
  upp[t] = r;
  if (o >= 6) p4[t] = h3;
  if (o >= 5) p3[t] = h2;
  p2[t] = b;
  up[t] = a;
}

// upp = 1.0 upp + c u
__global__ void ti_finish_kernel(Ptrs u, double *upp, double c, long np, int nv) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= np * nv) return;
  const int v = (int)(t / np);
  const long i = t - (long)v * np;
  upp[t] = __dadd_rn(__dmul_rn(1.0, upp[t]), __dmul_rn(c, u.p[v][i]));
}

// move_overlap_nonparallel (move.c:603-640): the points of an old box that
// a new box of the same level also holds, copied for every variable; one
// thread per (point of the index range, variable)
__global__ void copy_range_kernel(Ptrs src, Ptrs dst, Box3 sb, Box3 db, int3 s0, int3 d0, int3 n, long npts) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= npts) return;
  const int v = blockIdx.y;
  const int i = (int)(t % n.x), j = (int)((t / n.x) % n.y), k = (int)(t / ((long)n.x * n.y));
  dst.p[v][at3(db, d0.x + i, d0.y + j, d0.z + k)] = src.p[v][at3(sb, s0.x + i, s0.y + j, s0.z + k)];
}

}  // namespace

// one fine box and the coarse box that holds it (BAM's box->pr): the
// restriction and prolongation geometry of the pair
struct FmrPair {
  int fbox, cbox;
  bool has_r, has_p;
  RGeom rg;
  PGeom pg;
  int nr, npro;
  int *d_plist;  // the prolonged points (offsets in the prolongation box), npro of them
};

struct nrgpu_fmr {
  int nl, nv;
  nrgpu_fmr_params p;
  nrgpu_level *L[kMaxLevels];
  std::vector<Box3> box[kMaxLevels];                   // the level's boxes
  std::vector<double> bx0[kMaxLevels];                 // their origins, 3 per box
  double dx[kMaxLevels][3];
  double dt[kMaxLevels];
  nrgpu_bssn_params bp[kMaxLevels];
  nrgpu_z4_params zp[kMaxLevels];
  std::vector<double> fp[kMaxLevels], fr[kMaxLevels];  // flagprolong, flagrestrict (level-wide)
  std::vector<FmrPair> pairs[kMaxLevels];              // per fine level, one per fine box
  double *up[kMaxLevels], *upp[kMaxLevels];  // u(n-1) copy and time interpolant
  // u(n-2), u(n-3), u(n-4) for time interpolation of orders 4-6 (u_p2, u_p3,
  // u_p4 of evolve.c:289-294), order_timeinterpolation - 3 of them
  double *hist[kMaxLevels][3];
  int iteration[kMaxLevels];
  // puncture tracking on the finest level (lmaxpunc = amr_lmax, grid.c:
  // 287-294): positions [3n] then the shift at the old positions [3n], and
  // the status of the last step per puncture
  int ntrack, track_fixz;
  double *d_track;
  int *d_tstatus;
  // the tracker per puncture (moving_puncture_track_method,
  // moving_punctures.c:123-180): the first next_ext punctures by the
  // extremum search on variable track_var, the rest by the shift integrator
  int track_method, track_var, track_max, track_fixz_ext;
  double track_minmove;
  // moving boxes: the caller's hook, called where the reference calls
  // move_box (main.c:428), and the levels whose pairs with their parent
  // wait to be set up again after a regrid of that parent
  nrgpu_fmr_move_fn move_fn;
  void *move_user;
  bool pair_stale[kMaxLevels];
  // graph of one coarse step for one set of state pointers
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  std::vector<double *> graph_u;
  // the graph is captured and replayed on the driver's own stream, ordered
  // after the caller's stream and before the caller's next work by events
  cudaStream_t gst;
  cudaEvent_t ev_in, ev_out;
};

namespace {

// coefficients_lagrange_N (lagrange.c:13-27) on unit spacing from 0
void lagrange(int n, double x, double *c) {
  for (int i = 0; i < n; i++) {
    double d = 1;
    for (int j = 0; j < n; j++)
      if (j != i) d *= (x - 0.0 - j * 1.0) / ((i - j) * 1.0);
    c[i] = d;
  }
}

// box.c:284-307
int parent_index(double cx0, double cdx, double fx0, double fdx, int fi) {
  return (int)(0.5 + (fx0 + fi * fdx - cx0) / cdx);
}
int point_index(double X0, double dX, double x0, double dx, int i) { return (int)((x0 + i * dx - X0) / dX); }

long hat(const Box3 &b, int i, int j, int k) { return b.off + i + (long)b.n[0] * (j + (long)b.n[1] * k); }

// the coarse box of level l-1 that holds every parent point of fine box fb
int parent_box(const nrgpu_fmr *F, int l, int fb) {
  const Box3 &f = F->box[l][fb];
  const double *fx0 = &F->bx0[l][3 * fb];
  for (int cb = 0; cb < (int)F->box[l - 1].size(); ++cb) {
    const Box3 &c = F->box[l - 1][cb];
    const double *cx0 = &F->bx0[l - 1][3 * cb];
    bool ok = true;
    for (int d = 0; d < 3 && ok; ++d) {
      const int lo = parent_index(cx0[d], F->dx[l - 1][d], fx0[d], F->dx[l][d], 0);
      const int hi = parent_index(cx0[d], F->dx[l - 1][d], fx0[d], F->dx[l][d], f.n[d] - 1);
      ok = lo >= 0 && hi < c.n[d];
    }
    if (ok) return cb;
  }
  return -1;
}

// setRPflags (flag.c:122-255) of one fine box and its parent box, then the
// bounding boxes of restrict_varlist_boxtobox_N and prolong_varlist_boxtobox_N
// (interpolate_boxtobox_N.c:870-1370, forallboxes(lf)).  With several fine
// boxes the reference sets each box's flagrestrict on a ghost parent of that
// box; here each pair's coarse flags are kept apart (cr) for its restriction
// box, and their union goes to the level's flagrestrict.
int setup_one_pair(nrgpu_fmr *F, int l, int fbi, std::vector<double> &cr) {
  FmrPair P;
  P.fbox = fbi;
  P.cbox = parent_box(F, l, fbi);
  if (P.cbox < 0) return nrgpu_set_error(NRGPU_ERR_ARG, "box %d of level %d does not nest in level %d", fbi, l, l - 1);
  const Box3 &f = F->box[l][fbi], &c = F->box[l - 1][P.cbox];
  const double *fx0 = &F->bx0[l][3 * fbi], *cx0 = &F->bx0[l - 1][3 * P.cbox];
  const int nbuf = F->p.nbuffer, b = F->p.order_RP / 2;
  const long npf = (long)f.n[0] * f.n[1] * f.n[2];
  std::vector<double> &fp = F->fp[l];
  std::fill(cr.begin(), cr.end(), 0.0);
  for (int k = 0; k < f.n[2]; k++)
    for (int j = 0; j < f.n[1]; j++)
      for (int i = 0; i < f.n[0]; i++) {
        const int idx[3] = {i, j, k};
        long m[3];
        for (int d = 0; d < 3; d++) {
          const double lo = fx0[d], hi = fx0[d] + (f.n[d] - 1) * F->dx[l][d];
          const double x = fx0[d] + idx[d] * F->dx[l][d];
          m[d] = npf;
          int n = (int)(1.5 + (x - lo) / F->dx[l][d]);
          if (n <= nbuf) m[d] = n;
          n = (int)(1.5 - (x - hi) / F->dx[l][d]);
          if (n <= nbuf) m[d] = n;
        }
        long ii = m[0] < m[1] ? m[0] : m[1];
        ii = ii < m[2] ? ii : m[2];
        fp[hat(f, i, j, k)] = ii < npf ? (double)ii : 0.0;
      }
  for (int pass = 0; pass < 2; pass++)
    for (int k = 0; k < f.n[2]; k++)
      for (int j = 0; j < f.n[1]; j++)
        for (int i = 0; i < f.n[0]; i++) {
          const int pi = parent_index(cx0[0], F->dx[l - 1][0], fx0[0], F->dx[l][0], i);
          const int pj = parent_index(cx0[1], F->dx[l - 1][1], fx0[1], F->dx[l][1], j);
          const int pk = parent_index(cx0[2], F->dx[l - 1][2], fx0[2], F->dx[l][2], k);
          const double p = fp[hat(f, i, j, k)];
          double &r = cr[hat(c, pi, pj, pk)];
          if (pass == 0 && p == 0) r = 3;
          if (pass == 1) {
            if (p >= 3) r = 2;
            else if (p == 2) r = 1;
          }
        }
  for (int k = 0; k < c.n[2]; k++)
    for (int j = 0; j < c.n[1]; j++)
      for (int i = 0; i < c.n[0]; i++)
        if (cr[hat(c, i, j, k)] != 0) F->fr[l - 1][hat(c, i, j, k)] = cr[hat(c, i, j, k)];
  // restriction box (the parent box's points with this pair's flag >= 3)
  int ic[6] = {1 << 30, -(1 << 30), 1 << 30, -(1 << 30), 1 << 30, -(1 << 30)};
  long n = 0;
  for (int k = 0; k < c.n[2]; k++)
    for (int j = 0; j < c.n[1]; j++)
      for (int i = 0; i < c.n[0]; i++)
        if (cr[hat(c, i, j, k)] >= 3) {
          const int idx[3] = {i, j, k};
          for (int d = 0; d < 3; d++) {
            ic[2 * d] = idx[d] < ic[2 * d] ? idx[d] : ic[2 * d];
            ic[2 * d + 1] = idx[d] > ic[2 * d + 1] ? idx[d] : ic[2 * d + 1];
          }
          n++;
        }
  P.has_r = n > 0;
  P.nr = 0;
  if (n) {
    RGeom &G = P.rg;
    memcpy(G.ic, ic, sizeof ic);
    for (int d = 0; d < 3; d++) {
      const int lo = point_index(fx0[d], F->dx[l][d], cx0[d], F->dx[l - 1][d], ic[2 * d]) - b + 1;
      const int hi = point_index(fx0[d], F->dx[l][d], cx0[d], F->dx[l - 1][d], ic[2 * d + 1]) + b;
      if (lo < 0 || hi >= f.n[d])
        return nrgpu_set_error(NRGPU_ERR_ARG, "restriction: boxes too small (level %d)", l);
      G.if0[d] = lo;
    }
    lagrange(F->p.order_RP, F->p.order_RP / 2.0 - 0.5, G.w);
    P.nr = (ic[1] - ic[0] + 1) * (ic[3] - ic[2] + 1) * (ic[5] - ic[4] + 1);
  }
  // prolongation boxes
  PGeom &Q = P.pg;
  int fb[6] = {1 << 30, -(1 << 30), 1 << 30, -(1 << 30), 1 << 30, -(1 << 30)};
  int f0[6] = {1 << 30, -(1 << 30), 1 << 30, -(1 << 30), 1 << 30, -(1 << 30)};
  n = 0;
  for (int k = 0; k < f.n[2]; k++)
    for (int j = 0; j < f.n[1]; j++)
      for (int i = 0; i < f.n[0]; i++) {
        const int idx[3] = {i, j, k};
        const double p = fp[hat(f, i, j, k)];
        int *bb = (p > 0 && nbuf >= p) ? fb : f0;
        if (bb == fb) n++;
        for (int d = 0; d < 3; d++) {
          bb[2 * d] = idx[d] < bb[2 * d] ? idx[d] : bb[2 * d];
          bb[2 * d + 1] = idx[d] > bb[2 * d + 1] ? idx[d] : bb[2 * d + 1];
        }
      }
  P.has_p = n > 0;
  P.npro = 0;
  P.d_plist = nullptr;
  if (n) {
    memcpy(Q.fb, fb, sizeof fb);
    memcpy(Q.f0, f0, sizeof f0);
    for (int d = 0; d < 3; d++) {
      const int lo = point_index(cx0[d], F->dx[l - 1][d], fx0[d], F->dx[l][d], fb[2 * d]) - b + 1;
      const int hi = point_index(cx0[d], F->dx[l - 1][d], fx0[d], F->dx[l][d], fb[2 * d + 1]) + b;
      if (lo < 0 || hi >= c.n[d])
        return nrgpu_set_error(NRGPU_ERR_ARG, "prolongation: boxes too small (level %d)", l);
      if ((fb[2 * d + 1] - fb[2 * d] + 1) % 2)
        return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "level %d is not made of whole parent cells", l);
      // the output pairs start on a lower child (fine point a quarter coarse
      // cell below its parent), as prolong_boxtobox_N assumes
      if (point_index(cx0[d], F->dx[l - 1][d], fx0[d], F->dx[l][d], fb[2 * d]) !=
          parent_index(cx0[d], F->dx[l - 1][d], fx0[d], F->dx[l][d], fb[2 * d]) - 1)
        return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "level %d is not aligned with its parent's cells", l);
      Q.cs[d] = lo;
    }
    lagrange(F->p.order_RP, F->p.order_RP / 2.0 - 0.25, Q.c1);
    lagrange(F->p.order_RP, F->p.order_RP / 2.0 - 0.75, Q.c2);
    // the points written: every point of the box but the pairs whose first
    // point lies in the inner box (prolong_boxtobox_N's test)
    std::vector<int> list;
    const int nI = fb[1] - fb[0] + 1, nJ = fb[3] - fb[2] + 1, nK = fb[5] - fb[4] + 1;
    for (int tk = 0; tk < nK; ++tk)
      for (int tj = 0; tj < nJ; ++tj)
        for (int ti = 0; ti < nI; ++ti) {
          const int i0 = fb[0] + 2 * (ti / 2), j = fb[2] + tj, k = fb[4] + tk;
          if (i0 >= f0[0] && i0 <= f0[1] && j >= f0[2] && j <= f0[3] && k >= f0[4] && k <= f0[5]) continue;
          list.push_back(ti + nI * (tj + nJ * tk));
        }
    P.npro = (int)list.size();
    P.d_plist = nullptr;
    if (P.npro) {
      NRGPU_CUDA_TRY(cudaMalloc(&P.d_plist, sizeof(int) * list.size()));
      NRGPU_CUDA_TRY(cudaMemcpy(P.d_plist, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice));
    }
    P.has_p = P.npro > 0;
  }
  F->pairs[l].push_back(P);
  return NRGPU_OK;
}

// the pairs of level l with level l-1
int setup_pair(nrgpu_fmr *F, int l) {
  F->fp[l].assign(F->L[l]->npoints, 0.0);
  F->fr[l - 1].assign(F->L[l - 1]->npoints, 0.0);
  for (FmrPair &P : F->pairs[l]) cudaFree(P.d_plist);
  F->pairs[l].clear();
  std::vector<double> cr(F->L[l - 1]->npoints, 0.0);
  for (int fb = 0; fb < (int)F->box[l].size(); ++fb) {
    const int e = setup_one_pair(F, l, fb, cr);
    if (e) return e;
  }
  return NRGPU_OK;
}

int fill(Ptrs *P, double *const *u, int nv) {
  for (int v = 0; v < kMaxVars; ++v) P->p[v] = v < nv ? u[v] : nullptr;
  for (int v = 0; v < nv; ++v)
    if (!u[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null variable pointer %d", v);
  return NRGPU_OK;
}

// restrict_prolong_varlist between level l and its parent (nbuffer 3):
// every pair restricted, then every pair prolonged (inject.c:63-100)
int restrict_prolong(nrgpu_fmr *F, int l, const Ptrs &uc, const Ptrs &uf, cudaStream_t st, int nvars = -1) {
  const int o = F->p.order_RP;
  const int nv = nvars < 0 ? F->nv : nvars;
  for (const FmrPair &P : F->pairs[l]) {
    if (!P.has_r) continue;
    const Box3 &cb = F->box[l - 1][P.cbox], &fb = F->box[l][P.fbox];
    const dim3 g((P.nr + 127) / 128, nv);
    if (o == 2) restrict_kernel<2><<<g, 128, 0, st>>>(uc, uf, cb, fb, P.rg, P.nr);
    else if (o == 4) restrict_kernel<4><<<g, 128, 0, st>>>(uc, uf, cb, fb, P.rg, P.nr);
    else restrict_kernel<6><<<g, 128, 0, st>>>(uc, uf, cb, fb, P.rg, P.nr);
    NRGPU_CUDA_TRY(cudaGetLastError());
  }
  for (const FmrPair &P : F->pairs[l]) {
    if (!P.has_p) continue;
    const Box3 &cb = F->box[l - 1][P.cbox], &fb = F->box[l][P.fbox];
    const dim3 g((P.npro + 127) / 128, nv);
    if (o == 2) prolong_kernel<2><<<g, 128, 0, st>>>(uc, uf, cb, fb, P.pg, P.d_plist, P.npro);
    else if (o == 4) prolong_kernel<4><<<g, 128, 0, st>>>(uc, uf, cb, fb, P.pg, P.d_plist, P.npro);
    else prolong_kernel<6><<<g, 128, 0, st>>>(uc, uf, cb, fb, P.pg, P.d_plist, P.npro);
    NRGPU_CUDA_TRY(cudaGetLastError());
  }
  return NRGPU_OK;
}

Ptrs upp_ptrs(nrgpu_fmr *F, int l) {
  Ptrs P;
  const long np = F->L[l]->npoints;
  for (int v = 0; v < kMaxVars; ++v) P.p[v] = v < F->nv ? F->upp[l] + (long)v * np : nullptr;
  return P;
}

// one step of level l: evolve() with the time interpolation of a level with
// a child around the RK4 stages, then the algebraic constraints
// first shift component in the evolved list: betax is variable 18 of BSSN
// (bssn.c:315-322) and 19 of Z4c (z4.c:234-242)
int shift_index(const nrgpu_fmr *F) { return F->p.system == NRGPU_SYSTEM_BSSN ? 18 : 19; }

// how many of the tracked punctures (the first ones) the extremum search
// moves: all for "ext", the first for "extint", none for "int"
int n_extremum(const nrgpu_fmr *F) {
  if (!F->ntrack) return 0;
  return F->track_method == 0 ? F->ntrack : (F->track_method == 2 ? 1 : 0);
}

int step_level(nrgpu_fmr *F, int l, double *const *u, cudaStream_t st) {
  const bool child = l < F->nl - 1;
  const long np = F->L[l]->npoints;
  Ptrs U;
  int e = fill(&U, u, F->nv);
  if (e) return e;
  const unsigned nb = (unsigned)((np * F->nv + 255) / 256);
  int o = 0;
  if (child) {
    o = F->iteration[l] + 2 > F->p.order_timeinterpolation ? F->p.order_timeinterpolation : F->iteration[l] + 2;
    if (o <= 3) {
      const double ca = o == 2 ? 0.5 : 0.75, cb = o == 2 ? 0.0 : -0.125;
      ti_start_kernel<<<nb, 256, 0, st>>>(U, F->up[l], F->upp[l], ca, cb, np, F->nv);
    } else {
      ti_start_hist_kernel<<<nb, 256, 0, st>>>(U, F->up[l], F->upp[l], F->hist[l][0], F->hist[l][1],
                                               F->hist[l][2], o, np, F->nv);
    }
    NRGPU_CUDA_TRY(cudaGetLastError());
  }
  // the integrator reads the shift one step earlier at the old positions
  // (betax_p in moving_punctures_integrate.c:62-64): taken before the step
  const int next = n_extremum(F), nint = F->ntrack - next;
  if (l == F->nl - 1 && nint > 0 &&
      (e = nrgpu_track_before_step(F->L[l], u + shift_index(F), F->p.order_RP, nint, F->d_track + 3 * next,
                                   F->d_track + 3 * F->ntrack + 3 * next, st)))
    return e;
  if (F->p.system == NRGPU_SYSTEM_BSSN) e = nrgpu_bssn_rk4_stages(F->L[l], u, F->dt[l], &F->bp[l], st);
  else e = nrgpu_z4_rk4_stages(F->L[l], u, F->dt[l], &F->zp[l], st);
  if (e) return e;
  if (child) {
    static const double cfin[7] = {0, 0, 1.0 / 2, 3. / 8, 5. / 16, 35. / 128, 63. / 256};
    ti_finish_kernel<<<nb, 256, 0, st>>>(U, F->upp[l], cfin[o], np, F->nv);
    NRGPU_CUDA_TRY(cudaGetLastError());
  }
  if (F->p.system == NRGPU_SYSTEM_BSSN) e = nrgpu_bssn_algcon(F->L[l], u, &F->bp[l], st);
  else e = nrgpu_z4_algcon(F->L[l], u, &F->zp[l], st);
  if (e) return e;
  F->iteration[l]++;
  return NRGPU_OK;
}

// advance_levelandsublevels (main.c:397-418)
int advance(nrgpu_fmr *F, int l, double *const *u, cudaStream_t st) {
  int e = step_level(F, l, u + l * F->nv, st);
  if (e) return e;
  if (l < F->nl - 1) {
    if ((e = advance(F, l + 1, u, st))) return e;
    if (l >= F->p.lbo && (e = advance(F, l + 1, u, st))) return e;
  }
  if (l > 0) {
    // parentaligned (inject.c:10-21): dequal of the level times
    const double tl = F->iteration[l] * F->dt[l], tp = F->iteration[l - 1] * F->dt[l - 1];
    const bool aligned = !(tl < tp - 1e-10 || tp < tl - 1e-10);
    Ptrs uc, uf;
    if ((e = fill(&uf, u + l * F->nv, F->nv))) return e;
    if (aligned) {
      if ((e = fill(&uc, u + (l - 1) * F->nv, F->nv))) return e;
    } else {
      uc = upp_ptrs(F, l - 1);
    }
    if ((e = restrict_prolong(F, l, uc, uf, st))) return e;
  }
  // ANALYZE of the level (main.c:420-423): track_puncture on the finest level
  if (l == F->nl - 1 && F->ntrack) {
    const int next = n_extremum(F), nint = F->ntrack - next;
    if (next && (e = nrgpu_track_extremum_on(F->L[l], u[l * F->nv + F->track_var], F->track_max, F->track_minmove,
                                             F->p.order_RP, F->track_fixz_ext, next, F->d_track, F->d_tstatus,
                                             st)))
      return e;
    if (nint && (e = nrgpu_track_after_step(F->L[l], u + l * F->nv + shift_index(F), F->dt[l], F->p.order_RP,
                                            F->track_fixz, nint, F->d_track + 3 * next,
                                            F->d_track + 3 * F->ntrack + 3 * next, F->d_tstatus + next, st)))
      return e;
  }
  // move_box(g, l + 1) (move.c:808-856): the levels above l may move once l
  // and its sublevels are done, unless l is aligned in time with its parent
  if (F->move_fn && l + 1 < F->nl) {
    bool go = l == 0;
    if (!go) {
      const double tl = F->iteration[l] * F->dt[l], tp = F->iteration[l - 1] * F->dt[l - 1];
      go = tl < tp - 1e-10;
    }
    if (go) {
      const int r = F->move_fn(F->move_user, F, l + 1, (void *)st);
      if (r) return r < 0 ? r : nrgpu_set_error(NRGPU_ERR_ARG, "move hook of level %d returned %d", l + 1, r);
      for (int q = 1; q < F->nl; ++q)
        if (F->pair_stale[q])
          return nrgpu_set_error(NRGPU_ERR_ARG, "level %d was not set up again after its parent moved", q);
    }
  }
  return NRGPU_OK;
}

// ---- moving boxes: one level to a new set of boxes ---------------------------
// move_overlap (move.c:712-800) for every time level of the level: the new
// points are prolonged from the parent (prolong_varlist with flag -3 or -1,
// interpolate_boxtobox_N.c:870-1010, order_RP), then every point that an old
// box also holds is copied from it.  The parent's state is the new one when
// the parent moved first (levels move coarsest first, move.c:874-983).
struct Buffers {
  Ptrs p;
  bool ok;
};

// the state of level p during a regrid of levels lmin..: the new buffers if
// p moved in this regrid, else the current ones
double *const *unew_or_u(const nrgpu_fmr *F, int lmin, int p, double *const *u, double *const *unew,
                         const nrgpu_level_desc *desc) {
  if (p >= lmin && desc[p - lmin].nboxes > 0) return unew + (long)(p - lmin) * F->nv;
  return u + (long)p * F->nv;
}

Buffers level_set(double *base, long np, int nv) {
  Buffers b;
  b.ok = base != nullptr;
  for (int v = 0; v < kMaxVars; ++v) b.p.p[v] = base && v < nv ? base + (long)v * np : nullptr;
  return b;
}

// index range of the overlap of two boxes of one level (box_overlap_range,
// move.c:518-566): false when empty
bool overlap_range(const Box3 &a, const double *ax0, const Box3 &b, const double *bx0, const double *dx, int *ia,
                   int *ib) {
  for (int d = 0; d < 3; ++d) {
    const double alo = ax0[d], ahi = ax0[d] + (a.n[d] - 1) * dx[d];
    const double blo = bx0[d], bhi = bx0[d] + (b.n[d] - 1) * dx[d];
    const double lo = alo > blo ? alo : blo, hi = ahi < bhi ? ahi : bhi;
    if (hi < lo - 1e-10 * dx[d]) return false;
    ia[2 * d] = (int)floor((lo - alo + 1e-10) / dx[d]);
    ia[2 * d + 1] = (int)floor((hi - alo + 1e-10) / dx[d]);
    ib[2 * d] = (int)floor((lo - blo + 1e-10) / dx[d]);
    ib[2 * d + 1] = (int)floor((hi - blo + 1e-10) / dx[d]);
  }
  return true;
}

template <int N>
void launch_prolong(const Ptrs &uc, const Ptrs &uf, const Box3 &cb, const Box3 &fb, const PGeom &G, const int *list,
                    int n, int nv, cudaStream_t st) {
  prolong_kernel<N><<<dim3((n + 127) / 128, nv), 128, 0, st>>>(uc, uf, cb, fb, G, list, n);
}

int regrid_level(nrgpu_fmr *F, int m, const nrgpu_level_desc &d, double *const *uold, double *const *unew,
                 double *const *uparent, cudaStream_t st) {
  if (d.symmetry) return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "level %d: symmetry grids", m);
  if (d.dx != F->dx[m][0] || d.dy != F->dx[m][1] || d.dz != F->dx[m][2])
    return nrgpu_set_error(NRGPU_ERR_ARG, "level %d: a move keeps the grid spacing", m);
  for (int v = 0; v < F->nv; ++v)
    if (!unew[v] || !uold[v] || !uparent[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "level %d: null state pointer", m);
  const int nv = F->nv;
  const bool parent_role = m < F->nl - 1;
  const int nh = F->p.order_timeinterpolation > 3 ? F->p.order_timeinterpolation - 3 : 0;
  // the old level
  std::vector<Box3> obox = F->box[m];
  std::vector<double> obx0 = F->bx0[m];
  nrgpu_level *oL = F->L[m];
  const long onp = oL->npoints;
  // the new level
  nrgpu_level *nL = nullptr;
  int e = nrgpu_level_create(&d, &nL);
  if (e) return e;
  double *scr;
  if ((e = nrgpu_level_scratch(nL, &scr))) {
    nrgpu_level_destroy(nL);
    return e;
  }
  int blk[3];
  if (!nrgpu_level_get_block(oL, blk)) nrgpu_level_block(nL, blk[0], blk[1], blk[2]);
  nrgpu_level_tile(nL, nrgpu_level_tile(oL, -1));
  nrgpu_level_queue(nL, nrgpu_level_queue(oL, -1));
  const long nnp = d.npoints;
  // time levels of a parent level: u_p, u_pp and u_p2..u_p4 (evolve.c:
  // 250-258), moved with u (move.c:930-939)
  double *nup = nullptr, *nupp = nullptr, *nhist[3] = {nullptr, nullptr, nullptr};
  auto fail = [&](int err) {
    cudaFree(nup);
    cudaFree(nupp);
    for (int h = 0; h < 3; ++h) cudaFree(nhist[h]);
    nrgpu_level_destroy(nL);
    F->box[m] = obox;
    F->bx0[m] = obx0;
    return err;
  };
  if (parent_role) {
    const size_t bytes = sizeof(double) * nv * (size_t)nnp;
    bool ok = cudaMalloc(&nup, bytes) == cudaSuccess && cudaMalloc(&nupp, bytes) == cudaSuccess;
    for (int h = 0; h < nh && ok; ++h) ok = cudaMalloc(&nhist[h], bytes) == cudaSuccess;
    if (!ok) {
      cudaGetLastError();
      return fail(nrgpu_set_error(NRGPU_ERR_NOMEM, "time levels of the moved level %d", m));
    }
  }
  F->box[m].clear();
  F->bx0[m].clear();
  for (int b = 0; b < d.nboxes; ++b) {
    F->box[m].push_back(Box3{{d.box[b].m, d.box[b].n, d.box[b].o}, (long)d.box[b].noffset});
    F->bx0[m].push_back(d.box[b].x0);
    F->bx0[m].push_back(d.box[b].y0);
    F->bx0[m].push_back(d.box[b].z0);
  }
  // the buffer sets: (parent source, old, new)
  const long pnp = F->L[m - 1]->npoints;
  struct Set {
    Buffers par, old, neu;
  };
  std::vector<Set> sets;
  {
    Set u;
    for (int v = 0; v < kMaxVars; ++v) {
      u.par.p.p[v] = v < nv ? uparent[v] : nullptr;
      u.old.p.p[v] = v < nv ? uold[v] : nullptr;
      u.neu.p.p[v] = v < nv ? unew[v] : nullptr;
    }
    u.par.ok = u.old.ok = u.neu.ok = true;
    sets.push_back(u);
  }
  if (parent_role) {
    sets.push_back(Set{level_set(F->up[m - 1], pnp, nv), level_set(F->up[m], onp, nv), level_set(nup, nnp, nv)});
    sets.push_back(Set{level_set(F->upp[m - 1], pnp, nv), level_set(F->upp[m], onp, nv), level_set(nupp, nnp, nv)});
    for (int h = 0; h < nh; ++h)
      sets.push_back(Set{level_set(F->hist[m - 1][h], pnp, nv), level_set(F->hist[m][h], onp, nv),
                         level_set(nhist[h], nnp, nv)});
  }
  const int o = F->p.order_RP, b = o / 2;
  std::vector<int *> lists;
  for (int j = 0; j < d.nboxes && !e; ++j) {
    const Box3 &f = F->box[m][j];
    const double *fx0 = &F->bx0[m][3 * j];
    // the points an old box holds are copied, the others prolonged
    const long nfp = (long)f.n[0] * f.n[1] * f.n[2];
    std::vector<char> held(nfp, 0);
    for (int i = 0; i < (int)obox.size(); ++i) {
      int io[6], in[6];
      if (!overlap_range(obox[i], &obx0[3 * i], f, fx0, F->dx[m], io, in)) continue;
      for (int k = in[4]; k <= in[5]; ++k)
        for (int jj = in[2]; jj <= in[3]; ++jj)
          for (int ii = in[0]; ii <= in[1]; ++ii) held[ii + (long)f.n[0] * (jj + (long)f.n[1] * k)] = 1;
    }
    std::vector<int> list;
    for (long q = 0; q < nfp; ++q)
      if (!held[q]) list.push_back((int)q);
    if (list.empty()) continue;
    const int cbi = parent_box(F, m, j);
    if (cbi < 0) {
      e = nrgpu_set_error(NRGPU_ERR_ARG, "moved box %d of level %d does not nest in level %d", j, m, m - 1);
      break;
    }
    const Box3 &c = F->box[m - 1][cbi];
    const double *cx0 = &F->bx0[m - 1][3 * cbi];
    PGeom G;
    for (int dd = 0; dd < 3; ++dd) {
      G.fb[2 * dd] = 0;
      G.fb[2 * dd + 1] = f.n[dd] - 1;
      G.f0[2 * dd] = 1 << 30;
      G.f0[2 * dd + 1] = -(1 << 30);
      const int lo = point_index(cx0[dd], F->dx[m - 1][dd], fx0[dd], F->dx[m][dd], 0) - b + 1;
      const int hi = point_index(cx0[dd], F->dx[m - 1][dd], fx0[dd], F->dx[m][dd], f.n[dd] - 1) + b;
      if (lo < 0 || hi >= c.n[dd]) e = nrgpu_set_error(NRGPU_ERR_ARG, "moved level %d: boxes too small", m);
      else if (f.n[dd] % 2 || point_index(cx0[dd], F->dx[m - 1][dd], fx0[dd], F->dx[m][dd], 0) !=
                                  parent_index(cx0[dd], F->dx[m - 1][dd], fx0[dd], F->dx[m][dd], 0) - 1)
        e = nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "moved level %d is not aligned with its parent's cells", m);
      G.cs[dd] = lo;
    }
    if (e) break;
    lagrange(o, o / 2.0 - 0.25, G.c1);
    lagrange(o, o / 2.0 - 0.75, G.c2);
    int *dl = nullptr;
    if (cudaMalloc(&dl, sizeof(int) * list.size()) != cudaSuccess ||
        cudaMemcpy(dl, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(dl);
      e = nrgpu_set_error(NRGPU_ERR_NOMEM, "prolongation list of the moved level %d", m);
      break;
    }
    lists.push_back(dl);
    for (const Set &S : sets) {
      if (o == 2) launch_prolong<2>(S.par.p, S.neu.p, c, f, G, dl, (int)list.size(), nv, st);
      else if (o == 4) launch_prolong<4>(S.par.p, S.neu.p, c, f, G, dl, (int)list.size(), nv, st);
      else launch_prolong<6>(S.par.p, S.neu.p, c, f, G, dl, (int)list.size(), nv, st);
    }
    if (cudaGetLastError() != cudaSuccess) e = nrgpu_set_error(NRGPU_ERR_CUDA, "prolongation of the moved level %d", m);
  }
  // copy what the old boxes hold (all pairs of old and new boxes)
  for (int j = 0; j < d.nboxes && !e; ++j)
    for (int i = 0; i < (int)obox.size() && !e; ++i) {
      int io[6], in[6];
      if (!overlap_range(obox[i], &obx0[3 * i], F->box[m][j], &F->bx0[m][3 * j], F->dx[m], io, in)) continue;
      const int3 s0 = make_int3(io[0], io[2], io[4]), d0 = make_int3(in[0], in[2], in[4]);
      const int3 n = make_int3(io[1] - io[0] + 1, io[3] - io[2] + 1, io[5] - io[4] + 1);
      const long npts = (long)n.x * n.y * n.z;
      for (const Set &S : sets)
        copy_range_kernel<<<dim3((unsigned)((npts + 255) / 256), nv), 256, 0, st>>>(S.old.p, S.neu.p, obox[i],
                                                                                      F->box[m][j], s0, d0, n, npts);
      if (cudaGetLastError() != cudaSuccess) e = nrgpu_set_error(NRGPU_ERR_CUDA, "copy into the moved level %d", m);
    }
  // the old buffers are read above: the stream finishes before they go
  if (!e && cudaStreamSynchronize(st) != cudaSuccess) e = nrgpu_set_error(NRGPU_ERR_CUDA, "regrid of level %d", m);
  for (int *dl : lists) cudaFree(dl);
  if (e) return fail(e);
  nrgpu_level_destroy(oL);
  F->L[m] = nL;
  if (parent_role) {
    cudaFree(F->up[m]);
    cudaFree(F->upp[m]);
    F->up[m] = nup;
    F->upp[m] = nupp;
    for (int h = 0; h < 3; ++h) {
      cudaFree(F->hist[m][h]);
      F->hist[m][h] = nhist[h];
    }
  }
  return NRGPU_OK;
}

}  // namespace

extern "C" int nrgpu_fmr_params_default(nrgpu_fmr_params *p) {
  if (!p) return nrgpu_set_error(NRGPU_ERR_ARG, "null params");
  p->system = NRGPU_SYSTEM_Z4C;
  p->lbo = 0;
  p->order_timeinterpolation = 3;
  p->order_RP = 4;
  p->nbuffer = 3;
  p->use_graph = 1;
  p->autotune = 1;
  return NRGPU_OK;
}

extern "C" int nrgpu_fmr_destroy(nrgpu_fmr *F) {
  if (!F) return NRGPU_OK;
  if (F->exec) cudaGraphExecDestroy(F->exec);
  if (F->graph) cudaGraphDestroy(F->graph);
  if (F->gst) cudaStreamDestroy(F->gst);
  if (F->ev_in) cudaEventDestroy(F->ev_in);
  if (F->ev_out) cudaEventDestroy(F->ev_out);
  for (int l = 0; l < F->nl; ++l) {
    for (FmrPair &P : F->pairs[l]) cudaFree(P.d_plist);
    cudaFree(F->up[l]);
    cudaFree(F->upp[l]);
    for (int h = 0; h < 3; ++h) cudaFree(F->hist[l][h]);
    nrgpu_level_destroy(F->L[l]);
  }
  cudaFree(F->d_track);
  cudaFree(F->d_tstatus);
  delete F;
  return NRGPU_OK;
}

extern "C" int nrgpu_fmr_create(int nl, const nrgpu_level_desc *levels, const double *dt, const void *sysparams,
                                const nrgpu_fmr_params *p, nrgpu_fmr **out) {
  if (!levels || !dt || !sysparams || !p || !out || nl < 1 || nl > kMaxLevels)
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad arguments (1 <= nlevels <= %d)", kMaxLevels);
  if (p->system != NRGPU_SYSTEM_BSSN && p->system != NRGPU_SYSTEM_Z4C)
    return nrgpu_set_error(NRGPU_ERR_ARG, "system %d", p->system);
  if (p->order_timeinterpolation < 2 || p->order_timeinterpolation > 6)
    return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "order_timeinterpolation %d (2 to 6)", p->order_timeinterpolation);
  if (p->order_RP != 2 && p->order_RP != 4 && p->order_RP != 6)
    return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "order_RP %d (2, 4 or 6)", p->order_RP);
  if (p->nbuffer < 1 || p->lbo < 0) return nrgpu_set_error(NRGPU_ERR_ARG, "nbuffer %d, lbo %d", p->nbuffer, p->lbo);
  nrgpu_fmr *F = new nrgpu_fmr();
  memset(F->L, 0, sizeof F->L);
  memset(F->up, 0, sizeof F->up);
  memset(F->upp, 0, sizeof F->upp);
  memset(F->hist, 0, sizeof F->hist);
  memset(F->iteration, 0, sizeof F->iteration);
  F->graph = nullptr;
  F->exec = nullptr;
  F->gst = nullptr;
  F->ev_in = F->ev_out = nullptr;
  F->ntrack = F->track_fixz = 0;
  F->track_method = 1;  // the shift integrator ("int")
  F->move_fn = nullptr;
  F->move_user = nullptr;
  memset(F->pair_stale, 0, sizeof F->pair_stale);
  F->d_track = nullptr;
  F->d_tstatus = nullptr;
  F->nl = nl;
  F->p = *p;
  F->nv = p->system == NRGPU_SYSTEM_BSSN ? NRGPU_NV : NRGPU_Z4_NVARS;
  int e = NRGPU_OK;
  for (int l = 0; l < nl && !e; ++l) {
    const nrgpu_level_desc &d = levels[l];
    if (d.nboxes < 1 || !d.box) e = nrgpu_set_error(NRGPU_ERR_ARG, "level %d: no boxes", l);
    else if (d.symmetry)
      e = nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "level %d: symmetry grids in the refinement driver", l);
    else if (dt[l] <= 0) e = nrgpu_set_error(NRGPU_ERR_ARG, "level %d: dt %g", l, dt[l]);
    if (e) break;
    F->box[l].clear();
    F->bx0[l].clear();
    for (int b = 0; b < d.nboxes; ++b) {
      F->box[l].push_back(Box3{{d.box[b].m, d.box[b].n, d.box[b].o}, (long)d.box[b].noffset});
      F->bx0[l].push_back(d.box[b].x0);
      F->bx0[l].push_back(d.box[b].y0);
      F->bx0[l].push_back(d.box[b].z0);
    }
    F->dx[l][0] = d.dx; F->dx[l][1] = d.dy; F->dx[l][2] = d.dz;
    F->dt[l] = dt[l];
    if (p->system == NRGPU_SYSTEM_BSSN) F->bp[l] = ((const nrgpu_bssn_params *)sysparams)[l];
    else F->zp[l] = ((const nrgpu_z4_params *)sysparams)[l];
    if ((e = nrgpu_level_create(&d, &F->L[l]))) break;
    double *scr;
    if ((e = nrgpu_level_scratch(F->L[l], &scr))) break;  // no allocation later, inside a graph capture
    if (l > 0 && (e = setup_pair(F, l))) break;
    if (p->autotune == 2) nrgpu_level_tile(F->L[l], 1);
    if (p->autotune == 1 &&
        (e = nrgpu_level_autotune(F->L[l], p->system,
                                  p->system == NRGPU_SYSTEM_BSSN ? (const void *)&F->bp[l] : (const void *)&F->zp[l],
                                  nullptr, nullptr)))
      break;
    if (l < nl - 1) {
      const size_t bytes = sizeof(double) * F->nv * (size_t)d.npoints;
      if (cudaMalloc(&F->up[l], bytes) != cudaSuccess || cudaMalloc(&F->upp[l], bytes) != cudaSuccess) {
        cudaGetLastError();
        e = nrgpu_set_error(NRGPU_ERR_NOMEM, "time interpolation buffers of level %d", l);
      } else if (cudaMemset(F->up[l], 0, bytes) != cudaSuccess || cudaMemset(F->upp[l], 0, bytes) != cudaSuccess) {
        e = nrgpu_set_error(NRGPU_ERR_CUDA, "memset");
      }
      for (int h = 0; h < p->order_timeinterpolation - 3 && !e; ++h) {
        if (cudaMalloc(&F->hist[l][h], bytes) != cudaSuccess) {
          cudaGetLastError();
          F->hist[l][h] = nullptr;
          e = nrgpu_set_error(NRGPU_ERR_NOMEM, "time levels of level %d", l);
        } else if (cudaMemset(F->hist[l][h], 0, bytes) != cudaSuccess) {
          e = nrgpu_set_error(NRGPU_ERR_CUDA, "memset");
        }
      }
    }
  }
  if (!e && (cudaStreamCreateWithFlags(&F->gst, cudaStreamNonBlocking) != cudaSuccess ||
             cudaEventCreateWithFlags(&F->ev_in, cudaEventDisableTiming) != cudaSuccess ||
             cudaEventCreateWithFlags(&F->ev_out, cudaEventDisableTiming) != cudaSuccess))
    e = nrgpu_set_error(NRGPU_ERR_CUDA, "stream/event creation");
  if (e) {
    nrgpu_fmr_destroy(F);
    return e;
  }
  *out = F;
  return NRGPU_OK;
}

extern "C" int nrgpu_fmr_flags(nrgpu_fmr *F, int l, double *flagprolong, double *flagrestrict) {
  if (!F || l < 0 || l >= F->nl) return nrgpu_set_error(NRGPU_ERR_ARG, "bad level");
  const size_t np = (size_t)F->L[l]->npoints;
  if (flagprolong) {
    if (l == 0) memset(flagprolong, 0, sizeof(double) * np);
    else memcpy(flagprolong, F->fp[l].data(), sizeof(double) * np);
  }
  if (flagrestrict) {
    if (l == F->nl - 1) memset(flagrestrict, 0, sizeof(double) * np);
    else memcpy(flagrestrict, F->fr[l].data(), sizeof(double) * np);
  }
  return NRGPU_OK;
}

extern "C" int nrgpu_fmr_restrict_prolong(nrgpu_fmr *F, int lfine, double *const *uc, double *const *uf,
                                          void *stream) {
  if (!F || !uc || !uf || lfine < 1 || lfine >= F->nl) return nrgpu_set_error(NRGPU_ERR_ARG, "bad arguments");
  Ptrs C, P;
  int e;
  if ((e = fill(&C, uc, F->nv)) || (e = fill(&P, uf, F->nv))) return e;
  return restrict_prolong(F, lfine, C, P, (cudaStream_t)stream);
}

extern "C" int nrgpu_fmr_restrict_prolong_vars(nrgpu_fmr *F, int lfine, int nvars, double *const *uc,
                                               double *const *uf, void *stream) {
  if (!F || !uc || !uf || lfine < 1 || lfine >= F->nl || nvars < 1 || nvars > kMaxVars)
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad arguments (1 <= nvars <= %d)", kMaxVars);
  Ptrs C, P;
  for (int v = 0; v < kMaxVars; ++v) {
    C.p[v] = v < nvars ? uc[v] : nullptr;
    P.p[v] = v < nvars ? uf[v] : nullptr;
  }
  for (int v = 0; v < nvars; ++v)
    if (!uc[v] || !uf[v]) return nrgpu_set_error(NRGPU_ERR_ARG, "null variable pointer %d", v);
  return restrict_prolong(F, lfine, C, P, (cudaStream_t)stream, nvars);
}

extern "C" int nrgpu_fmr_block(nrgpu_fmr *F, int l, int *block) {
  if (!F || l < 0 || l >= F->nl) return nrgpu_set_error(NRGPU_ERR_ARG, "no level %d", l);
  return nrgpu_level_get_block(F->L[l], block);
}

extern "C" int nrgpu_fmr_iteration(nrgpu_fmr *F, int l) {
  if (!F || l < 0 || l >= F->nl) return -1;
  return F->iteration[l];
}

extern "C" int nrgpu_fmr_advance(nrgpu_fmr *F, double *const *u, int nsteps, void *stream) {
  if (!F || !u || nsteps < 0) return nrgpu_set_error(NRGPU_ERR_ARG, "bad arguments");
  const cudaStream_t st = (cudaStream_t)stream;
  const int ntot = F->nl * F->nv;
  for (int s = 0; s < nsteps; ++s) {
    // the launch sequence of a coarse step is the same for every step once
    // no level is in its first iteration (time interpolation order) and
    // the state pointers are the same
    bool steady = true;
    const int full = F->p.order_timeinterpolation - 2 > 1 ? F->p.order_timeinterpolation - 2 : 1;
    for (int l = 0; l < F->nl; ++l) steady = steady && F->iteration[l] >= full;
    if (!F->p.use_graph || !steady || F->move_fn) {
      int e = advance(F, 0, u, st);
      if (e) return e;
      continue;
    }
    if (!F->exec || F->graph_u.size() != (size_t)ntot || memcmp(F->graph_u.data(), u, sizeof(double *) * ntot)) {
      if (F->exec) cudaGraphExecDestroy(F->exec);
      if (F->graph) cudaGraphDestroy(F->graph);
      F->exec = nullptr;
      F->graph = nullptr;
      int it[kMaxLevels];
      memcpy(it, F->iteration, sizeof it);
      NRGPU_CUDA_TRY(cudaStreamBeginCapture(F->gst, cudaStreamCaptureModeThreadLocal));
      int e = advance(F, 0, u, F->gst);
      cudaGraph_t g = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(F->gst, &g);
      memcpy(F->iteration, it, sizeof it);  // the capture ran nothing
      if (e) {
        if (g) cudaGraphDestroy(g);
        return e;
      }
      if (ce != cudaSuccess) return nrgpu_set_error(NRGPU_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
      F->graph = g;
      NRGPU_CUDA_TRY(cudaGraphInstantiate(&F->exec, g, 0));
      F->graph_u.assign(u, u + ntot);
    }
    NRGPU_CUDA_TRY(cudaEventRecord(F->ev_in, st));
    NRGPU_CUDA_TRY(cudaStreamWaitEvent(F->gst, F->ev_in, 0));
    NRGPU_CUDA_TRY(cudaGraphLaunch(F->exec, F->gst));
    NRGPU_CUDA_TRY(cudaEventRecord(F->ev_out, F->gst));
    NRGPU_CUDA_TRY(cudaStreamWaitEvent(st, F->ev_out, 0));
    // the iteration counters advance as the recursion would have
    for (int l = 0; l < F->nl; ++l) {
      int times = 1;
      for (int q = 1; q <= l; ++q) times *= (q - 1 >= F->p.lbo) ? 2 : 1;
      F->iteration[l] += times;
    }
  }
  return NRGPU_OK;
}

extern "C" int nrgpu_fmr_set_move(nrgpu_fmr *F, nrgpu_fmr_move_fn fn, void *user) {
  if (!F) return nrgpu_set_error(NRGPU_ERR_ARG, "null hierarchy");
  F->move_fn = fn;
  F->move_user = user;
  return NRGPU_OK;
}

extern "C" int nrgpu_fmr_regrid(nrgpu_fmr *F, int lmin, int nlev, const nrgpu_level_desc *desc, double *const *u,
                                double *const *unew, void *stream) {
  if (!F || !desc || !u || !unew || lmin < 1 || nlev < 1 || lmin + nlev > F->nl)
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad regrid arguments (levels 1 to %d)", F ? F->nl - 1 : 0);
  const cudaStream_t st = (cudaStream_t)stream;
  bool moved = false;
  for (int i = 0; i < nlev; ++i) {
    const int m = lmin + i;
    int e;
    if (desc[i].nboxes > 0) {
      if ((e = regrid_level(F, m, desc[i], u + (long)m * F->nv, unew + (long)i * F->nv, unew_or_u(F, lmin, m - 1, u,
                                                                                                  unew, desc),
                            st)))
        return e;
      F->pair_stale[m] = true;
      if (m + 1 < F->nl) F->pair_stale[m + 1] = true;
      moved = true;
    }
    if (F->pair_stale[m]) {
      if ((e = setup_pair(F, m))) return e;
      F->pair_stale[m] = false;
    }
  }
  // a child of the last level given keeps its boxes but gets new pairs
  const int c = lmin + nlev;
  if (c < F->nl && F->pair_stale[c]) {
    const int e = setup_pair(F, c);
    if (e) return e;
    F->pair_stale[c] = false;
  }
  if (moved) {
    if (F->exec) cudaGraphExecDestroy(F->exec);
    if (F->graph) cudaGraphDestroy(F->graph);
    F->exec = nullptr;
    F->graph = nullptr;
    F->graph_u.clear();
  }
  return NRGPU_OK;
}

// ---- checkpoint of the hierarchy's own state (no counterpart) -------------------
// The reference's checkpoint (checkpoint.c:14-165) writes the level variables;
// here the caller owns those, and the hierarchy owns the iteration counters,
// and for every level with a child the previous step's copy and the time
// interpolant.  Layout: a header (magic, version, levels, variables, the
// levels' point counts), the counters, then per parent level u(n-1) and upp.
namespace {
constexpr uint32_t kCkptMagic = 0x4652474e;  // "NGRF"
// 2: the tracked positions at the end; 3: the older time levels of
// interpolation orders 4-6 after each level's u(n-1) and interpolant
uint32_t ckpt_version(const nrgpu_fmr *F) { return F->p.order_timeinterpolation > 3 ? 3 : 2; }
int ckpt_nbuf(const nrgpu_fmr *F) { return 2 + (F->p.order_timeinterpolation > 3 ? F->p.order_timeinterpolation - 3 : 0); }
size_t ckpt_bytes(const nrgpu_fmr *F) {
  size_t b = sizeof(uint32_t) * 4 + sizeof(long) * F->nl + sizeof(int) * F->nl;
  for (int l = 0; l < F->nl - 1; ++l) b += ckpt_nbuf(F) * sizeof(double) * F->nv * (size_t)F->L[l]->npoints;
  b += sizeof(int) + sizeof(double) * 3 * F->ntrack;
  return b;
}
}  // namespace

extern "C" int nrgpu_fmr_state_size(nrgpu_fmr *F, size_t *bytes) {
  if (!F || !bytes) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  *bytes = ckpt_bytes(F);
  return NRGPU_OK;
}

extern "C" int nrgpu_fmr_save(nrgpu_fmr *F, void *host, size_t bytes) {
  if (!F || !host || bytes < ckpt_bytes(F)) return nrgpu_set_error(NRGPU_ERR_ARG, "buffer of %zu bytes", bytes);
  NRGPU_CUDA_TRY(cudaDeviceSynchronize());
  char *c = (char *)host;
  const uint32_t h[4] = {kCkptMagic, ckpt_version(F), (uint32_t)F->nl, (uint32_t)F->nv};
  memcpy(c, h, sizeof h);
  c += sizeof h;
  for (int l = 0; l < F->nl; ++l, c += sizeof(long)) {
    const long np = F->L[l]->npoints;
    memcpy(c, &np, sizeof np);
  }
  memcpy(c, F->iteration, sizeof(int) * F->nl);
  c += sizeof(int) * F->nl;
  for (int l = 0; l < F->nl - 1; ++l) {
    const size_t b = sizeof(double) * F->nv * (size_t)F->L[l]->npoints;
    NRGPU_CUDA_TRY(cudaMemcpy(c, F->up[l], b, cudaMemcpyDeviceToHost));
    c += b;
    NRGPU_CUDA_TRY(cudaMemcpy(c, F->upp[l], b, cudaMemcpyDeviceToHost));
    c += b;
    for (int q = 0; q < ckpt_nbuf(F) - 2; ++q, c += b)
      NRGPU_CUDA_TRY(cudaMemcpy(c, F->hist[l][q], b, cudaMemcpyDeviceToHost));
  }
  memcpy(c, &F->ntrack, sizeof(int));
  c += sizeof(int);
  if (F->ntrack) NRGPU_CUDA_TRY(cudaMemcpy(c, F->d_track, sizeof(double) * 3 * F->ntrack, cudaMemcpyDeviceToHost));
  return NRGPU_OK;
}

extern "C" int nrgpu_fmr_load(nrgpu_fmr *F, const void *host, size_t bytes) {
  if (!F || !host || bytes < ckpt_bytes(F)) return nrgpu_set_error(NRGPU_ERR_ARG, "buffer of %zu bytes", bytes);
  const char *c = (const char *)host;
  uint32_t h[4];
  memcpy(h, c, sizeof h);
  c += sizeof h;
  if (h[0] != kCkptMagic || h[1] != ckpt_version(F) || h[2] != (uint32_t)F->nl || h[3] != (uint32_t)F->nv)
    return nrgpu_set_error(NRGPU_ERR_ARG, "checkpoint of another hierarchy (levels %u, variables %u)", h[2], h[3]);
  for (int l = 0; l < F->nl; ++l, c += sizeof(long)) {
    long np;
    memcpy(&np, c, sizeof np);
    if (np != F->L[l]->npoints) return nrgpu_set_error(NRGPU_ERR_ARG, "checkpoint level %d: %ld points", l, np);
  }
  int it[kMaxLevels];
  memcpy(it, c, sizeof(int) * F->nl);
  c += sizeof(int) * F->nl;
  {
    size_t off = 0;
    for (int l = 0; l < F->nl - 1; ++l) off += ckpt_nbuf(F) * sizeof(double) * F->nv * (size_t)F->L[l]->npoints;
    int nt;
    memcpy(&nt, c + off, sizeof nt);
    if (nt != F->ntrack)
      return nrgpu_set_error(NRGPU_ERR_ARG, "checkpoint tracks %d punctures, the hierarchy %d", nt, F->ntrack);
  }
  NRGPU_CUDA_TRY(cudaDeviceSynchronize());
  for (int l = 0; l < F->nl - 1; ++l) {
    const size_t b = sizeof(double) * F->nv * (size_t)F->L[l]->npoints;
    NRGPU_CUDA_TRY(cudaMemcpy(F->up[l], c, b, cudaMemcpyHostToDevice));
    c += b;
    NRGPU_CUDA_TRY(cudaMemcpy(F->upp[l], c, b, cudaMemcpyHostToDevice));
    c += b;
    for (int q = 0; q < ckpt_nbuf(F) - 2; ++q, c += b)
      NRGPU_CUDA_TRY(cudaMemcpy(F->hist[l][q], c, b, cudaMemcpyHostToDevice));
  }
  c += sizeof(int);
  if (F->ntrack) NRGPU_CUDA_TRY(cudaMemcpy(F->d_track, c, sizeof(double) * 3 * F->ntrack, cudaMemcpyHostToDevice));
  memcpy(F->iteration, it, sizeof(int) * F->nl);
  return NRGPU_OK;
}

// ---- puncture tracking ----------------------------------------------------------
namespace {
// the captured coarse step changes: capture it again at the next advance
void drop_graph(nrgpu_fmr *F) {
  if (F->exec) cudaGraphExecDestroy(F->exec);
  if (F->graph) cudaGraphDestroy(F->graph);
  F->exec = nullptr;
  F->graph = nullptr;
  F->graph_u.clear();
}
}  // namespace

extern "C" int nrgpu_fmr_track(nrgpu_fmr *F, int n, const double *pos, int fixz) {
  if (!F || n < 0 || n > NRGPU_MAX_PUNCTURES || (n && !pos))
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad arguments (0 <= n <= %d)", NRGPU_MAX_PUNCTURES);
  NRGPU_CUDA_TRY(cudaDeviceSynchronize());
  cudaFree(F->d_track);
  cudaFree(F->d_tstatus);
  F->d_track = nullptr;
  F->d_tstatus = nullptr;
  F->ntrack = 0;
  drop_graph(F);
  if (!n) return NRGPU_OK;
  if (cudaMalloc(&F->d_track, sizeof(double) * 6 * n) != cudaSuccess ||
      cudaMalloc(&F->d_tstatus, sizeof(int) * n) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(F->d_track);
    F->d_track = nullptr;
    return nrgpu_set_error(NRGPU_ERR_NOMEM, "tracking buffers");
  }
  NRGPU_CUDA_TRY(cudaMemcpy(F->d_track, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
  NRGPU_CUDA_TRY(cudaMemset(F->d_tstatus, 0, sizeof(int) * n));
  F->ntrack = n;
  F->track_fixz = fixz ? 1 : 0;
  return NRGPU_OK;
}

extern "C" int nrgpu_fmr_track_method(nrgpu_fmr *F, int method, int var, int find_max, double minmove,
                                      int fixz_ext) {
  if (!F) return nrgpu_set_error(NRGPU_ERR_ARG, "null hierarchy");
  if (method < 0 || method > 2)
    return nrgpu_set_error(NRGPU_ERR_ARG, "tracking method %d (0 ext, 1 int, 2 extint)", method);
  if (method != 1 && (var < 0 || var >= F->nv))
    return nrgpu_set_error(NRGPU_ERR_ARG, "tracked variable %d (0..%d)", var, F->nv - 1);
  if (method != 1 && !(minmove >= 0.0)) return nrgpu_set_error(NRGPU_ERR_ARG, "minmove %g", minmove);
  NRGPU_CUDA_TRY(cudaDeviceSynchronize());
  F->track_method = method;
  F->track_var = method == 1 ? 0 : var;
  F->track_max = find_max ? 1 : 0;
  F->track_minmove = minmove;
  F->track_fixz_ext = fixz_ext ? 1 : 0;
  drop_graph(F);
  return NRGPU_OK;
}

extern "C" int nrgpu_fmr_punctures(nrgpu_fmr *F, double *pos, int *status) {
  if (!F || !pos) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  if (!F->ntrack) return nrgpu_set_error(NRGPU_ERR_ARG, "no punctures tracked");
  NRGPU_CUDA_TRY(cudaDeviceSynchronize());
  NRGPU_CUDA_TRY(cudaMemcpy(pos, F->d_track, sizeof(double) * 3 * F->ntrack, cudaMemcpyDeviceToHost));
  if (status) NRGPU_CUDA_TRY(cudaMemcpy(status, F->d_tstatus, sizeof(int) * F->ntrack, cudaMemcpyDeviceToHost));
  return NRGPU_OK;
}
