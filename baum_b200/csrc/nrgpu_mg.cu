// nrgpu_mg.cu -- the puncture initial-data multigrid on B200 (FP64).
//
// Restates the reference's FAS multigrid for the Hamiltonian constraint in
// puncture form, L(u) = Laplace(u) + b (1 + a (1+u))^-7 = 0
// (PunctureSolve.c:21-138; multigrid.c:35-123; solve.c:20-161;
// fasmg.c:41-122; relax.c:174-190; residual.c:13-75;
// restrictprolong.c:21-122; exactsolve.c:18-77; makestack.c:36-170;
// robin.c:29-223), for one cubic box with a Robin outer boundary.
//
// Device design:
//  * every stack level is a cube of m^3 points stored x fastest; the
//    relaxation is undamped Jacobi, done as ping-pong between two arrays
//    (the reference copies u to v and writes u; the values are the same);
//  * the Robin condition is a gather over the boundary points with the normal
//    neighbour and the factors 1-c, 1+c precomputed at set-up;
//  * the coarse-grid right-hand side of FAS, fH = R fh + L R uh - R L uh,
//    is one fused kernel;
//  * the coarsest level (4^3 .. 10^3 points) is solved "exactly" by one
//    thread block that sweeps, checks its residual and stops on the device;
//  * residual norms are two-pass deterministic block reductions (warp
//    shuffles, then one block) into a device scalar;
//  * a device flag marks convergence of the finest level: every kernel of a
//    V-cycle returns at once when it is set, so cycles are enqueued in
//    batches (and captured as a CUDA graph) and the host reads the flag and
//    the cycle counter once per batch.  The cycle count is exact.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "nrgpu_common.cuh"

namespace {

struct MgLevel {
  int m;
  long np;
  double dx, x0;
  double *u, *u2, *v, *w, *f, *a, *b;  // u2: ping-pong partner of u
  int nb;                              // boundary points
  int *bidx, *bnrm;                    // boundary point, its Robin normal neighbour
  double *bc1, *bc2;                   // 1-c, 1+c of the u condition (far limit 0)
};

struct MgStatus {
  double res;       // last finest-level residual (RMS over inner points)
  int done;         // finest level converged: the rest of the batch is skipped
  int ncycles;      // V cycles performed on the level being cycled
  int exact_sweeps; // sweeps of the last coarsest solve
  int pad;
};

constexpr int RB = 256;  // threads per block of the grid kernels

__device__ __forceinline__ bool inner(int i, int j, int k, int m) {
  return i > 0 && j > 0 && k > 0 && i < m - 1 && j < m - 1 && k < m - 1;
}

// Robin / Dirichlet gather on the boundary (set_boundary_robin): with far
// limit 0 the Robin value is u_n (1-c)/(1+c); falloff 0 gives -u_n
// (each kernel below is a per-point function, *_at(t, ...), called by one
// grid thread per point, or in block-stride loops by the one-block bottom
// of the V cycle, bottom_vcycle_kernel)
__device__ __forceinline__ void robin_at(int t, double *u, const int *__restrict__ bidx,
                                         const int *__restrict__ bnrm, const double *__restrict__ c1,
                                         const double *__restrict__ c2, int nb, int dirichlet) {
  if (t >= nb) return;
  const double un = u[bnrm[t]];
  u[bidx[t]] = dirichlet ? -un : un * c1[t] / c2[t];
}
__global__ void robin_kernel(double *u, const int *__restrict__ bidx, const int *__restrict__ bnrm,
                             const double *__restrict__ c1, const double *__restrict__ c2, int nb, int dirichlet,
                             const int *__restrict__ done) {
  if (done && *done) return;
  robin_at(blockIdx.x * blockDim.x + threadIdx.x, u, bidx, bnrm, c1, c2, nb, dirichlet);
}

// w^-7 and w^-8 by multiplication: the reference's pow(w, -7.0) and
// pow(w, -8.0) (PunctureSolve.c:38-41) within a few ulp, at a few FLOPs
// instead of an FP64 pow (log + exp) per point and sweep
__device__ __forceinline__ double inv_pow7(double w) {
  const double r = 1.0 / w, r2 = r * r, r4 = r2 * r2;
  return r4 * r2 * r;
}
__device__ __forceinline__ double inv_pow8(double w) {
  const double r = 1.0 / w, r2 = r * r, r4 = r2 * r2;
  return r4 * r4;
}

// the puncture operator at an inner point
__device__ __forceinline__ double lop_point(const double *__restrict__ u, long q, int m, double cc, double cx,
                                            double a, double b) {
  const long mm = (long)m * m;
  return cc * u[q] + cx * (u[q - 1] + u[q + 1]) + cx * (u[q - m] + u[q + m]) + cx * (u[q - mm] + u[q + mm]) +
         b * inv_pow7(1.0 + a * (1.0 + u[q]));
}

// The boundary condition fused into the kernel that produces the inner
// values it reads.  Set_boundary_robin writes u[b] = u[n] (1-c)/(1+c) (or
// -u[n] for the Dirichlet correction) from the boundary point's inward normal
// neighbour n, which is always an inner point.  A fused kernel runs np + nb
// threads: thread q < np computes inner point q, thread np + t recomputes the
// value of the normal neighbour of boundary point t with the same
// arithmetic and writes the boundary value from it.  Out-of-place kernels
// only (the recomputation reads the kernel's inputs, never its outputs), so
// the result is bit-identical to the kernel followed by robin_kernel.
struct RobinFuse {
  const int *bidx, *bnrm;
  const double *c1, *c2;
  int nb;         // 0: no boundary threads
  int dirichlet;  // -u[n] instead of u[n] c1 / c2
};

// thread -> (point whose value is computed, boundary slot or -1); false past the end
__device__ __forceinline__ bool fused_point(int t, int np, const RobinFuse &R, int &q, int &slot) {
  if (t < np) {
    q = t;
    slot = -1;
    return true;
  }
  if (t < np + R.nb) {
    slot = t - np;
    q = R.bnrm[slot];
    return true;
  }
  return false;
}
__device__ __forceinline__ void fused_store(double *out, int q, int slot, double v, const RobinFuse &R) {
  if (slot < 0) out[q] = v;
  else out[R.bidx[slot]] = R.dirichlet ? -v : v * R.c1[slot] / R.c2[slot];
}

// (i, j, k) of point q of an m^3 cube from FP64 products with rm = 1/m and
// rmm = 1/m^2 instead of integer divisions: (q + 1/2) / m^2 lies at least
// 1/(2 m^2) from an integer, far above the products' rounding, so the
// truncations are the exact quotients
__device__ __forceinline__ void cube_ijk(int q, int m, double rm, double rmm, int &i, int &j, int &k) {
  k = (int)(((double)q + 0.5) * rmm);
  const int r = q - k * m * m;
  j = (int)(((double)r + 0.5) * rm);
  i = r - j * m;
}

// the same with the reciprocals formed here (1/m rounded, squared: the
// margin above holds with that product's rounding too)
__device__ __forceinline__ void cube_ijk(int q, int m, int &i, int &j, int &k) {
  const double rm = 1.0 / m;
  cube_ijk(q, m, rm, rm * rm, i, j, k);
}

// one Jacobi sweep un = uo + (f - L uo)/L_ii on inner points (Lpuncture_GS),
// followed by the Robin condition on un (relax.c:19-43 then robin.c:146-223)
__device__ __forceinline__ void jacobi_at(int t, const double *__restrict__ uo, double *__restrict__ un,
                                          const double *__restrict__ f, const double *__restrict__ a,
                                          const double *__restrict__ b, int m, double cx, const RobinFuse &R,
                                          double rm, double rmm) {
  int q, slot;
  if (!fused_point(t, m * m * m, R, q, slot)) return;
  int i, j, k;
  cube_ijk(q, m, rm, rmm, i, j, k);
  if (!inner(i, j, k, m)) return;
  const double cc = -2.0 * (cx + cx + cx);
  const double aq = a[q], bq = b[q], uq = uo[q];
  const double lu = lop_point(uo, q, m, cc, cx, aq, bq);
  const double lii = cc - 7.0 * bq * aq * inv_pow8(1.0 + aq * (1.0 + uq));
  fused_store(un, q, slot, uq + (f[q] - lu) / lii, R);
}
__global__ void jacobi_kernel(const double *__restrict__ uo, double *__restrict__ un, const double *__restrict__ f,
                              const double *__restrict__ a, const double *__restrict__ b, int m, double cx,
                              RobinFuse R, const int *__restrict__ done, double rm, double rmm) {
  if (done && *done) return;
  jacobi_at(blockIdx.x * blockDim.x + threadIdx.x, uo, un, f, a, b, m, cx, R, rm, rmm);
}

// a damped Jacobi sweep un = uo + omega (f - L uo)/L_ii with the Robin
// condition fused in: the smoothing of an initial guess before the V cycles
// (nrgpu_mg_smooth; no counterpart in the reference, whose sweeps are
// undamped)
__global__ void damped_jacobi_kernel(const double *__restrict__ uo, double *__restrict__ un,
                                     const double *__restrict__ f, const double *__restrict__ a,
                                     const double *__restrict__ b, int m, double cx, double omega, RobinFuse R) {
  int q, slot;
  if (!fused_point(blockIdx.x * blockDim.x + threadIdx.x, m * m * m, R, q, slot)) return;
  int i, j, k;
  cube_ijk(q, m, i, j, k);
  if (!inner(i, j, k, m)) return;
  const double cc = -2.0 * (cx + cx + cx);
  const double aq = a[q], bq = b[q], uq = uo[q];
  const double lu = lop_point(uo, q, m, cc, cx, aq, bq);
  const double lii = cc - 7.0 * bq * aq * inv_pow8(1.0 + aq * (1.0 + uq));
  fused_store(un, q, slot, uq + omega * ((f[q] - lu) / lii), R);
}

// block partial sums of (L u - f)^2 over inner points
__global__ void residual_partial_kernel(const double *__restrict__ u, const double *__restrict__ f,
                                        const double *__restrict__ a, const double *__restrict__ b, int m,
                                        double cx, double *partial, const int *__restrict__ done) {
  if (done && *done) return;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const long np = (long)m * m * m;
  double s = 0.0;
  if (q < np) {
    int i, j, k;
    cube_ijk(q, m, i, j, k);
    if (inner(i, j, k, m)) {
      const double r = lop_point(u, q, m, -2.0 * (cx + cx + cx), cx, a[q], b[q]) - f[q];
      s = r * r;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double ws[RB / 32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < RB / 32 ? ws[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
}

// final reduction, RMS over the n inner points; when tol >= 0 this is the
// convergence test of a V-cycle loop: res <= tol sets done, else counts a cycle
__global__ void residual_final_kernel(const double *__restrict__ partial, int nparts, long ninner, MgStatus *st,
                                      double tol, int count, int vnmax) {
  if (st->done) return;
  double s = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += partial[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ double ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += ws[w];
    const double res = sqrt(t / (double)ninner);
    st->res = res;
    if (count) {
      if (res <= tol) st->done = 1;        // converged: no further cycle
      else if (st->ncycles >= vnmax) st->done = 2;  // cycle budget spent
      else st->ncycles += 1;               // one more cycle follows
    }
  }
}

// 8-point average of the fine children of inner coarse points
// (mg_restrict_var), with the Robin condition on the result when R.nb > 0
__global__ void restrict_kernel(const double *__restrict__ fv, double *__restrict__ cv, int mf, int mc, int off,
                                RobinFuse R, const int *__restrict__ done) {
  if (done && *done) return;
  int q, slot;
  if (!fused_point(blockIdx.x * blockDim.x + threadIdx.x, mc * mc * mc, R, q, slot)) return;
  int I, J, K;
  cube_ijk(q, mc, I, J, K);
  if (!inner(I, J, K, mc)) return;
  const long mf2 = (long)mf * mf;
  const long f0 = (long)(2 * I - off) + mf * (long)(2 * J - off) + mf2 * (long)(2 * K - off);
  fused_store(cv, q, slot,
              0.125 * (fv[f0] + fv[f0 + 1 + mf + mf2] + fv[f0 + 1] + fv[f0 + mf] + fv[f0 + mf2] + fv[f0 + 1 + mf] +
                       fv[f0 + 1 + mf2] + fv[f0 + mf + mf2]),
              R);
}

// finetocoarse (solve.c) in one pass over the coarse points: uH = R uh
// (mg_restrict_var) with the Robin condition, and the two restrictions of
// the FAS right-hand side, R fh into fH and R L uh into vH, with L uh
// (Lpuncture_nonlin) evaluated at the eight children.  The children of the
// inner coarse points are exactly the inner fine points, so every fine
// operator value is computed once; the sums run in the order of
// mg_restrict_var's eight terms.
__device__ __forceinline__ void fine_to_coarse_at(int t, const double *__restrict__ uh,
                                                  const double *__restrict__ fh, const double *__restrict__ ah,
                                                  const double *__restrict__ bh, double *__restrict__ uH,
                                                  double *__restrict__ RfH, double *__restrict__ RluH, int mf, int mc,
                                                  int off, double cxh, const RobinFuse &R) {
  int q, slot;
  if (!fused_point(t, mc * mc * mc, R, q, slot)) return;
  int I, J, K;
  cube_ijk(q, mc, I, J, K);
  if (!inner(I, J, K, mc)) return;
  const long mf2 = (long)mf * mf;
  const long f0 = (long)(2 * I - off) + mf * (long)(2 * J - off) + mf2 * (long)(2 * K - off);
  const long c[8] = {f0, f0 + 1 + mf + mf2, f0 + 1, f0 + mf, f0 + mf2, f0 + 1 + mf, f0 + 1 + mf2, f0 + mf + mf2};
  fused_store(uH, q, slot,
              0.125 * (uh[c[0]] + uh[c[1]] + uh[c[2]] + uh[c[3]] + uh[c[4]] + uh[c[5]] + uh[c[6]] + uh[c[7]]), R);
  if (slot >= 0) return;
  const double cch = -2.0 * (cxh + cxh + cxh);
  double lu[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) lu[n] = lop_point(uh, c[n], mf, cch, cxh, ah[c[n]], bh[c[n]]);
  RluH[q] = 0.125 * (lu[0] + lu[1] + lu[2] + lu[3] + lu[4] + lu[5] + lu[6] + lu[7]);
  RfH[q] = 0.125 * (fh[c[0]] + fh[c[1]] + fh[c[2]] + fh[c[3]] + fh[c[4]] + fh[c[5]] + fh[c[6]] + fh[c[7]]);
}
__global__ void fine_to_coarse_kernel(const double *__restrict__ uh, const double *__restrict__ fh,
                                      const double *__restrict__ ah, const double *__restrict__ bh,
                                      double *__restrict__ uH, double *__restrict__ RfH, double *__restrict__ RluH,
                                      int mf, int mc, int off, double cxh, RobinFuse R, const int *__restrict__ done) {
  if (done && *done) return;
  fine_to_coarse_at(blockIdx.x * blockDim.x + threadIdx.x, uh, fh, ah, bh, uH, RfH, RluH, mf, mc, off, cxh, R);
}

// the FAS coarse right-hand side fH = R fh + (L uH - R L uh) at inner coarse
// points (fH holds R fh, RluH holds R L uh), and wH = uH at every point
__device__ __forceinline__ void coarse_rhs_at(int q, const double *__restrict__ uH, double *__restrict__ fH,
                                              const double *__restrict__ RluH, double *__restrict__ wH,
                                              const double *__restrict__ aH, const double *__restrict__ bH, int mc,
                                              double cxH) {
  if (q >= mc * mc * mc) return;
  wH[q] = uH[q];
  int I, J, K;
  cube_ijk(q, mc, I, J, K);
  if (!inner(I, J, K, mc)) return;
  const double luH = lop_point(uH, q, mc, -2.0 * (cxH + cxH + cxH), cxH, aH[q], bH[q]);
  fH[q] = fH[q] + (luH - RluH[q]);
}
__global__ void coarse_rhs_kernel(const double *__restrict__ uH, double *__restrict__ fH,
                                  const double *__restrict__ RluH, double *__restrict__ wH,
                                  const double *__restrict__ aH, const double *__restrict__ bH, int mc, double cxH,
                                  const int *__restrict__ done) {
  if (done && *done) return;
  coarse_rhs_at(blockIdx.x * blockDim.x + threadIdx.x, uH, fH, RluH, wH, aH, bH, mc, cxH);
}

// wH = uH (all points), vH = uH - wH helpers
__global__ void copy_kernel(const double *__restrict__ s, double *__restrict__ d, long n, const int *__restrict__ done) {
  if (done && *done) return;
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) d[q] = s[q];
}
__device__ __forceinline__ void sub_inner_at(int t, const double *__restrict__ x, const double *__restrict__ y,
                                             double *__restrict__ r, int m, const RobinFuse &R) {
  int q, slot;
  if (!fused_point(t, m * m * m, R, q, slot)) return;
  int i, j, k;
  cube_ijk(q, m, i, j, k);
  if (inner(i, j, k, m)) fused_store(r, q, slot, x[q] - y[q], R);
}
__global__ void sub_inner_kernel(const double *__restrict__ x, const double *__restrict__ y, double *__restrict__ r,
                                 int m, RobinFuse R, const int *__restrict__ done) {
  if (done && *done) return;
  sub_inner_at(blockIdx.x * blockDim.x + threadIdx.x, x, y, r, m, R);
}

// trilinear prolongation of the coarse correction, added to the inner fine
// points (mg_prolong_var + add); weights 1/4, 3/4 from the cell-centred
// staggering, coarse index ci = floor((i + off') / 2)
__device__ __forceinline__ void prolong_add_at(int q, const double *__restrict__ cv, double *__restrict__ uf,
                                               int mf, int mc, double fx0, double fdx, double cx0, double cdx,
                                               int add) {
  if (q >= mf * mf * mf) return;
  int i, j, k;
  cube_ijk(q, mf, i, j, k);
  if (!inner(i, j, k, mf)) return;
  const double xf = fx0 + i * fdx, yf = fx0 + j * fdx, zf = fx0 + k * fdx;
  const int ci = (int)((xf - cx0) / cdx), cj = (int)((yf - cx0) / cdx), ck = (int)((zf - cx0) / cdx);
  const double kx1 = (xf - (cx0 + ci * cdx)) / cdx, ky1 = (yf - (cx0 + cj * cdx)) / cdx,
               kz1 = (zf - (cx0 + ck * cdx)) / cdx;
  const double kx0 = 1 - kx1, ky0 = 1 - ky1, kz0 = 1 - kz1;
  const long mc2 = (long)mc * mc;
  const long c0 = ci + (long)mc * cj + mc2 * ck;
  const double p = kx0 * ky0 * kz0 * cv[c0] + kx1 * ky0 * kz0 * cv[c0 + 1] + kx0 * ky1 * kz0 * cv[c0 + mc] +
                   kx1 * ky1 * kz0 * cv[c0 + 1 + mc] + kx0 * ky0 * kz1 * cv[c0 + mc2] +
                   kx1 * ky0 * kz1 * cv[c0 + 1 + mc2] + kx0 * ky1 * kz1 * cv[c0 + mc + mc2] +
                   kx1 * ky1 * kz1 * cv[c0 + 1 + mc + mc2];
  uf[q] = add ? uf[q] + p : p;
}
__global__ void prolong_add_kernel(const double *__restrict__ cv, double *__restrict__ uf, int mf, int mc,
                                   double fx0, double fdx, double cx0, double cdx, int add,
                                   const int *__restrict__ done) {
  if (done && *done) return;
  prolong_add_at(blockIdx.x * blockDim.x + threadIdx.x, cv, uf, mf, mc, fx0, fdx, cx0, cdx, add);
}

// "exact" solve of the coarsest level in one thread block (exactsolve):
// findres, then Jacobi sweeps (each followed by the Robin condition) until
// the residual drops below tol/10 after at least nmin sweeps, at most nmax
__device__ void block_robin(double *u, const int *bidx, const int *bnrm, const double *c1, const double *c2, int nb) {
  for (int t = threadIdx.x; t < nb; t += blockDim.x) u[bidx[t]] = u[bnrm[t]] * c1[t] / c2[t];
}
__device__ double block_residual(const double *u, const double *f, const double *a, const double *b, int m, double cx,
                                 double *red) {
  const long np = (long)m * m * m;
  double s = 0.0;
  long n = 0;
  for (long q = threadIdx.x; q < np; q += blockDim.x) {
    const int i = q % m, j = (q / m) % m, k = q / (m * m);
    if (!inner(i, j, k, m)) continue;
    const double r = lop_point(u, q, m, -2.0 * (cx + cx + cx), cx, a[q], b[q]) - f[q];
    s += r * r;
  }
  n = (long)(m - 2) * (m - 2) * (m - 2);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
  __syncthreads();
  return sqrt(t / (double)n);
}
__global__ void exact_solve_kernel(double *u, double *u2, const double *f, const double *a, const double *b, int m,
                                   double cx, const int *bidx, const int *bnrm, const double *c1, const double *c2,
                                   int nb, int nmin, int nmax, double tol10, MgStatus *st) {
  if (st->done) return;
  __shared__ double red[32];
  const long np = (long)m * m * m;
  // findres applies the Robin condition to u first (Lpuncture_nonlin)
  block_robin(u, bidx, bnrm, c1, c2, nb);
  __syncthreads();
  double *uo = u, *un = u2;
  int i;
  for (i = 1; i <= nmax; ++i) {
    const double cc = -2.0 * (cx + cx + cx);
    for (long q = threadIdx.x; q < np; q += blockDim.x) {
      const int ii = q % m, jj = (q / m) % m, kk = q / (m * m);
      if (!inner(ii, jj, kk, m)) { un[q] = uo[q]; continue; }
      const double lu = lop_point(uo, q, m, cc, cx, a[q], b[q]);
      const double lii = cc - 7.0 * b[q] * a[q] * inv_pow8(1.0 + a[q] * (1.0 + uo[q]));
      un[q] = uo[q] + (f[q] - lu) / lii;
    }
    __syncthreads();
    block_robin(un, bidx, bnrm, c1, c2, nb);
    __syncthreads();
    double *t = uo; uo = un; un = t;
    if (i >= nmin) {
      const double r = block_residual(uo, f, a, b, m, cx, red);
      if (r < tol10) break;
    }
  }
  // leave the result in u
  if (uo != u) {
    for (long q = threadIdx.x; q < np; q += blockDim.x) u[q] = uo[q];
    __syncthreads();
  }
  if (threadIdx.x == 0) st->exact_sweeps = i;
}

// The coarsest solve by one warp with the whole level in shared memory
// (levels of up to NRGPU_MG_WARP_SOLVE_MAX points): the sweeps, Robin
// updates and residual tests of exact_solve_kernel, synchronised by
// __syncwarp instead of block barriers and global-memory round trips.  The
// coarsest level is a handful of inner points (8 on the 4^3 level) swept up
// to exact_nmax times per V cycle, so the sweep's latency is the cost.
constexpr int NRGPU_MG_WARP_SOLVE_MAX = 1000;
// run by the 32 threads of one warp (lane = threadIdx.x & 31), sm: the
// level's shared-memory copy (warp_solve_smem bytes)
__device__ void exact_solve_warp(double *u, const double *f, const double *a, const double *b, int m, double cx,
                                 const int *bidx, const int *bnrm, const double *c1, const double *c2, int nb,
                                 int nmin, int nmax, double tol10, MgStatus *st, double *sm) {
  const int np = m * m * m, lane = threadIdx.x & 31;
  double *su = sm, *sv = su + np, *sa = sv + np, *sb = sa + np, *sf = sb + np, *sc1 = sf + np, *sc2 = sc1 + nb;
  int *sbi = (int *)(sc2 + nb), *sbn = sbi + nb;
  for (int q = lane; q < np; q += 32) {
    su[q] = u[q];
    sa[q] = a[q];
    sb[q] = b[q];
    sf[q] = f[q];
  }
  for (int t = lane; t < nb; t += 32) {
    sc1[t] = c1[t];
    sc2[t] = c2[t];
    sbi[t] = bidx[t];
    sbn[t] = bnrm[t];
  }
  __syncwarp();
  // findres applies the Robin condition to u first (Lpuncture_nonlin)
  for (int t = lane; t < nb; t += 32) su[sbi[t]] = su[sbn[t]] * sc1[t] / sc2[t];
  const int mi = m - 2, ni = mi * mi * mi;
  int *sq = sbn + nb;  // the inner points' indices
  for (int p = lane; p < ni; p += 32) sq[p] = (1 + p % mi) + m * ((1 + (p / mi) % mi) + m * (1 + p / (mi * mi)));
  __syncwarp();
  const double cc = -2.0 * (cx + cx + cx);
  double *uo = su, *un = sv;
  // Pass `it` evaluates L u_{it-1} once: its residual is the test after
  // sweep it-1 (from nmin sweeps on), and the same value gives sweep it.
  // This is the reference's sweep-then-test loop with the operator of the
  // test shared by the next sweep; results are identical.
  int it;
  for (it = 1; it <= nmax + 1; ++it) {
    double s = 0.0;
    for (int p = lane; p < ni; p += 32) {
      const int q = sq[p];
      const double aq = sa[q], bq = sb[q], uq = uo[q];
      const double lu = lop_point(uo, q, m, cc, cx, aq, bq);
      const double r = lu - sf[q];
      s += r * r;
      if (it <= nmax) {
        const double lii = cc - 7.0 * bq * aq * inv_pow8(1.0 + aq * (1.0 + uq));
        un[q] = uq + (sf[q] - lu) / lii;
      }
    }
    if (it - 1 >= nmin && it > 1) {  // the first test follows the first sweep
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (sqrt(s / (double)ni) < tol10) {
        it -= 1;  // sweeps done
        break;
      }
    }
    if (it > nmax) break;  // nmax sweeps and no pass: the loop ends at nmax + 1
    __syncwarp();
    // every point outside the inner cube is a boundary point: the Robin
    // condition writes all of them from the new inner values
    for (int t = lane; t < nb; t += 32) un[sbi[t]] = un[sbn[t]] * sc1[t] / sc2[t];
    __syncwarp();
    double *tt = uo;
    uo = un;
    un = tt;
  }
  __syncwarp();
  for (int q = lane; q < np; q += 32) u[q] = uo[q];
  if (lane == 0) st->exact_sweeps = it;
}
__global__ void __launch_bounds__(32) exact_solve_warp_kernel(double *u, const double *f, const double *a,
                                                              const double *b, int m, double cx, const int *bidx,
                                                              const int *bnrm, const double *c1, const double *c2,
                                                              int nb, int nmin, int nmax, double tol10, MgStatus *st) {
  if (st->done) return;
  extern __shared__ double sm[];
  exact_solve_warp(u, f, a, b, m, cx, bidx, bnrm, c1, c2, nb, nmin, nmax, tol10, st, sm);
}

static size_t warp_solve_smem(int m, int nb) {
  const size_t np = (size_t)m * m * m, ni = (size_t)(m - 2) * (m - 2) * (m - 2);
  return sizeof(double) * (5 * np + 2 * (size_t)nb) + sizeof(int) * (2 * (size_t)nb + ni);
}

// The bottom of the V cycle in one thread block: every level of at most
// NRGPU_MG_BOTTOM_MAX points (10^3 and 6^3 of the 130^3 stack, and the 4^3
// coarsest) runs the same steps as vcycle() with the same per-point
// functions, in block-stride loops separated by __syncthreads, instead of
// ~25 kernels of a few hundred threads.  Each level's u returns to its entry
// buffer, as in vcycle().  (With the 18^3 level in the block too, one
// block's sweeps took as long as the launches they replaced.)
constexpr int NRGPU_MG_BOTTOM_MAX = 1000;
constexpr int NRGPU_MG_BOTTOM_THREADS = 512;
constexpr int NRGPU_MG_MAXLEV = 16;
struct MgDev {
  int m, nb;
  double dx, x0;
  double *u, *u2, *v, *w, *f, *a, *b;
  const int *bidx, *bnrm;
  const double *bc1, *bc2;
};

__global__ void __launch_bounds__(NRGPU_MG_BOTTOM_THREADS)
    bottom_vcycle_kernel(const MgDev *__restrict__ lv, int top, int npre, int npost, int exact_nmin, int exact_nmax,
                         double tol10, MgStatus *st, const int *__restrict__ done) {
  if (done && *done) return;
  extern __shared__ double sm[];
  const int tid = threadIdx.x, nt = blockDim.x;
  double *U[NRGPU_MG_MAXLEV], *U2[NRGPU_MG_MAXLEV];
  for (int l = 0; l <= top; ++l) {
    U[l] = lv[l].u;
    U2[l] = lv[l].u2;
  }
  // down: pre-sweeps, restriction and the FAS right-hand side
  for (int l = top; l >= 1; --l) {
    const MgDev &h = lv[l], &H = lv[l - 1];
    const int np = h.m * h.m * h.m, npH = H.m * H.m * H.m;
    const double cx = 1 / (h.dx * h.dx), cxH = 1 / (H.dx * H.dx);
    const double rm = 1.0 / h.m, rmm = 1.0 / ((double)h.m * h.m);
    const RobinFuse Rh = {h.bidx, h.bnrm, h.bc1, h.bc2, h.nb, 0}, RH = {H.bidx, H.bnrm, H.bc1, H.bc2, H.nb, 0};
    for (int s = 0; s < npre; ++s) {
      for (int t = tid; t < np + h.nb; t += nt) jacobi_at(t, U[l], U2[l], h.f, h.a, h.b, h.m, cx, Rh, rm, rmm);
      __syncthreads();
      double *x = U[l];
      U[l] = U2[l];
      U2[l] = x;
    }
    if (npre == 0) {
      for (int t = tid; t < h.nb; t += nt) robin_at(t, U[l], h.bidx, h.bnrm, h.bc1, h.bc2, h.nb, 0);
      __syncthreads();
    }
    for (int t = tid; t < npH + H.nb; t += nt)
      fine_to_coarse_at(t, U[l], h.f, h.a, h.b, U[l - 1], H.f, H.v, h.m, H.m, 1, cx, RH);
    __syncthreads();
    for (int t = tid; t < npH; t += nt) coarse_rhs_at(t, U[l - 1], H.f, H.v, H.w, H.a, H.b, H.m, cxH);
    __syncthreads();
  }
  // the coarsest level, by the first warp
  if (tid < 32) {
    const MgDev &c = lv[0];
    exact_solve_warp(U[0], c.f, c.a, c.b, c.m, 1 / (c.dx * c.dx), c.bidx, c.bnrm, c.bc1, c.bc2, c.nb, exact_nmin,
                     exact_nmax, tol10, st, sm);
  }
  __syncthreads();
  // up: correction, prolongation, Robin condition, post-sweeps
  for (int l = 1; l <= top; ++l) {
    const MgDev &h = lv[l], &H = lv[l - 1];
    const int np = h.m * h.m * h.m, npH = H.m * H.m * H.m;
    const double cx = 1 / (h.dx * h.dx);
    const double rm = 1.0 / h.m, rmm = 1.0 / ((double)h.m * h.m);
    const RobinFuse Rh = {h.bidx, h.bnrm, h.bc1, h.bc2, h.nb, 0}, RHd = {H.bidx, H.bnrm, H.bc1, H.bc2, H.nb, 1};
    for (int t = tid; t < npH + H.nb; t += nt) sub_inner_at(t, U[l - 1], H.w, H.v, H.m, RHd);
    __syncthreads();
    for (int t = tid; t < np; t += nt) prolong_add_at(t, H.v, U[l], h.m, H.m, h.x0, h.dx, H.x0, H.dx, 1);
    __syncthreads();
    for (int t = tid; t < h.nb; t += nt) robin_at(t, U[l], h.bidx, h.bnrm, h.bc1, h.bc2, h.nb, 0);
    __syncthreads();
    for (int s = 0; s < npost; ++s) {
      for (int t = tid; t < np + h.nb; t += nt) jacobi_at(t, U[l], U2[l], h.f, h.a, h.b, h.m, cx, Rh, rm, rmm);
      __syncthreads();
      double *x = U[l];
      U[l] = U2[l];
      U2[l] = x;
    }
    if (U[l] != h.u) {
      for (int t = tid; t < np; t += nt) h.u[t] = U[l][t];
      __syncthreads();
      U2[l] = U[l];
      U[l] = h.u;
    }
  }
}

__global__ void robin_factors_kernel(const int *bidx, const int *bnrm, double *c1, double *c2, int nb, int m, double x0,
                                     double dx, double falloff) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nb) return;
  const int q = bidx[t], n = bnrm[t];
  const int i = q % m, j = (q / m) % m, k = q / (m * m);
  const int ni = n % m, nj = (n / m) % m, nk = n / (m * m);
  const double x1 = x0 + i * dx, y1 = x0 + j * dx, z1 = x0 + k * dx;
  const double xa = x0 + ni * dx, ya = x0 + nj * dx, za = x0 + nk * dx;
  const double x = 0.5 * (x1 + xa), y = 0.5 * (y1 + ya), z = 0.5 * (z1 + za);
  const double vx = x1 - xa, vy = y1 - ya, vz = z1 - za;
  const double c = 0.5 * falloff * (vx * x + vy * y + vz * z) / (x * x + y * y + z * z);
  c1[t] = 1 - c;
  c2[t] = 1 + c;
}

// Brill-Lindquist + Bowen-York coefficients (SetMWBL, SetBYK,
// SetPunctureCoefficients): a = 1/(psi - 1), b = a^7 K_ij K^ij / 8
struct Punctures {
  int n;
  double mass[8], pos[8][3], mom[8][3], spin[8][3];
};
__global__ void coefficients_kernel(Punctures P, int m, double dx, double *a, double *b) {
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long)m * m * m) return;
  const int i = q % m, j = (q / m) % m, k = q / ((long)m * m);
  const double x0 = -(m - 1) * dx / 2;
  const double x = x0 + i * dx, y = x0 + j * dx, z = x0 + k * dx;
  double p = 0.0, K[6] = {0, 0, 0, 0, 0, 0};
  for (int n = 0; n < P.n; ++n) {
    const double xi = x - P.pos[n][0], yi = y - P.pos[n][1], zi = z - P.pos[n][2];
    double r = sqrt(xi * xi + yi * yi + zi * zi);
    if (!(r < -1e-10 || 0.0 < r - 1e-10)) r = 1e-13;  // dequal(r,0) -> EPSZERO
    p += P.mass[n] * (1 / r) * 0.5;
    const double N[3] = {xi / r, yi / r, zi / r};
    const double *Pm = P.mom[n], *S = P.spin[n];
    const double NP = N[0] * Pm[0] + N[1] * Pm[1] + N[2] * Pm[2];
    const double eNS[3] = {N[1] * S[2] - N[2] * S[1], N[2] * S[0] - N[0] * S[2], N[0] * S[1] - N[1] * S[0]};
    int c = 0;
    for (int s = 0; s < 3; ++s)
      for (int t = s; t < 3; ++t, ++c)
        K[c] += 1.5 / (r * r) * (N[s] * Pm[t] + N[t] * Pm[s] - ((s == t) - N[s] * N[t]) * NP) -
                3.0 / (r * r * r) * (eNS[s] * N[t] + eNS[t] * N[s]);
  }
  const double psi = p + 1.0;
  const double aq = 1 / (psi - 1);
  const double K2 = K[0] * K[0] + K[3] * K[3] + K[5] * K[5] + 2 * K[1] * K[1] + 2 * K[2] * K[2] + 2 * K[4] * K[4];
  a[q] = aq;
  b[q] = 0.125 * pow(aq, 7.0) * K2;
}

unsigned nblk(long n) { return (unsigned)((n + RB - 1) / RB); }

}  // namespace

// ---- host side ----------------------------------------------------------------
struct nrgpu_mg {
  int nl;  // levels, 0 = coarsest
  MgLevel lv[16];
  nrgpu_mg_params p;
  MgStatus *st;       // device
  double *partial;    // device block partial sums (finest level size)
  int npartial;
  cudaStream_t stream;  // library-owned (captured into CUDA graphs)
  cudaGraph_t graph[16];
  cudaGraphExec_t exec[16];
  // the one-block bottom of the V cycle: levels 0..bottom (0: not used)
  int bottom;
  MgDev *d_lv;
};

// stack sizes (coarsegridsize, makestack.c:36-79) for one process
static int stack_sizes(int m, int size_nmin, int levels_nmax, int *sizes) {
  int n = 0, l = 1;
  sizes[n++] = m;
  while (n < 16) {
    if (levels_nmax != -1 && l > levels_nmax) break;
    if ((m - 2) % 4) break;
    const int mnew = m / 2 + 1;
    if (mnew < size_nmin || mnew < 4) break;
    sizes[n++] = m = mnew;
    l++;
  }
  return n;
}

// find_robin_normal (robin.c:29-143) on the host: averaged unit directions to
// the inner members of the 27-neighbourhood, then the grid direction with the
// largest projection (first maximum in loop order)
static void robin_normals(int m, std::vector<int> &bidx, std::vector<int> &bnrm) {
  auto isb = [m](int i, int j, int k) { return i == 0 || j == 0 || k == 0 || i == m - 1 || j == m - 1 || k == m - 1; };
  for (int k = 0; k < m; ++k)
    for (int j = 0; j < m; ++j)
      for (int i = 0; i < m; ++i) {
        if (!isb(i, j, k)) continue;
        double vx = 0, vy = 0, vz = 0, mx = 0;
        int best = -1;
        for (int pass = 0; pass < 2; ++pass)
          for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b)
              for (int c = 0; c < 3; ++c) {
                const int ii = i + a - 1, jj = j + b - 1, kk = k + c - 1;
                if (ii < 0 || jj < 0 || kk < 0 || ii >= m || jj >= m || kk >= m) continue;
                if (isb(ii, jj, kk)) continue;
                const double s = sqrt((double)((a - 1) * (a - 1) + (b - 1) * (b - 1) + (c - 1) * (c - 1)));
                if (pass == 0) {
                  vx += (a - 1) / s; vy += (b - 1) / s; vz += (c - 1) / s;
                } else {
                  const double dot = (vx * (a - 1) + vy * (b - 1) + vz * (c - 1)) / s;
                  if (dot > mx) { mx = dot; best = ii + m * (jj + m * kk); }
                }
              }
        bidx.push_back(i + m * (j + m * k));
        bnrm.push_back(best);
      }
}

extern "C" void nrgpu_mg_params_default(nrgpu_mg_params *p) {
  if (!p) return;
  p->npre = 3;
  p->npost = 3;
  p->exact_nmin = 10;
  p->exact_nmax = 200;
  p->vcycle_nmin = 0;
  p->vcycle_nmax = 2000;
  p->fullV = 1;
  p->size_nmin = 4;
  p->levels_nmax = -1;
  p->tol = 1e-10;
  p->falloff = 1.0;
  p->batch = 8;
}

extern "C" int nrgpu_mg_destroy(nrgpu_mg *M) {
  if (!M) return NRGPU_OK;
  for (int l = 0; l < M->nl; ++l) {
    MgLevel &L = M->lv[l];
    cudaFree(L.u); cudaFree(L.u2); cudaFree(L.v); cudaFree(L.w); cudaFree(L.f); cudaFree(L.a); cudaFree(L.b);
    cudaFree(L.bidx); cudaFree(L.bnrm); cudaFree(L.bc1); cudaFree(L.bc2);
    if (M->exec[l]) cudaGraphExecDestroy(M->exec[l]);
    if (M->graph[l]) cudaGraphDestroy(M->graph[l]);
  }
  cudaFree(M->st);
  cudaFree(M->partial);
  cudaFree(M->d_lv);
  if (M->stream) cudaStreamDestroy(M->stream);
  free(M);
  return NRGPU_OK;
}

extern "C" int nrgpu_mg_create(int m, double dx, const nrgpu_mg_params *p, nrgpu_mg **out) {
  if (!p || !out || m < 4 || !(dx > 0)) return nrgpu_set_error(NRGPU_ERR_ARG, "bad multigrid arguments");
  if (p->npre < 0 || p->npost < 0 || p->exact_nmax < 1 || p->vcycle_nmax < 1 || p->batch < 1)
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad multigrid parameters");
  if ((long)m * m * m > 0x7fffffffL) return nrgpu_set_error(NRGPU_ERR_ARG, "box too large");
  int sizes[16];
  const int nl = stack_sizes(m, p->size_nmin, p->levels_nmax, sizes);
  nrgpu_mg *M = (nrgpu_mg *)calloc(1, sizeof(nrgpu_mg));
  if (!M) return nrgpu_set_error(NRGPU_ERR_NOMEM, "host allocation");
  M->nl = nl;
  M->p = *p;
  bool ok = true;
  for (int l = 0; l < nl && ok; ++l) {
    MgLevel &L = M->lv[l];
    L.m = sizes[nl - 1 - l];
    L.np = (long)L.m * L.m * L.m;
    L.dx = dx * (double)(1 << (nl - 1 - l));
    L.x0 = -(L.m - 1) * L.dx / 2;
    const size_t by = sizeof(double) * L.np;
    ok = cudaMalloc(&L.u, by) == cudaSuccess && cudaMalloc(&L.u2, by) == cudaSuccess &&
         cudaMalloc(&L.v, by) == cudaSuccess && cudaMalloc(&L.w, by) == cudaSuccess &&
         cudaMalloc(&L.f, by) == cudaSuccess && cudaMalloc(&L.a, by) == cudaSuccess &&
         cudaMalloc(&L.b, by) == cudaSuccess;
    if (!ok) break;
    std::vector<int> bi, bn;
    robin_normals(L.m, bi, bn);
    L.nb = (int)bi.size();
    ok = cudaMalloc(&L.bidx, sizeof(int) * L.nb) == cudaSuccess && cudaMalloc(&L.bnrm, sizeof(int) * L.nb) == cudaSuccess &&
         cudaMalloc(&L.bc1, sizeof(double) * L.nb) == cudaSuccess &&
         cudaMalloc(&L.bc2, sizeof(double) * L.nb) == cudaSuccess;
    if (!ok) break;
    cudaMemcpy(L.bidx, bi.data(), sizeof(int) * L.nb, cudaMemcpyHostToDevice);
    cudaMemcpy(L.bnrm, bn.data(), sizeof(int) * L.nb, cudaMemcpyHostToDevice);
    robin_factors_kernel<<<nblk(L.nb), RB>>>(L.bidx, L.bnrm, L.bc1, L.bc2, L.nb, L.m, L.x0, L.dx, p->falloff);
    for (double *z : {L.u, L.u2, L.v, L.w, L.f, L.a, L.b}) cudaMemset(z, 0, by);
  }
  if (ok && M->lv[0].np <= NRGPU_MG_WARP_SOLVE_MAX) {
    const size_t sm = warp_solve_smem(M->lv[0].m, M->lv[0].nb);
    if (sm > 48 * 1024)
      ok = cudaFuncSetAttribute(exact_solve_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) ==
               cudaSuccess &&
           cudaFuncSetAttribute(bottom_vcycle_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) ==
               cudaSuccess;
    // the one-block bottom: the levels above the coarsest with at most
    // NRGPU_MG_BOTTOM_MAX points
    int top = 0;
    while (top + 1 < nl && M->lv[top + 1].np <= NRGPU_MG_BOTTOM_MAX) ++top;
    if (ok && top >= 1) {
      MgDev dv[NRGPU_MG_MAXLEV];
      for (int l = 0; l <= top; ++l) {
        const MgLevel &L = M->lv[l];
        dv[l] = MgDev{L.m, L.nb, L.dx, L.x0, L.u, L.u2, L.v, L.w, L.f, L.a, L.b, L.bidx, L.bnrm, L.bc1, L.bc2};
      }
      ok = cudaMalloc(&M->d_lv, sizeof(MgDev) * (top + 1)) == cudaSuccess &&
           cudaMemcpy(M->d_lv, dv, sizeof(MgDev) * (top + 1), cudaMemcpyHostToDevice) == cudaSuccess;
      if (ok) M->bottom = top;
    }
  }
  M->npartial = (int)nblk(M->lv[nl - 1].np);
  ok = ok && cudaStreamCreateWithFlags(&M->stream, cudaStreamNonBlocking) == cudaSuccess &&
       cudaMalloc(&M->st, sizeof(MgStatus)) == cudaSuccess &&
       cudaMalloc(&M->partial, sizeof(double) * M->npartial) == cudaSuccess;
  if (!ok || cudaDeviceSynchronize() != cudaSuccess) {
    cudaGetLastError();
    nrgpu_mg_destroy(M);
    return nrgpu_set_error(NRGPU_ERR_NOMEM, "multigrid stack allocation failed");
  }
  *out = M;
  return NRGPU_OK;
}

// ---- the cycle ------------------------------------------------------------------
static void robin_u(nrgpu_mg *M, MgLevel &L, double *u, const int *done) {
  robin_kernel<<<nblk(L.nb), RB, 0, M->stream>>>(u, L.bidx, L.bnrm, L.bc1, L.bc2, L.nb, 0, done);
}
static double cxof(const MgLevel &L) { return 1 / (L.dx * L.dx); }
static RobinFuse robin_of(const MgLevel &L, int dirichlet) {
  return RobinFuse{L.bidx, L.bnrm, L.bc1, L.bc2, L.nb, dirichlet};
}
static const RobinFuse kNoRobin = {nullptr, nullptr, nullptr, nullptr, 0, 0};

// Jacobi sweeps, each with its Robin condition fused in
static void sweeps(nrgpu_mg *M, MgLevel &L, int n, const int *done) {
  for (int s = 0; s < n; ++s) {
    jacobi_kernel<<<nblk(L.np + L.nb), RB, 0, M->stream>>>(L.u, L.u2, L.f, L.a, L.b, L.m, cxof(L), robin_of(L, 0),
                                                           done, 1.0 / L.m, 1.0 / ((double)L.m * L.m));
    std::swap(L.u, L.u2);
  }
}

// the children of coarse point I are the fine points 2I-1 and 2I in each
// direction: the stack levels are centred with m_fine = 2 m_coarse - 2, so
// box_child_index gives (int)(2I - 1/2) = 2I - 1 for the inner I
constexpr int kChildOff = 1;

static void vcycle(nrgpu_mg *M, int l, const int *done) {
  if (l >= 1 && l <= M->bottom) {
    bottom_vcycle_kernel<<<1, NRGPU_MG_BOTTOM_THREADS, warp_solve_smem(M->lv[0].m, M->lv[0].nb), M->stream>>>(
        M->d_lv, l, M->p.npre, M->p.npost, M->p.exact_nmin, M->p.exact_nmax, M->p.tol / 10, M->st, done);
    return;
  }
  MgLevel &h = M->lv[l];
  if (l == 0) {
    if (h.np <= NRGPU_MG_WARP_SOLVE_MAX)
      exact_solve_warp_kernel<<<1, 32, warp_solve_smem(h.m, h.nb), M->stream>>>(
          h.u, h.f, h.a, h.b, h.m, cxof(h), h.bidx, h.bnrm, h.bc1, h.bc2, h.nb, M->p.exact_nmin, M->p.exact_nmax,
          M->p.tol / 10, M->st);
    else
      exact_solve_kernel<<<1, 256, 0, M->stream>>>(h.u, h.u2, h.f, h.a, h.b, h.m, cxof(h), h.bidx, h.bnrm, h.bc1,
                                                  h.bc2, h.nb, M->p.exact_nmin, M->p.exact_nmax, M->p.tol / 10,
                                                  M->st);
    return;
  }
  MgLevel &H = M->lv[l - 1];
  const int off = kChildOff;
  double *const u_entry = h.u;
  sweeps(M, h, M->p.npre, done);
  // finetocoarse: Lpuncture_nonlin's Robin call on u repeats what the last
  // sweep wrote (boundary values from the same inner values), so it is only
  // needed without pre-sweeps
  if (M->p.npre == 0) robin_u(M, h, h.u, done);
  fine_to_coarse_kernel<<<nblk(H.np + H.nb), RB, 0, M->stream>>>(h.u, h.f, h.a, h.b, H.u, H.f, H.v, h.m, H.m, off,
                                                                 cxof(h), robin_of(H, 0), done);
  coarse_rhs_kernel<<<nblk(H.np), RB, 0, M->stream>>>(H.u, H.f, H.v, H.w, H.a, H.b, H.m, cxof(H), done);
  vcycle(M, l - 1, done);
  // coarsetofine
  sub_inner_kernel<<<nblk(H.np + H.nb), RB, 0, M->stream>>>(H.u, H.w, H.v, H.m, robin_of(H, 1), done);
  prolong_add_kernel<<<nblk(h.np), RB, 0, M->stream>>>(H.v, h.u, h.m, H.m, h.x0, h.dx, H.x0, H.dx, 1, done);
  robin_u(M, h, h.u, done);
  sweeps(M, h, M->p.npost, done);
  // an odd number of sweeps leaves u in the partner array: move it back so
  // that every cycle starts and ends on the same buffers (graph replay)
  if (h.u != u_entry) {
    copy_kernel<<<nblk(h.np), RB, 0, M->stream>>>(h.u, u_entry, h.np, done);
    std::swap(h.u, h.u2);
  }
}

// residual test of level l (restau): Robin on u, RMS of L u - f
static void restau(nrgpu_mg *M, int l, int count) {
  MgLevel &h = M->lv[l];
  const int *done = count ? &M->st->done : nullptr;
  robin_u(M, h, h.u, done);
  residual_partial_kernel<<<nblk(h.np), RB, 0, M->stream>>>(h.u, h.f, h.a, h.b, h.m, cxof(h), M->partial, done);
  residual_final_kernel<<<1, 1024, 0, M->stream>>>(M->partial, (int)nblk(h.np), (long)(h.m - 2) * (h.m - 2) * (h.m - 2),
                                                  M->st, M->p.tol, count, M->p.vcycle_nmax);
}

extern "C" int nrgpu_mg_solve(nrgpu_mg *M, const double *a, const double *b, double *u, int *ncycles, double *normres,
                              void *stream) {
  if (!M || !a || !b || !u) return nrgpu_set_error(NRGPU_ERR_ARG, "null multigrid argument");
  if (M->p.vcycle_nmin != 0) return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "mg_vcycle_nmin must be 0");
  // the caller's stream is drained first; the solve runs on the solver's own
  // stream, which can be captured into CUDA graphs
  NRGPU_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  const int top = M->nl - 1;
  MgLevel &T = M->lv[top];
  const size_t by = sizeof(double) * T.np;
  NRGPU_CUDA_TRY(cudaMemcpyAsync(T.u, u, by, cudaMemcpyDeviceToDevice, M->stream));
  NRGPU_CUDA_TRY(cudaMemcpyAsync(T.a, a, by, cudaMemcpyDeviceToDevice, M->stream));
  NRGPU_CUDA_TRY(cudaMemcpyAsync(T.b, b, by, cudaMemcpyDeviceToDevice, M->stream));
  // initializestack: restrict coefficients and u down the stack; v, w, f = 0
  for (int l = top; l > 0; --l) {
    MgLevel &h = M->lv[l], &H = M->lv[l - 1];
    const int off = kChildOff;
    restrict_kernel<<<nblk(H.np), RB, 0, M->stream>>>(h.a, H.a, h.m, H.m, off, kNoRobin, nullptr);
    restrict_kernel<<<nblk(H.np), RB, 0, M->stream>>>(h.b, H.b, h.m, H.m, off, kNoRobin, nullptr);
    restrict_kernel<<<nblk(H.np), RB, 0, M->stream>>>(h.u, H.u, h.m, H.m, off, kNoRobin, nullptr);
  }
  for (int l = 0; l <= top; ++l) {
    MgLevel &L = M->lv[l];
    cudaMemsetAsync(L.v, 0, sizeof(double) * L.np, M->stream);
    cudaMemsetAsync(L.w, 0, sizeof(double) * L.np, M->stream);
    cudaMemsetAsync(L.f, 0, sizeof(double) * L.np, M->stream);
  }
  MgStatus h_st;
  const int batch = M->p.batch;
  for (int l = M->p.fullV ? 0 : top; l <= top; ++l) {
    NRGPU_CUDA_TRY(cudaMemsetAsync(M->st, 0, sizeof(MgStatus), M->stream));
    if (l == 0) {
      // the coarsest level is tested once and, unless the test passes,
      // solved once (solve.c:56-91: "for l == 0, solve is exact")
      restau(M, 0, 1);
      vcycle(M, 0, nullptr);
    } else {
      // V cycles in batches: test, cycle, test, cycle, ... ; the device flag
      // turns the rest of a batch into no-ops once the test passes
      int cycles = 0;
      for (;;) {
        if (!M->exec[l]) {
          cudaGraph_t g;
          NRGPU_CUDA_TRY(cudaStreamBeginCapture(M->stream, cudaStreamCaptureModeThreadLocal));
          for (int s = 0; s < batch; ++s) {
            restau(M, l, 1);
            vcycle(M, l, &M->st->done);
          }
          NRGPU_CUDA_TRY(cudaStreamEndCapture(M->stream, &g));
          M->graph[l] = g;
          NRGPU_CUDA_TRY(cudaGraphInstantiate(&M->exec[l], g, 0));
        }
        NRGPU_CUDA_TRY(cudaGraphLaunch(M->exec[l], M->stream));
        NRGPU_CUDA_TRY(cudaMemcpyAsync(&h_st, M->st, sizeof h_st, cudaMemcpyDeviceToHost, M->stream));
        NRGPU_CUDA_TRY(cudaStreamSynchronize(M->stream));
        cycles = h_st.ncycles;
        if (h_st.done) break;
      }
      if (l == top) {
        if (ncycles) *ncycles = cycles;
        if (normres) *normres = h_st.res;
      }
    }
    if (l < top) {
      // prolong_u: trilinear onto the inner points of the next level, Robin
      MgLevel &H = M->lv[l], &h = M->lv[l + 1];
      prolong_add_kernel<<<nblk(h.np), RB, 0, M->stream>>>(H.u, h.u, h.m, H.m, h.x0, h.dx, H.x0, H.dx, 0, nullptr);
      robin_u(M, h, h.u, nullptr);
    }
  }
  NRGPU_CUDA_TRY(cudaMemcpyAsync(u, T.u, by, cudaMemcpyDeviceToDevice, M->stream));
  NRGPU_CUDA_TRY(cudaStreamSynchronize(M->stream));
  NRGPU_CUDA_TRY(cudaGetLastError());
  // like the reference, running out of V cycles is not an error: the caller
  // sees ncycles == vcycle_nmax and normres > tol
  return NRGPU_OK;
}

extern "C" int nrgpu_mg_smooth(nrgpu_mg *M, const double *a, const double *b, double *u, int nsweeps, double omega,
                               void *stream) {
  if (!M || !a || !b || !u || nsweeps < 0 || !(omega > 0.0 && omega <= 1.0))
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad smoothing arguments (nsweeps >= 0, 0 < omega <= 1)");
  NRGPU_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  MgLevel &T = M->lv[M->nl - 1];
  const size_t by = sizeof(double) * T.np;
  NRGPU_CUDA_TRY(cudaMemcpyAsync(T.u, u, by, cudaMemcpyDeviceToDevice, M->stream));
  NRGPU_CUDA_TRY(cudaMemcpyAsync(T.a, a, by, cudaMemcpyDeviceToDevice, M->stream));
  NRGPU_CUDA_TRY(cudaMemcpyAsync(T.b, b, by, cudaMemcpyDeviceToDevice, M->stream));
  NRGPU_CUDA_TRY(cudaMemsetAsync(T.f, 0, by, M->stream));
  for (int s = 0; s < nsweeps; ++s) {
    damped_jacobi_kernel<<<nblk(T.np + T.nb), RB, 0, M->stream>>>(T.u, T.u2, T.f, T.a, T.b, T.m, cxof(T), omega,
                                                                   robin_of(T, 0));
    std::swap(T.u, T.u2);
  }
  NRGPU_CUDA_TRY(cudaMemcpyAsync(u, T.u, by, cudaMemcpyDeviceToDevice, M->stream));
  NRGPU_CUDA_TRY(cudaStreamSynchronize(M->stream));
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}

extern "C" int nrgpu_puncture_coefficients(int m, double dx, int npunc, const double *mass, const double *pos,
                                           const double *mom, const double *spin, double *a, double *b, void *stream) {
  if (m < 2 || npunc < 1 || npunc > 8 || !mass || !pos || !mom || !spin || !a || !b)
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad puncture arguments (1..8 punctures)");
  Punctures P;
  memset(&P, 0, sizeof P);
  P.n = npunc;
  for (int n = 0; n < npunc; ++n) {
    P.mass[n] = mass[n];
    for (int c = 0; c < 3; ++c) {
      P.pos[n][c] = pos[3 * n + c];
      P.mom[n][c] = mom[3 * n + c];
      P.spin[n][c] = spin[3 * n + c];
    }
  }
  coefficients_kernel<<<nblk((long)m * m * m), RB, 0, (cudaStream_t)stream>>>(P, m, dx, a, b);
  NRGPU_CUDA_TRY(cudaGetLastError());
  return NRGPU_OK;
}
