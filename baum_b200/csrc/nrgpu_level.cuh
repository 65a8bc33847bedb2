// nrgpu_level.cuh -- device mirror of a BAM level (tL, bam_amr.h:46-74).
#pragma once
#include "nrgpu_common.cuh"

// one point with a non-zero boundary flag: linear index, box-local ijk,
// box number and flag; the boundary kernels walk this list
struct FlagPoint {
  int ijk, i, j, k;
  int box, flag;
};

// z slabs of the pipelined host-buffer step (nrgpu_bssn_evolve_host)
#define NRGPU_HOST_SLABS 8

// a symmetry ghost (SYMBOUND point), its mirror image and the reflected
// axes (bit 0 x, 1 y, 2 z): the value is the mirror's times the variable's
// parity under those reflections
struct SymPoint {
  int dst, src, mask;
};

struct nrgpu_level {
  int device;
  int nboxes;
  int npoints;
  double dx, dy, dz;
  BoxGeo *hbox;            // host copy of the boxes
  int *d_boundary;         // [npoints] flags on the device
  FlagPoint *d_flagpts;    // points with flag != 0
  int nflagpts;
  // flag-0 points within 2 of a box face (the order ladder: lower-order
  // stencils there), sorted by that distance d (FlagPoint.flag = d);
  // nladder[d] = points with distance <= d
  FlagPoint *d_ladder;
  int nladder[3];
  BoxGeo *d_box;           // boxes on the device
  int *d_status;           // [0]: NaN flag, [1]: inner point without stencil room
  // RK4 scratch: three full 24-variable lists, allocated on first use
  double *scratch;
  size_t scratch_points;
  // staging buffer of a box whose size has no compile-time-stride kernel
  // (pad_copy_kernel), allocated with the scratch when a box needs it
  double *pad;
  size_t pad_doubles;
  int pad_tried;
  // device copy of a host state for the host-buffer entry points
  double *hoststate;
  // points with boundary flag 0, and the norm reduction buffer (first use)
  long ninner;
  double *d_red;
  // partials and results of the 0d output reductions (first use)
  double *d_red0d;
  // extents of the rhs kernels' 128-thread blocks (x, y, z)
  int blk[3];
  // reflection symmetry: the axes (desc.symmetry), the ghost list, and the
  // rhs list of the unfused RK stages of a symmetry grid (first use)
  int symmetry, nsym;
  SymPoint *d_sym;
  double *rsym;
  // side stream of the boundary kernel, which runs beside the interior
  // kernel of the same stage (first use)
  cudaStream_t side;
  cudaEvent_t ev_fork, ev_join;
  // copy and compute streams, and per-slab events, of the pipelined
  // host-buffer step (created on first use)
  cudaStream_t hs_copy, hs_comp;
  cudaEvent_t hev_in[NRGPU_HOST_SLABS], hev_out[NRGPU_HOST_SLABS];
  // interior rhs over TMA-staged tiles (1) instead of per-point global
  // loads (0), where the level and the parameters allow it; the tensor maps
  // of recently used variable lists (host memory, first use)
  int tile;
  // 1: the Z4c interior of all boxes in one persistent launch over a queue
  // of tiles (nrgpu_level_queue), where the boxes allow it
  int queue;
  void *tma_cache;
  int nsm;   // multiprocessors of the level's device
};

// library-internal pieces shared by the entry points and the mesh-refinement
// driver (nrgpu_bssn.cu)
int nrgpu_bssn_rk4_stages(nrgpu_level *L, double *const *u, double dt, const nrgpu_bssn_params *p,
                          cudaStream_t st);
int nrgpu_z4_rk4_stages(nrgpu_level *L, double *const *u, double dt, const nrgpu_z4_params *p, cudaStream_t st);
int nrgpu_z4_algcon(nrgpu_level *L, double *const *u, const nrgpu_z4_params *p, cudaStream_t st);
// set_boundary's background branch for Z4c and the RK4 step that it needs
// (the state's copy kept apart from the extrapolated stage input)
// (nrgpu_z4bg.cu)
int nrgpu_z4_background_extrapolate(nrgpu_level *L, double *const *u, cudaStream_t st);
int nrgpu_z4_background_boundary(nrgpu_level *L, double *const *unew, double *const *upre, double c,
                                 double *const *ucur, const nrgpu_z4_params *p, cudaStream_t st);
int nrgpu_z4_rk4_background(nrgpu_level *L, double *const *u, double dt, const nrgpu_z4_params *p, cudaStream_t st);
// the level's three RK4 scratch lists, allocated on first use (nrgpu_lib.cu)
int nrgpu_level_scratch(nrgpu_level *L, double **out);
// the box sizes with a compile-time-stride Z4c rhs kernel; a box of another
// size up to the largest is staged into a copy with the strides of the next
// one (nrgpu_level_pad)
constexpr int kPadSizes[] = {66, 72, 104, 136, 162, 168, 194};
// the staging size of an m x n box: 0 when it has a kernel of its own or is
// too large
inline int nrgpu_pad_size(int m, int n) {
  if (m == n)
    for (int c : kPadSizes)
      if (c == m) return 0;
  for (int c : kPadSizes)
    if (c >= m && c >= n) return c;
  return 0;
}
void nrgpu_level_pad(nrgpu_level *L);
// set_boundary_symmetry on a list of nv variables of the given system
// (NRGPU_SYSTEM_BSSN / _Z4C); nothing without symmetry (nrgpu_bssn.cu)
int nrgpu_level_symmetry(nrgpu_level *L, double *const *u, int system, cudaStream_t st);
// the side stream of the boundary kernel (nrgpu_lib.cu)
int nrgpu_level_side(nrgpu_level *L);
// the two halves of a tracking step for a driver that keeps no copy of the
// previous shift: before the step the shift at the old positions into b1,
// after it the corrector passes from b1 (nrgpu_track.cu)
// the extremum search on the given stream (no device switch: graph capture)
int nrgpu_track_extremum_on(nrgpu_level *L, const double *var, int find_max, double minmove, int order, int fixz,
                            int n, double *pos, int *status, cudaStream_t st);
int nrgpu_track_before_step(nrgpu_level *L, const double *const *beta, int order, int n, const double *pos,
                            double *b1, cudaStream_t st);
int nrgpu_track_after_step(nrgpu_level *L, const double *const *beta, double dt, int order, int fixz, int n,
                           double *pos, const double *b1, int *status, cudaStream_t st);
