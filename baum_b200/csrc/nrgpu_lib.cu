// nrgpu_lib.cu -- library state, errors, level mirrors and host-buffer calls.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "nrgpu_level.cuh"

static thread_local char g_err[512] = "";

int nrgpu_set_error(int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
  return code;
}

extern "C" int nrgpu_abi_version(void) { return NRGPU_ABI_VERSION; }

extern "C" const char *nrgpu_last_error(void) { return g_err; }

extern "C" int nrgpu_init(int device) {
  int n = 0;
  NRGPU_CUDA_TRY(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return nrgpu_set_error(NRGPU_ERR_ARG, "device %d of %d", device, n);
  NRGPU_CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  NRGPU_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED, "built for sm_100a, device is sm_%d%d",
                                               prop.major, prop.minor);
  return NRGPU_OK;
}

extern "C" void nrgpu_bssn_params_default(nrgpu_bssn_params *p) {
  if (!p) return;
  memset(p, 0, sizeof *p);
  p->order_centered = 4;
  p->order_advection = 4;
  p->advection_lopsided = 1;
  p->advection_lopsided6 = 3;  // reference default (bam_amr.c:52)
  p->order_dissipation = 6;
  p->dissfactor = 0.1 / 64.0;  // dissipation_factor / 2^order_dissipation (evolve.c:503)
  p->forceKzerofactor = 1.0;   // Getv("bssn_forceKzero","no") for the default "no"
  p->subtractA = 1;
  p->normalizedetg = 1;
  p->oploglapse = 1;
  p->oplogwithshift = 1;
  p->gamma0factor = 1.0;
  p->withGadv = p->withShiftadv = p->withBadv = p->withB = 1.0;
  p->lapseharmonicf = 2.0;
  p->shiftgammacoeff = 0.75;
  p->shiftdriver = 2.0;
  p->chiDivFloor = -1000.0;
  p->chipsipower = -4.0;
  // VarNameSetBoundaryInfo (bssn.c:269-311); gauge speed sqrt(2) for 1+log
  const double vg = 1.4142135623730951;
  for (int v = 0; v < NRGPU_BSSN_NVARS; ++v) { p->bc_var0[v] = 0.0; p->bc_speed[v] = 1.0; }
  const int unit[5] = {0, 3, 5, 6, 17};
  for (int i = 0; i < 5; ++i) p->bc_var0[unit[i]] = 1.0;
  p->bc_speed[13] = p->bc_speed[6] = p->bc_speed[17] = vg;
}

extern "C" int nrgpu_level_create(const nrgpu_level_desc *d, nrgpu_level **out) {
  if (!d || !out || !d->box || !d->boundary || d->nboxes < 1 || d->npoints < 1)
    return nrgpu_set_error(NRGPU_ERR_ARG, "bad level description");
  long total = 0;
  for (int b = 0; b < d->nboxes; ++b) {
    const nrgpu_box &bx = d->box[b];
    if (bx.m < 1 || bx.n < 1 || bx.o < 1 || bx.noffset != total)
      return nrgpu_set_error(NRGPU_ERR_ARG, "box %d: bad size or offset", b);
    total += (long)bx.m * bx.n * bx.o;
  }
  if (total != d->npoints || total > 0x7fffffffL)
    return nrgpu_set_error(NRGPU_ERR_ARG, "npoints %d does not match the boxes (%ld)", d->npoints, total);
  std::vector<FlagPoint> fl;
  for (int b = 0; b < d->nboxes; ++b) {
    const nrgpu_box &bx = d->box[b];
    for (int k = 0; k < bx.o; ++k)
      for (int j = 0; j < bx.n; ++j)
        for (int i = 0; i < bx.m; ++i) {
          const int ijk = bx.noffset + i + bx.m * (j + bx.n * k);
          const int f = d->boundary[ijk];
          if (f == 0) continue;
          if (f != NRGPU_PHYBOUND && f != NRGPU_REFBOUND && !(f == NRGPU_SYMBOUND && d->symmetry))
            return nrgpu_set_error(NRGPU_ERR_UNSUPPORTED,
                                   "boundary flag %d at point %d (0, PHYBOUND, REFBOUND, SYMBOUND with symmetry)", f,
                                   ijk);
          fl.push_back(FlagPoint{ijk, i, j, k, b, f});
        }
  }
  // flag-0 points within 2 of their box's faces, by distance: the interior
  // kernels compute the points where the full stencil order fits, a list
  // kernel the others (boundaryNaway ladder, bam_amr_loops_box.h:215-220)
  std::vector<FlagPoint> lad[3];
  for (int b = 0; b < d->nboxes; ++b) {
    const nrgpu_box &bx = d->box[b];
    for (int k = 0; k < bx.o; ++k)
      for (int j = 0; j < bx.n; ++j)
        for (int i = 0; i < bx.m; ++i) {
          const int dd = std::min(std::min(std::min(i, j), k), std::min(std::min(bx.m - 1 - i, bx.n - 1 - j),
                                                                         bx.o - 1 - k));
          if (dd > 2) continue;
          const int ijk = bx.noffset + i + bx.m * (j + bx.n * k);
          if (d->boundary[ijk] != 0) continue;
          lad[dd].push_back(FlagPoint{ijk, i, j, k, b, dd});
        }
  }
  std::vector<FlagPoint> ladder;
  int nlad[3];
  for (int q = 0; q < 3; ++q) {
    ladder.insert(ladder.end(), lad[q].begin(), lad[q].end());
    nlad[q] = (int)ladder.size();
  }
  // symmetry ghosts: set_boundary_reflection_one (symmetry.c:28-82) copies the
  // nneg = (int)(1 - lo / h) planes below zero from planes 2 nneg - 1 - n, axis
  // after axis; the result is the mirror image with the product of parities
  if (d->symmetry < 0 || d->symmetry > 7) return nrgpu_set_error(NRGPU_ERR_ARG, "symmetry mask %d", d->symmetry);
  std::vector<SymPoint> sym;
  for (int b = 0; b < d->nboxes && d->symmetry; ++b) {
    const nrgpu_box &bx = d->box[b];
    const int n3[3] = {bx.m, bx.n, bx.o};
    const double lo[3] = {bx.x0, bx.y0, bx.z0}, h[3] = {d->dx, d->dy, d->dz};
    int nneg[3];
    for (int a = 0; a < 3; ++a) {
      nneg[a] = (d->symmetry >> a & 1) && lo[a] < 0 ? (int)(1 - lo[a] / h[a]) : 0;
      if (2 * nneg[a] > n3[a]) return nrgpu_set_error(NRGPU_ERR_ARG, "box %d: no mirror for the symmetry ghosts", b);
    }
    for (int k = 0; k < bx.o; ++k)
      for (int j = 0; j < bx.n; ++j)
        for (int i = 0; i < bx.m; ++i) {
          int idx[3] = {i, j, k}, src[3] = {i, j, k}, mask = 0;
          for (int a = 0; a < 3; ++a)
            if (idx[a] < nneg[a]) {
              mask |= 1 << a;
              src[a] = 2 * nneg[a] - 1 - idx[a];
            }
          if (!mask) continue;
          sym.push_back(SymPoint{bx.noffset + i + bx.m * (j + bx.n * k),
                                 bx.noffset + src[0] + bx.m * (src[1] + bx.n * src[2]), mask});
        }
  }
  nrgpu_level *L = (nrgpu_level *)calloc(1, sizeof(nrgpu_level));
  if (!L) return nrgpu_set_error(NRGPU_ERR_NOMEM, "host allocation");
  cudaGetDevice(&L->device);
  L->nboxes = d->nboxes;
  L->npoints = d->npoints;
  L->dx = d->dx; L->dy = d->dy; L->dz = d->dz;
  L->hbox = (BoxGeo *)malloc(sizeof(BoxGeo) * d->nboxes);
  for (int b = 0; b < d->nboxes; ++b)
    L->hbox[b] = BoxGeo{d->box[b].m, d->box[b].n, d->box[b].o, d->box[b].noffset, d->box[b].x0, d->box[b].y0,
                        d->box[b].z0};
  L->nflagpts = (int)fl.size();
  for (int q = 0; q < 3; ++q) L->nladder[q] = nlad[q];
  L->ninner = (long)d->npoints - (long)fl.size();
  L->blk[0] = 32; L->blk[1] = 4; L->blk[2] = 1;
  if (cudaDeviceGetAttribute(&L->nsm, cudaDevAttrMultiProcessorCount, L->device) != cudaSuccess || L->nsm < 1)
    L->nsm = 148;
  L->symmetry = d->symmetry;
  L->nsym = (int)sym.size();
  bool ok = cudaMalloc(&L->d_boundary, sizeof(int) * d->npoints) == cudaSuccess &&
            cudaMalloc(&L->d_box, sizeof(BoxGeo) * d->nboxes) == cudaSuccess &&
            cudaMalloc(&L->d_status, sizeof(int) * 4) == cudaSuccess &&
            (fl.empty() || cudaMalloc(&L->d_flagpts, sizeof(FlagPoint) * fl.size()) == cudaSuccess) &&
            (ladder.empty() || cudaMalloc(&L->d_ladder, sizeof(FlagPoint) * ladder.size()) == cudaSuccess) &&
            (sym.empty() || cudaMalloc(&L->d_sym, sizeof(SymPoint) * sym.size()) == cudaSuccess);
  if (ok)
    ok = cudaMemcpy(L->d_boundary, d->boundary, sizeof(int) * d->npoints, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(L->d_box, L->hbox, sizeof(BoxGeo) * d->nboxes, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(L->d_status, 0, sizeof(int) * 4) == cudaSuccess &&
         (fl.empty() ||
          cudaMemcpy(L->d_flagpts, fl.data(), sizeof(FlagPoint) * fl.size(), cudaMemcpyHostToDevice) == cudaSuccess) &&
         (ladder.empty() || cudaMemcpy(L->d_ladder, ladder.data(), sizeof(FlagPoint) * ladder.size(),
                                       cudaMemcpyHostToDevice) == cudaSuccess) &&
         (sym.empty() ||
          cudaMemcpy(L->d_sym, sym.data(), sizeof(SymPoint) * sym.size(), cudaMemcpyHostToDevice) == cudaSuccess);
  if (!ok) {
    nrgpu_level_destroy(L);
    return nrgpu_set_error(NRGPU_ERR_NOMEM, "device allocation of the level mirror failed");
  }
  *out = L;
  return NRGPU_OK;
}

extern "C" int nrgpu_level_destroy(nrgpu_level *L) {
  if (!L) return NRGPU_OK;
  cudaFree(L->d_boundary);
  cudaFree(L->d_box);
  cudaFree(L->d_status);
  cudaFree(L->d_flagpts);
  cudaFree(L->d_ladder);
  cudaFree(L->d_sym);
  cudaFree(L->rsym);
  cudaFree(L->scratch);
  cudaFree(L->pad);
  cudaFree(L->hoststate);
  cudaFree(L->d_red);
  cudaFree(L->d_red0d);
  for (int q = 0; q < NRGPU_HOST_SLABS; ++q) {
    if (L->hev_in[q]) cudaEventDestroy(L->hev_in[q]);
    if (L->hev_out[q]) cudaEventDestroy(L->hev_out[q]);
  }
  if (L->side) cudaStreamDestroy(L->side);
  if (L->ev_fork) cudaEventDestroy(L->ev_fork);
  if (L->ev_join) cudaEventDestroy(L->ev_join);
  if (L->hs_copy) cudaStreamDestroy(L->hs_copy);
  if (L->hs_comp) cudaStreamDestroy(L->hs_comp);
  free(L->tma_cache);
  free(L->hbox);
  free(L);
  return NRGPU_OK;
}

// three variable lists of RK4 scratch (room for the 25 Z4c variables),
// allocated once per level
// the staging buffer for boxes of up to 194 points per side without a
// compile-time-stride kernel of their own: 25 lists with strides (1, P, P P),
// P the next kernel size (kPadSizes); tried once per level, and a level
// without it runs those boxes with the run-time-stride kernel
void nrgpu_level_pad(nrgpu_level *L) {
  if (L->pad_tried) return;
  L->pad_tried = 1;
  size_t need = 0;
  for (int b = 0; b < L->nboxes; ++b) {
    const int P = nrgpu_pad_size(L->hbox[b].m, L->hbox[b].n);
    if (P > 0) need = std::max(need, (size_t)NRGPU_Z4_NVARS * P * P * L->hbox[b].o);
  }
  if (need && cudaMalloc(&L->pad, sizeof(double) * need) == cudaSuccess) {
    L->pad_doubles = need;
  } else {
    cudaGetLastError();
    L->pad = nullptr;
    L->pad_doubles = 0;
  }
}

int nrgpu_level_scratch(nrgpu_level *L, double **out) {
  if (!L->scratch) {
    const size_t bytes = sizeof(double) * 3 * NRGPU_Z4_NVARS * (size_t)L->npoints;
    if (cudaMalloc(&L->scratch, bytes) != cudaSuccess) {
      L->scratch = nullptr;
      cudaGetLastError();
      return nrgpu_set_error(NRGPU_ERR_NOMEM, "RK4 scratch of %zu bytes", bytes);
    }
    L->scratch_points = (size_t)L->npoints;
    nrgpu_level_pad(L);
  }
  *out = L->scratch;
  return NRGPU_OK;
}

int nrgpu_level_side(nrgpu_level *L) {
  if (L->side) return NRGPU_OK;
  NRGPU_CUDA_TRY(cudaStreamCreateWithFlags(&L->side, cudaStreamNonBlocking));
  NRGPU_CUDA_TRY(cudaEventCreateWithFlags(&L->ev_fork, cudaEventDisableTiming));
  NRGPU_CUDA_TRY(cudaEventCreateWithFlags(&L->ev_join, cudaEventDisableTiming));
  return NRGPU_OK;
}

extern "C" int nrgpu_level_nan_flag(nrgpu_level *L, int *flag) {
  if (!L || !flag) return nrgpu_set_error(NRGPU_ERR_ARG, "null argument");
  int h[2] = {0, 0};
  NRGPU_CUDA_TRY(cudaMemcpy(h, L->d_status, sizeof h, cudaMemcpyDeviceToHost));
  NRGPU_CUDA_TRY(cudaMemset(L->d_status, 0, sizeof h));
  *flag = h[0] & 1;
  if (h[0] & 2) return nrgpu_set_error(NRGPU_ERR_TIMEOUT, "a wait for a staged tile ran out of time");
  if (h[1]) return nrgpu_set_error(NRGPU_ERR_ARG, "an inner point had no room for its stencil");
  return NRGPU_OK;
}

