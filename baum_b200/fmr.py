"""Host-side mirror of the reference's mesh refinement around the evolution.

``Hierarchy`` holds the nested boxes of a grid (one or several separate
boxes per level, each made of whole cells of the coarser box that holds it:
the single-rank grid of amr = bo newfmr, amr_fmr = nestedboxes) on the device and advances them by coarse steps:
advance_levelandsublevels (main.c:397-418) with the time interpolation of
evolve (evolve.c:292-340, 371-380) and restrict_prolong_evolve
(inject.c:116-132).  ``restrict_prolong_varlist`` is inject.c:63-100 with
nbuffer 3.  All arithmetic runs in libnrgpu.so (nrgpu_fmr_*).
"""
import ctypes as C

import numpy as np
import torch

from . import abi
from .bssn import _ptrs, _stream


class Hierarchy:
    def __init__(self, levels, dt, sysparams, params=None):
        """levels: abi.Level per level, coarsest first; dt: per-level time
        steps; sysparams: per-level abi.BssnParams or abi.Z4Params."""
        self.levels = list(levels)  # regrid replaces entries of this copy
        self.params = params or abi.fmr_params(
            system=abi.SYSTEM_BSSN if isinstance(sysparams[0], abi.BssnParams) else abi.SYSTEM_Z4C)
        self.nv = abi.NVARS if self.params.system == abi.SYSTEM_BSSN else abi.Z4_NVARS
        nl = len(levels)
        self._descs = (abi.LevelDesc * nl)(*[lv.desc for lv in levels])
        self.dt = list(dt)
        self._dt = (C.c_double * nl)(*dt)
        self._sp = (type(sysparams[0]) * nl)(*sysparams)
        h = C.c_void_p()
        abi.check(abi.lib().nrgpu_fmr_create(nl, self._descs, self._dt, C.cast(self._sp, C.c_void_p),
                                             C.byref(self.params), C.byref(h)))
        self.handle = h
        self._uptrs = None

    def empty(self):
        """One zero (nvars, npoints) float64 CUDA tensor per level."""
        return [torch.zeros((self.nv, lv.npoints), dtype=torch.float64, device="cuda") for lv in self.levels]

    def flags(self, l):
        """(flagprolong, flagrestrict) of level l as numpy arrays."""
        n = self.levels[l].npoints
        fp, fr = np.zeros(n), np.zeros(n)
        dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
        abi.check(abi.lib().nrgpu_fmr_flags(self.handle, l, dp(fp), dp(fr)))
        return fp, fr

    def restrict_prolong_varlist(self, lfine, uc, uf, stream=None):
        abi.check(abi.lib().nrgpu_fmr_restrict_prolong(self.handle, lfine, _ptrs(uc, self.nv), _ptrs(uf, self.nv),
                                                       _stream(stream)))

    def restrict_prolong_vars(self, lfine, uc, uf, stream=None):
        """restrict_prolong_varlist with nbuffer 3 on other variables
        (set_boundary_refinement_cf, inject.c:179-189): uc, uf of shape
        (nvars, npoints) on levels lfine - 1 and lfine."""
        nv = uc.shape[0]
        abi.check(abi.lib().nrgpu_fmr_restrict_prolong_vars(self.handle, int(lfine), nv, _ptrs(uc, nv),
                                                            _ptrs(uf, nv), _stream(stream)))

    def advance(self, u, nsteps=1, stream=None):
        """nsteps coarse steps of the per-level states u (list of tensors)."""
        ptrs = [t.data_ptr() + v * t.stride(0) * 8 for t in u for v in range(self.nv)]
        for t in u:
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and t.shape[0] == self.nv):
                raise ValueError("each level state is a contiguous float64 CUDA tensor (nvars, npoints)")
        self._uptrs = abi.ptr_array(ptrs)
        self.move_error = None
        status = abi.lib().nrgpu_fmr_advance(self.handle, self._uptrs, int(nsteps), _stream(stream))
        if self.move_error is not None:
            raise self.move_error
        abi.check(status)
        return u

    def regrid(self, lmin, new_levels, u, stream=None):
        """Move levels lmin.. to new boxes (nrgpu_fmr_regrid; move_box,
        move.c:808-986): new_levels[i] is an abi.Level for level lmin + i, or
        None to keep it.  The moved levels' states in u (the list given to
        advance) are replaced by new tensors holding the moved data; inside
        a move hook the pointer table of the running advance is updated
        too."""
        nl = len(new_levels)
        descs = (abi.LevelDesc * nl)()
        fresh = []
        for i, lv in enumerate(new_levels):
            if lv is None:
                descs[i].nboxes = 0
                fresh.append(None)
            else:
                descs[i] = lv.desc
                fresh.append(torch.empty((self.nv, lv.npoints), dtype=torch.float64, device="cuda"))
        cur = [t.data_ptr() + v * t.stride(0) * 8 for t in u for v in range(self.nv)]
        new = []
        for t in fresh:
            new += [0] * self.nv if t is None else [t.data_ptr() + v * t.stride(0) * 8 for v in range(self.nv)]
        self._keep = (descs, new_levels)
        # inside a move hook the stream arrives as the raw handle
        st = C.c_void_p(stream) if isinstance(stream, int) else _stream(stream)
        abi.check(abi.lib().nrgpu_fmr_regrid(self.handle, int(lmin), nl, descs, abi.ptr_array(cur),
                                             abi.ptr_array(new), st))
        for i, t in enumerate(fresh):
            if t is None:
                continue
            l = lmin + i
            u[l] = t
            self.levels[l] = new_levels[i]
            if self._uptrs is not None:
                for v in range(self.nv):
                    self._uptrs[l * self.nv + v] = t.data_ptr() + v * t.stride(0) * 8
        return u

    def set_move(self, fn):
        """fn(l, stream) is called where the reference calls move_box(g, l)
        during advance (nrgpu_fmr_set_move); it may call regrid(l.., ...) on
        the list being advanced.  None removes it."""
        if fn is None:
            self._move = None
            abi.check(abi.lib().nrgpu_fmr_set_move(self.handle, None, None))
            return

        def hook(user, fmr, l, stream):
            try:
                fn(int(l), stream)
                return 0
            except Exception as e:  # reported as an error of the advance
                self.move_error = e
                return -1  # NRGPU_ERR_ARG
        self._move = abi.FMR_MOVE_FN(hook)
        abi.check(abi.lib().nrgpu_fmr_set_move(self.handle, C.cast(self._move, C.c_void_p), None))

    def iteration(self, l):
        return abi.lib().nrgpu_fmr_iteration(self.handle, l)

    def block(self, l):
        """The rhs block shape (x, y, z) level l runs with (128 threads)."""
        b = (C.c_int * 3)()
        abi.check(abi.lib().nrgpu_fmr_block(self.handle, l, b))
        return tuple(b)

    def save(self):
        """The hierarchy's own state (iteration counters, previous-step
        copies, time interpolants) as a numpy byte array (nrgpu_fmr_save)."""
        n = C.c_size_t()
        abi.check(abi.lib().nrgpu_fmr_state_size(self.handle, C.byref(n)))
        buf = np.empty(n.value, dtype=np.uint8)
        abi.check(abi.lib().nrgpu_fmr_save(self.handle, buf.ctypes.data, n.value))
        return buf

    def load(self, buf):
        """Restore a state written by save() (nrgpu_fmr_load)."""
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        abi.check(abi.lib().nrgpu_fmr_load(self.handle, buf.ctypes.data, buf.size))

    def track(self, positions, fixz=False):
        """Track punctures from these start positions (n x 3) on the finest
        level during the following steps (nrgpu_fmr_track; track_puncture
        with the shift integrator); an empty list stops tracking."""
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        abi.check(abi.lib().nrgpu_fmr_track(self.handle, pos.shape[0],
                                            pos.ctypes.data_as(C.POINTER(C.c_double)), int(bool(fixz))))
        self.ntrack = pos.shape[0]

    TRACK_METHODS = {"ext": 0, "int": 1, "extint": 2}

    def track_method(self, method="int", var=None, find_max=False, minmove=0.01, fixz_ext=False):
        """The tracker per puncture (nrgpu_fmr_track_method,
        moving_puncture_track_method): "int" (the shift integrator), "ext"
        (the extremum search of variable var, the lapse by default, for every
        puncture) or "extint" (the search for the first puncture, the
        integrator for the rest)."""
        if var is None:
            var = 17 if self.params.system == abi.SYSTEM_BSSN else 18
        abi.check(abi.lib().nrgpu_fmr_track_method(self.handle, self.TRACK_METHODS[method], int(var),
                                                   int(bool(find_max)), float(minmove), int(bool(fixz_ext))))

    def punctures(self):
        """(positions n x 3, status per puncture) of the tracked punctures
        (nrgpu_fmr_punctures): bit 0 the last step integrated, bit 1 the new
        position lay on the level and was taken."""
        n = getattr(self, "ntrack", 0)
        pos = np.empty((n, 3))
        st = np.empty(n, dtype=np.int32)
        abi.check(abi.lib().nrgpu_fmr_punctures(self.handle, pos.ctypes.data_as(C.POINTER(C.c_double)),
                                                st.ctypes.data_as(C.POINTER(C.c_int))))
        return pos, st

    def close(self):
        if self.handle:
            abi.lib().nrgpu_fmr_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def nested_levels(sizes, dx0):
    """Boxes of a nested grid centred on the origin: sizes[l] points per
    direction on level l (level 0 with its physical boundary layer, 4n+2,
    grid.c:84-99; finer levels multiples of 4, so that each is made of whole
    parent cells), spacing dx0 / 2^l.  Flags as the reference sets them:
    PHYBOUND on the outer layer of level 0, REFBOUND on the outer layer of
    finer levels (box.c:543-552)."""
    out = []
    for l, m in enumerate(sizes):
        if l == 0 and m % 4 != 2:
            raise ValueError("level 0 has 4n+2 points per direction")
        if l > 0 and (m % 4 or m // 2 + 6 > sizes[l - 1]):
            raise ValueError("level %d: a multiple of 4 that nests in level %d with room for the stencils" % (l, l - 1))
        dx = dx0 / 2 ** l
        x0 = -0.5 * (m - 1) * dx
        i = np.arange(m)
        edge = (i == 0) | (i == m - 1)
        e3 = edge[None, None, :] | edge[None, :, None] | edge[:, None, None]
        flags = np.where(e3, 1 if l == 0 else -1, 0).astype(np.int32).ravel()
        out.append(abi.Level([(m, m, m, x0, x0, x0)], dx, flags))
    return out
