"""Loader for the CPU oracle (oracle/nr_oracle.c -> oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, never by the product package.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from baum_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "nr_oracle.c")
MGSRC = os.path.join(HERE, "mg_oracle.c")
ADMSRC = os.path.join(HERE, "adm_oracle.c")
FMRSRC = os.path.join(HERE, "fmr_oracle.c")
TRACKSRC = os.path.join(HERE, "track_oracle.c")


def build(force=False):
    """Compile the restatement with gcc (-O2, OpenMP, no fast-math)."""
    deps = [SRC, MGSRC, ADMSRC, FMRSRC, TRACKSRC, os.path.join(HERE, "..", "include", "nrgpu.h")]
    if not force and os.path.exists(SO) and all(os.path.getmtime(SO) >= os.path.getmtime(d) for d in deps):
        return SO
    cmd = ["gcc", "-O2", "-std=gnu99", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
           SRC, MGSRC, ADMSRC, FMRSRC, TRACKSRC, "-o", SO, "-lm"]
    subprocess.run(cmd, check=True)
    return SO


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(SO)
        pp = C.POINTER(C.c_void_p)
        LD = C.POINTER(abi.LevelDesc)
        BP = C.POINTER(abi.BssnParams)
        for name, args in {
            "oracle_bssn_rhs": [LD, pp, pp, C.c_double, pp, BP],
            "oracle_bssn_boundary": [LD, pp, pp, C.c_double, pp, BP],
            "oracle_bssn_algcon": [LD, pp, BP],
            "oracle_bssn_rk4_step": [LD, pp, C.c_double, BP],
            "oracle_bssn_evolve": [LD, pp, C.c_double, C.c_int, BP],
            "oracle_z4_rhs": [LD, pp, pp, C.c_double, pp, C.POINTER(abi.Z4Params)],
            "oracle_z4_boundary": [LD, pp, pp, C.c_double, pp, C.POINTER(abi.Z4Params)],
            "oracle_z4_evolve": [LD, pp, C.c_double, C.c_int, C.POINTER(abi.Z4Params)],
            "oracle_to_adm": [LD, pp, pp, C.c_double],
            "oracle_fmr_flags": [LD, LD, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)],
            "oracle_fmr_restrict_prolong": [LD, LD, C.c_int, pp, pp, C.c_int, C.c_int],
            "oracle_adm_constraints": [LD, pp, pp, C.c_int, C.c_int],
            "oracle_norms": [LD, pp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)],
            "oracle_track_extremum": [LD, C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                                      C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int)],
            "oracle_track_punctures": [LD, pp, pp, C.c_double, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int),
                                       C.POINTER(C.c_int)],
        }.items():
            f = getattr(L, name)
            f.restype = C.c_int
            f.argtypes = args
        _lib = L
    return _lib


def _ptrs(arr):
    """24 row pointers of a C-contiguous (24, npoints) float64 array."""
    assert arr.dtype == np.float64 and arr.flags.c_contiguous
    base = arr.ctypes.data
    stride = arr.strides[0]
    return abi.ptr_array([base + i * stride for i in range(arr.shape[0])])


def bssn_rhs(level, u, params, c=0.0, upre=None, out=None):
    """rhs (inner points) + radiative boundary of u[24, npoints] (c = 0)."""
    out = np.zeros_like(u) if out is None else out
    upre = u if upre is None else upre
    pu, pn, pp_ = _ptrs(u), _ptrs(out), _ptrs(upre)
    e = lib().oracle_bssn_rhs(C.byref(level.desc), pn, pp_, c, pu, C.byref(params))
    if e:
        raise RuntimeError("oracle rhs failed")
    lib().oracle_bssn_boundary(C.byref(level.desc), pn, pp_, c, pu, C.byref(params))
    return out


def bssn_evolve(level, u, dt, nsteps, params):
    """nsteps RK4 steps of u[24, npoints] in place."""
    e = lib().oracle_bssn_evolve(C.byref(level.desc), _ptrs(u), dt, nsteps, C.byref(params))
    if e:
        raise RuntimeError("oracle evolve failed")
    return u


def puncture_coefficients(m, dx, binary):
    """a, b of the oracle on the m^3 cube."""
    L = lib()
    n = m ** 3
    a = np.zeros(n)
    b = np.zeros(n)
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    L.oracle_puncture_coefficients(m, C.c_double(dx), len(binary.mass), dp(binary.mass), dp(binary.pos),
                                   dp(binary.mom), dp(binary.spin), dp(a), dp(b))
    return a, b


def mg_solve(m, dx, a, b, u=None, params=None):
    """The oracle multigrid; returns (u, V cycles, residual history)."""
    from baum_b200 import abi
    p = params or abi.mg_params()
    L = lib()
    u = np.zeros(m ** 3) if u is None else np.ascontiguousarray(u, dtype=np.float64).copy()
    hist = np.zeros(p.vcycle_nmax + 1)
    nl = C.c_int()
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    L.oracle_mg_solve.restype = C.c_int
    n = L.oracle_mg_solve(m, C.c_double(dx), dp(np.ascontiguousarray(a)), dp(np.ascontiguousarray(b)), dp(u),
                          p.npre, p.npost, p.exact_nmin, p.exact_nmax, p.vcycle_nmin, p.vcycle_nmax, p.fullV,
                          p.size_nmin, p.levels_nmax, C.c_double(p.tol), dp(hist), C.byref(nl))
    return u, n, hist[:n + 1]


def z4_rhs(level, u, params, c=0.0, upre=None, out=None):
    """Z4c rhs (inner points) + radiative boundary of u[25, npoints]."""
    out = np.zeros_like(u) if out is None else out
    upre = u if upre is None else upre
    pu, pn, pp_ = _ptrs(u), _ptrs(out), _ptrs(upre)
    if lib().oracle_z4_rhs(C.byref(level.desc), pn, pp_, c, pu, C.byref(params)):
        raise RuntimeError("oracle z4 rhs failed")
    lib().oracle_z4_boundary(C.byref(level.desc), pn, pp_, c, pu, C.byref(params))
    return out


def z4_evolve(level, u, dt, nsteps, params):
    if lib().oracle_z4_evolve(C.byref(level.desc), _ptrs(u), dt, nsteps, C.byref(params)):
        raise RuntimeError("oracle z4 evolve failed")
    return u


def to_adm(level, u, chipsipower=-4.0):
    """ADM g_ij, K_ij (12, npoints) from a BSSN or Z4c state (first 14 rows)."""
    adm = np.zeros((12, u.shape[1]))
    lib().oracle_to_adm(C.byref(level.desc), _ptrs(np.ascontiguousarray(u)), _ptrs(adm), chipsipower)
    return adm


def adm_constraints(level, adm, order_centered, mode=0, out=None):
    """ham, mom_i (and normham, normmom_i for mode 1 / 2 = term by term) on
    the flag-0 points; other points of out are left as they are."""
    nout = 8 if mode else 4
    out = np.zeros((nout, adm.shape[1])) if out is None else out
    if lib().oracle_adm_constraints(C.byref(level.desc), _ptrs(np.ascontiguousarray(adm)), _ptrs(out),
                                    order_centered, mode):
        raise RuntimeError("oracle constraints failed")
    return out


def norms(level, v):
    """(RMS, max |.|) of each row of v over the flag-0 points."""
    v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1, level.npoints)
    n2 = np.zeros(v.shape[0])
    ni = np.zeros(v.shape[0])
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    lib().oracle_norms(C.byref(level.desc), _ptrs(v), v.shape[0], dp(n2), dp(ni))
    return n2, ni


def fmr_flags(coarse, fine, nbuffer):
    """(flagprolong of the fine level, flagrestrict of the coarse level)."""
    fp = np.zeros(fine.npoints)
    cr = np.zeros(coarse.npoints)
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    if lib().oracle_fmr_flags(C.byref(coarse.desc), C.byref(fine.desc), nbuffer, dp(fp), dp(cr)):
        raise RuntimeError("fine level does not nest in the coarse one")
    return fp, cr


def fmr_restrict_prolong(coarse, fine, uc, uf, order=4, nbuffer=3):
    """restrict_prolong_varlist in place on uc (nv, npc) and uf (nv, npf)."""
    e = lib().oracle_fmr_restrict_prolong(C.byref(coarse.desc), C.byref(fine.desc), uc.shape[0], _ptrs(uc),
                                          _ptrs(uf), order, nbuffer)
    if e:
        raise RuntimeError("oracle restrict/prolong failed (%d)" % e)


class FmrState:
    """Host state of a multi-level evolution for the oracle driver: per
    level u, the previous step's copy and the time interpolant.

    advance() restates advance_levelandsublevels (main.c:397-418): step the
    level, then its child twice (once for levels below lbo), then restrict
    and prolong with the parent (restrict_prolong_evolve, inject.c:116-132;
    the parent's u when both are at the same time, parentaligned
    inject.c:10-21, else its time interpolant).  snap(l, iteration, u) is
    called right after each level step, where the reference's POST_EVOLVE
    functions run."""

    def __init__(self, levels, u0, system, params, dt, lbo=0, order_ti=3, order_rp=4, nbuffer=3):
        self.levels, self.system, self.params = levels, system, params
        self.nv = u0[0].shape[0]
        self.u = [np.ascontiguousarray(x, dtype=np.float64).copy() for x in u0]
        self.up = [np.zeros_like(x) for x in self.u]
        self.upp = [np.zeros_like(x) for x in self.u]
        # u(n-2), u(n-3), u(n-4) for time interpolation of orders 4-6
        self.hist = [[np.zeros_like(x) for _ in range(max(0, order_ti - 3))] for x in self.u]
        self.dt = [float(x) for x in dt]
        self.iteration = [0] * len(levels)
        self.lbo, self.order_ti, self.order_rp, self.nbuffer = lbo, order_ti, order_rp, nbuffer

    def step_level(self, l):
        f = lib().oracle_fmr_evolve_level_h
        f.restype = C.c_int
        child = l < len(self.levels) - 1
        h = [_ptrs(x) for x in self.hist[l]] + [None] * (3 - len(self.hist[l]))
        e = f(C.byref(self.levels[l].desc), self.system, C.byref(self.params[l]), self.nv, _ptrs(self.u[l]),
              _ptrs(self.up[l]), _ptrs(self.upp[l]), h[0], h[1], h[2], C.c_double(self.dt[l]), self.iteration[l],
              int(child), self.order_ti)
        if e:
            raise RuntimeError("oracle level step failed (%d)" % e)
        self.iteration[l] += 1

    def _advance(self, l, snap):
        self.step_level(l)
        if snap:
            snap(l, self.iteration[l], self.u[l])
        if l < len(self.levels) - 1:
            self._advance(l + 1, snap)
            if l >= self.lbo:
                self._advance(l + 1, snap)
        if l > 0:
            tl = self.iteration[l] * self.dt[l]
            tp = self.iteration[l - 1] * self.dt[l - 1]
            aligned = not (tl < tp - 1e-10 or tp < tl - 1e-10)
            uc = self.u[l - 1] if aligned else self.upp[l - 1]
            fmr_restrict_prolong(self.levels[l - 1], self.levels[l], uc, self.u[l], self.order_rp, self.nbuffer)

    def advance(self, nsteps=1, snap=None):
        for _ in range(nsteps):
            self._advance(0, snap)
        return self.u


def track_punctures(level, beta, beta_p, dt, pos, order=4, fixz=0):
    """track_moving_puncture_integrate for each row of pos (n x 3): the new
    positions, the integrator's return values and the position test."""
    beta = np.ascontiguousarray(beta, dtype=np.float64)
    beta_p = np.ascontiguousarray(beta_p, dtype=np.float64)
    pold = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    n = pold.shape[0]
    pnew = np.zeros_like(pold)
    moved = np.zeros(n, dtype=np.int32)
    inside = np.zeros(n, dtype=np.int32)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    e = lib().oracle_track_punctures(C.byref(level.desc), _ptrs(beta), _ptrs(beta_p), dt, order, int(fixz), n,
                                     pold.ctypes.data_as(dp), pnew.ctypes.data_as(dp), moved.ctypes.data_as(ip),
                                     inside.ctypes.data_as(ip))
    if e:
        raise RuntimeError("oracle_track_punctures: %d" % e)
    return pnew, moved, inside


def track_extremum(level, var, pos, order=4, find_max=0, minmove=0.01, fixz=0):
    """track_moving_puncture_extremum for each row of pos (n x 3): the new
    positions and the position test."""
    var = np.ascontiguousarray(var, dtype=np.float64)
    pold = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
    n = pold.shape[0]
    pnew = np.zeros_like(pold)
    inside = np.zeros(n, dtype=np.int32)
    dp = C.POINTER(C.c_double)
    e = lib().oracle_track_extremum(C.byref(level.desc), var.ctypes.data, int(find_max), minmove, order, int(fixz), n,
                                    pold.ctypes.data_as(dp), pnew.ctypes.data_as(dp),
                                    inside.ctypes.data_as(C.POINTER(C.c_int)))
    if e:
        raise RuntimeError("oracle_track_extremum: %d" % e)
    return pnew, inside
