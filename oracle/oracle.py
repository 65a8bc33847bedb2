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


def build(force=False):
    """Compile the restatement with gcc (-O2, OpenMP, no fast-math)."""
    deps = [SRC, MGSRC, ADMSRC, os.path.join(HERE, "..", "include", "nrgpu.h")]
    if not force and os.path.exists(SO) and all(os.path.getmtime(SO) >= os.path.getmtime(d) for d in deps):
        return SO
    cmd = ["gcc", "-O2", "-std=gnu99", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
           SRC, MGSRC, ADMSRC, "-o", SO, "-lm"]
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
            "oracle_adm_constraints": [LD, pp, pp, C.c_int, C.c_int],
            "oracle_norms": [LD, pp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)],
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
