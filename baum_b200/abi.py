"""ctypes mirror of include/nrgpu.h and the loader of the CUDA library.

The library is the product: ``baum_b200/libnrgpu.so`` built from
``baum_b200/csrc`` for sm_100a.  There is no fallback; :func:`lib` raises if
the library is missing or cannot be loaded.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.environ.get("NRGPU_LIBRARY") or os.path.join(HERE, "libnrgpu.so")
NVARS = 24

# BSSN evolve-list order (reference bssn.c:315-322)
BSSN_VARS = ["g11", "g12", "g13", "g22", "g23", "g33", "chi", "A11", "A12", "A13", "A22", "A23",
             "A33", "K", "G1", "G2", "G3", "alpha", "beta1", "beta2", "beta3", "B1", "B2", "B3"]
# the same list under the reference's variable names (bam_bssn.c, bam_adm.c)
BSSN_BAM_NAMES = ["bssn_gxx", "bssn_gxy", "bssn_gxz", "bssn_gyy", "bssn_gyz", "bssn_gzz",
                  "bssn_chi", "bssn_Axx", "bssn_Axy", "bssn_Axz", "bssn_Ayy", "bssn_Ayz",
                  "bssn_Azz", "bssn_K", "bssn_Gx", "bssn_Gy", "bssn_Gz", "alpha", "betax",
                  "betay", "betaz", "betadotx", "betadoty", "betadotz"]

NRGPU_OK = 0
ERRORS = {-1: "bad argument", -2: "CUDA error", -3: "NaN/Inf in rhs", -4: "out of device memory",
          -5: "unsupported", -6: "device wait timed out"}
PHYBOUND = 1


class Box(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("o", C.c_int), ("noffset", C.c_int),
                ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double)]


class LevelDesc(C.Structure):
    _fields_ = [("nboxes", C.c_int), ("box", C.POINTER(Box)), ("npoints", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("boundary", C.POINTER(C.c_int)), ("symmetry", C.c_int)]


class BssnParams(C.Structure):
    _fields_ = [("order_centered", C.c_int), ("order_advection", C.c_int),
                ("advection_lopsided", C.c_int), ("advection_lopsided6", C.c_int),
                ("order_dissipation", C.c_int), ("dissfactor", C.c_double),
                ("forceKzerofactor", C.c_double), ("subtractA", C.c_int),
                ("normalizedetg", C.c_int), ("oploglapse", C.c_int), ("oploglapse2", C.c_int),
                ("oplogwithshift", C.c_int), ("harmoniclapse", C.c_int),
                ("gamma0factor", C.c_double), ("gamma2factor", C.c_double),
                ("withGadv", C.c_double), ("withShiftadv", C.c_double),
                ("withBadv", C.c_double), ("withB", C.c_double),
                ("lapseharmonicf", C.c_double), ("shiftalphapower", C.c_double),
                ("shiftgammacoeff", C.c_double), ("shiftGalphapower", C.c_double),
                ("shiftdriver", C.c_double), ("chiDivFloor", C.c_double),
                ("chipsipower", C.c_double), ("bc_var0", C.c_double * NVARS),
                ("bc_speed", C.c_double * NVARS)]


def getv(value, token):
    """The reference's token test of a parameter string (GetvFlag,
    parameters.c:883-900): only the FIRST occurrence of token as a substring
    is examined, and it counts only if it is a whole word.  So "withB" is
    false in "withBadv withB" but true in "withB withBadv"."""
    i = value.find(token)
    if i < 0:
        return 0
    start = i == 0 or value[i - 1] == " "
    j = i + len(token)
    end = j == len(value) or value[j] == " "
    return 1 if start and end else 0


def bssn_params_from_par(lapse="1+log withshift", shift="gamma0 withGadv withBadv withShiftadv", **over):
    """Factors of bssn_rhs_movpunc_N from the bssn_lapse / bssn_shift strings
    (bssn_rhs_movpunc_N.c:117-131)."""
    f = dict(oploglapse=getv(lapse, "1+log"), oploglapse2=getv(lapse, "1+log2"),
             oplogwithshift=getv(lapse, "withshift"), harmoniclapse=getv(lapse, "harmonic"),
             gamma0factor=float(getv(shift, "gamma0")), gamma2factor=float(getv(shift, "gamma2")),
             withGadv=float(getv(shift, "withGadv")), withShiftadv=float(getv(shift, "withShiftadv")),
             withBadv=float(getv(shift, "withBadv")), withB=float(not getv(shift, "withoutB")))
    f.update(over)
    return bssn_params(**f)


def bssn_params(**over):
    """Parameters of the single-puncture BSSN workload: 1+log withshift,
    gamma0 withGadv withBadv withShiftadv, shiftdriver 2, 4th-order centred
    and lopsided advection, KO6 with dissipation_factor 0.1 (dissfactor =
    0.1/2^6, evolve.c:503), radiative boundary speeds from bssn.c:288-311."""
    p = BssnParams()
    p.order_centered = 4
    p.order_advection = 4
    p.advection_lopsided = 1
    p.advection_lopsided6 = 3  # reference default, bam_amr.c:52
    p.order_dissipation = 6
    p.dissfactor = 0.1 / 2.0 ** 6
    p.forceKzerofactor = 1.0  # Getv("bssn_forceKzero","no") is 1 for the default "no"
    p.subtractA = 1
    p.normalizedetg = 1
    p.oploglapse, p.oploglapse2, p.oplogwithshift, p.harmoniclapse = 1, 0, 1, 0
    p.gamma0factor, p.gamma2factor = 1.0, 0.0
    p.withGadv = p.withShiftadv = p.withBadv = p.withB = 1.0
    p.lapseharmonicf = 2.0
    p.shiftalphapower = 0.0
    p.shiftgammacoeff = 0.75
    p.shiftGalphapower = 0.0
    p.shiftdriver = 2.0
    p.chiDivFloor = -1000.0
    p.chipsipower = -4.0
    for k, v in over.items():
        setattr(p, k, v)
    set_bc_from_gauge(p)
    return p


def set_bc_from_gauge(p):
    """Far limits and speeds of VarNameSetBoundaryInfo (bssn.c:269-311)."""
    if p.oploglapse:
        vg = p.lapseharmonicf ** 0.5
    elif p.oploglapse2:
        vg = (4.0 / 3.0) ** 0.5
    else:
        vg = 1.0
    var0 = [0.0] * NVARS
    speed = [1.0] * NVARS
    for i in (0, 3, 5, 6, 17):   # gxx gyy gzz chi alpha -> far limit 1
        var0[i] = 1.0
    for i in (13, 6, 17):        # K chi alpha travel at the gauge speed
        speed[i] = vg
    p.bc_var0[:] = var0
    p.bc_speed[:] = speed


Z4_NVARS = 25
# Z4c evolve-list order (reference z4.c:234-242)
Z4_VARS = ["g11", "g12", "g13", "g22", "g23", "g33", "chi", "A11", "A12", "A13", "A22", "A23", "A33",
           "Khat", "G1", "G2", "G3", "Theta", "alpha", "beta1", "beta2", "beta3", "B1", "B2", "B3"]


class Z4Params(C.Structure):
    _fields_ = [("order_centered", C.c_int), ("order_advection", C.c_int),
                ("advection_lopsided", C.c_int), ("advection_lopsided6", C.c_int),
                ("order_dissipation", C.c_int), ("dissfactor", C.c_double),
                ("kappa1", C.c_double), ("kappa2", C.c_double), ("zeroThetaRHS", C.c_double),
                ("useNPTs", C.c_int), ("subtractA", C.c_int), ("normalizedetg", C.c_int),
                ("oploglapse", C.c_int), ("oploglapse2", C.c_int), ("oplogwithshift", C.c_int),
                ("harmoniclapse", C.c_int), ("gamma0factor", C.c_double), ("gamma2factor", C.c_double),
                ("withGadv", C.c_double), ("withShiftadv", C.c_double), ("withBadv", C.c_double),
                ("withB", C.c_double), ("lapseharmonicf", C.c_double), ("shiftalphapower", C.c_double),
                ("shiftgammacoeff", C.c_double), ("shiftdriver", C.c_double), ("chiDivFloor", C.c_double),
                ("chipsipower", C.c_double), ("bc_var0", C.c_double * Z4_NVARS),
                ("bc_speed", C.c_double * Z4_NVARS), ("precision", C.c_int), ("boundary", C.c_int)]


def z4_params(**over):
    """Z4c settings of the precision-sweep and FMR workloads: z4_lapse =
    1+log withshift, z4_shift = gamma0 withGadv withBadv withShiftadv withB,
    shiftdriver 2, shiftgammacoeff 0.75, kappa1 = 0.02, kappa2 = 0, Theta
    evolved (z4_zeroThetaRHS default "no" reads as 1), no non-principal
    terms, 4th order + KO6 with dissipation_factor 0.1; boundary far limits
    and speeds of z4.c:204-228."""
    p = Z4Params()
    p.order_centered = p.order_advection = 4
    p.advection_lopsided = 1
    p.advection_lopsided6 = 3
    p.order_dissipation = 6
    p.dissfactor = 0.1 / 2.0 ** 6
    p.kappa1, p.kappa2 = 0.02, 0.0
    p.zeroThetaRHS = 1.0
    p.useNPTs = 0
    p.subtractA = p.normalizedetg = 1
    p.oploglapse, p.oploglapse2, p.oplogwithshift, p.harmoniclapse = 1, 0, 1, 0
    p.gamma0factor, p.gamma2factor = 1.0, 0.0
    p.withGadv = p.withShiftadv = p.withBadv = p.withB = 1.0
    p.lapseharmonicf = 2.0
    p.shiftalphapower = 0.0
    p.shiftgammacoeff = 0.75
    p.shiftdriver = 2.0
    p.chiDivFloor = -1000.0
    p.chipsipower = -4.0
    for k, v in over.items():
        setattr(p, k, v)
    vg = p.lapseharmonicf ** 0.5 if p.oploglapse else ((4.0 / 3.0) ** 0.5 if p.oploglapse2 else 1.0)
    var0 = [0.0] * Z4_NVARS
    speed = [1.0] * Z4_NVARS
    for i in (0, 3, 5, 6, 18):   # gxx gyy gzz chi alpha
        var0[i] = 1.0
    for i in (13, 6, 18):        # Khat chi alpha
        speed[i] = vg
    p.bc_var0[:] = var0
    p.bc_speed[:] = speed
    return p


def z4_params_from_par(lapse="1+log withshift", shift="gamma0 withGadv withBadv withShiftadv withB", **over):
    """Factors of z4_rhs_movpunc_N from the z4_lapse / z4_shift strings
    (z4_rhs_movpunc_N.m:610-626), with the reference's token semantics."""
    f = dict(oploglapse=getv(lapse, "1+log"), oploglapse2=getv(lapse, "1+log2"),
             oplogwithshift=getv(lapse, "withshift"), harmoniclapse=getv(lapse, "harmonic"),
             gamma0factor=float(getv(shift, "gamma0")), gamma2factor=float(getv(shift, "gamma2")),
             withGadv=float(getv(shift, "withGadv")), withShiftadv=float(getv(shift, "withShiftadv")),
             withBadv=float(getv(shift, "withBadv")), withB=float(getv(shift, "withB")))
    f.update(over)
    return z4_params(**f)


class MgParams(C.Structure):
    _fields_ = [("npre", C.c_int), ("npost", C.c_int), ("exact_nmin", C.c_int), ("exact_nmax", C.c_int),
                ("vcycle_nmin", C.c_int), ("vcycle_nmax", C.c_int), ("fullV", C.c_int),
                ("size_nmin", C.c_int), ("levels_nmax", C.c_int), ("tol", C.c_double),
                ("falloff", C.c_double), ("batch", C.c_int)]


class FmrParams(C.Structure):
    _fields_ = [("system", C.c_int), ("lbo", C.c_int), ("order_timeinterpolation", C.c_int),
                ("order_RP", C.c_int), ("nbuffer", C.c_int), ("use_graph", C.c_int),
                ("autotune", C.c_int)]


SYSTEM_BSSN, SYSTEM_Z4C = 0, 1


def fmr_params(**over):
    """amr = bo with lbo 0, order_timeinterpolation 3, order_RP 4,
    amr_nbuffer 3, Z4c, coarse steps replayed from a CUDA graph, each
    level's rhs block shape picked by the autotuner."""
    p = FmrParams(SYSTEM_Z4C, 0, 3, 4, 3, 1, 1)
    for k, v in over.items():
        setattr(p, k, v)
    return p


def mg_params(**over):
    """The puncture-solve settings of the binary-puncture workload:
    mg_relax_npre = npost = 3, mg_exact_nmin/nmax = 10/200, mg_size_nmin = 4,
    mg_vcycle_nmax = 2000, full-V cycling, tolerance 1e-10, Robin falloff 1."""
    p = MgParams(3, 3, 10, 200, 0, 2000, 1, 4, -1, 1e-10, 1.0, 8)
    for k, v in over.items():
        setattr(p, k, v)
    return p


class Level:
    """Host-side description of a level (keeps the ctypes arrays alive)."""

    def __init__(self, boxes, dx, boundary, dy=None, dz=None, symmetry=0):
        import numpy as np
        self.boxes = (Box * len(boxes))()
        off = 0
        for i, b in enumerate(boxes):
            m, n, o, x0, y0, z0 = b
            self.boxes[i] = Box(m, n, o, off, x0, y0, z0)
            off += m * n * o
        self.npoints = off
        self.boundary = np.ascontiguousarray(boundary, dtype=np.int32)
        assert self.boundary.size == off
        self.desc = LevelDesc(len(boxes), self.boxes, off, dx, dy or dx, dz or dx,
                              self.boundary.ctypes.data_as(C.POINTER(C.c_int)), int(symmetry))
        self.dx = dx

    @staticmethod
    def single_box(n, dx):
        """A cubic single box of n^3 points, centred (grid.c:84-105), with
        the outer layer flagged PHYBOUND (flag.c:23-36)."""
        import numpy as np
        x0 = -(n - 1) * dx / 2
        b = np.zeros((n, n, n), dtype=np.int32)
        b[0, :, :] = b[-1, :, :] = b[:, 0, :] = b[:, -1, :] = b[:, :, 0] = b[:, :, -1] = PHYBOUND
        return Level([(n, n, n, x0, x0, x0)], dx, b.ravel())

    def coords(self):
        import numpy as np
        xs, ys, zs = [], [], []
        for b in self.boxes:
            i = np.arange(b.m)
            j = np.arange(b.n)
            k = np.arange(b.o)
            z, y, x = np.meshgrid(b.z0 + k * self.desc.dz, b.y0 + j * self.desc.dy,
                                  b.x0 + i * self.desc.dx, indexing="ij")
            xs.append(x.ravel()); ys.append(y.ravel()); zs.append(z.ravel())
        return np.concatenate(xs), np.concatenate(ys), np.concatenate(zs)


# nrgpu_fmr_move_fn: int (*)(void *user, nrgpu_fmr *fmr, int l, void *stream)
FMR_MOVE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p)


def ptr_array(ptrs):
    arr = (C.c_void_p * len(ptrs))()
    for i, p in enumerate(ptrs):
        arr[i] = p
    return arr


_lib = None


def lib():
    """Load libnrgpu.so; raise if it is absent (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise RuntimeError("libnrgpu.so not built: run python -c 'import __graft_entry__ as g; g.build()'")
    L = C.CDLL(LIBPATH)
    vp = C.c_void_p
    pp = C.POINTER(C.c_void_p)
    sig = {
        "nrgpu_abi_version": (C.c_int, []),
        "nrgpu_last_error": (C.c_char_p, []),
        "nrgpu_init": (C.c_int, [C.c_int]),
        "nrgpu_bssn_params_default": (None, [C.POINTER(BssnParams)]),
        "nrgpu_level_create": (C.c_int, [C.POINTER(LevelDesc), C.POINTER(vp)]),
        "nrgpu_level_destroy": (C.c_int, [vp]),
        "nrgpu_bssn_rhs": (C.c_int, [vp, pp, pp, C.c_double, pp, C.POINTER(BssnParams), vp]),
        "nrgpu_bssn_boundary": (C.c_int, [vp, pp, pp, C.c_double, pp, C.POINTER(BssnParams), vp]),
        "nrgpu_bssn_algcon": (C.c_int, [vp, pp, C.POINTER(BssnParams), vp]),
        "nrgpu_vladd": (C.c_int, [vp, C.c_int, pp, C.c_double, pp, C.c_double, pp, vp]),
        "nrgpu_bssn_rk4_step": (C.c_int, [vp, pp, C.c_double, C.POINTER(BssnParams), vp]),
        "nrgpu_bssn_evolve_host": (C.c_int, [vp, pp, C.c_int, C.c_double, C.POINTER(BssnParams)]),
        "nrgpu_level_nan_flag": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "nrgpu_probe_fp64_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_float)]),
        "nrgpu_z4_rhs": (C.c_int, [vp, pp, pp, C.c_double, pp, C.POINTER(Z4Params), vp]),
        "nrgpu_z4_boundary": (C.c_int, [vp, pp, pp, C.c_double, pp, C.POINTER(Z4Params), vp]),
        "nrgpu_z4_rk4_step": (C.c_int, [vp, pp, C.c_double, C.POINTER(Z4Params), vp]),
        "nrgpu_mg_params_default": (None, [C.POINTER(MgParams)]),
        "nrgpu_mg_create": (C.c_int, [C.c_int, C.c_double, C.POINTER(MgParams), C.POINTER(vp)]),
        "nrgpu_mg_destroy": (C.c_int, [vp]),
        "nrgpu_mg_solve": (C.c_int, [vp, vp, vp, vp, C.POINTER(C.c_int), C.POINTER(C.c_double), vp]),
        "nrgpu_mg_smooth": (C.c_int, [vp, vp, vp, vp, C.c_int, C.c_double, vp]),
        "nrgpu_to_adm": (C.c_int, [vp, pp, pp, C.c_double, vp]),
        "nrgpu_adm_constraints": (C.c_int, [vp, pp, pp, C.c_int, C.c_int, vp]),
        "nrgpu_norms": (C.c_int, [vp, pp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), vp]),
        "nrgpu_output0d": (C.c_int, [vp, pp, C.c_int, C.POINTER(C.c_double), vp]),
        "nrgpu_mlp_nparams": (C.c_int, []),
        "nrgpu_mlp_create": (C.c_int, [C.c_int, C.POINTER(vp)]),
        "nrgpu_mlp_destroy": (C.c_int, [vp]),
        "nrgpu_mlp_set_params": (C.c_int, [vp, C.POINTER(C.c_float), C.c_int]),
        "nrgpu_mlp_get_params": (C.c_int, [vp, C.POINTER(C.c_float), C.c_int]),
        "nrgpu_mlp_set_conditions": (C.c_int, [vp, C.POINTER(C.c_double), C.c_int]),
        "nrgpu_mlp_features": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, C.c_double, vp]),
        "nrgpu_mlp_copy_features": (C.c_int, [vp, C.c_int, C.POINTER(C.c_uint16)]),
        "nrgpu_mlp_train_step": (C.c_int, [vp, vp, C.c_int, C.c_float, C.c_int, C.POINTER(C.c_float), vp]),
        "nrgpu_mlp_gradients": (C.c_int, [vp, C.POINTER(C.c_float), C.c_int]),
        "nrgpu_mlp_forward": (C.c_int, [vp, C.c_int, vp, vp]),
        "nrgpu_mlp_predict_u": (C.c_int, [vp, C.POINTER(C.c_double), C.c_int, C.c_double, C.c_double, vp, vp]),
        "nrgpu_mlp_predict_u_fp32": (C.c_int, [vp, C.POINTER(C.c_double), C.c_int, C.c_double, C.c_double, vp, vp]),
        "nrgpu_mlp_predict_u_tc": (C.c_int, [vp, C.POINTER(C.c_double), C.c_int, C.c_double, C.c_double, vp, vp]),
        "nrgpu_mlp_tc_status": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "nrgpu_fmr_params_default": (C.c_int, [C.POINTER(FmrParams)]),
        "nrgpu_fmr_create": (C.c_int, [C.c_int, C.POINTER(LevelDesc), C.POINTER(C.c_double), vp,
                                       C.POINTER(FmrParams), C.POINTER(vp)]),
        "nrgpu_fmr_destroy": (C.c_int, [vp]),
        "nrgpu_fmr_flags": (C.c_int, [vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "nrgpu_fmr_restrict_prolong": (C.c_int, [vp, C.c_int, pp, pp, vp]),
        "nrgpu_fmr_advance": (C.c_int, [vp, pp, C.c_int, vp]),
        "nrgpu_fmr_iteration": (C.c_int, [vp, C.c_int]),
        "nrgpu_fmr_block": (C.c_int, [vp, C.c_int, C.POINTER(C.c_int)]),
        "nrgpu_fmr_state_size": (C.c_int, [vp, C.POINTER(C.c_size_t)]),
        "nrgpu_fmr_save": (C.c_int, [vp, vp, C.c_size_t]),
        "nrgpu_fmr_load": (C.c_int, [vp, vp, C.c_size_t]),
        "nrgpu_fmr_track": (C.c_int, [vp, C.c_int, C.POINTER(C.c_double), C.c_int]),
        "nrgpu_fmr_track_method": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int]),
        "nrgpu_fmr_punctures": (C.c_int, [vp, C.POINTER(C.c_double), C.POINTER(C.c_int)]),
        "nrgpu_fmr_set_move": (C.c_int, [vp, vp, vp]),
        "nrgpu_fmr_restrict_prolong_vars": (C.c_int, [vp, C.c_int, C.c_int, pp, pp, vp]),
        "nrgpu_adm_mass_integrands": (C.c_int, [vp, pp, vp, vp, pp, vp]),
        "nrgpu_psi4": (C.c_int, [vp, pp, vp, pp, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), vp, vp, vp,
                                 vp]),
        "nrgpu_psi4_rescale": (C.c_int, [vp, vp, vp, C.POINTER(C.c_double), vp]),
        "nrgpu_psi4_modes": (C.c_int, [vp, vp, vp, C.POINTER(C.c_double), C.c_int, C.c_int,
                                       C.POINTER(C.c_double), C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.POINTER(C.c_double), vp]),
        "nrgpu_sphere_integral": (C.c_int, [vp, vp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                            C.c_int, C.c_int, C.POINTER(C.c_double), vp]),
        "nrgpu_fmr_regrid": (C.c_int, [vp, C.c_int, C.c_int, C.POINTER(LevelDesc), pp, pp, vp]),
        "nrgpu_track_punctures": (C.c_int, [vp, pp, pp, C.c_double, C.c_int, C.c_int, C.c_int, vp, vp, vp]),
        "nrgpu_track_punctures_extremum": (C.c_int, [vp, vp, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, vp, vp,
                                                     vp]),
        "nrgpu_level_autotune": (C.c_int, [vp, C.c_int, vp, vp, C.POINTER(C.c_int)]),
        "nrgpu_level_block": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
        "nrgpu_level_get_block": (C.c_int, [vp, C.POINTER(C.c_int)]),
        "nrgpu_level_tile": (C.c_int, [vp, C.c_int]),
        "nrgpu_level_queue": (C.c_int, [vp, C.c_int]),
        "nrgpu_puncture_coefficients": (C.c_int, [C.c_int, C.c_double, C.c_int, C.POINTER(C.c_double),
                                                  C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                  C.POINTER(C.c_double), vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status):
    if status != NRGPU_OK:
        msg = lib().nrgpu_last_error()
        raise RuntimeError("nrgpu error %d (%s): %s" % (status, ERRORS.get(status, "?"),
                                                        msg.decode() if msg else ""))
    return status
