"""Host-side mirror of the reference's ADM diagnostics over the C ABI.

``bssn_to_adm_vl`` / ``z4_to_adm_vl`` (bssn.c:132-197, z4.c:93-124) fill the
ADM metric and extrinsic curvature from the conformal variables at
POST_EVOLVE; ``computeadmconstraints`` (adm.c:14-74) evaluates
``adm_constraints_N`` on them at output time; the 0d output reduces the
results with ``bampi_allreduce_norm2`` / ``_normInf`` (reduce.c:209-266,
output0d.c:62-73).  A variable list here is a contiguous float64 CUDA
tensor of shape (nvars, npoints); all arithmetic runs in libnrgpu.so.
"""
import ctypes as C

import numpy as np
import torch

from . import abi
from .bssn import _ptrs, _stream

ADM_VARS = ["adm_gxx", "adm_gxy", "adm_gxz", "adm_gyy", "adm_gyz", "adm_gzz",
            "adm_Kxx", "adm_Kxy", "adm_Kxz", "adm_Kyy", "adm_Kyz", "adm_Kzz"]
CON_VARS = ["ham", "momx", "momy", "momz", "normham", "normmomx", "normmomy", "normmomz"]

# adm_normalizedConstraints (bam_adm.c:40) -> constraint mode
PLAIN, NORMALIZED, TERMBYTERM = 0, 1, 2


def normalized_mode(value):
    """The mode for a value of adm_normalizedConstraints, with the
    reference's token tests (adm_constraints_N.c:62-63)."""
    if not abi.getv(value, "yes"):
        return PLAIN
    return TERMBYTERM if abi.getv(value, "TermByTerm") else NORMALIZED


def bssn_to_adm_vl(dl, u, adm=None, chipsipower=-4.0, stream=None):
    """ADM g_ij, K_ij (12, npoints) from a BSSN (24) or Z4c (25) state."""
    if not (u.is_cuda and u.dtype == torch.float64 and u.is_contiguous() and u.dim() == 2 and u.shape[0] >= 14):
        raise ValueError("u is a contiguous float64 CUDA tensor of shape (>= 14, npoints)")
    adm = dl.empty(12) if adm is None else adm
    abi.check(abi.lib().nrgpu_to_adm(dl.handle, _ptrs(u, u.shape[0]), _ptrs(adm, 12), float(chipsipower),
                                     _stream(stream)))
    return adm


z4_to_adm_vl = bssn_to_adm_vl


def adm_constraints_N(dl, ucon, uadm, order_centered, mode=PLAIN, stream=None):
    """ham, mom_i (+ normalised ones for mode != PLAIN) into ucon on the
    flag-0 points (adm_constraints_N.c:22)."""
    nout = 8 if mode else 4
    if ucon.shape[0] < nout:
        raise ValueError("ucon needs %d rows" % nout)
    abi.check(abi.lib().nrgpu_adm_constraints(dl.handle, _ptrs(uadm, 12), _ptrs(ucon, ucon.shape[0]),
                                              int(order_centered), int(mode), _stream(stream)))
    return ucon


def norms(dl, v, stream=None):
    """(norm2, normInf) numpy arrays of each row of v over the flag-0 points."""
    n = v.shape[0]
    n2 = np.zeros(n)
    ni = np.zeros(n)
    dp = lambda x: x.ctypes.data_as(C.POINTER(C.c_double))
    abi.check(abi.lib().nrgpu_norms(dl.handle, _ptrs(v, n), n, dp(n2), dp(ni), _stream(stream)))
    return n2, ni


# the output types of write_level_0d (utility/output/output0d.c:58-62)
OUTPUT0D_TYPES = ("max", "min", "norm", "normInf", "integral")


def write_level_0d(dl, v, stream=None):
    """The 0d output scalars of each row of v over the flag-0 points
    (nrgpu_output0d): a (nrows, 5) numpy array, columns in the order of
    OUTPUT0D_TYPES."""
    n = v.shape[0]
    out = np.zeros((n, 5))
    abi.check(abi.lib().nrgpu_output0d(dl.handle, _ptrs(v, n), n, out.ctypes.data_as(C.POINTER(C.c_double)),
                                       _stream(stream)))
    return out


def computeadmconstraints(dl, u, order_centered, mode=PLAIN, chipsipower=-4.0, stream=None):
    """to_adm + constraints + norms of one level: returns (adm, con,
    {name: (norm2, normInf)}), the numbers the reference writes to its
    ham / mom 0d output files."""
    adm = bssn_to_adm_vl(dl, u, chipsipower=chipsipower, stream=stream)
    con = dl.empty(8 if mode else 4)
    adm_constraints_N(dl, con, adm, order_centered, mode, stream)
    n2, ni = norms(dl, con, stream)
    return adm, con, {name: (n2[i], ni[i]) for i, name in enumerate(CON_VARS[:con.shape[0]])}


MASS_VARS = ["ADM_mass_integrand", "ADM_mass_integrand_chi", "ADM_mass_Pxint", "ADM_mass_Pyint",
             "ADM_mass_Pzint", "ADM_mass_Jxint", "ADM_mass_Jyint", "ADM_mass_Jzint"]


def adm_mass_integrands(dl, uadm, trK, chi, out=None, stream=None):
    """The eight integrands of ADM_mass (ADM_mass.c:80-87) into out (8,
    npoints; zero where not computed when out is None) at the flag-0 points,
    from the ADM metric and curvature uadm (12, npoints) and the evolved
    trace K and chi (npoints each)."""
    out = torch.zeros((8, dl.level.npoints), dtype=torch.float64, device="cuda") if out is None else out
    for t in (trK, chi):
        if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
            raise ValueError("trK and chi are contiguous float64 CUDA tensors")
    abi.check(abi.lib().nrgpu_adm_mass_integrands(dl.handle, _ptrs(uadm, 12), C.c_void_p(trK.data_ptr()),
                                                  C.c_void_p(chi.data_ptr()), _ptrs(out, 8), _stream(stream)))
    return out


def integral_over_sphere(dl, f, r, ntheta, nphi, order, center=(0.0, 0.0, 0.0), stream=None):
    """integral_over_sphere_Simpson (Integral_over_sphere.c:197-357) of the
    level array f (npoints) over the sphere of radius r; 0 when a point of
    the sphere cannot be interpolated on the level."""
    res = C.c_double()
    abi.check(abi.lib().nrgpu_sphere_integral(dl.handle, C.c_void_p(f.data_ptr()), float(center[0]),
                                              float(center[1]), float(center[2]), float(r), int(ntheta), int(nphi),
                                              int(order), C.byref(res), _stream(stream)))
    return res.value


def sphere_safely_inside(level, r, order_RP):
    """centered_sphere_safely_inside_level (main/amr/points.c:188-250): a
    one-box level whose bounding box (mirrored about the symmetry planes)
    holds the sphere of radius r + order_RP dx about the origin."""
    if len(level.boxes) > 1:
        return False
    b = level.boxes[0]
    rr = r + order_RP * level.dx
    lo = [b.x0, b.y0, b.z0]
    hi = [b.x0 + (b.m - 1) * level.dx, b.y0 + (b.n - 1) * level.desc.dy, b.z0 + (b.o - 1) * level.desc.dz]
    for d in range(3):
        if level.desc.symmetry >> d & 1:
            lo[d] = -hi[d]
    return all(not (-rr < lo[d] - 1e-10 or hi[d] < rr - 1e-10) for d in range(3))


def _origin(o):
    return (C.c_double * 3)(*[float(v) for v in o])


def psi4(dl, uadm, alpha, beta, order_centered, kinnersley=False, flat=False, origin=(0.0, 0.0, 0.0), out=None,
         csqr=True, stream=None):
    """rpsi4, ipsi4, Csqr (3, npoints) of curvature_invariants_N at the
    flag-0 points (zeros elsewhere when out is None) from the ADM metric and
    curvature uadm (12, npoints), the lapse (npoints) and the shift (3,
    npoints)."""
    out = torch.zeros((3, dl.level.npoints), dtype=torch.float64, device="cuda") if out is None else out
    abi.check(abi.lib().nrgpu_psi4(dl.handle, _ptrs(uadm, 12), C.c_void_p(alpha.data_ptr()), _ptrs(beta, 3),
                                   int(order_centered), int(bool(kinnersley)), int(bool(flat)), _origin(origin),
                                   C.c_void_p(out[0].data_ptr()), C.c_void_p(out[1].data_ptr()),
                                   C.c_void_p(out[2].data_ptr()) if csqr else None, _stream(stream)))
    return out


def rescale_psi4(dl, p, origin=(0.0, 0.0, 0.0), stream=None):
    """rescale_psi4 (Invariants.c:263-284) on rows 0, 1 of p."""
    abi.check(abi.lib().nrgpu_psi4_rescale(dl.handle, C.c_void_p(p[0].data_ptr()), C.c_void_p(p[1].data_ptr()),
                                           _origin(origin), _stream(stream)))


def psi4_modes(dl, p, radii, lmin=2, lmax=4, ntheta=47, nphi=46, order=4, origin=(0.0, 0.0, 0.0), stream=None):
    """compute_modes (Invariants.c:367-540): (len(radii), nmodes, 2) with the
    modes in the reference's column order (l ascending, m = -l..l)."""
    nr = len(radii)
    lnum, mnum = lmax - lmin + 1, 2 * lmax + 1
    buf = np.zeros(nr * lnum * mnum * 2)
    rad = (C.c_double * nr)(*[float(r) for r in radii])
    abi.check(abi.lib().nrgpu_psi4_modes(dl.handle, C.c_void_p(p[0].data_ptr()), C.c_void_p(p[1].data_ptr()),
                                         _origin(origin), int(lmin), int(lmax), rad, nr, int(ntheta), int(nphi),
                                         int(order), buf.ctypes.data_as(C.POINTER(C.c_double)), _stream(stream)))
    buf = buf.reshape(nr, lnum, mnum, 2)
    cols = [buf[:, l - lmin, m + l, :] for l in range(lmin, lmax + 1) for m in range(-l, l + 1)]
    return np.stack(cols, axis=1)
