"""Analytic puncture data for the evolution workloads.

Brill-Lindquist conformal factor psi = 1 + sum_n m_n / (2 r_n) with no
elliptic correction (punctures_solver = none: PunctureData,
Punctures.c:439; SetMWBL, ConformalFactor.c:147), turned into BSSN variables
the way bssn_startup does it (bssn.c:260-420, adm_to_bssn): g~ = delta,
chi = psi^-4, A~ = K = Gamma~ = 0, precollapsed lapse alpha = psi^-2
(bssn_initial_lapse = oochi05, bssn.c:370-380), zero shift and B.
"""
import numpy as np

from . import abi


def brill_lindquist_state(level, punctures):
    """punctures: list of (mass, x, y, z).  Returns a (24, npoints) array."""
    x, y, z = level.coords()
    psi = np.ones_like(x)
    for m, px, py, pz in punctures:
        r = np.sqrt((x - px) ** 2 + (y - py) ** 2 + (z - pz) ** 2)
        psi += m / (2.0 * r)
    u = np.zeros((abi.NVARS, x.size))
    u[0] = u[3] = u[5] = 1.0
    u[6] = psi ** -4
    u[17] = psi ** -2
    return u


def z4_brill_lindquist_state(level, punctures):
    """The same data in the Z4c evolve list (Khat = K = 0, Theta = 0 inserted
    before alpha, z4.c:234-242).  Returns a (25, npoints) array."""
    b = brill_lindquist_state(level, punctures)
    u = np.zeros((abi.Z4_NVARS, b.shape[1]))
    u[:17] = b[:17]
    u[18:] = b[17:]
    return u


def schwarzschild_c1(n_inner=64, dx=0.25):
    """The single-puncture workload: nxyz = n_inner gives an (n_inner+2)^3
    box (grid.c:84-99), M = 1 at the origin (never on a grid point)."""
    lev = abi.Level.single_box(n_inner + 2, dx)
    return lev, brill_lindquist_state(lev, [(1.0, 0.0, 0.0, 0.0)])


class Binary:
    """Puncture parameters (ReadPunctureParameters, Punctures.c:221-248):
    masses, positions, Bowen-York momenta and spins, one row per puncture."""

    def __init__(self, mass, pos, mom, spin):
        self.mass = np.ascontiguousarray(mass, dtype=np.float64)
        self.pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        self.mom = np.ascontiguousarray(mom, dtype=np.float64).reshape(-1, 3)
        self.spin = np.ascontiguousarray(spin, dtype=np.float64).reshape(-1, 3)

    @staticmethod
    def sample(rng):
        """One parameter set of the binary-puncture workload: m1, m2 in
        U(0.3, 0.7), separation d in U(4, 12) on the x axis, momenta
        +-P in y with P in U(0, 0.15), spins in U(-0.2, 0.2) per axis."""
        m = rng.uniform(0.3, 0.7, 2)
        d = rng.uniform(4.0, 12.0)
        P = rng.uniform(0.0, 0.15)
        return Binary(m, [[d / 2, 0, 0], [-d / 2, 0, 0]], [[0, P, 0], [0, -P, 0]], rng.uniform(-0.2, 0.2, (2, 3)))

    def vector(self):
        """Flat conditioning vector (masses, positions, momenta, spins)."""
        return np.concatenate([self.mass, self.pos.ravel(), self.mom.ravel(), self.spin.ravel()])


def _dp(a):
    import ctypes as C
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Multigrid:
    """The puncture multigrid on the device (nrgpu_mg_*): the reference's
    multigrid(level, u, f, v, c, ..., Lpuncture_nonlin, Lpuncture_GS)
    (multigrid.c:35) for one cube of m^3 points, spacing dx."""

    def __init__(self, m, dx, params=None):
        import ctypes as C
        self.m, self.dx = m, dx
        self.params = params or abi.mg_params()
        h = C.c_void_p()
        abi.check(abi.lib().nrgpu_mg_create(m, dx, C.byref(self.params), C.byref(h)))
        self.handle = h

    def coefficients(self, binary, stream=None):
        """a, b as (m^3,) float64 CUDA tensors."""
        import ctypes as C
        import torch
        n = self.m ** 3
        a = torch.empty(n, dtype=torch.float64, device="cuda")
        b = torch.empty(n, dtype=torch.float64, device="cuda")
        s = C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)
        abi.check(abi.lib().nrgpu_puncture_coefficients(
            self.m, self.dx, len(binary.mass), _dp(binary.mass), _dp(binary.pos), _dp(binary.mom),
            _dp(binary.spin), C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()), s))
        return a, b

    def solve(self, a, b, u, stream=None):
        """Solve in place; returns (V cycles on the finest level, RMS residual)."""
        import ctypes as C
        import torch
        nc, res = C.c_int(), C.c_double()
        s = C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)
        abi.check(abi.lib().nrgpu_mg_solve(self.handle, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                           C.c_void_p(u.data_ptr()), C.byref(nc), C.byref(res), s))
        return nc.value, res.value

    def smooth(self, a, b, u, nsweeps, omega=2.0 / 3.0, stream=None):
        """nsweeps damped Jacobi sweeps of the puncture equation on u (in
        place), each with the Robin condition: smoothing of a guess."""
        import ctypes as C
        import torch
        s = C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)
        abi.check(abi.lib().nrgpu_mg_smooth(self.handle, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                            C.c_void_p(u.data_ptr()), int(nsweeps), float(omega), s))

    def close(self):
        if self.handle:
            abi.lib().nrgpu_mg_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
