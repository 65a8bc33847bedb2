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


def schwarzschild_c1(n_inner=64, dx=0.25):
    """The single-puncture workload: nxyz = n_inner gives an (n_inner+2)^3
    box (grid.c:84-99), M = 1 at the origin (never on a grid point)."""
    lev = abi.Level.single_box(n_inner + 2, dx)
    return lev, brill_lindquist_state(lev, [(1.0, 0.0, 0.0, 0.0)])
