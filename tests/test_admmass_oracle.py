"""The CPU restatement of the ADM mass analysis (oracle/admmass_oracle.py)
pinned to the reference's own integrands and sphere integrals
(tests/golden/admmass_*.npz): one box, and three nested levels whose
integrands are filled from parents and children before the integration
(ADM_mass.c:100-104, set_boundary_refinement_cf)."""
import numpy as np

from admmass_common import NPHI, NTHETA, ORDER, check_integrals, check_integrands, load
from baum_b200 import adm
from oracle import admmass_oracle as ao
from oracle import oracle


def oracle_run(name):
    g, levels = load(name)
    f = [ao.integrands(lv, g["inputs_l%d" % l]) for l, lv in enumerate(levels)]
    for l in range(len(levels) - 1, 0, -1):
        oracle.fmr_restrict_prolong(levels[l - 1], levels[l], f[l - 1], f[l], 4, 3)
    return g, levels, f


def rows(level, f, radii):
    return [(r, [ao.sphere_integral(level, f[v], r, NTHETA, NPHI, ORDER) for v in range(8)]) for r in radii
            if adm.sphere_safely_inside(level, r, 4)]


def test_oracle_adm_mass_one_box_matches_reference():
    g, levels, f = oracle_run("admmass_box")
    check_integrands(g, 0, f[0])
    check_integrals(g, 0, rows(levels[0], f[0], [2.0, 3.0]))


def test_oracle_adm_mass_three_levels_matches_reference():
    g, levels, f = oracle_run("admmass_fmr")
    for l, lv in enumerate(levels):
        check_integrands(g, l, f[l])
        check_integrals(g, l, rows(lv, f[l], [1.0, 2.5, 3.5]))
    # the coarse level's spheres read the children's restricted integrands:
    # without the restriction its r = 1 mass differs
    raw = ao.integrands(levels[0], g["inputs_l0"])
    m = ao.sphere_integral(levels[0], raw[0], 1.0, NTHETA, NPHI, ORDER)
    assert abs(m - g["integrals_l0"][0, 1]) > 1e-3 * abs(g["integrals_l0"][0, 1])
