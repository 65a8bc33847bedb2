"""The ADM mass analysis on the device (nrgpu_adm_mass_integrands,
nrgpu_fmr_restrict_prolong_vars, nrgpu_sphere_integral) against the
reference's integrands and integrals (tests/golden/admmass_*.npz): one box,
and three nested levels filled from parents and children before the
integration (ADM_mass.c:100-104).  Same bounds as the oracle's pin:
integrands 1e-12 of each field's size, integrals 1e-11 of the row's mass."""
import numpy as np
import pytest
import torch

from admmass_common import NPHI, NTHETA, ORDER, check_integrals, check_integrands, load
from baum_b200 import abi, adm, bssn, fmr

pytestmark = pytest.mark.gpu


def device_run(name):
    g, levels = load(name)
    dls = [bssn.DeviceLevel(lv) for lv in levels]
    f = []
    for l, dl in enumerate(dls):
        x = torch.from_numpy(np.ascontiguousarray(g["inputs_l%d" % l])).cuda()
        f.append(adm.adm_mass_integrands(dl, x[:12].contiguous(), x[12].contiguous(), x[13].contiguous()))
    if len(levels) > 1:
        H = fmr.Hierarchy(levels, [0.1 / 2 ** l for l in range(len(levels))], [abi.bssn_params()] * len(levels),
                          abi.fmr_params(system=abi.SYSTEM_BSSN, use_graph=0, autotune=0))
        for l in range(len(levels) - 1, 0, -1):
            H.restrict_prolong_vars(l, f[l - 1], f[l])
        H.close()
    torch.cuda.synchronize()
    return g, levels, dls, f


def rows(dl, level, f, radii):
    return [(r, [adm.integral_over_sphere(dl, f[v], r, NTHETA, NPHI, ORDER) for v in range(8)]) for r in radii
            if adm.sphere_safely_inside(level, r, 4)]


def test_adm_mass_one_box_matches_reference(gpu):
    g, levels, dls, f = device_run("admmass_box")
    check_integrands(g, 0, f[0].cpu().numpy())
    check_integrals(g, 0, rows(dls[0], levels[0], f[0], [2.0, 3.0]))
    for dl in dls:
        dl.close()


def test_adm_mass_three_levels_matches_reference(gpu):
    g, levels, dls, f = device_run("admmass_fmr")
    for l, lv in enumerate(levels):
        check_integrands(g, l, f[l].cpu().numpy())
        check_integrals(g, l, rows(dls[l], lv, f[l], [1.0, 2.5, 3.5]))
    for dl in dls:
        dl.close()


def test_sphere_integral_of_a_polynomial(gpu):
    """The Simpson rule over the solid angle (the integrands carry their own
    R^2) of fields that 4th-order Lagrange interpolation reproduces: f = 1
    gives 4 pi up to the rule's error, f = z gives 0 and f = x^2 gives
    4 pi r^2 / 3; a sphere reaching past the level gives 0, as the
    reference."""
    lev = abi.Level.single_box(40, 0.25)
    dl = bssn.DeviceLevel(lev)
    x, y, z = (torch.from_numpy(c).cuda() for c in lev.coords())
    r = 2.0
    one = adm.integral_over_sphere(dl, torch.ones_like(x), r, 31, 60, 4)
    assert abs(one - 4 * np.pi) < 1e-3 * 4 * np.pi
    assert abs(adm.integral_over_sphere(dl, z.contiguous(), r, 31, 60, 4)) < 1e-12
    x2 = adm.integral_over_sphere(dl, (x * x).contiguous(), r, 31, 60, 4)
    assert abs(x2 - 4 * np.pi * r ** 2 / 3) < 2e-3 * 4 * np.pi * r ** 2 / 3
    assert adm.integral_over_sphere(dl, torch.ones_like(x), 5.0, 31, 60, 4) == 0.0
    dl.close()
