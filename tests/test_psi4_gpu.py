"""Psi4 on the device (nrgpu_psi4, nrgpu_psi4_rescale, nrgpu_psi4_modes)
against the reference's Invariants project (tests/golden/psi4_*.npz, made
by tests/golden/make_golden.py from its curvature_invariants_N and
compute_modes output): rpsi4 and ipsi4 (restricted, prolonged and times r)
and Csqr at 2048 sampled points per level, and the l = 2..4 spin-weight -2
modes at every radius the reference computed.  One box, and three nested
levels.  Bounds: the fields 1e-10 of each field's largest sampled value
(second derivatives of the metric at dx = 0.1-0.8, rounded in another
order), the modes 1e-10 of the largest mode at that radius."""
import numpy as np
import pytest
import torch

from admmass_common import levels_of
from conftest import load_golden
from baum_b200 import abi, adm, bssn, fmr

pytestmark = pytest.mark.gpu

RADII = {"psi4_box": [2.0, 3.0], "psi4_fmr": [1.0, 2.5, 3.5]}


def device_run(name):
    g = load_golden(name)
    levels = levels_of(g)
    dls = [bssn.DeviceLevel(lv) for lv in levels]
    p = []
    for l, dl in enumerate(dls):
        x = torch.from_numpy(np.ascontiguousarray(g["inputs_l%d" % l])).cuda()
        p.append(adm.psi4(dl, x[:12].contiguous(), x[12].contiguous(), x[13:16].contiguous(), 4))
    if len(levels) > 1:
        H = fmr.Hierarchy(levels, [0.1 / 2 ** l for l in range(len(levels))], [abi.bssn_params()] * len(levels),
                          abi.fmr_params(system=abi.SYSTEM_BSSN, use_graph=0, autotune=0))
        for l in range(len(levels) - 1, 0, -1):
            H.restrict_prolong_vars(l, p[l - 1], p[l])
        H.close()
    for dl, q in zip(dls, p):
        adm.rescale_psi4(dl, q)
    torch.cuda.synchronize()
    return g, levels, dls, p


def check(name):
    g, levels, dls, p = device_run(name)
    for l, lv in enumerate(levels):
        idx = g["sample_l%d" % l]
        want = g["psi4_l%d" % l]
        got = p[l].cpu().numpy()[:, idx]
        err = np.abs(got - want).max(axis=1) / np.abs(want).max(axis=1)
        assert err.max() < 1e-10, (l, err)
        radii = [r for r in RADII[name] if adm.sphere_safely_inside(lv, r, 4)]
        want_m = g["modes_l%d" % l]
        assert len(radii) == want_m.shape[0], (l, radii, want_m.shape)
        got_m = adm.psi4_modes(dls[l], p[l], radii)
        for n in range(len(radii)):
            scale = np.abs(want_m[n]).max()
            e = np.abs(got_m[n] - want_m[n]).max() / scale
            assert e < 1e-10, (l, radii[n], e)
    for dl in dls:
        dl.close()


def test_psi4_one_box_matches_reference(gpu):
    check("psi4_box")


def test_psi4_three_levels_matches_reference(gpu):
    check("psi4_fmr")
