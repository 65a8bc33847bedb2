"""The CPU restatement of the Z4c "background" box boundary
(oracle/z4bg_oracle.py) pinned to the reference's own rhs and states
(tests/golden/z4_bg_*.npz): the state extrapolated onto the boundary before
the rhs, the radiative (radcentered) and CPBC2 conditions one point inside
the box, the rhs extrapolated onto the boundary, and 3 written-out RK4 steps
with algcon."""
import numpy as np
import pytest

from conftest import golden_level, load_golden, relerr
from oracle import z4bg_oracle as zb
from test_z4_oracle_pin import z4_case

MODES = sorted(zb.MODES)


def params():
    p, _ = z4_case("z4_fourier_o4")
    return p


@pytest.mark.parametrize("mode", MODES)
def test_rhs_matches_reference(mode):
    g = load_golden("z4_bg_%s_rhs" % mode)
    lev = golden_level(g)
    u = np.ascontiguousarray(g["state_it0_l0"]).copy()
    r = zb.rhs(lev, u, params(), mode)
    assert relerr(r, g["rhs_it0_l0"]).max() < 1e-13
    # the boundary rhs itself, one point inside the box, to rounding
    pts = zb.ladder(lev)
    ref = g["rhs_it0_l0"]
    err = np.abs(r[7:18, pts] - ref[7:18, pts]).max(axis=1) / np.abs(ref[7:18]).max(axis=1)
    assert err.max() < 1e-14


@pytest.mark.parametrize("mode", MODES)
def test_rk4_matches_reference(mode):
    g = load_golden("z4_bg_%s" % mode)
    lev = golden_level(g)
    u = np.ascontiguousarray(g["state_it0_l0"]).copy()
    zb.evolve(lev, u, float(g["dt"]), 3, params(), mode)
    assert relerr(u, g["state_it3_l0"]).max() < 1e-13


def test_extrapolation_is_linear_on_faces_and_idempotent():
    """A field linear in x, y, z is reproduced exactly on every PHYBOUND
    point (faces, edges, corners), and a second extrapolation changes
    nothing."""
    g = load_golden("z4_bg_rad_rhs")
    lev = golden_level(g)
    x, y, z = lev.coords()
    f = np.stack([1.0 + 0.5 * x - 0.25 * y + 0.125 * z])
    u = np.where(lev.boundary == 1, 7.0, f)
    zb.extrapolate(lev, u)
    assert np.abs(u - f).max() < 1e-13
    v = zb.extrapolate(lev, u.copy())
    assert np.array_equal(u, v)


def test_ladder_is_the_flag0_shell_one_inside():
    g = load_golden("z4_bg_rad_rhs")
    lev = golden_level(g)
    b = lev.boxes[0]
    pts = zb.ladder(lev)
    assert len(pts) == (b.m - 2) * (b.n - 2) * (b.o - 2) - (b.m - 4) * (b.n - 4) * (b.o - 4)
    assert (lev.boundary[pts] == 0).all()


def test_cpbc_without_perturbation_keeps_flat_space():
    """Minkowski data (unit metric, lapse, chi, everything else zero): the
    CPBC2 rhs vanishes at every boundary point."""
    g = load_golden("z4_bg_cpbc_rhs")
    lev = golden_level(g)
    u = np.zeros((25, lev.npoints))
    for v in (0, 3, 5, 6, 18):
        u[v] = 1.0
    bc = zb.cpbc_rhs(lev, u, zb.ladder(lev), params())
    assert np.abs(bc).max() == 0.0
