"""The mesh-refinement oracle against the reference (golden dumps of a
3-level Berger-Oliger Z4c run): refinement flags exactly, and every level's
state after its steps, with restriction, prolongation and time
interpolation in between, within 2e-11 of each field's size.  The RHS is
not reproduced bit for bit, and its rounding differences accumulate over
the 14 level steps; the fields compared are of size 1e-2..1, so this is an
absolute difference of 1e-13 or less."""
import numpy as np
import pytest

from conftest import load_golden
from baum_b200 import abi, synthetic
from oracle import oracle

FMR_TOL = 2e-11


def fmr_case(name="z4_fmr3"):
    """Levels (with all their boxes), initial states, per-level parameters
    and time steps of a 3-level golden run: dissipation_factor 0.1 on level 0 and 0.2 x 0.1 on
    finer levels (get_dissipation_factor, evolve.c:486-530, with
    amr_move_lcube = 0 and physics without "Z4d"), dt = dtfac dx."""
    g = load_golden(name)
    levels, u0, params, dt = [], [], [], []
    for l in range(3):
        boxes = [(int(b[0]), int(b[1]), int(b[2]), b[4], b[5], b[6]) for b in g["boxes_l%d" % l]]
        lev = abi.Level(boxes, float(g["dx_l%d" % l]), g["boundary_l%d" % l])
        x, y, z = lev.coords()
        levels.append(lev)
        u0.append(synthetic.fourier_state(x, y, z, abi.Z4_NVARS, synthetic.Z4_UNIT, 8, 0.05, 16.0, 1))
        params.append(abi.z4_params_from_par(dissfactor=(0.1 if l == 0 else 0.02) / 2 ** 6))
        dt.append(0.25 * float(g["dx_l%d" % l]))
    return g, levels, u0, params, dt


def test_flags_match_reference():
    g, levels, _, _, _ = fmr_case()
    for l in (1, 2):
        fp, cr = oracle.fmr_flags(levels[l - 1], levels[l], 3)
        assert np.array_equal(fp, g["flagprolong_l%d" % l])
        assert np.array_equal(cr, g["flagrestrict_l%d" % (l - 1)])


def check_snapshots(g, run, tol=FMR_TOL):
    seen = []

    def snap(l, it, u):
        key = "state_it%d_l%d" % (it, l)
        if key in g:
            ref = g[key]
            got = u[g["vars"]]
            err = np.abs(got - ref).max(axis=1) / np.abs(ref).max(axis=1)
            assert err.max() < tol, (key, err)
            seen.append(key)
    run(snap)
    assert sorted(seen) == sorted(k for k in g if k.startswith("state_it"))


def test_three_level_evolution_matches_reference():
    g, levels, u0, params, dt = fmr_case()
    st = oracle.FmrState(levels, u0, 1, params, dt)
    check_snapshots(g, lambda snap: st.advance(2, snap))


def test_binary_grid_flags_match_reference():
    """The binary's grid: level 2 is two boxes, each with its own
    flagprolong (from its own bounding box); level 1 is one box."""
    g, levels, _, _, _ = fmr_case("z4_fmr3_binary")
    assert levels[2].desc.nboxes == 2
    for l in (1, 2):
        fp, cr = oracle.fmr_flags(levels[l - 1], levels[l], 3)
        assert np.array_equal(fp, g["flagprolong_l%d" % l])
    fp, cr = oracle.fmr_flags(levels[0], levels[1], 3)
    assert np.array_equal(cr, g["flagrestrict_l0"])


def test_binary_grid_evolution_matches_reference():
    """Two coarse steps of the binary's grid (level 2 in two boxes): chi and
    alpha of every level at the end, against the reference's dumps."""
    g, levels, u0, params, dt = fmr_case("z4_fmr3_binary")
    st = oracle.FmrState(levels, u0, 1, params, dt)
    check_snapshots(g, lambda snap: st.advance(2, snap))


@pytest.mark.parametrize("order,steps", [(4, 4), (6, 6)])
def test_time_interpolation_orders_4_and_6_match_reference(order, steps):
    """order_timeinterpolation 4 and 6 (evolve.c:298-340: the half-step
    interpolant from u(n+1) and three to five earlier time levels, shifted
    back each step): the reference's 3-level run for enough coarse steps
    that level 0 reaches the full order; every level within the same
    tolerance as the 3rd-order runs."""
    g, levels, u0, params, dt = fmr_case("z4_fmr3_ti%d" % order)
    st = oracle.FmrState(levels, u0, 1, params, dt, order_ti=order)
    check_snapshots(g, lambda snap: st.advance(steps, snap))
