"""The tracker's oracle (oracle/track_oracle.c) against the reference's own
tracker: tests/golden/track_*.npz hold the positions that
track_moving_puncture_integrate (Gauge/moving_punctures_integrate.c:29-100)
returned, run by the reference inside its evolution from a list of start
positions, with the current and previous shift it read.  The oracle must
return the same positions bit for bit, the same integrator return value and
the same position test (xyzinsidelevel, main/amr/points.c:121-133)."""
import os

import numpy as np
import pytest

from baum_b200 import abi
from oracle import oracle

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# case -> (order_RP, grid symmetry of the level)
TRACK_CASES = {"track_box": (4, 0), "track_box_rp2": (2, 0), "track_box_rp6": (6, 0),
               "track_octant": (4, 7), "track_fmr_binary": (4, 0)}


def track_fixture(case):
    """(level, beta, beta_p, dt, result rows, alpha) of a tracking fixture:
    the fields are the reference's, zero away from the start positions."""
    g = np.load(os.path.join(GOLDEN, case + ".npz"))
    tag = [k[:-7] for k in g.files if k.endswith("_result")][0]
    boxes = [(int(b[0]), int(b[1]), int(b[2]), b[4], b[5], b[6]) for b in g[tag + "_boxes"]]
    h = g[tag + "_h"]
    level = abi.Level(boxes, float(h[0]), g[tag + "_boundary"].astype(np.int32), dy=float(h[1]), dz=float(h[2]),
                      symmetry=TRACK_CASES[case][1])
    full = np.zeros((7, level.npoints))
    full[:, g[tag + "_idx"]] = g[tag + "_beta"]
    return level, full[:3].copy(), full[3:6].copy(), float(h[3]), g[tag + "_result"], full[6].copy()


@pytest.mark.parametrize("case", sorted(TRACK_CASES))
def test_oracle_matches_reference_tracker(case):
    level, beta, beta_p, dt, res, _ = track_fixture(case)
    order = TRACK_CASES[case][0]
    for fix in (0, 2):
        rows = res[res[:, 0] == fix]
        pnew, moved, inside = oracle.track_punctures(level, beta, beta_p, dt, rows[:, 2:5], order, fixz=fix == 2)
        assert np.array_equal(moved, rows[:, 1].astype(np.int32))
        assert np.array_equal(inside, rows[:, 8].astype(np.int32))
        assert np.array_equal(pnew, rows[:, 5:8]), np.abs(pnew - rows[:, 5:8]).max()


@pytest.mark.parametrize("case", sorted(TRACK_CASES))
def test_oracle_matches_reference_extremum_search(case):
    """track_moving_puncture_extremum on the lapse (minimum, minimal move
    0.01 dx), z free (rows 10) and pinned (rows 11): bit for bit."""
    level, _, _, _, res, alpha = track_fixture(case)
    for fix in (10, 11):
        rows = res[res[:, 0] == fix]
        assert len(rows)
        pnew, inside = oracle.track_extremum(level, alpha, rows[:, 2:5], TRACK_CASES[case][0], fixz=fix == 11)
        assert np.array_equal(inside, rows[:, 8].astype(np.int32))
        assert np.array_equal(pnew, rows[:, 5:8]), np.abs(pnew - rows[:, 5:8]).max()


def test_fixtures_cover_the_edge_cases():
    """Moved and unmoved positions (cubes that leave a box, points below a
    symmetry plane), new positions off the level, several boxes."""
    seen = {"unmoved_cube": False, "half": False, "off_level": False, "moved": False}
    for case in TRACK_CASES:
        level, _, _, _, res, _ = track_fixture(case)
        res = res[res[:, 0] < 10]
        moved = np.any(res[:, 2:5] != res[:, 5:8], axis=1)
        seen["moved"] |= bool(moved.any())
        seen["unmoved_cube"] |= bool(np.any(~moved & (res[:, 1] == 1) & (res[:, 8] == 1)))
        seen["half"] |= bool(np.any(res[:, 1] == 0))
        seen["off_level"] |= bool(np.any(res[:, 8] == 0))
    assert all(seen.values()), seen
    assert track_fixture("track_fmr_binary")[0].desc.nboxes == 2
