"""Puncture tracking on the GPU through the C ABI (nrgpu_track_punctures,
nrgpu_fmr_track): the level tracker against the reference's own tracker
results bit for bit, and tracking inside a mesh-refinement run against the
oracle driver with the oracle tracker after every finest-level step."""
import numpy as np
import pytest
import torch

from test_fmr_oracle_pin import fmr_case
from test_track_oracle_pin import TRACK_CASES, track_fixture
from baum_b200 import abi, fmr, tracking
from baum_b200.bssn import DeviceLevel
from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", sorted(TRACK_CASES))
def test_level_tracker_matches_reference(gpu, case):
    level, beta, beta_p, dt, res, alpha = track_fixture(case)
    dl = DeviceLevel(level)
    b = torch.from_numpy(beta).cuda()
    bp = torch.from_numpy(beta_p).cuda()
    for fix in (0, 2):
        rows = res[res[:, 0] == fix]
        pos = torch.from_numpy(np.ascontiguousarray(rows[:, 2:5])).cuda()
        st = tracking.track_moving_puncture_integrate(dl, b, bp, dt, pos, order=TRACK_CASES[case][0],
                                                      fixz=fix == 2).cpu().numpy()
        inside = rows[:, 8] == 1
        assert np.array_equal(st & 1, rows[:, 1].astype(np.int32))
        assert np.array_equal((st >> 1) & 1, inside.astype(np.int32))
        # the reference's new position where it lies on the level, else the old one
        want = np.where(inside[:, None], rows[:, 5:8], rows[:, 2:5])
        assert np.array_equal(pos.cpu().numpy(), want)
    # the extremum search on the lapse, z free and pinned
    a = torch.from_numpy(alpha).cuda()
    for fix in (10, 11):
        rows = res[res[:, 0] == fix]
        pos = torch.from_numpy(np.ascontiguousarray(rows[:, 2:5])).cuda()
        st = tracking.track_moving_puncture_extremum(dl, a, pos, order=TRACK_CASES[case][0],
                                                     fixz=fix == 11).cpu().numpy()
        inside = rows[:, 8] == 1
        assert np.array_equal((st >> 1) & 1, inside.astype(np.int32))
        want = np.where(inside[:, None], rows[:, 5:8], rows[:, 2:5])
        assert np.array_equal(pos.cpu().numpy(), want)
    dl.close()


class TrackedState(oracle.FmrState):
    """The oracle driver with track_puncture after each finest-level step
    and its restriction/prolongation (ANALYZE, main.c:420-423)."""

    def __init__(self, *a, pos, ib=19, next_=0, ia=18, **k):
        super().__init__(*a, **k)
        self.pos, self.ib = np.array(pos, dtype=np.float64), ib
        # the first next_ punctures by the extremum search on variable ia
        self.next, self.ia = next_, ia

    def _advance(self, l, snap):
        last = l == len(self.levels) - 1
        if last:
            beta_p = self.u[l][self.ib:self.ib + 3].copy()
        super()._advance(l, snap)
        if last:
            new = self.pos.copy()
            k = self.next
            if k < len(self.pos):
                pnew, _, inside = oracle.track_punctures(self.levels[l], self.u[l][self.ib:self.ib + 3], beta_p,
                                                         self.dt[l], self.pos[k:], self.order_rp)
                new[k:] = np.where(inside[:, None] == 1, pnew, self.pos[k:])
            if k:
                pnew, inside = oracle.track_extremum(self.levels[l], self.u[l][self.ia], self.pos[:k], self.order_rp)
                new[:k] = np.where(inside[:, None] == 1, pnew, self.pos[:k])
            self.pos = new


START = [[2.75, 0.1, -0.2], [-2.6, 0.3, 0.1], [0.6, 0.2, 0.1]]


def test_fmr_tracking_matches_oracle(gpu):
    """Two coarse steps of the binary's 3-level Z4c grid (level 2 in two
    boxes) with three tracked punctures: positions within 1e-11 of the
    oracle driver's (the level states agree to the driver tolerance, 2e-11
    relative), graph replay and plain launches identical, and a checkpoint
    taken after the first step resumes the positions bit for bit."""
    g, levels, u0, params, dt = fmr_case("z4_fmr3_binary")
    st = TrackedState(levels, u0, 1, params, dt, pos=START)
    st.advance(2)
    runs = []
    for use_graph in (0, 1):
        H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(use_graph=use_graph))
        H.track(START)
        u = [torch.from_numpy(x.copy()).cuda() for x in u0]
        H.advance(u, 1)
        ck = H.save()
        u1 = [x.clone() for x in u]
        H.advance(u, 1)
        pos, status = H.punctures()
        runs.append(pos)
        assert np.all(status == 3), status
        # resume from the checkpoint
        H.load(ck)
        H.advance(u1, 1)
        assert np.array_equal(H.punctures()[0], pos)
        H.close()
    assert np.array_equal(runs[0], runs[1])
    assert np.abs(runs[0] - st.pos).max() <= 1e-11, np.abs(runs[0] - st.pos).max()
    assert np.abs(st.pos - np.array(START)).max() > 1e-4  # the punctures moved


@pytest.mark.parametrize("method", ["ext", "extint"])
def test_fmr_extremum_tracking_matches_oracle(gpu, method):
    """moving_puncture_track_method = ext / extint inside the refinement
    run: the extremum search on the lapse for every puncture, or for the
    first one and the shift integrator for the rest, after every
    finest-level step; two coarse steps of the binary's 3-level grid against
    the oracle driver with the oracle trackers, graph replay and plain
    launches identical."""
    g, levels, u0, params, dt = fmr_case("z4_fmr3_binary")
    start = [[-2.6, 0.1, 0.05], [2.75, 0.1, -0.2], [0.6, 0.2, 0.1]]
    nx = len(start) if method == "ext" else 1
    st = TrackedState(levels, u0, 1, params, dt, pos=start, next_=nx)
    st.advance(2)
    runs = []
    for use_graph in (0, 1):
        H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(use_graph=use_graph))
        H.track(start)
        H.track_method(method)
        u = [torch.from_numpy(x.copy()).cuda() for x in u0]
        H.advance(u, 2)
        pos, status = H.punctures()
        assert np.all(status & 1), status
        runs.append(pos)
        H.close()
    assert np.array_equal(runs[0], runs[1])
    assert np.abs(runs[0] - st.pos).max() <= 1e-9, np.abs(runs[0] - st.pos).max()
    assert np.abs(st.pos[:nx] - np.array(start)[:nx]).max() > 1e-4  # the searched punctures moved
