"""The Z4c box work-queue kernel (nrgpu_level_queue): the interior of all
boxes of a level in one persistent launch, the blocks taking tiles from an
atomic counter.  Each point is computed by the same code as the per-box
launch, so the rhs and the RK4 steps are bit-identical with the queue on and
off: two and three 72^3 boxes (the full form's puncture boxes) at 4th and
6th order, in the rhs, add-linear and RK4 epilogues."""
import numpy as np
import pytest
import torch

from baum_b200 import abi, synthetic, z4

pytestmark = pytest.mark.gpu


def boxes_level(nboxes, m=72, dx=0.25):
    """nboxes boxes of m^3 points side by side in x, each with its outer
    layer flagged (PHYBOUND)."""
    i = np.arange(m)
    edge = (i == 0) | (i == m - 1)
    one = (edge[None, None, :] | edge[None, :, None] | edge[:, None, None]).astype(np.int32).ravel()
    boxes = [(m, m, m, -0.5 * m * dx + 0.1 + b * (m + 3) * dx, -0.5 * m * dx + 0.1, -0.5 * m * dx + 0.1)
             for b in range(nboxes)]
    return abi.Level(boxes, dx, np.concatenate([one] * nboxes))


def state(lev):
    x, y, z = lev.coords()
    u = synthetic.fourier_state(x, y, z, abi.Z4_NVARS, synthetic.Z4_UNIT, 8, 0.02, 24.0, 11)
    u[19] += 0.1 * np.sin(0.2 * y)  # a shift, so that every lopsided row takes part
    return u


@pytest.mark.parametrize("nboxes,order", [(2, 4), (3, 6), (2, 6)])
def test_queue_kernel_is_identical_to_per_box_launches(gpu, nboxes, order):
    lev = boxes_level(nboxes)
    u0 = state(lev)
    p = abi.z4_params(order_centered=order, order_advection=order)
    runs = []
    for on in (0, 1):
        dl = z4.DeviceLevel(lev)
        assert dl.queue(on) == on
        u = torch.from_numpy(u0.copy()).cuda()
        r = dl.empty(25)
        z4.evolve_rhs(dl, r, u, 0.0, u, p)
        n = dl.empty(25)
        z4.evolve_rhs(dl, n, u, 0.01, u, p)  # add-linear form
        for _ in range(2):
            z4.evolve_rk_rk4(dl, u, 0.05, p)
        torch.cuda.synchronize()
        assert not dl.nan_flag()
        runs.append([t.cpu().numpy() for t in (r, n, u)])
        dl.close()
    for a, b in zip(*runs):
        assert np.isfinite(a).all()
        assert np.array_equal(a, b)
    assert np.abs(runs[0][2] - u0).max() > 1e-6  # the state evolved


def test_queue_needs_equal_boxes_of_a_kernel_size(gpu):
    """A level of unequal boxes runs one launch per box with the queue
    switched on (same results as off)."""
    lev = abi.Level([(72, 72, 72, -9.1, -9.1, -9.1), (66, 66, 66, 10.1, -8.3, -8.3)], 0.25,
                    np.concatenate([boxes_level(1, 72).boundary, boxes_level(1, 66).boundary]))
    u0 = state(lev)
    p = abi.z4_params()
    out = []
    for on in (0, 1):
        dl = z4.DeviceLevel(lev)
        dl.queue(on)
        u = torch.from_numpy(u0.copy()).cuda()
        z4.evolve_rk_rk4(dl, u, 0.05, p)
        torch.cuda.synchronize()
        out.append(u.cpu().numpy())
        dl.close()
    assert np.isfinite(out[0]).all()
    assert np.array_equal(out[0], out[1])
