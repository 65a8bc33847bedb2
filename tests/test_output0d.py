"""The 0d output scalars (write_level_0d, utility/output/output0d.c:28-116:
max, min, norm, normInf, integral over the points with boundary flag 0)
against the reference's own values, written by the dump harness for its
evolved list after a state dump (tests/golden/red0d_*.npz, a box and an
octant grid whose SYMBOUND points are left out).  The CPU test restates the
reductions in numpy against the reference; the GPU test runs
nrgpu_output0d through the C ABI: max, min and normInf bit for bit; the
norm in the reference's form, sqrt(sum u^2 / (nvars n)) sqrt(nvars), within
5e-15 relative (the reference's own sequential sum is 1.6e-15 from the exact
one on these cases, and the device sums in another order); the integral,
times pow(dx, 3), within 1e-13 of the sum of |u| dx^3."""
import math
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = {"red0d_box": 0, "red0d_octant": 7}


def case(name):
    from baum_b200 import abi
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    boxes = [(int(b[0]), int(b[1]), int(b[2]), b[4], b[5], b[6]) for b in g["boxes"]]
    return abi.Level(boxes, float(g["dx"]), g["boundary"], symmetry=CASES[name]), g


def check(got, ref, g):
    """got, ref: (nvars, 5).  The sums are compared relative to the sum of
    |u| dx^3, the scale of their rounding (an integral of a field that
    changes sign cancels far below it)."""
    u = g["state"][:, g["boundary"] == 0]
    for t in (0, 1, 3):
        assert np.array_equal(got[:, t], ref[:, t]), t
    assert np.all(np.abs(got[:, 2] - ref[:, 2]) <= 5e-15 * ref[:, 2]), np.abs(got[:, 2] - ref[:, 2]) / ref[:, 2]
    scale = np.abs(u).sum(1) * float(g["dx"]) ** 3
    assert np.all(np.abs(got[:, 4] - ref[:, 4]) <= 1e-13 * scale), np.abs(got[:, 4] - ref[:, 4]) / scale


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_reference(name):
    level, g = case(name)
    u = g["state"][:, g["boundary"] == 0]
    nv = u.shape[0]
    got = np.stack([u.max(1), u.min(1), np.sqrt((u * u).sum(1) / (nv * u.shape[1])) * math.sqrt(nv),
                    np.abs(u).max(1), u.sum(1) * math.pow(float(g["dx"]), 3)], axis=1)
    check(got, g["result"].T, g)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_matches_reference(gpu, name):
    import torch
    from baum_b200 import adm
    from baum_b200.bssn import DeviceLevel
    level, g = case(name)
    dl = DeviceLevel(level)
    u = torch.from_numpy(np.ascontiguousarray(g["state"])).cuda()
    check(adm.write_level_0d(dl, u), g["result"].T, g)
    dl.close()
