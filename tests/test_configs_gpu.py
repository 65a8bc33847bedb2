"""Parity at the shapes the benchmark times.

The Z4c rhs kernel is compiled with fixed box strides for the boxes of the
benchmarked grids (162^3: the precision-sweep box and level 0 of the batched
refinement grid; 168^3, 136^3, 104^3, 72^3: its finer levels; 194^3 and
136^3 at 6th order: the levels of the full form's grid, 72^3 at 6th order its
moving puncture boxes; 106^3 and 98^3: boxes of other sizes, staged into
a copy with the strides of the next size).  Each instance is run here
on a single box of its size through the C ABI and compared with the CPU
oracle (1e-12 relative per variable, the bar of every rhs parity test): the
precision-sweep box at its full size (160^3 inner points, 6th order) for
two RK4 steps, the others for one.  The batched 7-level grid itself is
compared with the oracle at reduced size (the same uneven pattern of
levels, every level stepped 2^l times per coarse step, restriction,
prolongation and time interpolation in between), and at its full size
through the stored oracle state that the benchmark also reports against.
The refinement levels are held to workloads.level_tolerance(l): 2e-11 of
each field's size on level 0, 4x per finer level, the growth of the
rounding of second differences with 1/dx^2.
"""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN, relerr
from baum_b200 import abi, fmr, punctures, workloads, z4
from oracle import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-12


def shifted_binary(lev, sep):
    """Brill-Lindquist binary (m = 0.5 each at x = +-sep) in the Z4c list
    with a smooth shift and Theta, so that advection, the shift terms and
    every lopsided row take part."""
    u = punctures.z4_brill_lindquist_state(lev, [(0.5, sep, 0.0, 0.0), (0.5, -sep, 0.0, 0.0)])
    x, y, z = lev.coords()
    L = 0.5 * (x.max() - x.min())
    u[19] = 0.05 * np.sin(2.1 * x / L) * np.cos(1.3 * z / L)
    u[20] = -0.04 * np.cos(1.7 * y / L + 0.4 * x / L)
    u[21] = 0.03 * np.sin(0.9 * z / L - 1.1 * y / L)
    u[17] = 1e-3 * np.cos(1.9 * (x + y) / L)
    return u


@pytest.mark.parametrize("m,order,steps", [(162, 6, 2), (162, 4, 1), (168, 4, 1), (136, 4, 1), (104, 4, 1),
                                           (72, 6, 1), (136, 6, 1), (194, 6, 1), (106, 6, 1), (98, 4, 1)])
def test_fixed_stride_instance_matches_oracle(gpu, m, order, steps):
    dx = 24.0 / (m - 2)
    lev = abi.Level.single_box(m, dx)
    u0 = shifted_binary(lev, 5.0)
    p = abi.z4_params(order_centered=order, order_advection=order)
    dl = z4.DeviceLevel(lev)
    u = torch.from_numpy(u0.copy()).cuda()
    dt = 0.25 * dx
    for _ in range(steps):
        z4.evolve_rk_rk4(dl, u, dt, p)
    torch.cuda.synchronize()
    assert not dl.nan_flag()
    got = u.cpu().numpy()
    dl.close()
    del u
    torch.cuda.empty_cache()
    uo = oracle.z4_evolve(lev, np.ascontiguousarray(u0), dt, steps, p)
    err = relerr(got, uo)
    assert err.max() < TOL, (m, order, err.max(), int(err.argmax()))


def test_seven_level_grid_matches_oracle(gpu):
    """The batched workload's hierarchy at reduced size, two coarse steps
    (the first with 2nd-order time interpolation, the second with 3rd),
    graph replay and tuned launch shapes as the benchmark runs it."""
    levels, params, dt = workloads.fmr_setup(workloads.FMR_SIZES_SMALL)
    u0 = [workloads.fmr_state_host(lev) for lev in levels]
    H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(use_graph=1, autotune=1))
    u = [torch.from_numpy(x.copy()).cuda() for x in u0]
    H.advance(u, 1)
    H.advance(u, 1)
    assert [H.iteration(l) for l in range(7)] == [2 ** (l + 1) for l in range(7)]
    got = [x.cpu().numpy() for x in u]
    H.close()
    st = oracle.FmrState(levels, u0, 1, params, dt)
    st.advance(2)
    for l in range(7):
        err = np.abs(got[l] - st.u[l]).max(axis=1) / np.maximum(np.abs(st.u[l]).max(axis=1), 1e-8)
        assert err.max() < workloads.level_tolerance(l), (l, err.max())


def test_benchmarked_seven_level_grid_matches_stored_oracle_state(gpu):
    fixture = os.path.join(GOLDEN, "fmr_c3_oracle.npz")
    levels, params, dt = workloads.fmr_setup()
    H = fmr.Hierarchy(levels, dt, params)
    u = [workloads.fmr_state_device(lev) for lev in levels]
    H.advance(u, 1)
    torch.cuda.synchronize()
    H.close()
    e_pts, e_sum = workloads.stored_state_deviation(u, fixture)
    for l in range(7):
        assert e_pts[l] < workloads.level_tolerance(l) and e_sum[l] < 1e-12, (l, e_pts, e_sum)
