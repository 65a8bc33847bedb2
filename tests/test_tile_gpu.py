"""The BSSN interior rhs over TMA-staged tiles (nrgpu_level_tile) against the
reference's outputs and the CPU oracle, at the tolerance of every rhs parity
test (1e-12 relative per variable).

Both forms are run: one block per tile, and the persistent kernel (one
block per SM walking the tiles).  The staged-tile kernel stages each field's 22 x 10 x 10 box (a 16 x 4 x 4
tile and a halo of 3) in shared memory with one TMA load and forms the same
terms as the per-point kernel in another order, so it is compared with the
reference and the oracle, not bit for bit with the per-point kernel.  The
cases cover partial tiles in every direction, the order ladder at box edges
(2nd order one point in), KO4 and KO6, the c != 0 branch, the fused RK4
stages, the host-buffer slabs (planes k0..k1 of a box), symmetry grids, a
level of several boxes, and the boxes the kernel does not cover (odd row
length, an advection shift it has no halo for), where the per-point kernel
runs instead.
"""
import numpy as np
import pytest
import torch

from conftest import GOLDEN_SYMMETRY, golden_level, load_golden, relerr
from baum_b200 import abi, bssn, fmr, punctures, synthetic
from oracle import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-12

CASES = {
    "bssn_fourier_o4": dict(),
    "bssn_fourier_o4_ko4": dict(order_dissipation=4, dissfactor=0.1 / 16),
}


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def tiled(lev, mode):
    dl = bssn.DeviceLevel(lev)
    assert dl.tile(mode) == mode
    return dl


MODES = pytest.mark.parametrize("mode", [1, 2], ids=["per_tile", "persistent"])


@pytest.mark.parametrize("case", sorted(CASES))
@MODES
def test_tile_rhs_and_rk4_match_reference(gpu, case, mode):
    """The reference's rhs; its RK4 states where the fixture holds them,
    else the oracle's."""
    g = load_golden(case)
    lev = golden_level(g)
    p = abi.bssn_params(**CASES[case])
    dl = tiled(lev, mode)
    u = to_dev(g["state_it0_l0"])
    r = dl.empty()
    bssn.evolve_rhs(dl, r, u, 0.0, u, p)
    torch.cuda.synchronize()
    assert relerr(r.cpu().numpy(), g["rhs_it0_l0"]).max() < TOL
    for _ in range(2):
        bssn.evolve_rk_rk4(dl, u, float(g["dt"]), p)
    torch.cuda.synchronize()
    want = g["state_it2_l0"] if "state_it2_l0" in g else \
        oracle.bssn_evolve(lev, np.ascontiguousarray(g["state_it0_l0"]), float(g["dt"]), 2, p)
    assert relerr(u.cpu().numpy(), want).max() < TOL
    assert not dl.nan_flag()


@MODES
def test_tile_puncture_rk4_matches_reference(gpu, mode):
    g = load_golden("bssn_punc_o4")
    lev = golden_level(g)
    p = abi.bssn_params()
    dl = tiled(lev, mode)
    u = to_dev(g["state_it0_l0"])
    for _ in range(4):
        bssn.evolve_rk_rk4(dl, u, float(g["dt"]), p)
    torch.cuda.synchronize()
    assert relerr(u.cpu().numpy(), g["state_it4_l0"]).max() < TOL


@MODES
def test_tile_c1_schwarzschild_50_steps_matches_oracle(gpu, mode):
    """The benchmarked workload at full size: 64^3 inner points, 50 RK4
    steps with the staged-tile rhs."""
    lev, u0 = punctures.schwarzschild_c1()
    p = abi.bssn_params()
    dt = 0.25 * 0.25
    dl = tiled(lev, mode)
    u = to_dev(u0)
    for _ in range(50):
        bssn.evolve_rk_rk4(dl, u, dt, p)
    torch.cuda.synchronize()
    uo = oracle.bssn_evolve(lev, np.ascontiguousarray(u0), dt, 50, p)
    err = relerr(u.cpu().numpy(), uo)
    assert err.max() < TOL, err
    assert not dl.nan_flag()


@pytest.mark.parametrize("m,order", [(40, 4), (40, 6), (26, 4)])
@MODES
def test_tile_partial_tiles_and_orders_match_oracle(gpu, m, order, mode):
    """38 inner points per side (partial tiles in x, y and z), 24 (one
    partial tile in x); 4th order with lopsided advection and KO6, 6th order
    with the centred 6th-order advection; the order ladder near every face.
    Fourier data with a non-zero shift."""
    lev = abi.Level.single_box(m, 0.4)
    x, y, z = lev.coords()
    u0 = synthetic.fourier_state(x, y, z, abi.NVARS, synthetic.BSSN_UNIT, 8, 0.05, 16.0, 9)
    over = dict(order_centered=order, order_advection=order, advection_lopsided6=3) if order == 6 else {}
    p = abi.bssn_params(**over)
    dl = tiled(lev, mode)
    u = to_dev(u0)
    r = dl.empty()
    bssn.evolve_rhs(dl, r, u, 0.0, u, p)
    ro = oracle.bssn_rhs(lev, np.ascontiguousarray(u0), p)
    assert relerr(r.cpu().numpy(), ro).max() < TOL
    un = to_dev(u0)
    pre = u0 * 1.01
    bssn.evolve_rhs(dl, un, to_dev(pre), 0.05, u, p)
    ra = oracle.bssn_rhs(lev, np.ascontiguousarray(u0), p, c=0.05, upre=np.ascontiguousarray(pre), out=u0.copy())
    assert relerr(un.cpu().numpy(), ra).max() < TOL
    for _ in range(2):
        bssn.evolve_rk_rk4(dl, u, 0.1, p)
    torch.cuda.synchronize()
    uo = oracle.bssn_evolve(lev, np.ascontiguousarray(u0), 0.1, 2, p)
    assert relerr(u.cpu().numpy(), uo).max() < TOL
    assert not dl.nan_flag()


@MODES
def test_tile_host_buffer_slabs_equal_device_path(gpu, mode):
    """The host-buffer step launches the interior in z slabs (planes
    k0..k1); with the staged-tile rhs it equals the device step bit for bit."""
    lev, u0 = punctures.schwarzschild_c1(n_inner=40, dx=0.5)
    p = abi.bssn_params()
    dl = tiled(lev, mode)
    u = to_dev(u0)
    for _ in range(2):
        bssn.evolve_rk_rk4(dl, u, 0.125, p)
    h = np.ascontiguousarray(u0.copy())
    bssn.evolve_host(dl, h, 2, 0.125, p)
    assert np.array_equal(h, u.cpu().numpy())


@pytest.mark.parametrize("case,steps", [("bssn_punc_octant", 4), ("bssn_fourier_bitant", 2)])
@MODES
def test_tile_symmetry_grids_match_reference(gpu, case, steps, mode):
    g = load_golden(case)
    lev = golden_level(g, GOLDEN_SYMMETRY[case])
    p = abi.bssn_params()
    dl = tiled(lev, mode)
    u = to_dev(g["state_it0_l0"])
    r = dl.empty()
    bssn.evolve_rhs(dl, r, u, 0.0, u, p)
    torch.cuda.synchronize()
    assert relerr(r.cpu().numpy(), g["rhs_it0_l0"], floor=1e-3).max() < TOL
    for _ in range(steps):
        bssn.evolve_rk_rk4(dl, u, float(g["dt"]), p)
    torch.cuda.synchronize()
    assert relerr(u.cpu().numpy(), g["state_it%d_l0" % steps]).max() < TOL


def test_tile_refinement_levels_match_oracle(gpu):
    """A 3-level BSSN hierarchy (REFBOUND outer layers on the finer levels)
    with the staged-tile rhs on every level, 2 coarse steps."""
    from test_fmr_oracle_pin import FMR_TOL
    levels = fmr.nested_levels([22, 28, 24], 0.5)
    params = [abi.bssn_params(dissfactor=(0.1 if l == 0 else 0.02) / 64) for l in range(3)]
    dt = [0.125 / 2 ** l for l in range(3)]
    u0 = []
    for lev in levels:
        x, y, z = lev.coords()
        u0.append(synthetic.fourier_state(x, y, z, abi.NVARS, synthetic.BSSN_UNIT, 8, 0.05, 16.0, 3))
    H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(system=abi.SYSTEM_BSSN, autotune=2))
    u = [to_dev(x) for x in u0]
    H.advance(u, 2)
    st = oracle.FmrState(levels, u0, 0, params, dt)
    st.advance(2)
    for l in range(3):
        a, b = u[l].cpu().numpy(), st.u[l]
        err = np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-8)
        assert err.max() < FMR_TOL, (l, err.max())
    H.close()


def test_tile_falls_back_where_it_does_not_apply(gpu):
    """An odd row length (rows not on 16-byte boundaries) and a 4th-order
    advection shift of 0 (taps 4 points out, beyond the halo): the per-point
    kernel runs, bit for bit what it gives with the tiles off."""
    for m, over in ((37, {}), (40, dict(advection_lopsided=0))):
        lev = abi.Level.single_box(m, 0.4)
        x, y, z = lev.coords()
        u0 = synthetic.fourier_state(x, y, z, abi.NVARS, synthetic.BSSN_UNIT, 8, 0.05, 16.0, 4)
        p = abi.bssn_params(**over)
        out = []
        for on in (0, 1):
            dl = bssn.DeviceLevel(lev)
            dl.tile(on)
            u = to_dev(u0)
            bssn.evolve_rk_rk4(dl, u, 0.1, p)
            torch.cuda.synchronize()
            out.append(u.cpu().numpy())
        assert np.array_equal(out[0], out[1])
