"""Parity of the CUDA BSSN path (through the C ABI) with the reference's
outputs (golden fixtures) and with the CPU oracle.

Tolerance: 1e-12 relative per variable (max-norm of the difference over the
max-norm of the reference variable; fields that are round-off noise in the
reference are compared against a floor of 1e-8, i.e. absolutely)."""
import numpy as np
import pytest
import torch

from conftest import golden_level, load_golden, relerr
from baum_b200 import abi, bssn, punctures
from oracle import oracle

pytestmark = pytest.mark.gpu
TOL = 1e-12

CASES = {
    "bssn_fourier_o4": dict(),
    "bssn_fourier_o6": dict(order_centered=6, order_advection=6, advection_lopsided6=2),
    "bssn_fourier_o4_ko4": dict(order_dissipation=4, dissfactor=0.1 / 16),
}


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("case", sorted(CASES))
def test_rhs_matches_reference_and_oracle(gpu, case):
    g = load_golden(case)
    lev = golden_level(g)
    p = abi.bssn_params(**CASES[case])
    dl = bssn.DeviceLevel(lev)
    u = to_dev(g["state_it0_l0"])
    r = dl.empty()
    bssn.evolve_rhs(dl, r, u, 0.0, u, p)
    torch.cuda.synchronize()
    r = r.cpu().numpy()
    assert relerr(r, g["rhs_it0_l0"]).max() < TOL
    ro = oracle.bssn_rhs(lev, np.ascontiguousarray(g["state_it0_l0"]), p)
    assert relerr(r, ro).max() < TOL
    assert not dl.nan_flag()


@pytest.mark.parametrize("case,steps", [("bssn_fourier_o4", 2), ("bssn_fourier_o6", 1), ("bssn_punc_o4", 4)])
def test_rk4_matches_reference(gpu, case, steps):
    g = load_golden(case)
    lev = golden_level(g)
    p = abi.bssn_params(**CASES.get(case, {}))
    dl = bssn.DeviceLevel(lev)
    u = to_dev(g["state_it0_l0"])
    for _ in range(steps):
        bssn.evolve_rk_rk4(dl, u, float(g["dt"]), p)
    torch.cuda.synchronize()
    assert relerr(u.cpu().numpy(), g["state_it%d_l0" % steps]).max() < TOL


def test_addlinear_matches_oracle(gpu):
    """c != 0 branch: unew = upre + c*rhs with trace removal and det
    normalisation (bssn_rhs_movpunc_N.m:432-450)."""
    g = load_golden("bssn_fourier_o4")
    lev = golden_level(g)
    p = abi.bssn_params()
    dl = bssn.DeviceLevel(lev)
    u0 = np.ascontiguousarray(g["state_it0_l0"])
    pre = u0 * 1.01
    u, up, un = to_dev(u0), to_dev(pre), to_dev(u0)
    bssn.evolve_rhs(dl, un, up, 0.05, u, p)
    ro = oracle.bssn_rhs(lev, u0, p, c=0.05, upre=np.ascontiguousarray(pre), out=u0.copy())
    assert relerr(un.cpu().numpy(), ro).max() < TOL


@pytest.mark.parametrize("n_inner,order", [(98, 4), (70, 6)])
def test_staged_box_matches_oracle(gpu, n_inner, order):
    """Boxes of sizes without a compile-time-stride kernel of their own
    (100^3 and 72^3 with the boundary layer: staged into copies with the
    strides of 104, and the 72 kernel itself at 6th order): the puncture
    box at dx = 0.25 with a shift, 2 RK4 steps, every variable within 1e-12
    of the oracle."""
    lev, u0 = punctures.schwarzschild_c1(n_inner, 0.25)
    x, _, _ = lev.coords()
    u0[18] = 0.05 * np.sin(0.3 * x)
    p = abi.bssn_params(**(CASES["bssn_fourier_o6"] if order == 6 else {}))
    dt = 0.25 * 0.25
    dl = bssn.DeviceLevel(lev)
    u = to_dev(u0)
    for _ in range(2):
        bssn.evolve_rk_rk4(dl, u, dt, p)
    torch.cuda.synchronize()
    uo = oracle.bssn_evolve(lev, np.ascontiguousarray(u0), dt, 2, p)
    err = relerr(u.cpu().numpy(), uo)
    assert err.max() < TOL, err
    assert not dl.nan_flag()


def test_c1_schwarzschild_50_steps_matches_oracle(gpu):
    """The single-puncture workload at full size: 64^3 inner points, dx=0.25,
    RK4 with dt = 0.25 dx, 50 steps, every variable within 1e-12."""
    lev, u0 = punctures.schwarzschild_c1()
    p = abi.bssn_params()
    dt = 0.25 * 0.25
    dl = bssn.DeviceLevel(lev)
    u = to_dev(u0)
    for _ in range(50):
        bssn.evolve_rk_rk4(dl, u, dt, p)
    torch.cuda.synchronize()
    ug = u.cpu().numpy()
    uo = oracle.bssn_evolve(lev, np.ascontiguousarray(u0), dt, 50, p)
    err = relerr(ug, uo)
    assert err.max() < TOL, err
    assert not dl.nan_flag()


@pytest.mark.parametrize("n_inner,nsteps,order", [(24, 3, 4), (24, 1, 4), (24, 0, 4), (40, 1, 6), (30, 2, 6),
                                                   (10, 2, 4)])
def test_evolve_host_matches_device_path(gpu, n_inner, nsteps, order):
    """The host-buffer call equals the device step bit for bit: z slabs
    whose 2D-copy upload and download overlap the first and last stages
    (a (24, n) host array), whole-variable copies (separate host arrays),
    and a box below 16 planes (not cut into slabs)."""
    lev, u0 = punctures.schwarzschild_c1(n_inner=n_inner, dx=0.5)
    p = abi.bssn_params(**(CASES["bssn_fourier_o6"] if order == 6 else {}))
    dl = bssn.DeviceLevel(lev)
    u = to_dev(u0)
    for _ in range(nsteps):
        bssn.evolve_rk_rk4(dl, u, 0.125, p)
    h = np.ascontiguousarray(u0.copy())
    bssn.evolve_host(dl, h, nsteps, 0.125, p)
    assert np.array_equal(h, u.cpu().numpy())
    # one array per variable at irregular gaps (no common pitch: whole-variable copies)
    n = u0.shape[1]
    buf = np.zeros(abi.NVARS * n + abi.NVARS ** 2)
    rows = [buf[v * n + v * v:(v + 1) * n + v * v] for v in range(abi.NVARS)]
    for v in range(abi.NVARS):
        rows[v][:] = u0[v]
    bssn.evolve_host(dl, rows, nsteps, 0.125, p)
    assert np.array_equal(np.stack(rows), h)
    assert not dl.nan_flag()


def test_nan_in_state_raises_flag(gpu):
    """A NaN planted in the input state (host side) is reported by the device
    flag after the rhs (the reference prints it, check.c:235)."""
    g = load_golden("bssn_fourier_o4")
    lev = golden_level(g)
    p = abi.bssn_params()
    dl = bssn.DeviceLevel(lev)
    s = np.ascontiguousarray(g["state_it0_l0"]).copy()
    s[13, 555] = np.nan
    u = to_dev(s)
    r = dl.empty()
    bssn.evolve_rhs(dl, r, u, 0.0, u, p)
    assert dl.nan_flag()
    assert not dl.nan_flag()   # reading clears it


def test_bad_arguments_are_refused(gpu):
    g = load_golden("bssn_fourier_o4")
    lev = golden_level(g)
    dl = bssn.DeviceLevel(lev)
    u = to_dev(g["state_it0_l0"])
    with pytest.raises(RuntimeError):
        bssn.evolve_rhs(dl, u.clone(), u, 0.0, u, abi.bssn_params(order_centered=8, order_advection=8))
    with pytest.raises(RuntimeError):
        bssn.evolve_rhs(dl, u.clone(), u, 0.0, u, abi.bssn_params(order_advection=6))


@pytest.mark.parametrize("case,steps", [("bssn_punc_octant", 4), ("bssn_fourier_bitant", 2)])
def test_symmetry_grids_match_reference(gpu, case, steps):
    """set_boundary_symmetry on the GPU: the octant puncture (reflections
    about x, y, z = 0) and the bitant Fourier data (z only): the rhs with its
    boundary, the RK4 steps, and the host-buffer call against the reference.
    The octant puncture's near-zero rhs fields are compared absolutely below
    1e-3 (round-off noise of ~1e-17)."""
    from conftest import GOLDEN_SYMMETRY
    g = load_golden(case)
    lev = golden_level(g, GOLDEN_SYMMETRY[case])
    p = abi.bssn_params()
    dl = bssn.DeviceLevel(lev)
    u = to_dev(g["state_it0_l0"])
    r = dl.empty()
    bssn.evolve_rhs(dl, r, u, 0.0, u, p)
    torch.cuda.synchronize()
    assert relerr(r.cpu().numpy(), g["rhs_it0_l0"], floor=1e-3).max() < TOL
    for _ in range(steps):
        bssn.evolve_rk_rk4(dl, u, float(g["dt"]), p)
    torch.cuda.synchronize()
    assert relerr(u.cpu().numpy(), g["state_it%d_l0" % steps]).max() < TOL
    h = np.ascontiguousarray(g["state_it0_l0"]).copy()
    bssn.evolve_host(dl, h, steps, float(g["dt"]), p)
    assert np.array_equal(h, u.cpu().numpy())
    assert not dl.nan_flag()


def test_z4_octant_matches_oracle(gpu):
    """The Z4c system on the octant grid of the golden puncture: 3 RK4 steps
    of the Brill-Lindquist puncture against the oracle (the same
    reflections, with Theta before alpha in the Z4c list)."""
    from conftest import GOLDEN_SYMMETRY
    from baum_b200 import z4
    g = load_golden("bssn_punc_octant")
    lev = golden_level(g, GOLDEN_SYMMETRY["bssn_punc_octant"])
    b = np.ascontiguousarray(g["state_it0_l0"])
    u0 = np.zeros((25, b.shape[1]))
    u0[:17] = b[:17]
    u0[18:] = b[17:]
    p = abi.z4_params()
    dl = z4.DeviceLevel(lev)
    u = to_dev(u0)
    for _ in range(3):
        z4.evolve_rk_rk4(dl, u, float(g["dt"]), p)
    torch.cuda.synchronize()
    uo = oracle.z4_evolve(lev, np.ascontiguousarray(u0.copy()), float(g["dt"]), 3, p)
    assert relerr(u.cpu().numpy(), uo).max() < TOL
