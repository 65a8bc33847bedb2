"""The Z4c "background" box boundaries on the device against the reference
(tests/golden/z4_bg_*.npz): set_boundary's background branch with the
radiative condition on centred stencils (boundary = background
radcentered, z4_boundary_box_rad) and with the constraint-preserving CPBC2
(boundary = background, z4_boundary_box).  One rhs evaluation with the
boundary callback (the rhs at every point, the extrapolated rhs on the
boundary included), and 3 RK4 steps with algcon, every variable within
1e-12 of the reference; and a larger box against the oracle
(oracle/z4bg_oracle.py)."""
import numpy as np
import pytest
import torch

from conftest import golden_level, load_golden, relerr
from baum_b200 import abi, synthetic, z4
from oracle import z4bg_oracle
from test_z4_oracle_pin import z4_case

pytestmark = pytest.mark.gpu
TOL = 1e-12
MODES = {"rad": 1, "cpbc": 2}


def params(mode):
    p, _ = z4_case("z4_fourier_o4")
    p.boundary = MODES[mode]
    return p


@pytest.mark.parametrize("mode", sorted(MODES))
def test_background_rhs_matches_reference(gpu, mode):
    g = load_golden("z4_bg_%s_rhs" % mode)
    dl = z4.DeviceLevel(golden_level(g))
    u = torch.from_numpy(np.ascontiguousarray(g["state_it0_l0"])).cuda()
    r = dl.empty(25)
    z4.evolve_rhs(dl, r, u, 0.0, u, params(mode))
    torch.cuda.synchronize()
    assert relerr(r.cpu().numpy(), g["rhs_it0_l0"]).max() < TOL


@pytest.mark.parametrize("mode", sorted(MODES))
def test_background_rk4_matches_reference(gpu, mode):
    g = load_golden("z4_bg_%s" % mode)
    dl = z4.DeviceLevel(golden_level(g))
    u = torch.from_numpy(np.ascontiguousarray(g["state_it0_l0"])).cuda()
    for _ in range(3):
        z4.evolve_rk_rk4(dl, u, float(g["dt"]), params(mode))
    torch.cuda.synchronize()
    assert relerr(u.cpu().numpy(), g["state_it3_l0"]).max() < TOL
    assert not dl.nan_flag()


def box_level(npts, dx):
    """One box of npts^3 points centred on the origin, PHYBOUND on its outer
    layer."""
    i = np.arange(npts)
    edge = (i == 0) | (i == npts - 1)
    flags = (edge[None, None, :] | edge[None, :, None] | edge[:, None, None]).astype(np.int32).ravel()
    x0 = -(npts - 1) * dx / 2
    return abi.Level([(npts, npts, npts, x0, x0, x0)], dx, flags)


@pytest.mark.parametrize("mode", sorted(MODES))
def test_background_matches_oracle_on_a_larger_box(gpu, mode):
    """A 42^3 box with a Fourier perturbation of flat space: the rhs with the
    boundary and one RK4 step against the oracle."""
    lev = box_level(42, 0.4)
    x, y, z = lev.coords()
    u0 = synthetic.fourier_state(x, y, z, abi.Z4_NVARS, synthetic.Z4_UNIT, 8, 0.05, 16.0, 7)
    p = params(mode)
    dl = z4.DeviceLevel(lev)
    u = torch.from_numpy(u0.copy()).cuda()
    r = dl.empty(25)
    z4.evolve_rhs(dl, r, u, 0.0, u, p)
    want = z4bg_oracle.rhs(lev, u0.copy(), p, mode)
    torch.cuda.synchronize()
    assert relerr(r.cpu().numpy(), want).max() < TOL
    u = torch.from_numpy(u0.copy()).cuda()
    z4.evolve_rk_rk4(dl, u, 0.1, p)
    want = z4bg_oracle.evolve(lev, u0.copy(), 0.1, 1, p, mode)
    torch.cuda.synchronize()
    assert relerr(u.cpu().numpy(), want).max() < TOL
