"""Convergence of the evolution with resolution, on the GPU through the C ABI.

The data are the gauge wave of the Apples-with-Apples testbeds (the
reference's AwA project, utility/AwA): flat space in the harmonic slicing
with the metric ds^2 = -H dt^2 + H dx^2 + dy^2 + dz^2,
H = 1 - A sin(2 pi (x - t) / d), zero shift.  It is an exact solution of the
Einstein equations (the constraints hold), so at time T every evolved
variable is known in closed form and the Hamiltonian constraint vanishes.
Here A = 0.1, d = 8, on boxes of 33^3, 65^3 and 129^3 points (h = 0.5, 0.25,
0.125; x in [-8, 8], the coarser points shared by the finer boxes), RK4 with
dt = h / 4 to T = 1, radiative boundaries; errors are measured where
|x|, |y|, |z| <= 4.

Expected: errors falling by 2^p per halving of h for p-th order stencils.
Measured factors are asserted within [0.75, 1.25] x 2^p:
* BSSN, 4th order + KO6 (the benchmark's discretisation): fields and
  max|H| x 16;
* Z4c, 4th order + KO6: fields x 16;
* BSSN, 6th order without dissipation (KO6 would add an h^5 term): fields
  x 64.
"""
import numpy as np
import pytest
import torch

from baum_b200 import abi, adm, bssn, z4

pytestmark = pytest.mark.gpu

A, D, T = 0.1, 8.0, 1.0
SIZES = [(33, 0.5), (65, 0.25), (129, 0.125)]


def gauge_wave(level, t, system):
    """The exact state at time t in the BSSN (24) or Z4c (25) list."""
    x, _, _ = level.coords()
    ph = 2.0 * np.pi * (x - t) / D
    H = 1.0 - A * np.sin(ph)
    dH = -A * (2.0 * np.pi / D) * np.cos(ph)     # d_x H
    Kxx = dH / (2.0 * np.sqrt(H))                # -d_t H / (2 alpha), d_t H = -d_x H
    K = Kxx / H
    chi = H ** (-1.0 / 3.0)
    b = np.zeros((abi.NVARS, x.size))
    b[0] = H ** (2.0 / 3.0)                      # g~xx
    b[3] = b[5] = H ** (-1.0 / 3.0)              # g~yy, g~zz
    b[6] = chi
    b[7] = chi * (2.0 / 3.0) * Kxx               # A~xx
    b[10] = b[12] = -chi * Kxx / (3.0 * H)       # A~yy, A~zz
    b[13] = K
    b[14] = (2.0 / 3.0) * H ** (-5.0 / 3.0) * dH  # G~x = -d_j g~^xj
    b[17] = np.sqrt(H)                           # alpha
    if system == "bssn":
        return b
    u = np.zeros((abi.Z4_NVARS, x.size))
    u[:17] = b[:17]      # Khat = K with Theta = 0
    u[18:] = b[17:]
    return u


HARMONIC = dict(oploglapse=0, oploglapse2=0, oplogwithshift=0, harmoniclapse=1, gamma0factor=0.0,
                gamma2factor=0.0, withB=1.0, shiftdriver=0.0)


def run(system, order, ko, m, h):
    lev = abi.Level.single_box(m, h)
    over = dict(HARMONIC, order_centered=order, order_advection=order, advection_lopsided6=3)
    if not ko:
        over["order_dissipation"] = 0
    if system == "bssn":
        p = abi.bssn_params(**over)
        mod = bssn
    else:
        p = abi.z4_params(**over)
        mod = z4
    dl = mod.DeviceLevel(lev)
    u = torch.from_numpy(gauge_wave(lev, 0.0, system)).cuda()
    dt = 0.25 * h
    for _ in range(int(round(T / dt))):
        mod.evolve_rk_rk4(dl, u, dt, p)
    torch.cuda.synchronize()
    assert not dl.nan_flag()
    x, y, z = lev.coords()
    inner = (np.abs(x) <= 4.0 + 1e-9) & (np.abs(y) <= 4.0 + 1e-9) & (np.abs(z) <= 4.0 + 1e-9)
    err = np.abs(u.cpu().numpy() - gauge_wave(lev, T, system))[:, inner].max()
    ham = None
    if system == "bssn":
        _, con, _ = adm.computeadmconstraints(dl, u, order)
        ham = np.abs(con[0].cpu().numpy()[inner]).max()
    dl.close()
    return err, ham


@pytest.mark.parametrize("system,order,ko", [("bssn", 4, True), ("z4c", 4, True), ("bssn", 6, False)],
                         ids=["bssn_o4_ko6", "z4c_o4_ko6", "bssn_o6"])
def test_gauge_wave_converges_at_the_stencil_order(gpu, system, order, ko):
    res = [run(system, order, ko, m, h) for m, h in SIZES]
    want = 2.0 ** order
    f_u = [res[i][0] / res[i + 1][0] for i in range(2)]
    assert all(0.75 * want <= f <= 1.25 * want for f in f_u), (f_u, [r[0] for r in res])
    if system == "bssn" and order == 4:
        f_h = [res[i][1] / res[i + 1][1] for i in range(2)]
        assert all(0.75 * want <= f <= 1.25 * want for f in f_h), (f_h, [r[1] for r in res])
