"""Parity of the CUDA ADM diagnostics (through the C ABI) with the reference
(golden dumps of bssn_to_adm / z4_to_adm and adm_constraints_N) and with the
CPU oracle; the constraint norms of an evolved puncture; convergence of the
Hamiltonian constraint on analytic data.

Tolerances: g_ij, K_ij within 1e-14 relative (two pow() per point);
ham and mom_i within 1e-11 of their largest value (they are sums of terms
much larger than the result); a normalised constraint c/D within the error
that allows in c divided by D; norm2 within 1e-13 relative (summation
order), normInf exact."""
import numpy as np
import pytest
import torch

from conftest import golden_level, load_golden, relerr
from test_adm_oracle_pin import CON_CASES, check_constraints
from baum_b200 import abi, adm, bssn, punctures
from oracle import oracle

pytestmark = pytest.mark.gpu


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("case", sorted(CON_CASES))
def test_to_adm_and_constraints_match_reference(gpu, case):
    g = load_golden(case)
    st, cn, order, mode = CON_CASES[case]
    lev = golden_level(g)
    dl = bssn.DeviceLevel(lev)
    u = to_dev(g[st])
    a = adm.bssn_to_adm_vl(dl, u)
    con = dl.empty(8 if mode else 4)
    adm.adm_constraints_N(dl, con, a, order, mode)
    torch.cuda.synchronize()
    ref = g[cn]
    assert relerr(a.cpu().numpy(), ref[:12]).max() < 1e-14
    inner = g["boundary"] == 0
    check_constraints(con.cpu().numpy()[:, inner], ref[12:20][:, inner])
    # the same constraints from the reference's own ADM variables
    con2 = dl.empty(8 if mode else 4)
    adm.adm_constraints_N(dl, con2, to_dev(ref[:12]), order, mode)
    check_constraints(con2.cpu().numpy()[:, inner], ref[12:20][:, inner])
    # flagged points are not written
    assert (con.cpu().numpy()[:, ~inner] == 0).all()


@pytest.mark.parametrize("order,mode", [(2, 0), (4, 1), (6, 2)])
def test_constraints_match_oracle_on_puncture(gpu, order, mode):
    lev, u0 = punctures.schwarzschild_c1(n_inner=40, dx=0.3)
    p = abi.bssn_params(order_centered=order, order_advection=order)
    dl = bssn.DeviceLevel(lev)
    u = to_dev(u0)
    for _ in range(3):
        bssn.evolve_rk_rk4(dl, u, 0.075, p)
    a = adm.bssn_to_adm_vl(dl, u)
    con = dl.empty(8 if mode else 4)
    adm.adm_constraints_N(dl, con, a, order, mode)
    torch.cuda.synchronize()
    ao = oracle.to_adm(lev, u.cpu().numpy())
    assert relerr(a.cpu().numpy(), ao).max() < 1e-14
    co = oracle.adm_constraints(lev, ao, order, mode)
    inner = lev.boundary == 0
    check_constraints(con.cpu().numpy()[:, inner], co[:, inner])


def test_norms_match_oracle(gpu):
    g = load_golden("bssn_punc_con")
    lev = golden_level(g)
    dl = bssn.DeviceLevel(lev)
    con = g["con_it3_l0"][12:20]
    n2, ni = adm.norms(dl, to_dev(con))
    o2, oi = oracle.norms(lev, con)
    np.testing.assert_allclose(n2, o2, rtol=1e-13)
    np.testing.assert_array_equal(ni, oi)
    # bit-reproducible from call to call
    n2b, nib = adm.norms(dl, to_dev(con))
    assert np.array_equal(n2, n2b) and np.array_equal(ni, nib)


def test_evolved_puncture_constraint_norms_match_oracle(gpu):
    """computeadmconstraints after 20 RK4 steps of the 64^3 single-puncture
    workload: norms of ham and mom_i from the GPU evolution + diagnostics
    against the oracle's evolution + diagnostics."""
    lev, u0 = punctures.schwarzschild_c1()
    p = abi.bssn_params()
    dl = bssn.DeviceLevel(lev)
    u = to_dev(u0)
    for _ in range(20):
        bssn.evolve_rk_rk4(dl, u, 0.0625, p)
    _, con, nrm = adm.computeadmconstraints(dl, u, 4, adm.NORMALIZED)
    uo = oracle.bssn_evolve(lev, np.ascontiguousarray(u0), 0.0625, 20, p)
    co = oracle.adm_constraints(lev, oracle.to_adm(lev, uo), 4, 1)
    o2, oi = oracle.norms(lev, co)
    # the two evolutions agree to ~1e-12 of each field; ham and mom_i take
    # two derivatives of them, and a normalised constraint divides by a
    # denominator that passes close to zero near the puncture, which
    # amplifies that difference further
    for i, name in enumerate(adm.CON_VARS):
        tol = 1e-10 if i < 4 else 1e-8
        assert abs(nrm[name][0] - o2[i]) <= tol * o2[i] + 1e-15, name
        assert abs(nrm[name][1] - oi[i]) <= tol * oi[i] + 1e-15, name
    # the diagnostics alone, on the oracle's state: as tight as the kernels
    _, _, nrm2 = adm.computeadmconstraints(dl, to_dev(uo), 4, adm.NORMALIZED)
    for i, name in enumerate(adm.CON_VARS[:4]):
        assert abs(nrm2[name][0] - o2[i]) <= 1e-12 * o2[i], name


def test_hamiltonian_constraint_converges_on_brill_lindquist(gpu):
    """Time-symmetric Brill-Lindquist data satisfy ham = 0 exactly; the
    discrete ham away from the puncture falls with the centred order
    (measured with the oracle: ratios 15.0 at order 4, 64.6 at order 6)."""
    def rms_outside(n_inner, dx, order):
        lev = abi.Level.single_box(n_inner + 2, dx)
        u0 = punctures.brill_lindquist_state(lev, [(1.0, 0.0, 0.0, 0.0)])
        dl = bssn.DeviceLevel(lev)
        a = adm.bssn_to_adm_vl(dl, to_dev(u0))
        con = dl.empty(4)
        adm.adm_constraints_N(dl, con, a, order)
        x, y, z = lev.coords()
        r = np.sqrt(x ** 2 + y ** 2 + z ** 2)
        sel = (r > 2.0) & (np.maximum(np.maximum(abs(x), abs(y)), abs(z)) < 5.0)
        return np.sqrt((con.cpu().numpy()[0][sel] ** 2).mean())
    for order, lo, hi in [(4, 11.0, 22.0), (6, 40.0, 90.0)]:
        ratio = rms_outside(64, 0.25, order) / rms_outside(128, 0.125, order)
        assert lo < ratio < hi, (order, ratio)


def test_bad_arguments_are_refused(gpu):
    lev, u0 = punctures.schwarzschild_c1(n_inner=8, dx=0.5)
    dl = bssn.DeviceLevel(lev)
    a = dl.empty(12)
    with pytest.raises(RuntimeError, match="order_centered"):
        adm.adm_constraints_N(dl, dl.empty(4), a, 8)
    with pytest.raises(RuntimeError, match="mode"):
        adm.adm_constraints_N(dl, dl.empty(8), a, 4, 3)
    with pytest.raises(RuntimeError, match="nvars"):
        adm.norms(dl, dl.empty(33))
