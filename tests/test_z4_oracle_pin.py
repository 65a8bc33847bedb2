"""The Z4c oracle against the reference (golden fixtures): rhs and RK4, with
the reference's first-occurrence token semantics for z4_shift."""
import numpy as np
import pytest

from conftest import golden_level, load_golden, relerr
from oracle import oracle
from baum_b200 import abi

Z4_CASES = {
    "z4_fourier_o4": (dict(), 2, "gamma0 withGadv withBadv withShiftadv withB"),
    "z4_fourier_o4_B": (dict(order_dissipation=4, dissfactor=0.1 / 16), 1, "gamma0 withB withGadv withBadv withShiftadv"),
    "z4_fourier_o6": (dict(order_centered=6, order_advection=6), 1, "gamma0 withGadv withBadv withShiftadv withB"),
}


def z4_case(case):
    over, steps, shift = Z4_CASES[case]
    return abi.z4_params_from_par(shift=shift, **over), steps


def test_token_semantics_of_the_reference():
    assert abi.getv("gamma0 withGadv withBadv withShiftadv withB", "withB") == 0
    assert abi.getv("gamma0 withB withGadv withBadv", "withB") == 1
    assert abi.getv("1+log withshift", "1+log") == 1
    assert abi.getv("1+log2 withshift", "1+log") == 0


@pytest.mark.parametrize("case", sorted(Z4_CASES))
def test_z4_oracle_matches_reference(case):
    g = load_golden(case)
    lev = golden_level(g)
    p, steps = z4_case(case)
    u = np.ascontiguousarray(g["state_it0_l0"])
    assert relerr(oracle.z4_rhs(lev, u, p), g["rhs_it0_l0"]).max() < 1e-13
    u2 = oracle.z4_evolve(lev, u.copy(), float(g["dt"]), steps, p)
    assert relerr(u2, g["state_it%d_l0" % steps]).max() < 1e-13
