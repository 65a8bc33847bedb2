"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from oracle/_ref/bam)."""
import numpy as np
import pytest

from conftest import GOLDEN_SYMMETRY, golden_level, load_golden, relerr
from oracle import oracle
from baum_b200 import abi, punctures

RHS_CASES = {
    "bssn_fourier_o4": dict(),
    "bssn_fourier_o6": dict(order_centered=6, order_advection=6, advection_lopsided6=2),
    "bssn_fourier_o4_ko4": dict(order_dissipation=4, dissfactor=0.1 / 16),
}


@pytest.mark.parametrize("case", sorted(RHS_CASES))
def test_oracle_rhs_matches_reference(case):
    g = load_golden(case)
    lev = golden_level(g)
    p = abi.bssn_params(**RHS_CASES[case])
    u = np.ascontiguousarray(g["state_it0_l0"])
    r = oracle.bssn_rhs(lev, u, p)
    err = relerr(r, g["rhs_it0_l0"])
    assert err.max() < 1e-13, err


@pytest.mark.parametrize("case,steps", [("bssn_fourier_o4", 2), ("bssn_fourier_o6", 1), ("bssn_punc_o4", 4)])
def test_oracle_rk4_matches_reference(case, steps):
    g = load_golden(case)
    lev = golden_level(g)
    over = RHS_CASES.get(case, {})
    p = abi.bssn_params(**over)
    u = np.ascontiguousarray(g["state_it0_l0"])
    oracle.bssn_evolve(lev, u, float(g["dt"]), steps, p)
    err = relerr(u, g["state_it%d_l0" % steps])
    assert err.max() < 1e-13, err


def test_brill_lindquist_matches_reference_initial_data():
    g = load_golden("bssn_punc_o4")
    lev = golden_level(g)
    u = punctures.brill_lindquist_state(lev, [(1.0, 0.0, 0.0, 0.0)])
    # Gamma~ of the reference is round-off noise (~1e-16) from adm_to_bssn
    err = relerr(u, g["state_it0_l0"], floor=1e-3)
    assert err.max() < 1e-12, err


def test_oracle_detects_a_planted_mistake():
    """A wrong KO factor in the oracle must be visible against the golden rhs
    (the comparison is sensitive enough to catch a real defect)."""
    g = load_golden("bssn_fourier_o4")
    lev = golden_level(g)
    p = abi.bssn_params(dissfactor=0.1 / 64 * 1.001)
    r = oracle.bssn_rhs(lev, np.ascontiguousarray(g["state_it0_l0"]), p)
    assert relerr(r, g["rhs_it0_l0"]).max() > 1e-9


@pytest.mark.parametrize("case,steps", [("bssn_punc_octant", 4), ("bssn_fourier_bitant", 2)])
def test_oracle_symmetry_grids_match_reference(case, steps):
    """set_boundary_symmetry: the puncture on an octant grid (reflections
    about x, y and z = 0) and the Fourier data on a bitant grid (z only):
    the rhs with its boundary and the RK4 steps against the reference."""
    g = load_golden(case)
    lev = golden_level(g, GOLDEN_SYMMETRY[case])
    p = abi.bssn_params()
    u = np.ascontiguousarray(g["state_it0_l0"])
    r = oracle.bssn_rhs(lev, u, p)
    # the puncture's rhs of g~ (A~ = 0, no shift) and Gamma~ is round-off
    # noise, ~1e-17: compared absolutely below 1e-3.  The puncture's steep
    # data next to the origin carry the round-off of a different operation
    # order to 1e-13 of K; a missing or wrong reflection is an O(1) error
    assert relerr(r, g["rhs_it0_l0"], floor=1e-3).max() < 1e-12
    oracle.bssn_evolve(lev, u, float(g["dt"]), steps, p)
    err = relerr(u, g["state_it%d_l0" % steps])
    assert err.max() < 1e-12, err
    # the reflections matter: without them the rhs at the ghosts differs
    r0 = oracle.bssn_rhs(golden_level(g), np.ascontiguousarray(g["state_it0_l0"]), p)
    assert relerr(r0, g["rhs_it0_l0"], floor=1e-3).max() > 1e-6
