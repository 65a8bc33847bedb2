"""The ADM diagnostics of the oracle against the reference (golden dumps of
bssn_to_adm / z4_to_adm, adm_constraints_N with normalised constraints, and
the flag-0 norms of reduce.c)."""
import numpy as np
import pytest

from conftest import golden_level, load_golden, relerr
from oracle import oracle

# case: (state dump, constraint dump, order_centered, normalisation mode)
CON_CASES = {
    "bssn_punc_con": ("state_it3_l0", "con_it3_l0", 4, 1),
    "z4_fourier_con": ("state_it2_l0", "con_it2_l0", 6, 2),
}


def con_case(case):
    g = load_golden(case)
    st, cn, order, mode = CON_CASES[case]
    return g, golden_level(g), np.ascontiguousarray(g[st]), g[cn], order, mode


def check_constraints(out, ref, tol=1e-11):
    """ham and mom_i to tol relative to their largest value; a normalised
    constraint c/D to the error that allows in c, divided by D (D is read
    off the reference as c / (c/D))."""
    err = np.abs(out - ref)
    scale = np.abs(ref[:4]).max(axis=1)
    assert (err[:4].max(axis=1) / scale).max() < tol
    for a in range(out.shape[0] - 4):
        nz = ref[4 + a] != 0
        den = np.full(ref.shape[1], np.inf)
        den[nz] = np.abs(ref[a, nz] / ref[4 + a, nz])
        assert (err[4 + a] <= tol * scale[a] / den + 1e-14).all()


@pytest.mark.parametrize("case", sorted(CON_CASES))
def test_to_adm_matches_reference(case):
    g, lev, u, con, order, mode = con_case(case)
    adm = oracle.to_adm(lev, u, -4.0)
    assert relerr(adm, con[:12]).max() < 1e-15


@pytest.mark.parametrize("case", sorted(CON_CASES))
def test_constraints_match_reference(case):
    g, lev, u, con, order, mode = con_case(case)
    inner = g["boundary"] == 0
    out = oracle.adm_constraints(lev, np.ascontiguousarray(con[:12]), order, mode)
    check_constraints(out[:, inner], con[12:20][:, inner])


@pytest.mark.parametrize("case", sorted(CON_CASES))
def test_norms_of_reference_constraints(case):
    g, lev, u, con, order, mode = con_case(case)
    inner = g["boundary"] == 0
    n2, ninf = oracle.norms(lev, con[12:16])
    ref = con[12:16][:, inner]
    np.testing.assert_allclose(n2, np.sqrt((ref ** 2).mean(axis=1)), rtol=1e-14)
    np.testing.assert_array_equal(ninf, np.abs(ref).max(axis=1))


def test_oracle_hamiltonian_converges_on_brill_lindquist():
    """ham = 0 for time-symmetric Brill-Lindquist data; away from the
    puncture the discrete ham falls as h^4 at order 4."""
    from baum_b200 import abi, punctures

    def rms(n, dx, order):
        lev = abi.Level.single_box(n + 2, dx)
        u0 = punctures.brill_lindquist_state(lev, [(1.0, 0.0, 0.0, 0.0)])
        con = oracle.adm_constraints(lev, oracle.to_adm(lev, u0), order, 0)
        x, y, z = lev.coords()
        sel = (np.sqrt(x ** 2 + y ** 2 + z ** 2) > 2.0) & (np.maximum(np.maximum(abs(x), abs(y)), abs(z)) < 5.0)
        return np.sqrt((con[0][sel] ** 2).mean())
    assert 12.0 < rms(32, 0.5, 4) / rms(64, 0.25, 4) < 21.0
