"""The CPU multigrid oracle against the reference's own puncture solve
(golden fixture from tests/golden/make_golden.py)."""
import numpy as np

from conftest import load_golden
from oracle import oracle
from baum_b200 import abi, punctures

BINARY_34 = punctures.Binary([0.5, 0.6], [[2.1, 0, 0], [-2.6, 0, 0]], [[0, 0.1, 0], [0, -0.1, 0]],
                             [[0, 0, 0.1], [-0.05, 0, 0.08]])


def test_mg_oracle_reproduces_reference_cycles_and_solution():
    g = load_golden("mg_binary_34")
    m, dx = int(g["m"]), float(g["dx"])
    a, b = oracle.puncture_coefficients(m, dx, BINARY_34)
    u, n, hist = oracle.mg_solve(m, dx, a, b)
    assert n == int(g["vcycles"])
    assert abs(hist[n] - float(g["residual"])) <= 1e-9 * float(g["residual"])
    assert np.abs(u - g["u"]).max() <= 1e-14 * np.abs(g["u"]).max()


def test_mg_oracle_stack_sizes():
    import ctypes as C
    L = oracle.lib()
    buf = (C.c_int * 32)()
    n = L.oracle_mg_stack_sizes(130, 4, -1, buf, 32)
    assert list(buf[:n]) == [130, 66, 34, 18, 10, 6, 4]
