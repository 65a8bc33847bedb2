"""Parity of the CUDA multigrid (through the C ABI) with the reference's
puncture solve (golden) and with the CPU oracle: the same number of V cycles
to the 1e-10 RMS residual, and the same u to 1e-10 relative."""
import numpy as np
import pytest
import torch

from conftest import load_golden
from oracle import oracle
from baum_b200 import abi, punctures
from test_mg_oracle_pin import BINARY_34

pytestmark = pytest.mark.gpu


def test_coefficients_match_oracle(gpu):
    mg = punctures.Multigrid(34, 0.5)
    a, b = mg.coefficients(BINARY_34)
    ao, bo = oracle.puncture_coefficients(34, 0.5, BINARY_34)
    assert np.abs(a.cpu().numpy() - ao).max() <= 1e-13 * np.abs(ao).max()
    assert np.abs(b.cpu().numpy() - bo).max() <= 1e-12 * np.abs(bo).max()


def test_mg_matches_reference_cycles_and_solution(gpu):
    g = load_golden("mg_binary_34")
    m, dx = int(g["m"]), float(g["dx"])
    mg = punctures.Multigrid(m, dx)
    a, b = mg.coefficients(BINARY_34)
    u = torch.zeros(m ** 3, dtype=torch.float64, device="cuda")
    n, res = mg.solve(a, b, u)
    assert n == int(g["vcycles"])
    assert res <= 1e-10
    assert np.abs(u.cpu().numpy() - g["u"]).max() <= 1e-10 * np.abs(g["u"]).max()


@pytest.mark.parametrize("batch", [1, 5])
def test_mg_cycle_count_independent_of_batching(gpu, batch):
    g = load_golden("mg_binary_34")
    m, dx = int(g["m"]), float(g["dx"])
    mg = punctures.Multigrid(m, dx, abi.mg_params(batch=batch))
    a, b = mg.coefficients(BINARY_34)
    u = torch.zeros(m ** 3, dtype=torch.float64, device="cuda")
    n, _ = mg.solve(a, b, u)
    assert n == int(g["vcycles"])


def test_mg_finest_only_cycles_match_oracle(gpu):
    """mg_typeofcycles != fullV: V cycles from the finest level only."""
    p = abi.mg_params(fullV=0)
    mg = punctures.Multigrid(34, 0.5, p)
    a, b = mg.coefficients(BINARY_34)
    u = torch.zeros(34 ** 3, dtype=torch.float64, device="cuda")
    n, _ = mg.solve(a, b, u)
    ao, bo = oracle.puncture_coefficients(34, 0.5, BINARY_34)
    uo, no, _ = oracle.mg_solve(34, 0.5, ao, bo, params=p)
    assert n == no
    assert np.abs(u.cpu().numpy() - uo).max() <= 1e-10 * np.abs(uo).max()


def test_mg_130_binary_matches_oracle(gpu):
    """The 129^3-cell grid of the binary-puncture workload (130^3 points,
    stack 130-66-34-18-10-6-4), one seeded parameter set, 40 V cycles (the
    oracle needs ~0.1 s per cycle at this size)."""
    rng = np.random.default_rng(2024)
    bi = punctures.Binary.sample(rng)
    m, dx = 130, 0.125
    p = abi.mg_params(vcycle_nmax=40)
    mg = punctures.Multigrid(m, dx, p)
    a, b = mg.coefficients(bi)
    u = torch.zeros(m ** 3, dtype=torch.float64, device="cuda")
    n, res = mg.solve(a, b, u)
    ao, bo = oracle.puncture_coefficients(m, dx, bi)
    uo, no, _ = oracle.mg_solve(m, dx, ao, bo, params=p)
    assert n == no, (n, no)
    assert np.abs(u.cpu().numpy() - uo).max() <= 1e-10 * np.abs(uo).max()
