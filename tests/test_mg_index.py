"""The multigrid kernels find a point's (i, j, k) in an m^3 cube from FP64
products with 1/m and 1/m^2 instead of integer divisions (cube_ijk in
baum_b200/csrc/nrgpu_mg.cu): k = trunc((q + 1/2) / m^2 as a product),
j likewise from the remainder.  The same IEEE operations in numpy give the
exact quotients for every point of every level of the 130^3 and 258^3
stacks, with 1/m^2 rounded once or formed as (1/m)^2."""
import numpy as np
import pytest


@pytest.mark.parametrize("m", [4, 6, 10, 18, 34, 66, 130, 258])
@pytest.mark.parametrize("squared", [False, True])
def test_product_decomposition_is_exact(m, squared):
    q = np.arange(m ** 3, dtype=np.int64)
    rm = 1.0 / m
    rmm = rm * rm if squared else 1.0 / (m * m)
    k = ((q.astype(np.float64) + 0.5) * rmm).astype(np.int64)
    r = q - k * m * m
    j = ((r.astype(np.float64) + 0.5) * rm).astype(np.int64)
    i = r - j * m
    assert np.array_equal(k, q // (m * m))
    assert np.array_equal(j, (q // m) % m)
    assert np.array_equal(i, q % m)
