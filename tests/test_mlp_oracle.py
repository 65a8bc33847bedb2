"""The warm-start network's CPU oracle: its analytic gradient against
central finite differences (plain float64), and its bf16 rounding."""
import numpy as np

from oracle import mlp_oracle as mo


def small_case(seed=3, n=48):
    rng = np.random.default_rng(seed)
    p = mo.init_params(rng)
    p[mo.OFF["w5"][0]:mo.OFF["w5"][0] + mo.HID] *= 30.0  # a non-trivial output layer
    cond = np.concatenate([[0.5, 0.6], [3, 0, 0, -3, 0, 0], [0, 0.1, 0, 0, -0.1, 0], rng.uniform(-0.2, 0.2, 6)])
    X = mo.features(cond, rng.integers(0, 34 ** 3, n), 34, 0.5, round_bf16=False)
    y = rng.standard_normal(n) * 0.1
    return p, X, y, rng


def test_gradient_matches_finite_differences():
    p, X, y, rng = small_case()
    _, g = mo.loss_and_grad(p, X, y, bf16_ops=False)
    idx = np.concatenate([rng.choice(mo.NPARAMS, 60, replace=False), [mo.NPARAMS - 1]])
    for i in idx:
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss_and_grad(pp, X, y, False)[0] - mo.loss_and_grad(pm, X, y, False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * np.abs(g).max() + 1e-7 * abs(g[i]), (i, fd, g[i])


def test_bf16_rounding_is_round_to_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -7, -2.5, 3.1415926])
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0            # tie -> even (down)
    assert r[2] == 1.0 + 2 ** -6                  # tie -> even (up)
    assert r[3] == 1.0 + 2 ** -7
    assert r[4] == -2.5
    assert abs(r[5] - 3.140625) < 1e-12


def test_bf16_gradient_is_close_to_exact():
    p, X, y, _ = small_case(5)
    _, g = mo.loss_and_grad(p, X, y, bf16_ops=False)
    _, gb = mo.loss_and_grad(p, X, y, bf16_ops=True)
    assert np.linalg.norm(gb - g) / np.linalg.norm(g) < 0.05


def test_layout_matches_the_library():
    from baum_b200 import abi, build
    build.build()
    assert abi.lib().nrgpu_mlp_nparams() == mo.NPARAMS
