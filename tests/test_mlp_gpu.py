"""The warm-start network on the GPU (nrgpu_mlp_*, BF16 tensor-core products
with FP32 accumulation) against its CPU FP64 oracle with the same BF16
operand rounding (oracle/mlp_oracle.py): features bit-exact, forward and
gradients within the FP32-accumulation error; training reduces the loss;
the trained weights shipped with the package predict u within 5 % on
binaries outside the training seeds; the FP32 inference matches an FP64
forward; the warm start (FP32 guess + damped Jacobi smoothing) lowers the
initial residual and at least halves the V cycles to 1e-10."""
import numpy as np
import pytest
import torch

from baum_b200 import warmstart
from baum_b200.punctures import Binary
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def case(n=2048, m=130, dx=0.125, seed=11):
    rng = np.random.default_rng(seed)
    bins = [Binary.sample(rng) for _ in range(3)]
    conds = np.array([warmstart.cond_vector(b) for b in bins])
    sets = rng.integers(0, 3, n).astype(np.int32)
    pts = rng.integers(0, m ** 3, n).astype(np.int32)
    return rng, conds, sets, pts, m, dx


def net_with(rng, conds, sets, pts, m, dx, scale_out=30.0):
    p = mo.init_params(rng)
    p[mo.OFF["w5"][0]:mo.OFF["w5"][0] + mo.HID] *= scale_out
    p32 = p.astype(np.float32)
    net = warmstart.Network(4096, p32)
    net.set_conditions(conds)
    net.features(torch.from_numpy(sets).cuda(), torch.from_numpy(pts).cuda(), m, dx)
    return net, p32.astype(np.float64)


def test_features_are_bit_exact(gpu):
    rng, conds, sets, pts, m, dx = case()
    net, _ = net_with(rng, conds, sets, pts, m, dx)
    X = net.copy_features(len(pts))
    Xo = mo.features(conds, pts, m, dx, set_idx=sets)
    assert np.array_equal(X, Xo)


def test_forward_matches_oracle(gpu):
    rng, conds, sets, pts, m, dx = case()
    net, p = net_with(rng, conds, sets, pts, m, dx)
    out = net.forward(len(pts)).cpu().numpy().astype(np.float64)
    ref, _ = mo.forward(p, mo.features(conds, pts, m, dx, set_idx=sets))
    assert np.abs(out - ref).max() <= 2e-3 * np.abs(ref).max()


def test_gradients_match_oracle(gpu):
    rng, conds, sets, pts, m, dx = case()
    net, p = net_with(rng, conds, sets, pts, m, dx)
    y = (0.1 * rng.standard_normal(len(pts))).astype(np.float32)
    loss = net.train_step(torch.from_numpy(y).cuda(), 0.0, update=False, want_loss=True)
    g = net.gradients().astype(np.float64)
    lo, go = mo.loss_and_grad(p, mo.features(conds, pts, m, dx, set_idx=sets), y.astype(np.float64))
    assert abs(loss - lo) <= 1e-4 * lo
    for name, (o, s) in mo.OFF.items():
        k = int(np.prod(s))
        a, b = g[o:o + k], go[o:o + k]
        assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b) + 1e-9, name
    # the parameters are untouched without update
    assert np.array_equal(net.params(), p.astype(np.float32))


def test_training_reduces_loss(gpu):
    rng, conds, sets, pts, m, dx = case(n=4096)
    net, _ = net_with(rng, conds, sets, pts, m, dx, scale_out=1.0)
    # a smooth target of the features: the first puncture's m / (r + m)
    X = mo.features(conds, pts, m, dx, set_idx=sets)
    y = torch.from_numpy((X[:, 7] - 0.3).astype(np.float32)).cuda()
    first = net.train_step(y, 1e-3, want_loss=True)
    for _ in range(300):
        last = net.train_step(y, 1e-3, want_loss=True)
    assert last < 0.05 * first


def test_predict_u_matches_oracle(gpu):
    net = warmstart.Network.load()
    b = Binary.sample(np.random.default_rng(99))
    m, dx = 66, 0.5
    u = net.predict_u(b, m, dx).cpu().numpy()
    idx = np.random.default_rng(1).integers(0, m ** 3, 4096)
    ref, _ = mo.forward(net.params().astype(np.float64), mo.features(warmstart.cond_vector(b), idx, m, dx))
    # the oracle rounds the same activations to BF16 after FP64 sums, the
    # device after FP32 sums: an activation may round to the neighbouring
    # BF16 value (2^-8 relative), hence a few 1e-3 of the largest output
    assert np.abs(u[idx] - net.uscale * ref).max() <= 5e-3 * np.abs(net.uscale * ref).max()


@pytest.mark.parametrize("m,dx", [(66, 0.5), (5, 1.0), (130, 0.25)])
def test_predict_u_tc_matches_oracle(gpu, m, dx):
    """The tensor-core forward (tcgen05.mma, TMEM accumulators, weights in
    shared memory) against the oracle's BF16 forward at sampled points and
    against the mma.sync path at every point: partial last tiles (66^3 =
    2246 tiles of 128 and 8 points), a cube smaller than one tile (5^3),
    and the warm start's 130^3 grid.  Same bound as the BF16 path: an
    activation may round to the neighbouring BF16 value, and SiLU uses the
    hardware tanh (relative error about 2^-11)."""
    net = warmstart.Network.load()
    b = Binary.sample(np.random.default_rng(97))
    u = net.predict_u_tc(b, m, dx).cpu().numpy()
    assert np.isfinite(u).all()
    idx = np.random.default_rng(3).integers(0, m ** 3, min(4096, m ** 3))
    ref, _ = mo.forward(net.params().astype(np.float64), mo.features(warmstart.cond_vector(b), idx, m, dx))
    ref = net.uscale * ref
    assert np.abs(u[idx] - ref).max() <= 5e-3 * np.abs(ref).max()
    u16 = net.predict_u(b, m, dx).cpu().numpy()
    assert np.abs(u - u16).max() <= 5e-3 * np.abs(u16).max()


def test_predict_u_tc_writes_into_a_given_buffer_and_repeats(gpu):
    """Into a caller's buffer (canaries around it untouched), twice with
    the same result: the kernel is deterministic (no atomics in the sums)."""
    net = warmstart.Network.load()
    b = Binary.sample(np.random.default_rng(96))
    m = 40
    buf = torch.full((m ** 3 + 2,), 7.0, dtype=torch.float64, device="cuda")
    net.predict_u_tc(b, m, 0.5, out=buf[1:1 + m ** 3])
    first = buf.clone()
    net.predict_u_tc(b, m, 0.5, out=buf[1:1 + m ** 3])
    assert buf[0].item() == 7.0 and buf[-1].item() == 7.0
    assert torch.equal(first, buf)


def test_predict_u_fp32_matches_fp64_forward(gpu):
    """The FP32 evaluation path against an FP64 forward of the same FP32
    weights on unrounded features (numpy): FP32 rounding only, far below
    the BF16 path's 2e-3."""
    net = warmstart.Network.load()
    b = Binary.sample(np.random.default_rng(98))
    m, dx = 66, 0.5
    u = net.predict_u_fp32(b, m, dx).cpu().numpy()
    idx = np.random.default_rng(2).integers(0, m ** 3, 4096)
    P = net.params().astype(np.float64)
    c = warmstart.cond_vector(b)
    h0 = -0.5 * (m - 1) * dx
    x = np.stack([h0 + (idx % m) * dx, h0 + (idx // m % m) * dx, h0 + (idx // (m * m)) * dx], 1)
    f = np.zeros((idx.size, 32))
    f[:, :3] = x / 8
    for q in range(2):
        d = x - c[2 + 3 * q:5 + 3 * q]
        r = np.sqrt((d * d).sum(1))
        g = 3 + 12 * q
        f[:, g:g + 3] = d / 8
        f[:, g + 3] = r / 8
        f[:, g + 4] = c[q] / (r + c[q])
        f[:, g + 5] = 2 * c[q]
        f[:, g + 6:g + 9] = 5 * c[8 + 3 * q:11 + 3 * q]
        f[:, g + 9:g + 12] = 5 * c[14 + 3 * q:17 + 3 * q]
    a, o = f, 0
    for l in range(4):
        k = 32 if l == 0 else 128
        W = P[o:o + k * 128].reshape(k, 128)
        bias = P[o + k * 128:o + k * 128 + 128]
        o += k * 128 + 128
        z = a @ W + bias
        a = z / (1 + np.exp(-z))
    ref = net.uscale * (a @ P[o:o + 128] + P[o + 128])
    assert np.abs(u[idx] - ref).max() <= 2e-5 * np.abs(ref).max()


STANDARD_BINARY = Binary([0.5, 0.5], [[4, 0, 0], [-4, 0, 0]], [[0, 0.1, 0], [0, -0.1, 0]], [[0, 0, 0.1], [0, 0, -0.1]])


def test_warm_start_is_close_and_lowers_the_initial_residual(gpu):
    """On binaries outside the training seeds, at the workload's 130^3 grid,
    the network's u is within 5 % (relative L2) of the multigrid solution,
    and the warm start (that u in FP32, smoothed) starts the V cycles from a
    lower RMS residual than u = 0."""
    from baum_b200 import abi
    from baum_b200.punctures import Multigrid
    net = warmstart.Network.load()
    rng = np.random.default_rng(424242)
    m, dx = warmstart.C2_M, warmstart.C2_DX
    mg = Multigrid(m, dx, abi.mg_params(fullV=0, vcycle_nmax=1))
    ref = Multigrid(m, dx, abi.mg_params(vcycle_nmax=300))
    for b in [STANDARD_BINARY, Binary.sample(rng)]:
        u_ref, _, _ = warmstart.solve_binary(ref, b)
        g = net.predict_u(b, m, dx)
        assert (g - u_ref).norm().item() <= 0.05 * u_ref.norm().item()
        # one V cycle from each start: the RMS residual is tested before it
        a, bb = mg.coefficients(b)
        r0 = mg.solve(a, bb, torch.zeros_like(g))[1]
        rg = mg.solve(a, bb, warmstart.warm_guess(net, mg, b, m, dx))[1]
        assert rg < r0, (rg, r0)
    mg.close()
    ref.close()


def test_warm_start_halves_vcycles(gpu):
    """The north-star target on the workload's grid (130^3, x in
    [-16.1, 16.1]): V cycles to the 1e-10 RMS residual from the warm start
    (the network's u in FP32, 32 damped Jacobi sweeps) at most half of
    those from u = 0, both V cycles and the reference's full-V.  The standard
    binary (measured 329 full-V, 342 V, 75 from the warm start) and a
    held-out draw (4760, 4831, 149)."""
    from baum_b200.punctures import Binary
    net = warmstart.Network.load()
    held = Binary.sample(np.random.default_rng(12))
    rows = warmstart.evaluate(net, [STANDARD_BINARY, held], nmax=8000, log=None)
    for r in rows:
        assert r["res_mlp"] <= 1e-10 and r["res_V"] <= 1e-10 and r["res_fullV"] <= 1e-10, r
        assert 2 * r["V_from_mlp"] <= min(r["V_from_zero"], r["fullV_from_zero"]), r
