"""CPU FP64 restatement of the warm-start network of libnrgpu (nrgpu_mlp.cu).

TEST INFRASTRUCTURE ONLY: imported by tests/ to check the CUDA kernels
(features, forward, gradients); never by the product package.

The network has no counterpart in the reference, so this file is its
oracle: the same features, layer layout and loss, evaluated in float64.
With ``bf16_ops=True`` every operand of a tensor-core product (features,
hidden activations, hidden weights, back-propagated pre-activation
gradients) is rounded to bfloat16 exactly as the kernels round it, and the
products are then accumulated in float64; with ``bf16_ops=False`` the
network is evaluated in plain float64, which is what the finite-difference
check of the analytic gradient uses.
"""
import numpy as np

IN, HID = 32, 128


def layout():
    """Offsets of the flat parameter vector: W1 [IN][HID], b1, W2..W4
    [HID][HID] with biases, w5 [HID], b5."""
    off, o = {}, 0
    for l in range(4):
        k = IN if l == 0 else HID
        off["W%d" % l] = (o, (k, HID))
        o += k * HID
        off["b%d" % l] = (o, (HID,))
        o += HID
    off["w5"] = (o, (HID,))
    o += HID
    off["b5"] = (o, (1,))
    o += 1
    return off, o


OFF, NPARAMS = layout()


def unpack(p):
    return {k: np.asarray(p[o:o + int(np.prod(s))], dtype=np.float64).reshape(s) for k, (o, s) in OFF.items()}


def pack(d):
    p = np.zeros(NPARAMS)
    for k, (o, s) in OFF.items():
        p[o:o + int(np.prod(s))] = np.asarray(d[k]).ravel()
    return p


def bf16(x):
    """Round to bfloat16 (round to nearest, ties to even) via float32."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64).reshape(f.shape)


def features(cond, pt, m, dx, set_idx=None, round_bf16=True):
    """Feature rows of grid points pt (x fastest) of the m^3 cube of spacing
    dx centred on the origin; cond is (nsets, 20) (m1 m2, pos 6, mom 6,
    spin 6), set_idx picks the binary of each row (default 0)."""
    cond = np.atleast_2d(np.asarray(cond, dtype=np.float64))
    pt = np.asarray(pt, dtype=np.int64)
    c = cond[np.zeros(len(pt), dtype=np.int64) if set_idx is None else np.asarray(set_idx)]
    h0 = -0.5 * (m - 1) * dx
    x = np.stack([h0 + (pt % m) * dx, h0 + ((pt // m) % m) * dx, h0 + (pt // (m * m)) * dx], axis=1)
    s = 1.0 / 8.0
    f = np.zeros((len(pt), IN))
    f[:, 0:3] = x * s
    for q in range(2):
        mq = c[:, q]
        d = x - c[:, 2 + 3 * q:5 + 3 * q]
        r = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
        b = 3 + 12 * q
        f[:, b:b + 3] = d * s
        f[:, b + 3] = r * s
        f[:, b + 4] = mq / (r + mq)
        f[:, b + 5] = 2.0 * mq
        f[:, b + 6:b + 9] = 5.0 * c[:, 8 + 3 * q:11 + 3 * q]
        f[:, b + 9:b + 12] = 5.0 * c[:, 14 + 3 * q:17 + 3 * q]
    return bf16(f) if round_bf16 else f


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, X, bf16_ops=True):
    """Returns (out, cache) for feature rows X."""
    P = unpack(p)
    r = bf16 if bf16_ops else (lambda v: np.asarray(v, dtype=np.float64))
    A = [r(X)]
    Z = []
    for l in range(4):
        z = A[-1] @ r(P["W%d" % l]) + P["b%d" % l]
        Z.append(z)
        A.append(r(silu(z)))
    out = A[-1] @ P["w5"] + P["b5"][0]
    return out, (A, Z, P, r)


def loss_and_grad(p, X, y, bf16_ops=True):
    """MSE loss mean((out - y)^2) and its gradient in the flat layout."""
    out, (A, Z, P, r) = forward(p, X, bf16_ops)
    n = len(y)
    loss = np.mean((out - y) ** 2)
    d = 2.0 * (out - y) / n
    g = {"w5": A[4].T @ d, "b5": np.array([d.sum()])}
    dZ = r(np.outer(d, P["w5"]) * dsilu(Z[3]))
    for l in range(3, -1, -1):
        g["W%d" % l] = A[l].T @ dZ
        g["b%d" % l] = dZ.sum(axis=0)
        if l == 0:
            break
        dA = dZ @ r(P["W%d" % l]).T
        dZ = r(dA * dsilu(Z[l - 1]))
    return loss, pack(g)


def init_params(rng):
    """Normal weights of variance 1/fan_in, zero biases, a small output layer."""
    d = {}
    for l in range(4):
        k = IN if l == 0 else HID
        d["W%d" % l] = rng.standard_normal((k, HID)) / np.sqrt(k)
        d["b%d" % l] = np.zeros(HID)
    d["w5"] = 0.01 * rng.standard_normal(HID)
    d["b5"] = np.zeros(1)
    return pack(d)
