"""Learned warm start of the puncture multigrid (no counterpart in the reference).

A coordinate MLP conditioned on the binary's parameters (masses, positions,
Bowen-York momenta and spins) predicts the correction u of the puncture
method; the multigrid then runs V cycles from that guess on the finest level
(cycle type "V", not the full-V driver, which would overwrite the guess from
the coarsest level up: solve.c:40,89-91, utility.c:61-82), to the same
1e-10 RMS residual.  The multigrid stays the arbiter: the guess only changes
where it starts.

Everything numeric runs in libnrgpu.so (nrgpu_mlp_*, nrgpu_mg_*): features,
the BF16 tensor-core products, the backward pass, Adam, the inference into
an FP64 u.  This module generates the training set with the GPU multigrid,
trains, evaluates and stores the weights.

    python -m baum_b200.warmstart --sets 2000 --out <dir>
"""
import argparse
import ctypes as C
import functools
import json
import os
import time

import numpy as np
import torch

from . import abi
from .punctures import Binary, Multigrid

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_c2.npz")
USCALE = 0.1
C2_M, C2_DX = 130, 0.25    # nxyz = 128 inner + Robin layer, x in [-16.1, 16.1]
# smoothing of the network's guess before the V cycles: damped Jacobi
# sweeps (the solver itself, undamped Jacobi in FAS V cycles, is unchanged).
# The guess's pointwise error carries grid-scale components that undamped
# Jacobi does not damp (its checkerboard amplification is -1); 32 sweeps at
# omega 2/3 remove them (measured: 8 sweeps 76-2276 V cycles on six binaries,
# 32 sweeps 75-1984; without them as many cycles as from u = 0)
NSMOOTH, OMEGA = 32, 2.0 / 3.0


def cond_vector(b):
    """The 20-double conditioning vector of a binary (two punctures)."""
    if len(b.mass) != 2:
        raise ValueError("the warm start is trained for two punctures")
    return np.concatenate([b.mass, b.pos.ravel(), b.mom.ravel(), b.spin.ravel()]).astype(np.float64)


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class Network:
    """The device network (nrgpu_mlp): parameters, training, inference."""

    def __init__(self, max_batch=16384, params=None, uscale=USCALE):
        L = abi.lib()
        self.nparams = L.nrgpu_mlp_nparams()
        h = C.c_void_p()
        abi.check(L.nrgpu_mlp_create(int(max_batch), C.byref(h)))
        self.handle, self.max_batch, self.uscale = h, max_batch, uscale
        if params is not None:
            self.set_params(params)

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        abi.check(abi.lib().nrgpu_mlp_set_params(self.handle, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))

    def params(self):
        p = np.zeros(self.nparams, dtype=np.float32)
        abi.check(abi.lib().nrgpu_mlp_get_params(self.handle, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))
        return p

    def gradients(self):
        g = np.zeros(self.nparams, dtype=np.float32)
        abi.check(abi.lib().nrgpu_mlp_gradients(self.handle, g.ctypes.data_as(C.POINTER(C.c_float)), g.size))
        return g

    def set_conditions(self, conds):
        """The (nsets, 20) table of conditioning vectors rows refer to."""
        conds = np.ascontiguousarray(np.atleast_2d(conds), dtype=np.float64)
        abi.check(abi.lib().nrgpu_mlp_set_conditions(self.handle, conds.ctypes.data_as(C.POINTER(C.c_double)),
                                                     conds.shape[0]))

    def features(self, set_idx, pt_idx, m, dx):
        """Feature rows of the batch: set_idx, pt_idx int32 CUDA tensors."""
        abi.check(abi.lib().nrgpu_mlp_features(self.handle, C.c_void_p(set_idx.data_ptr()),
                                               C.c_void_p(pt_idx.data_ptr()), int(pt_idx.numel()), int(m),
                                               float(dx), _stream()))

    def copy_features(self, n):
        """The last n feature rows as float64 (exact BF16 values)."""
        h = np.zeros((n, 32), dtype=np.uint16)
        abi.check(abi.lib().nrgpu_mlp_copy_features(self.handle, n, h.ctypes.data_as(C.POINTER(C.c_uint16))))
        return (h.astype(np.uint32) << 16).view(np.float32).astype(np.float64)

    def train_step(self, y, lr, update=True, want_loss=False):
        loss = C.c_float()
        abi.check(abi.lib().nrgpu_mlp_train_step(self.handle, C.c_void_p(y.data_ptr()), int(y.numel()),
                                                 float(lr), int(update), C.byref(loss) if want_loss else None,
                                                 _stream()))
        return loss.value if want_loss else None

    def forward(self, n):
        out = torch.empty(n, dtype=torch.float32, device="cuda")
        abi.check(abi.lib().nrgpu_mlp_forward(self.handle, int(n), C.c_void_p(out.data_ptr()), _stream()))
        return out

    def predict_u(self, binary, m, dx, out=None):
        """The warm start u (m^3 FP64 CUDA tensor) for one binary."""
        cv = cond_vector(binary)
        u = torch.empty(m ** 3, dtype=torch.float64, device="cuda") if out is None else out
        abi.check(abi.lib().nrgpu_mlp_predict_u(self.handle, cv.ctypes.data_as(C.POINTER(C.c_double)), int(m),
                                                float(dx), float(self.uscale), C.c_void_p(u.data_ptr()),
                                                _stream()))
        return u

    def predict_u_fp32(self, binary, m, dx, out=None):
        """The same prediction in FP32 from the FP32 master weights (no BF16
        rounding of features or activations)."""
        cv = cond_vector(binary)
        u = torch.empty(m ** 3, dtype=torch.float64, device="cuda") if out is None else out
        abi.check(abi.lib().nrgpu_mlp_predict_u_fp32(self.handle, cv.ctypes.data_as(C.POINTER(C.c_double)), int(m),
                                                     float(dx), float(self.uscale), C.c_void_p(u.data_ptr()),
                                                     _stream()))
        return u

    def predict_u_tc(self, binary, m, dx, out=None, check=True):
        """The BF16 prediction on the tensor cores (tcgen05): one kernel,
        weights resident in shared memory.  check=True synchronises and
        raises if a bounded wait inside the kernel ran out."""
        cv = cond_vector(binary)
        u = torch.empty(m ** 3, dtype=torch.float64, device="cuda") if out is None else out
        abi.check(abi.lib().nrgpu_mlp_predict_u_tc(self.handle, cv.ctypes.data_as(C.POINTER(C.c_double)), int(m),
                                                   float(dx), float(self.uscale), C.c_void_p(u.data_ptr()),
                                                   _stream()))
        if check:
            flag = C.c_int(0)
            abi.check(abi.lib().nrgpu_mlp_tc_status(self.handle, C.byref(flag)))
        return u

    def save(self, path, **meta):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez_compressed(path, params=self.params(), uscale=self.uscale, meta=json.dumps(meta))

    @staticmethod
    def load(path=WEIGHTS, max_batch=65536):
        z = np.load(path)
        return Network(max_batch, z["params"], float(z["uscale"]))

    def close(self):
        if self.handle:
            abi.lib().nrgpu_mlp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def init_params(rng):
    """Weights of variance 1/fan_in, zero biases, a small output layer (the
    flat layout of nrgpu_mlp: W1 [32][128], b1, W2..W4 [128][128] with
    biases, w5 [128], b5)."""
    parts = []
    for l in range(4):
        k = 32 if l == 0 else 128
        parts += [rng.standard_normal(k * 128) / np.sqrt(k), np.zeros(128)]
    parts += [0.01 * rng.standard_normal(128), np.zeros(1)]
    return np.concatenate(parts).astype(np.float32)


@functools.lru_cache(maxsize=2)
def grid_coords(m, dx):
    h0 = -0.5 * (m - 1) * dx
    i = np.arange(m ** 3)
    return h0 + (i % m) * dx, h0 + ((i // m) % m) * dx, h0 + (i // (m * m)) * dx


def sample_points(b, m, dx, n, rng, near=2.5, frac_near=0.5):
    """n grid points: a fraction frac_near within `near` of a puncture (where
    u varies fastest), the rest uniform over the cube."""
    x, y, z = grid_coords(m, dx)
    close = np.zeros(x.size, dtype=bool)
    for p in b.pos:
        close |= (x - p[0]) ** 2 + (y - p[1]) ** 2 + (z - p[2]) ** 2 < near * near
    cand = np.flatnonzero(close)
    k = int(n * frac_near)
    return np.concatenate([rng.integers(0, m ** 3, n - k), rng.choice(cand, k, replace=len(cand) < k)])


def solve_binary(mg, b, u=None):
    """GPU multigrid of binary b from u (zeros by default); returns (u,
    V cycles, residual)."""
    a, bb = mg.coefficients(b)
    if u is None:
        u = torch.zeros(mg.m ** 3, dtype=torch.float64, device="cuda")
    n, res = mg.solve(a, bb, u)
    return u, n, res


def generate(binaries, m=C2_M, dx=C2_DX, npts=16384, cycles=80, seed=0, frac_near=0.5, log=print):
    """Training set: each binary solved by the GPU full-V multigrid (capped
    at `cycles` V cycles, residual ~1e-8), npts sampled points per binary.
    Returns (conds[nsets,20], set_idx, pt_idx, y = u / USCALE)."""
    rng = np.random.default_rng(seed)
    mg = Multigrid(m, dx, abi.mg_params(vcycle_nmax=cycles))
    conds, sets, pts, ys = [], [], [], []
    t0 = time.time()
    for s, b in enumerate(binaries):
        u, n, res = solve_binary(mg, b)
        uh = u.cpu().numpy()
        idx = sample_points(b, m, dx, npts, rng, frac_near=frac_near)
        conds.append(cond_vector(b))
        sets.append(np.full(npts, s, dtype=np.int32))
        pts.append(idx.astype(np.int32))
        ys.append((uh[idx] / USCALE).astype(np.float32))
        if log and (s % 200 == 0 or s == len(binaries) - 1):
            log("  set %d/%d: %d V cycles, residual %.2e, max|u| %.3f (%.0f s)"
                % (s + 1, len(binaries), n, res, np.abs(uh).max(), time.time() - t0))
    mg.close()
    return np.array(conds), np.concatenate(sets), np.concatenate(pts), np.concatenate(ys)


def train(net, data, m=C2_M, dx=C2_DX, epochs=12, batch=16384, lr0=2e-3, lr1=2e-5, seed=1, log=print):
    """Adam with a cosine rate from lr0 to lr1 over all steps; the rows are
    reshuffled every epoch.  Returns the per-epoch mean sampled losses."""
    conds, sets, pts, ys = data
    net.set_conditions(conds)
    rng = np.random.default_rng(seed)
    n = (len(ys) // batch) * batch
    steps = epochs * (n // batch)
    hist, k = [], 0
    for e in range(epochs):
        perm = rng.permutation(len(ys))[:n]
        ds = torch.from_numpy(sets[perm]).cuda()
        dp = torch.from_numpy(pts[perm]).cuda()
        dy = torch.from_numpy(ys[perm]).cuda()
        tot, cnt = 0.0, 0
        for i in range(0, n, batch):
            lr = lr1 + 0.5 * (lr0 - lr1) * (1.0 + np.cos(np.pi * k / steps))
            net.features(ds[i:i + batch], dp[i:i + batch], m, dx)
            want = (i // batch) % 50 == 0
            l = net.train_step(dy[i:i + batch], lr, want_loss=want)
            if want:
                tot, cnt = tot + l, cnt + 1
            k += 1
        hist.append(tot / max(1, cnt))
        if log:
            log("  epoch %d: loss %.3e (lr %.1e)" % (e + 1, hist[-1], lr))
    torch.cuda.synchronize()
    return hist


def warm_guess(net, mg, b, m, dx, nsmooth=NSMOOTH, omega=OMEGA, path="fp32"):
    """The product warm start: the network's u in FP32 (path "fp32"), or in
    BF16 on the tensor cores (path "tc"), then nsmooth damped Jacobi sweeps
    on the finest level."""
    g = net.predict_u_tc(b, m, dx) if path == "tc" else net.predict_u_fp32(b, m, dx)
    if nsmooth:
        a, bb = mg.coefficients(b)
        mg.smooth(a, bb, g, nsmooth, omega)
    return g


def evaluate(net, binaries, m=C2_M, dx=C2_DX, nmax=2000, nsmooth=NSMOOTH, log=print):
    """V cycles (and ms) to 1e-10 for each binary from six starts: full-V
    from u = 0 (the reference's default), V cycles from u = 0, V cycles from
    the network's u as trained (BF16), in FP32, in FP32 followed by nsmooth
    damped Jacobi sweeps (the warm start, "V_from_mlp"), and the tensor-core
    BF16 u followed by the same sweeps ("V_from_mlp_tc").  A count of nmax
    means the cap was reached (res_* > 1e-10)."""
    mg = Multigrid(m, dx, abi.mg_params(vcycle_nmax=nmax))
    mgv = Multigrid(m, dx, abi.mg_params(vcycle_nmax=nmax, fullV=0))

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return r, 1e3 * (time.perf_counter() - t0)

    rows = []
    for b in binaries:
        (_, n_full, r_full), t_full = timed(lambda: solve_binary(mg, b))
        (u0, n_v, r_v), t_v = timed(lambda: solve_binary(mgv, b))
        g16, t_inf16 = timed(lambda: net.predict_u(b, m, dx))
        g32, t_inf32 = timed(lambda: net.predict_u_fp32(b, m, dx))
        _, t_inftc = timed(lambda: net.predict_u_tc(b, m, dx))
        gs, t_guess = timed(lambda: warm_guess(net, mgv, b, m, dx, nsmooth))
        gt, t_guess_tc = timed(lambda: warm_guess(net, mgv, b, m, dx, nsmooth, path="tc"))
        nrm = u0.norm().item()
        errs = [(g - u0).norm().item() / nrm for g in (g16, g32, gs)]
        (_, n_16, r_16), t_16 = timed(lambda: solve_binary(mgv, b, u=g16))
        (_, n_32, r_32), t_32 = timed(lambda: solve_binary(mgv, b, u=g32))
        (_, n_w, r_w), t_w = timed(lambda: solve_binary(mgv, b, u=gs))
        (_, n_t, r_t), t_t = timed(lambda: solve_binary(mgv, b, u=gt))
        rows.append({"cond": cond_vector(b).tolist(),
                     "fullV_from_zero": n_full, "V_from_zero": n_v, "V_from_mlp_bf16": n_16,
                     "V_from_mlp_fp32": n_32, "V_from_mlp": n_w, "V_from_mlp_tc": n_t, "res_mlp_tc": r_t,
                     "ms_mlp_tc": t_t + t_guess_tc, "inference_ms_tc": t_inftc, "guess_ms_tc": t_guess_tc,
                     "res_fullV": r_full, "res_V": r_v, "res_mlp_bf16": r_16, "res_mlp_fp32": r_32, "res_mlp": r_w,
                     "ms_fullV": t_full, "ms_V": t_v, "ms_mlp": t_w + t_guess,
                     "mlp_rel_l2_error_bf16": errs[0], "mlp_rel_l2_error_fp32": errs[1],
                     "mlp_rel_l2_error_smoothed": errs[2], "inference_ms_bf16": t_inf16, "inference_ms_fp32": t_inf32,
                     "guess_ms": t_guess, "nsmooth": nsmooth})
        if log:
            log("  fullV %4d  V %4d  V(mlp bf16) %4d  V(mlp fp32) %4d  V(mlp fp32 + %d sweeps) %4d  V(mlp tc + "
                "sweeps) %4d   |u_mlp-u|/|u| %.2e %.2e %.2e" % (n_full, n_v, n_16, n_32, nsmooth, n_w, n_t, *errs))
    mg.close()
    mgv.close()
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sets", type=int, default=2000)
    ap.add_argument("--heldout", type=int, default=12)
    ap.add_argument("--npts", type=int, default=16384)
    ap.add_argument("--cycles", type=int, default=80)
    ap.add_argument("--epochs", type=int, default=12)
    # training draws from this seed, held-out draws from seed + 1 + i; the
    # benchmark's draws come from another stream (seed 2024)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--frac-near", type=float, default=0.5)
    ap.add_argument("--eval-nmax", type=int, default=2000)
    ap.add_argument("--out", default=os.path.dirname(WEIGHTS))
    a = ap.parse_args()
    torch.cuda.set_device(0)
    abi.check(abi.lib().nrgpu_init(0))
    rng = np.random.default_rng(a.seed)
    train_b = [Binary.sample(rng) for _ in range(a.sets)]
    held_b = [Binary.sample(np.random.default_rng(a.seed + 1 + i)) for i in range(a.heldout)]
    t0 = time.time()
    print("generating %d solutions at %d^3" % (a.sets, C2_M), flush=True)
    data = generate(train_b, npts=a.npts, cycles=a.cycles, seed=a.seed, frac_near=a.frac_near)
    t_gen = time.time() - t0
    net = Network(16384, init_params(np.random.default_rng(a.seed + 7)))
    t0 = time.time()
    hist = train(net, data, epochs=a.epochs)
    t_train = time.time() - t0
    path = os.path.join(a.out, "warmstart_c2.npz")
    net.save(path, sets=a.sets, npts=a.npts, cycles=a.cycles, epochs=a.epochs, seed=a.seed, m=C2_M, dx=C2_DX,
             frac_near=a.frac_near)
    print("evaluating on %d held-out binaries" % a.heldout, flush=True)
    rows = evaluate(Network.load(path), held_b, nmax=a.eval_nmax)
    rep = {"train_seconds": t_train, "generate_seconds": t_gen, "loss_history": hist, "heldout": rows,
           "weights": path}
    with open(os.path.join(a.out, "warmstart_report.json"), "w") as f:
        json.dump(rep, f, indent=1)
    print(json.dumps({k: v for k, v in rep.items() if k != "heldout"}))


if __name__ == "__main__":
    main()
