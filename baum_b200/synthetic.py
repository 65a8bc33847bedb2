"""Synthetic evolution data: a flat background plus seeded Fourier modes.

The batched FMR workload starts every level from g~ = delta, chi = 1,
alpha = 1, all other fields 0, plus a sum of nmodes sine modes of amplitude
amp per field, with integer wave numbers in [-2, 2] per axis on a box of
length L and random coefficients and phases.  The draws come from a
splitmix64 stream in a fixed order (all wave vectors first, then per field
the (coefficient, phase) pair of each mode), so that the oracle harness of
the reference build and this module produce the same state from the same
seed.  Evaluated per point from the coordinates, the data are consistent
across refinement levels.
"""
import numpy as np

MASK = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed):
        self.state = seed & MASK

    def next(self):
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def uniform01(self):
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)


# rows whose background is 1: g~xx g~yy g~zz chi and alpha
BSSN_UNIT = (0, 3, 5, 6, 17)
Z4_UNIT = (0, 3, 5, 6, 18)


def fourier_state(x, y, z, nvars, unit_rows, nmodes=8, amp=1e-3, length=16.0, seed=1):
    """(nvars, npoints) state at the points (x, y, z)."""
    g = SplitMix64(seed)
    k = np.zeros((nmodes, 3))
    for m in range(nmodes):
        for i in range(3):
            n = int(g.next() % 5) - 2
            k[m, i] = 2.0 * np.pi * n / length
    u = np.zeros((nvars, x.size))
    for v in range(nvars):
        c = np.zeros(nmodes)
        ph = np.zeros(nmodes)
        for m in range(nmodes):
            c[m] = 2.0 * g.uniform01() - 1.0
            ph[m] = 2.0 * np.pi * g.uniform01()
        s = np.zeros(x.size)
        for m in range(nmodes):
            s += c[m] * np.sin(k[m, 0] * x + k[m, 1] * y + k[m, 2] * z + ph[m])
        u[v] = (1.0 if v in unit_rows else 0.0) + amp * s
    return u


def fourier_state_device(x, y, z, nvars, unit_rows, nmodes=8, amp=1e-3, length=16.0, seed=1):
    """The same state built on the device from CUDA coordinate tensors (the
    same draws; the sums run in torch, so the last bits may differ from
    fourier_state)."""
    import torch
    g = SplitMix64(seed)
    k = [[0.0] * 3 for _ in range(nmodes)]
    for m in range(nmodes):
        for i in range(3):
            k[m][i] = 2.0 * np.pi * (int(g.next() % 5) - 2) / length
    u = torch.empty((nvars, x.numel()), dtype=torch.float64, device=x.device)
    for v in range(nvars):
        cp = [(2.0 * g.uniform01() - 1.0, 2.0 * np.pi * g.uniform01()) for _ in range(nmodes)]
        s = torch.zeros_like(x)
        for m, (c, ph) in enumerate(cp):
            s += c * torch.sin(k[m][0] * x + k[m][1] * y + k[m][2] * z + ph)
        u[v] = (1.0 if v in unit_rows else 0.0) + amp * s
    return u
