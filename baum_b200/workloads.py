"""The benchmarked grids, defined once for the benchmark, the fixtures that
pin them and the parity tests.

Batched refinement workload: 7 nested 2:1 levels of uneven size, Z4c 4th
order + KO6, Berger-Oliger subcycling on every level, order_RP 4, amr_nbuffer
3, 3rd-order time interpolation, Fourier data of amplitude 1e-3 (8 modes) on
a flat background.  Level 0: 160^3 inner points and the physical boundary
layer; finer levels: interiors 128, 160, 96, 128, 64, 96 plus 4 points per
side (3 prolonged buffer points and the refinement boundary).  The
dissipation factor is 0.1 on level 0 and 0.2 x 0.1 on finer levels
(get_dissipation_factor, evolve.c:486-530: levels above amr_move_lcube = 0,
physics without "Z4d"), dt = dtfac dx with dtfac 0.25.
"""
import numpy as np

FMR_SIZES = [162, 136, 168, 104, 136, 72, 104]
FMR_DX0 = 0.5
# the same hierarchy shrunk so that the CPU oracle steps it in seconds: the
# same uneven pattern and nesting (every level made of whole parent cells,
# room for the stencils)
FMR_SIZES_SMALL = [42, 40, 44, 32, 40, 24, 32]

# the full form's grid without its moving boxes: 9 nested 2:1 levels, a
# 192^3-inner coarsest box and 128^3 interiors (plus 4 points per side) on
# the 8 finer levels, Z4c 6th order + KO6 (as the precision-sweep box)
C5_SIZES = [194] + [136] * 8
C5_DX0 = 0.5


def fmr_setup(sizes=None, dx0=None, order=4):
    """(levels, per-level Z4c parameters, per-level dt) of a nested grid."""
    from . import abi, fmr
    sizes = sizes or FMR_SIZES
    dx0 = dx0 or FMR_DX0
    levels = fmr.nested_levels(sizes, dx0)
    params = [abi.z4_params_from_par(dissfactor=(0.1 if l == 0 else 0.02) / 64, order_centered=order,
                                     order_advection=order) for l in range(len(levels))]
    dt = [0.25 * dx0 / 2 ** l for l in range(len(levels))]
    return levels, params, dt


def fmr_state_host(level):
    """Initial data of a level on the host (numpy, the oracle's input)."""
    from . import abi, synthetic
    x, y, z = level.coords()
    return synthetic.fourier_state(x, y, z, abi.Z4_NVARS, synthetic.Z4_UNIT, 8, 1e-3, 16.0, 1)


def fmr_state_device(level):
    """The same initial data built on the device (the last bits of the sines
    may differ from fmr_state_host)."""
    import torch
    from . import abi, synthetic
    x, y, z = (torch.from_numpy(c).cuda() for c in level.coords())
    return synthetic.fourier_state_device(x, y, z, abi.Z4_NVARS, synthetic.Z4_UNIT, 8, 1e-3, 16.0, 1)


def sample_points(npoints, n, seed):
    """Sorted distinct point indices at which a stored state is compared."""
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(npoints, size=min(n, npoints), replace=False)).astype(np.int64)


# Tolerance of a refinement level's state against the oracle, relative to
# each field's size: 2e-11 on level 0 (the pin of the 3-level runs against
# the reference), 4x per finer level.  The device and the oracle add the
# stencil terms in different orders; the rounding of a second difference of
# a field of unit background (g~, chi, alpha) is ~eps sum|w| |u| / dx^2, 4x
# per level, and reaches the fields of size 1e-3 through the rhs.  Measured
# on the 7-level grid after one coarse step: 6.5e-13 on level 0, 8e-10 on
# level 6 (Khat: 6e-13 absolute).
def level_tolerance(level):
    return 2e-11 * 4.0 ** level


def stored_state_deviation(u, fixture):
    """Deviation of device states u (one (nvars, npoints) tensor per level)
    from a stored state (tests/golden/make_fmr_c3_fixture.py), per level: at
    the sampled points relative to each field's size (its largest |u| over
    the level), and of the per-variable sums relative to the sums of |u|.
    Returns two lists, one entry per level."""
    import torch
    g = np.load(fixture)
    e_pts, e_sum = [], []
    for l in range(len(g["sizes"])):
        idx = torch.from_numpy(g["idx_l%d" % l]).to(u[l].device)
        a = u[l][:, idx].cpu().numpy()
        b = g["u_l%d" % l]
        e_pts.append(float((np.abs(a - b).max(axis=1) / np.maximum(g["max_l%d" % l], 1e-8)).max()))
        s = u[l].sum(dim=1).cpu().numpy()
        e_sum.append(float((np.abs(s - g["sum_l%d" % l]) / g["abssum_l%d" % l]).max()))
    return e_pts, e_sum
