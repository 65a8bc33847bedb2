"""Moving boxes on the device (nrgpu_fmr_regrid, nrgpu_fmr_set_move): the
data transfer of move_box (move.c:808-986) and move_overlap (move.c:712-800)
checked by properties that hold at any size, and the points in the
Berger-Oliger recursion where the hook runs (main.c:426-428 with the time
test of move.c:853-856).  The reference's own moving grid, driven through
BAM, is compared in tests/test_bam_binding_gpu.py.

* Every point of a moved level that an old box also held keeps its value
  bit for bit, in the state and in every time level of a parent level.
* Every other point is the parent's value prolonged at order_RP: with
  data that are a polynomial of degree 3 in each coordinate, 4th-order
  Lagrange prolongation reproduces it to rounding.
* A regrid to the same boxes changes nothing, and the following coarse
  steps are bit for bit those without it.
"""
import numpy as np
import pytest
import torch

from baum_b200 import abi, fmr

pytestmark = pytest.mark.gpu

SIZES = [26, 24, 24]
DX0 = 0.5


def poly(x, y, z, v):
    """Degree <= 3 in each coordinate, different per variable: a small
    perturbation of flat space (1 on the diagonal metric, chi and lapse of
    the Z4c list, synthetic.Z4_UNIT), so that the state also evolves."""
    from baum_b200 import synthetic
    a = 1.0 + 0.01 * v
    p = a * 1e-3 * (1.0 + 0.3 * x - 0.2 * y + 0.1 * z + 0.05 * x * x * y - 0.02 * z ** 3 + 0.01 * x * y * z
                    + 0.003 * (x * y) ** 2 * z)
    return p + (1.0 if v in synthetic.Z4_UNIT else 0.0)


def state_of(level, nv, marker=0.0):
    x, y, z = level.coords()
    out = np.stack([poly(x, y, z, v) for v in range(nv)])
    if marker:
        out = out + marker * np.sin(1.3 * x + 0.7 * y - 0.4 * z + np.arange(nv)[:, None])
    return out


def shifted(level, l, di, dj=0, dk=0):
    """The single box of a level moved by (di, dj, dk) points (multiples of
    2: whole parent cells), REFBOUND on its outer layer."""
    b = level.boxes[0]
    dx = level.dx
    m = b.m
    i = np.arange(m)
    edge = (i == 0) | (i == m - 1)
    e3 = edge[None, None, :] | edge[None, :, None] | edge[:, None, None]
    flags = np.where(e3, -1, 0).astype(np.int32).ravel()
    return abi.Level([(m, b.n, b.o, b.x0 + di * dx, b.y0 + dj * dx, b.z0 + dk * dx)], dx, flags)


def hierarchy(order_ti=3):
    levels = fmr.nested_levels(SIZES, DX0)
    params = [abi.z4_params(dissfactor=0.1 / 64) for _ in levels]
    dt = [0.125 / 2 ** l for l in range(len(levels))]
    fp = abi.fmr_params(system=abi.SYSTEM_Z4C, use_graph=0, order_timeinterpolation=order_ti, autotune=0)
    return fmr.Hierarchy(levels, dt, params, fp), levels


def ckpt_parts(buf, nps, nv, nh):
    """up, upp and the older time levels of every parent level from a
    nrgpu_fmr_save buffer (header, point counts, counters, then per parent
    level up, upp, hist...)."""
    nl = len(nps)
    off = 16 + 8 * nl + 4 * nl
    parts = []
    for l in range(nl - 1):
        n = nv * nps[l]
        arrs = []
        for _ in range(2 + nh):
            arrs.append(np.frombuffer(buf[off:off + 8 * n].tobytes(), dtype=np.float64).reshape(nv, nps[l]))
            off += 8 * n
        parts.append(arrs)
    return parts, off


def coords_key(level):
    x, y, z = level.coords()
    return {(round(a / level.dx * 4), round(b / level.dx * 4), round(c / level.dx * 4)): i
            for i, (a, b, c) in enumerate(zip(x, y, z))}


def check_moved(old_level, new_level, old_vals, new_vals, nv, tol=1e-12):
    """Held points copied bit for bit, the others the polynomial."""
    ko = coords_key(old_level)
    x, y, z = new_level.coords()
    held = np.zeros(new_level.npoints, dtype=bool)
    for i, key in enumerate(zip(*(np.round(np.array(c) / new_level.dx * 4).astype(int) for c in (x, y, z)))):
        j = ko.get(tuple(int(q) for q in key))
        if j is not None:
            held[i] = True
            assert np.array_equal(new_vals[:, i], old_vals[:, j])
    assert held.any() and (~held).any()
    want = np.stack([poly(x, y, z, v) for v in range(nv)])[:, ~held]
    err = np.abs(new_vals[:, ~held] - want).max() / np.abs(want).max()
    assert err < tol, err
    return held


def test_regrid_finest_level_copies_held_points_and_prolongs_the_rest(gpu):
    H, levels = hierarchy()
    nv = H.nv
    u = [torch.from_numpy(state_of(lv, nv, marker=1e-5 if l == 2 else 0.0)).cuda() for l, lv in enumerate(levels)]
    old2 = u[2].cpu().numpy().copy()
    new2 = shifted(levels[2], 2, 2, -2, 4)
    H.regrid(2, [new2], u)
    got = u[2].cpu().numpy()
    check_moved(levels[2], new2, old2, got, nv)
    # the flags of the moved level are those of a fresh hierarchy with the
    # same boxes
    fp, _ = H.flags(2)
    G = fmr.Hierarchy(levels[:2] + [new2], [0.125, 0.0625, 0.03125], [abi.z4_params()] * 3,
                      abi.fmr_params(system=abi.SYSTEM_Z4C, use_graph=0, autotune=0))
    fp2, _ = G.flags(2)
    _, fr1 = H.flags(1)
    _, fr2 = G.flags(1)
    assert np.array_equal(fp, fp2) and np.array_equal(fr1, fr2)
    G.close()
    H.close()


@pytest.mark.parametrize("order_ti", [3, 5])
def test_regrid_parent_level_moves_every_time_level(gpu, order_ti):
    """Level 1 (a parent) moves by one of its parent's cells in x and y;
    level 2 keeps its boxes.  The state and the time levels (u_p, u_pp and
    u_p2, u_p3 at order 5) follow the copy-or-prolong rule."""
    H, levels = hierarchy(order_ti)
    nv = H.nv
    nh = max(0, order_ti - 3)
    u = [torch.from_numpy(state_of(lv, nv, marker=2e-5 if l == 1 else 0.0)).cuda() for l, lv in enumerate(levels)]
    # time levels: the polynomial on level 0, the marked polynomial on level 1
    nps = [lv.npoints for lv in levels]
    buf = H.save()
    parts, _ = ckpt_parts(buf, nps, nv, nh)
    buf = buf.copy()
    off = 16 + 8 * 3 + 4 * 3
    for l in range(2):
        for q in range(2 + nh):
            a = state_of(levels[l], nv, marker=(3e-5 * (q + 1)) if l == 1 else 0.0)
            buf[off:off + a.nbytes] = np.frombuffer(a.tobytes(), dtype=np.uint8)
            off += a.nbytes
    H.load(buf)
    old_u1 = u[1].cpu().numpy().copy()
    old_parts, _ = ckpt_parts(H.save(), nps, nv, nh)
    new1 = shifted(levels[1], 1, 2, 2)
    H.regrid(1, [new1, None], u)
    check_moved(levels[1], new1, old_u1, u[1].cpu().numpy(), nv)
    new_parts, _ = ckpt_parts(H.save(), [lv.npoints for lv in H.levels], nv, nh)
    for q in range(2 + nh):
        check_moved(levels[1], new1, old_parts[1][q], new_parts[1][q], nv)
        assert np.array_equal(new_parts[0][q], old_parts[0][q])
    # the hierarchy steps on with the moved level
    H.advance(u, 1)
    torch.cuda.synchronize()
    assert all(bool(torch.isfinite(t).all()) for t in u)
    H.close()


def test_regrid_to_the_same_boxes_changes_nothing(gpu):
    """Levels 1 and 2 regridded onto their own boxes between two coarse
    steps: the state after the second step is bit for bit that of a run
    without the regrid."""
    from baum_b200 import synthetic
    runs = []
    for regrid in (False, True):
        H, levels = hierarchy()
        u = []
        for lv in levels:
            x, y, z = lv.coords()
            u.append(torch.from_numpy(synthetic.fourier_state(x, y, z, abi.Z4_NVARS, synthetic.Z4_UNIT, 8, 0.05,
                                                              16.0, 5)).cuda())
        H.advance(u, 1)
        if regrid:
            H.regrid(1, [shifted(levels[1], 1, 0), shifted(levels[2], 2, 0)], u)
        H.advance(u, 1)
        torch.cuda.synchronize()
        runs.append([t.cpu().numpy() for t in u])
        H.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


def test_move_hook_runs_where_the_reference_moves_boxes(gpu):
    """move_box(g, l + 1) after level l and its sublevels (main.c:428) when
    l = 0 or level l is not aligned with level l - 1: per coarse step of a
    4-level hierarchy, after the first substep of level 2 (hook 3), after
    the first substep of level 1 (hook 2, once its sublevels are done), after
    the first substep of level 2 again, then after level 0 (hook 1).  A
    hook that moves the finest box by one parent cell per call keeps the
    run going, with the pairs set up again each time."""
    levels = fmr.nested_levels([26, 24, 24, 24], DX0)
    params = [abi.z4_params(dissfactor=0.1 / 64) for _ in levels]
    dt = [0.125 / 2 ** l for l in range(4)]
    H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(system=abi.SYSTEM_Z4C, autotune=0))
    u = [torch.from_numpy(state_of(lv, H.nv)).cuda() for lv in levels]
    calls = []
    sign = [1]

    def hook(l, stream):
        calls.append((l, [H.iteration(q) for q in range(4)]))
        if l == 3:
            sign[0] = -sign[0]
            H.regrid(3, [shifted(H.levels[3], 3, 2 * sign[0])], u, stream)

    H.set_move(hook)
    H.advance(u, 2)
    torch.cuda.synchronize()
    assert [c[0] for c in calls] == [3, 2, 3, 1] * 2, calls
    assert calls[0][1] == [1, 1, 1, 2] and calls[3][1] == [1, 2, 4, 8]
    assert all(bool(torch.isfinite(t).all()) for t in u)
    H.set_move(None)
    H.close()
