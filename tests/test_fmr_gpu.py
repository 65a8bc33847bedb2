"""The mesh-refinement driver on the GPU (nrgpu_fmr_*) against the reference
(refinement flags of its 3-level run) and the CPU oracle (restriction and
prolongation bit for bit; the Berger-Oliger evolution of all levels within
the oracle's own tolerance to the reference), and the graph replay of the
coarse steps against plain launches."""
import numpy as np
import pytest
import torch

from conftest import load_golden
from test_fmr_oracle_pin import FMR_TOL, fmr_case
from baum_b200 import abi, fmr, synthetic
from oracle import oracle

pytestmark = pytest.mark.gpu


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_geometry_builder_matches_reference():
    g, levels, _, _, _ = fmr_case()
    built = fmr.nested_levels([18, 24, 24], 0.5)
    for a, b in zip(built, levels):
        assert np.array_equal(a.boundary, b.boundary)
        assert (a.boxes[0].m, a.boxes[0].x0, a.desc.dx) == (b.boxes[0].m, b.boxes[0].x0, b.desc.dx)


def test_flags_match_reference(gpu):
    g, levels, u0, params, dt = fmr_case()
    H = fmr.Hierarchy(levels, dt, params)
    for l in range(3):
        fp, fr = H.flags(l)
        assert np.array_equal(fp, g["flagprolong_l%d" % l])
        assert np.array_equal(fr, g["flagrestrict_l%d" % l])


@pytest.mark.parametrize("order", [2, 4, 6])
def test_restrict_prolong_is_bit_exact(gpu, order):
    levels = fmr.nested_levels([26, 32, 32], 0.5)
    params = [abi.z4_params()] * 3
    H = fmr.Hierarchy(levels, [0.1, 0.05, 0.025], params, abi.fmr_params(order_RP=order))
    rng = np.random.default_rng(order)
    for l in (1, 2):
        uc = rng.standard_normal((abi.Z4_NVARS, levels[l - 1].npoints))
        uf = rng.standard_normal((abi.Z4_NVARS, levels[l].npoints))
        dc, df = to_dev(uc), to_dev(uf)
        H.restrict_prolong_varlist(l, dc, df)
        oracle.fmr_restrict_prolong(levels[l - 1], levels[l], uc, uf, order, 3)
        assert np.array_equal(dc.cpu().numpy(), uc)
        assert np.array_equal(df.cpu().numpy(), uf)


def test_three_level_evolution_matches_oracle(gpu):
    g, levels, u0, params, dt = fmr_case()
    H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(use_graph=0))
    u = [to_dev(x) for x in u0]
    H.advance(u, 2)
    assert [H.iteration(l) for l in range(3)] == [2, 4, 8]
    st = oracle.FmrState(levels, u0, 1, params, dt)
    st.advance(2)
    for l in range(3):
        a, b = u[l].cpu().numpy(), st.u[l]
        err = np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-8)
        assert err.max() < FMR_TOL, (l, err.max())


def test_graph_replay_is_identical_to_launches(gpu):
    g, levels, u0, params, dt = fmr_case()
    runs = []
    for use_graph in (0, 1):
        H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(use_graph=use_graph))
        u = [to_dev(x) for x in u0]
        H.advance(u, 1)
        H.advance(u, 3)
        torch.cuda.synchronize()
        runs.append([x.cpu().numpy() for x in u])
        assert [H.iteration(l) for l in range(3)] == [4, 8, 16]
    for a, b in zip(*runs):
        assert np.array_equal(a, b)


def test_bssn_hierarchy_matches_oracle(gpu):
    levels = fmr.nested_levels([22, 28, 24], 0.5)
    params = [abi.bssn_params(dissfactor=(0.1 if l == 0 else 0.02) / 64) for l in range(3)]
    dt = [0.125 / 2 ** l for l in range(3)]
    u0 = []
    for lev in levels:
        x, y, z = lev.coords()
        u0.append(synthetic.fourier_state(x, y, z, abi.NVARS, synthetic.BSSN_UNIT, 8, 0.05, 16.0, 3))
    H = fmr.Hierarchy(levels, dt, params)
    u = [to_dev(x) for x in u0]
    H.advance(u, 2)
    st = oracle.FmrState(levels, u0, 0, params, dt)
    st.advance(2)
    for l in range(3):
        a, b = u[l].cpu().numpy(), st.u[l]
        err = np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-8)
        assert err.max() < FMR_TOL, (l, err.max())


def test_binary_grid_on_the_gpu(gpu):
    """The binary's grid of the reference (level 2 in two boxes around the
    punctures): flags and one restriction/prolongation bit for bit against
    the oracle, the first box's flagprolong against the reference, and two
    coarse steps of all levels within the oracle's tolerance, graph replay
    and plain launches identical."""
    g, levels, u0, params, dt = fmr_case("z4_fmr3_binary")
    assert levels[2].desc.nboxes == 2
    H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(use_graph=0))
    for l in (1, 2):
        fp, _ = H.flags(l)
        assert np.array_equal(fp, g["flagprolong_l%d" % l])
        _, cr = oracle.fmr_flags(levels[l - 1], levels[l], 3)
        assert np.array_equal(H.flags(l - 1)[1], cr)
    rng = np.random.default_rng(7)
    uc = rng.standard_normal((abi.Z4_NVARS, levels[1].npoints))
    uf = rng.standard_normal((abi.Z4_NVARS, levels[2].npoints))
    dc, df = to_dev(uc), to_dev(uf)
    H.restrict_prolong_varlist(2, dc, df)
    oracle.fmr_restrict_prolong(levels[1], levels[2], uc, uf, 4, 3)
    assert np.array_equal(dc.cpu().numpy(), uc)
    assert np.array_equal(df.cpu().numpy(), uf)
    H.close()
    st = oracle.FmrState(levels, u0, 1, params, dt)
    st.advance(2)
    runs = []
    for use_graph in (0, 1):
        H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(use_graph=use_graph))
        u = [to_dev(x) for x in u0]
        H.advance(u, 1)
        H.advance(u, 1)
        torch.cuda.synchronize()
        assert [H.iteration(l) for l in range(3)] == [2, 4, 8]
        runs.append([x.cpu().numpy() for x in u])
        H.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b)
    for l in range(3):
        a, b = runs[0][l], st.u[l]
        err = np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), 1e-8)
        assert err.max() < FMR_TOL, (l, err.max())


def test_checkpoint_resumes_bit_for_bit(gpu):
    """nrgpu_fmr_save / nrgpu_fmr_load: two coarse steps, a checkpoint, two
    more steps; a new hierarchy loaded from the checkpoint with the saved
    level states gives the same states bit for bit (graph replay on both
    sides).  A checkpoint of another hierarchy is refused."""
    g, levels, u0, params, dt = fmr_case()
    H = fmr.Hierarchy(levels, dt, params)
    u = [to_dev(x) for x in u0]
    H.advance(u, 2)
    buf = H.save()
    saved = [x.clone() for x in u]
    H.advance(u, 2)
    torch.cuda.synchronize()
    ref = [x.cpu().numpy() for x in u]
    H.close()
    H2 = fmr.Hierarchy(levels, dt, params)
    H2.load(buf)
    assert [H2.iteration(l) for l in range(3)] == [2, 4, 8]
    H2.advance(saved, 2)
    torch.cuda.synchronize()
    for a, b in zip(saved, ref):
        assert np.array_equal(a.cpu().numpy(), b)
    H2.close()
    H3 = fmr.Hierarchy(levels[:2], dt[:2], params[:2])
    with pytest.raises(RuntimeError):
        H3.load(buf)
    H3.close()


@pytest.mark.parametrize("order,steps", [(4, 4), (6, 6)])
def test_time_interpolation_orders_4_and_6(gpu, order, steps):
    """order_timeinterpolation 4 and 6 (evolve.c:298-340) on the device:
    every level against the oracle at the end (the oracle is pinned to the
    reference's 3-level runs at these orders, whose dumps precede each
    coarse step's last restriction), within the tolerance of the 3rd-order
    runs; graph replay equals plain launches bit for bit (the
    graph is captured once every level runs at the full order); a checkpoint
    taken half way resumes bit for bit (it carries the older time levels)."""
    g, levels, u0, params, dt = fmr_case("z4_fmr3_ti%d" % order)
    runs = []
    for use_graph in (0, 1):
        H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(order_timeinterpolation=order, use_graph=use_graph))
        u = [to_dev(x) for x in u0]
        H.advance(u, steps)
        torch.cuda.synchronize()
        runs.append([x.cpu().numpy() for x in u])
        H.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b)
    got = runs[1]
    st = oracle.FmrState(levels, u0, 1, params, dt, order_ti=order)
    st.advance(steps)
    for l in range(3):
        err = np.abs(got[l] - st.u[l]).max(axis=1) / np.maximum(np.abs(st.u[l]).max(axis=1), 1e-8)
        assert err.max() < FMR_TOL, (l, err.max())
    # checkpoint half way
    fp = abi.fmr_params(order_timeinterpolation=order)
    H = fmr.Hierarchy(levels, dt, params, fp)
    u = [to_dev(x) for x in u0]
    H.advance(u, steps // 2)
    buf = H.save()
    saved = [x.clone() for x in u]
    H.close()
    H2 = fmr.Hierarchy(levels, dt, params, fp)
    H2.load(buf)
    H2.advance(saved, steps - steps // 2)
    torch.cuda.synchronize()
    for a, b in zip(saved, got):
        assert np.array_equal(a.cpu().numpy(), b)
    H2.close()
