"""The rhs block-shape autotuner (nrgpu_level_autotune, nrgpu_level_block):
every 128- and 256-thread shape gives bit-identical states (one point per thread,
no reduction across threads), the tuner leaves the user's arrays alone,
and a mesh-refinement run with tuned shapes equals the untuned one."""
import numpy as np
import pytest
import torch

from baum_b200 import abi, bssn, fmr, synthetic, z4

pytestmark = pytest.mark.gpu
SHAPES = ((32, 4, 1), (64, 2, 1), (16, 8, 1), (8, 16, 1), (128, 1, 1), (16, 4, 2), (8, 8, 2), (32, 2, 2),
          (8, 4, 4), (4, 8, 4), (16, 2, 4), (4, 4, 8), (64, 4, 1), (32, 8, 1), (16, 8, 2), (32, 4, 2),
          (16, 4, 4), (8, 8, 4), (64, 2, 2), (128, 2, 1))


def fourier(level, nv, unit):
    x, y, z = level.coords()
    return synthetic.fourier_state(x, y, z, nv, unit, 8, 0.05, 16.0, 5)


@pytest.mark.parametrize("system", ["bssn", "z4c"])
def test_every_block_shape_gives_identical_states(gpu, system):
    lev = abi.Level.single_box(37, 0.4)   # 35 inner points per side: ragged in every shape
    if system == "bssn":
        mod, nv, p, u0 = bssn, abi.NVARS, abi.bssn_params(), fourier(lev, abi.NVARS, synthetic.BSSN_UNIT)
    else:
        mod, nv, p, u0 = z4, abi.Z4_NVARS, abi.z4_params(), fourier(lev, abi.Z4_NVARS, synthetic.Z4_UNIT)
    out = []
    for shape in SHAPES:
        dl = mod.DeviceLevel(lev)
        dl.set_block(*shape)
        assert dl.block() == shape
        u = torch.from_numpy(u0.copy()).cuda()
        for _ in range(2):
            mod.evolve_rk_rk4(dl, u, 0.05, p)
        torch.cuda.synchronize()
        out.append(u.cpu().numpy())
        dl.close()
    for o in out[1:]:
        assert np.array_equal(o, out[0])


def test_tuner_picks_a_shape_and_leaves_the_state(gpu):
    lev = abi.Level.single_box(70, 0.2)
    dl = z4.DeviceLevel(lev)
    u0 = fourier(lev, abi.Z4_NVARS, synthetic.Z4_UNIT)
    u = torch.from_numpy(u0.copy()).cuda()
    best = dl.autotune(abi.SYSTEM_Z4C, abi.z4_params())
    assert best in SHAPES
    assert np.array_equal(u.cpu().numpy(), u0)
    assert not dl.nan_flag()
    assert dl.block() == best
    with pytest.raises(RuntimeError):
        dl.set_block(48, 2, 1)
    with pytest.raises(RuntimeError):
        dl.set_block(32, 8, 2)
    with pytest.raises(RuntimeError):
        dl.autotune(7, abi.z4_params())


def test_tuned_hierarchy_equals_untuned(gpu):
    levels = fmr.nested_levels([30, 28, 24], 0.5)
    params = [abi.z4_params(dissfactor=0.02 / 64) for _ in range(3)]
    dt = [0.125 / 2 ** l for l in range(3)]
    u0 = [fourier(lv, abi.Z4_NVARS, synthetic.Z4_UNIT) for lv in levels]
    runs = []
    for tune in (0, 1):
        H = fmr.Hierarchy(levels, dt, params, abi.fmr_params(autotune=tune))
        if not tune:
            assert [H.block(l) for l in range(3)] == [(32, 4, 1)] * 3
        else:
            assert all(H.block(l) in SHAPES for l in range(3))
        u = [torch.from_numpy(x.copy()).cuda() for x in u0]
        H.advance(u, 2)
        torch.cuda.synchronize()
        runs.append([x.cpu().numpy() for x in u])
        H.close()
    for a, b in zip(*runs):
        assert np.array_equal(a, b)
