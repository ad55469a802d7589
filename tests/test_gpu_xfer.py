"""List transfer (zsph_set_list_transfer): the corrector's neighbour lists
made from the predictor's must give results bit-identical with the full
list build, step after step, whether the device takes the transfer or falls
back to the full build (displacements above half the skin, particles
leaving the grid, stale cell bounds after a lone last particle)."""
import numpy as np
import pytest

import zsph_b200 as z
from zsph_b200 import cases

pytestmark = pytest.mark.gpu

_FIELDS = ("pos", "vel", "rhop", "type", "table", "tmp_pos", "tmp_vel", "tmp_rhop")


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def _assert_identical(a, b, tag):
    x, y = a.download("old"), b.download("old")
    for k in _FIELDS:
        assert np.array_equal(_bits(getattr(x, k)), _bits(getattr(y, k))), f"{tag}: old.{k}"
    ta, tb = a.download_tmp(), b.download_tmp()
    for k in ta:
        assert np.array_equal(_bits(ta[k]), _bits(tb[k])), f"{tag}: tmp.{k}"


def _pair(c, skin=0.05):
    on = z.Solver.from_case(c)
    on.set_list_transfer(True, skin)
    off = z.Solver.from_case(c)  # the default: full list builds
    return on, off


@pytest.mark.parametrize("dx,steps,chunk", [(0.04, 400, 100), (0.02, 300, 50), (0.01, 100, 50)])
def test_transfer_bit_identical_dam_break(dx, steps, chunk):
    c = cases.dam_break(dx)
    on, off = _pair(c)
    for k in range(steps // chunk):
        on.run(chunk)
        off.run(chunk)
        _assert_identical(on, off, f"dam break dx={dx}, step {(k + 1) * chunk}")
    info = on.list_transfer_info()
    assert info["transferred"] + info["full_builds"] == steps
    assert info["transferred"] >= 0.9 * steps  # the collapsing column stays within the skin
    assert off.list_transfer_info() == {"transferred": 0, "full_builds": 0, "full_searches": 0}
    on.close()
    off.close()


def test_transfer_eager_steps_and_profiled_steps():
    c = cases.dam_break(0.02)
    on, off = _pair(c)
    on.run(100)
    off.run(100)
    for _ in range(5):
        on.step()
        off.step()
    on.step_profiled()
    off.step_profiled()
    on.sync()
    off.sync()
    _assert_identical(on, off, "eager and profiled steps")
    assert on.list_transfer_info()["transferred"] == 106
    names = [k for k, _ in on.step_profiled()]
    assert {"xfer_classify", "xfer_search", "nblist_xfer", "nblist_fallback"} <= set(names)
    on.close()
    off.close()


def test_zero_skin_always_builds_in_full():
    c = cases.dam_break(0.02)
    on, off = _pair(c, skin=0.0)
    on.run(60)
    off.run(60)
    _assert_identical(on, off, "skin 0")
    info = on.list_transfer_info()
    assert info["transferred"] == 0 and info["full_builds"] == 60
    on.close()
    off.close()


def test_particles_leaving_the_grid_fall_back():
    # fluid particles with random velocities in a box whose grid ends near
    # the walls: some leave the grid (killed by the corrector's hash)
    c = cases.random_cloud(6000, 17, kill_frac=0.02)
    c.state.vel[:] *= 40.0
    c.state.tmp_vel[:] = c.state.vel
    on, off = _pair(c)
    for k in range(4):
        on.run(10)
        off.run(10)
        _assert_identical(on, off, f"cloud, step {10 * (k + 1)}")
    info = on.list_transfer_info()
    assert info["full_builds"] > 0 and info["transferred"] + info["full_builds"] == 40
    on.close()
    off.close()


@pytest.mark.parametrize("stale", [None, "n-1", "mixed"])
def test_lone_last_particle_stale_bounds(stale):
    # a particle alone in the highest occupied cell: the cell bounds after it
    # keep earlier values (sort.cu), here zeros, n - 1 everywhere, or a mix;
    # the particles whose rows reach them search in full
    c = cases.random_cloud(3000, 7)
    c.state.pos[-1] = [0.2, 0.15, 0.36]
    c.state.tmp_pos[-1] = c.state.pos[-1]
    c.state.vel[-1] = 0.0
    c.state.tmp_vel[-1] = 0.0
    on, off = _pair(c)
    if stale is not None:
        n, G = on.n, on.G
        rng = np.random.default_rng(3)
        gs = np.full(G, n - 1, np.int32) if stale == "n-1" else rng.integers(-5, n + 5, G).astype(np.int32)
        ge = np.full(G, n - 1, np.int32) if stale == "n-1" else rng.integers(-5, n + 5, G).astype(np.int32)
        for sol in (on, off):
            sol.upload_tmp(grid_start=gs, grid_end=ge)
    on.run(20)
    off.run(20)
    _assert_identical(on, off, f"lone last particle, stale {stale}")
    info = on.list_transfer_info()
    assert info["transferred"] + info["full_builds"] == 20
    on.close()
    off.close()


@pytest.mark.parametrize("skin", [0.02, 0.2])
def test_other_skins_bit_identical(skin):
    c = cases.dam_break(0.02)
    on, off = _pair(c, skin=skin)
    on.run(200)
    off.run(200)
    _assert_identical(on, off, f"skin {skin}")
    assert on.list_transfer_info()["transferred"] > 0
    on.close()
    off.close()


def test_transfer_bit_identical_full_size():
    on, off = _pair(cases.config1())
    on.run(40)
    off.run(40)
    _assert_identical(on, off, "dam break dx=0.005, 40 steps")
    assert on.list_transfer_info()["transferred"] == 40
    on.close()
    off.close()
