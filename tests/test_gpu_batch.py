"""Batched form (zsph_create_batch) and the autotuner (zsph_autotune).

Every kernel launch of a batch covers all scenes; per scene the arithmetic,
the sorted order and the neighbour visit order are those of the scene run
alone, so the results are bit-identical.  The autotuner only changes launch
shapes (CTA sizes, register budgets, steps per graph), so a tuned run is
bit-identical too, and tuning leaves the state where it found it."""
import numpy as np
import pytest

import zsph_b200 as z
from zsph_b200 import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scenes():
    cs, draws = cases.batch_scenes(5, seed=11, fluid_range=(5000, 20000))
    return cs


def _rows(st, a, b):
    return {k: getattr(st, k)[a:b] for k in ("pos", "vel", "rhop", "type", "table")}


def test_batch_matches_each_scene_alone(scenes):
    nsteps = 12
    b = z.Solver.from_batch(scenes)
    b.run(nsteps)
    got = b.download("old")
    assert b.status() == 0
    off = 0
    for c in scenes:
        s = z.Solver.from_case(c)
        s.run(nsteps)
        want = s.download("old")
        g = _rows(got, off, off + c.n)
        for k, v in _rows(want, 0, c.n).items():
            assert np.array_equal(g[k], v), (c.name, k)
        off += c.n
        s.close()
    b.close()


def test_autotune_keeps_state_and_results(scenes):
    c = scenes[0]
    a, b = z.Solver.from_case(c), z.Solver.from_case(c)
    a.run(3)
    b.run(3)
    before = a.download("old")
    r = a.autotune(2)
    print("tune", r)
    assert r["candidates"] == 36 and r["ms_per_step"] > 0 and r["ms_per_step"] <= r["ms_default"] * 1.0001
    after = a.download("old")
    for k in ("pos", "vel", "rhop", "type", "table"):
        assert np.array_equal(getattr(before, k), getattr(after, k)), k
    a.run(9)  # tuned shapes, possibly several steps per graph replay
    b.run(9)
    x, y = a.download("old"), b.download("old")
    for k in ("pos", "vel", "rhop", "type", "table"):
        assert np.array_equal(getattr(x, k), getattr(y, k)), k
    a.close()
    b.close()


def test_autotune_batch(scenes):
    bt = z.Solver.from_batch(scenes)
    r = bt.autotune(2)
    print("batch tune", r)
    assert r["candidates"] == 36
    bt.run(5)
    assert bt.status() == 0
    bt.close()


def test_set_launch_shapes_applies_every_candidate_bit_identically(scenes):
    c = scenes[1]
    ref = z.Solver.from_case(c)
    ref.run(6)
    want = ref.download("old")
    ref.close()
    for cw, mb, spg, sg in ((2, 1, 4, 2), (4, 8, 1, 3), (2, 6, 4, 4), (0, 0, 0, 0), (4, 1, 1, 2)):
        s = z.Solver.from_case(c)
        s.set_launch_shapes(cw, mb, spg, sg)
        s.run(6)
        got = s.download("old")
        assert s.status() == 0
        for k in ("pos", "vel", "rhop", "type", "table"):
            assert np.array_equal(getattr(got, k), getattr(want, k)), (cw, mb, spg, sg, k)
        for bad in ((3, 0, 0, 0), (0, 5, 0, 0), (0, 0, 2, 0), (-1, 0, 0, 0), (0, 0, 0, 1), (0, 0, 0, 5)):
            with pytest.raises(z.ZsphError):
                s.set_launch_shapes(*bad)
        s.close()


# ---- persistent mode: the whole step in one cooperative launch --------------

def test_persistent_step_matches_the_separate_launches(scenes):
    """The persistent kernel runs the same stage code behind grid barriers:
    zsph_step and zsph_run give the separate launches' results bit for bit
    (hence each scene's result run alone), the tmp arrays included."""
    nsteps = 7
    ref = z.Solver.from_batch(scenes)
    ref.run(nsteps)
    want, want_t = ref.download("old"), ref.download_tmp()
    ref.close()
    for via_run in (True, False):
        b = z.Solver.from_batch(scenes)
        b.set_persistent(True)
        info = b.persistent_info()
        assert info["ctas"] >= 148
        if via_run:
            b.run(nsteps)
        else:
            for _ in range(nsteps):
                b.step()
        got, got_t = b.download("old"), b.download_tmp()
        assert b.status() == 0
        print("persistent", info, b.persistent_info())
        for k in ("pos", "vel", "rhop", "tmp_pos", "tmp_vel", "tmp_rhop", "type", "table"):
            assert np.array_equal(getattr(got, k), getattr(want, k)), (via_run, k)
        for k in ("hash", "index", "grid_start", "grid_end", "acc_drhodt", "dofv_grandrho"):
            assert np.array_equal(got_t[k], want_t[k]), (via_run, k)
        b.close()


def test_persistent_barrier_wait_is_bounded(scenes):
    """A barrier whose last arrival never comes: every CTA gives up after its
    bounded wait, the handle reports ZSPH_ETIMEOUT, and the context stays
    usable (a persistent run afterwards still succeeds)."""
    b = z.Solver.from_batch(scenes)
    b.set_persistent(True)
    rc = z.lib.zsph_persistent_barrier_test(b.h, 2000, None)
    assert rc == z.ZSPH_ETIMEOUT, z.last_error(b.h)
    assert b.status() == 0  # the self-test cleared the flag
    b.run(2)
    assert b.status() == 0
    assert np.all(np.isfinite(b.download("old").pos))
    with pytest.raises(z.ZsphError):
        z.Solver.from_case(scenes[0]).set_persistent(True)  # single-scene handles have no persistent mode
    b.close()
