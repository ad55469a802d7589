"""Learned-corrector form: the predictor-stage features against the CPU
oracle, training on snapshots of plain steps (the network must beat the
predictor-only corrector on held-out snapshots), the learned run with its
judge, and the fallback to the plain corrector when the network is wrong."""
import numpy as np
import pytest

import zsph_b200 as z
from oracle import pyoracle as po
from zsph_b200 import cases

pytestmark = pytest.mark.gpu

FEAT_TOL = 2e-3  # |gpu - oracle| per feature, relative to the feature's RMS over fluid rows


def _moving_state(dx=0.04, steps=60):
    c = cases.small(dx)
    sol = z.Solver.from_case(c)
    sol.run(steps)
    sol.sync()
    return c, sol


def test_features_match_oracle():
    c, sol = _moving_state()
    st = sol.download("old")
    prev = sol.download_tmp()["acc_drhodt"]  # the last corrector-stage values, old_'s order
    scale = sol.feature_scales()
    feats = sol.learn_features()  # predictor sub-step: features of new_'s order
    o = po.Oracle(c.json, st)
    o.search("old", "new")
    o.boundary("new", po.WALLS_FIRST)
    o.governing("new")
    want = o.features(scale, "new", acc_prev=prev)
    fluid = o.new["type"] == 1
    assert np.array_equal(sol.download("new").type, o.new["type"])
    assert np.all(feats[~fluid] == 0)
    for k in range(32):
        rms = np.sqrt(np.mean(want[fluid, k].astype(np.float64) ** 2)) + 1e-30
        err = np.max(np.abs(feats[fluid, k] - want[fluid, k])) / rms
        assert err < FEAT_TOL, (k, err)
    sol.close()


@pytest.fixture(scope="module")
def trained():
    c, sol = _moving_state(0.04, 40)
    count = sol.collect(160, 2, 80)
    assert count == 80
    net = z.Mlp(seed=7)
    stats = sol.train(net, epochs=30, batch_tiles=32, lr=2e-3, seed=1, val_frac=0.2)
    print("train", stats)
    yield c, sol, net, stats
    net.close()
    sol.close()


def test_training_beats_predictor_only(trained):
    """What the learned corrector gains: on held-out snapshots its
    corrector-stage values are closer to the plain corrector's than the
    predictor-stage values alone; the stats also report the extrapolation
    prior alone, the network's share of the gain."""
    _, _, _, s = trained
    assert s["snapshots_train"] == 64 and s["snapshots_val"] == 16
    assert s["loss_last"] < s["loss_first"]
    assert s["val_acc_rel_l2"] < s["val_acc_rel_l2_base"]
    assert s["val_drho_rel_l2"] < s["val_drho_rel_l2_base"]
    assert s["val_acc_rel_l2_extrap"] < s["val_acc_rel_l2_base"]


def test_learned_run_is_judged(trained):
    _, sol, net, _ = trained
    r = sol.run_learned(net, 40, judge_every=10, tol=1e-2)
    print("run", r)
    assert r["steps"] == 40 and r["judged"] == 4
    assert r["learned"] + r["plain"] == 36
    assert np.isfinite(r["err_max"]) and r["err_max"] > 0
    st = sol.download("old")
    assert np.all(np.isfinite(st.pos)) and np.all(np.isfinite(st.vel))
    assert sol.status() == 0


def test_untrained_network_falls_back():
    c, sol = _moving_state(0.04, 20)
    net = z.Mlp(seed=3)
    norm = net.norm
    norm["out_std"] = np.full(4, 50.0, np.float32)  # untrained and loud: far off the plain corrector
    net.norm = norm
    r = sol.run_learned(net, 30, judge_every=5, tol=1e-2)
    print("run", r)
    assert r["judged"] == 6 and r["fallbacks"] >= 1 and r["plain"] > 0
    assert r["err_max"] > 1e-2
    st = sol.download("old")
    assert np.all(np.isfinite(st.pos))
    net.close()
    sol.close()


def _by_id(st):
    ids = st.table + np.arange(len(st.table), dtype=np.int32)
    order = np.empty_like(ids)
    order[ids] = np.arange(len(ids), dtype=np.int32)
    return order


def test_list_reuse_fresh_corrector_matches_the_plain_corrector():
    """The corrector on the predictor's neighbour lists with a fresh boundary
    pass evaluates the plain corrector's equations at the predicted state;
    it differs only where a pair crossed the 2h radius during the half step
    (the lists miss pairs that entered, whose kernel weight is near zero) and
    in summation order.  Judged on every step, its accelerations agree with
    the plain corrector's to well below the 1e-2 tolerance (here exactly: no
    pair crossed the radius and no particle changed cell in a half step, so
    the plain corrector's search reproduced the same order)."""
    c, sol = _moving_state(0.04, 60)
    r = sol.run_learned(None, 20, judge_every=1, tol=1e-2, corrector=z.CORR_REUSE_FRESH, series=20)
    print("fresh", r)
    assert r["judged"] == 20 and r["fallbacks"] == 0 and len(r["err_series"]) == 20
    assert r["err_max"] < 1e-3
    assert sol.status() == 0
    sol.close()


def test_list_reuse_correctors_track_the_plain_run():
    """Unjudged runs of both list-reuse correctors stay close to the plain
    run by particle id (the lagged form further away than the fresh one), and
    the lagged form's judged error is reported honestly (nonzero)."""
    c, base = _moving_state(0.04, 60)
    start = base.download("old")
    base.run(30)
    ref = base.download("old")
    base.close()
    errs = {}
    for corr in (z.CORR_REUSE_FRESH, z.CORR_REUSE_LAGGED):
        sol = z.Solver.from_case(c)
        sol.upload(start)
        r = sol.run_learned(None, 30, judge_every=0, tol=1e-2, corrector=corr)
        assert r["learned"] == 30 and r["judged"] == 0
        st = sol.download("old")
        assert sol.status() == 0
        a, b = _by_id(st), _by_id(ref)
        fl = ref.type[b] == 1
        errs[corr] = float(np.abs(st.pos[a][fl] - ref.pos[b][fl]).max())
        sol.close()
    print("max |x - x_plain| after 30 steps:", errs)
    assert errs[z.CORR_REUSE_FRESH] < 1e-5
    assert errs[z.CORR_REUSE_FRESH] <= errs[z.CORR_REUSE_LAGGED] < 1e-3
    sol = z.Solver.from_case(c)
    sol.upload(start)
    r = sol.run_learned(None, 10, judge_every=2, tol=1.0, corrector=z.CORR_REUSE_LAGGED, series=5)
    print("lagged", r)
    assert r["judged"] == 5 and 0 < r["err_max"] < 1.0
    sol.close()
