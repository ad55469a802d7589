"""The learned-corrector features' CPU oracle on known answers: a fluid
particle deep inside the still dam-break column sees a full kernel support
(Shepard sum near 1, no wall contribution, vanishing gradient and velocity
terms); one next to the floor sees the wall layers."""
import numpy as np

from oracle import pyoracle as po
from zsph_b200 import cases


def test_feature_known_answers_at_rest():
    c = cases.small(0.04)
    o = po.Oracle(c.json, c.state, dtype=np.float64)
    o.search("old", "new")
    o.boundary("new", po.WALLS_FIRST)
    o.governing("new")
    f = o.features(np.ones(32, np.float32), "new")
    st = o.new
    pos, typ = st["pos"], st["type"]
    h = c.json.dx * c.json.h_factor
    fluid = typ == 1
    assert np.all(f[~fluid] == 0)
    # deep interior of the column (x, y in [0, 0.6], z in [0, 1.2] for the small case's water)
    deep = fluid & (pos[:, 0] > 3 * h) & (pos[:, 0] < 0.6 - 3 * h) & (pos[:, 1] > 3 * h) & (pos[:, 1] < 0.6 - 3 * h) \
        & (pos[:, 2] > 3 * h) & (pos[:, 2] < 1.2 - 3 * h)
    assert deep.sum() > 10
    d = f[deep]
    self_term = o.p.m / st["rhop"][deep, 0] * o.p.adh  # (m/rho_i) W(0): the sum runs over j != i
    assert np.all(np.abs(d[:, 0] + self_term - 1.0) < 0.05)  # Shepard sum over fluid
    assert np.all(d[:, 1] == 0)                       # no wall neighbours
    assert np.all(np.abs(d[:, 2:5]) * h < 0.05)       # symmetric support: no kernel-gradient sum
    assert np.all(d[:, 18:21] == 0)                   # at rest
    assert np.all(d[:, 25:28] == 0) and np.all(d[:, 31] == 0)  # no previous corrector value given
    # with one: D = predictor-stage value - previous corrector value of the same particle
    prev = np.random.default_rng(0).normal(size=(c.n, 4))
    f2 = o.features(np.ones(32, np.float32), "new", acc_prev=prev)
    src = o.tmp["index"][deep]
    assert np.allclose(f2[deep][:, 25:28], d[:, 14:17] - prev[src, :3])
    assert np.allclose(f2[deep][:, 31], d[:, 17] - prev[src, 3])
    # next to the floor: wall Shepard sum and an upward wall pressure force
    floor = fluid & (pos[:, 2] < 0.5 * c.json.dx + 1e-6) & (pos[:, 0] > 3 * h) & (pos[:, 0] < 0.6 - 3 * h) \
        & (pos[:, 1] > 3 * h) & (pos[:, 1] < 0.6 - 3 * h)
    assert floor.sum() > 5
    assert np.all(f[floor, 1] > 0.2)
    assert np.all(f[floor, 30] > 0)
