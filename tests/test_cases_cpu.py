"""The synthetic workloads on the CPU: the floating-body case and the
batched form's seeded scene draw have the sizes and obey the rules the
documentation states (no randomness except the seeded draw)."""
import numpy as np

import zsph_b200 as z
from zsph_b200 import cases


def test_floating_body_case_counts():
    c = cases.config2()
    assert (c.n, c.n_fluid, c.n_wall) == (2440708, 2000000, 432708)
    assert int(np.sum(c.state.type == 2)) == 8000
    b = c.body
    assert b["count"] == 8000 and b["first"] == c.n_fluid + c.n_wall
    assert abs(b["mass"] - 500.0 * 0.2 ** 3) < 1e-9  # 0.2 m cube of density 500 kg/m^3


def test_batch_scene_draw_is_seeded_and_obeys_its_rules():
    cs, draws = cases.batch_scenes(256, seed=2026)
    assert len(cs) == len(draws) == 256
    assert sum(c.n_fluid for c in cs) == 4912694 and sum(c.n for c in cs) == 11533280
    for c, d in zip(cs, draws):
        assert 0.2 <= d["w"] <= 0.6 and 0.5 <= d["aspect"] <= 2.0 and 0.01 <= d["dx"] <= 0.02
        assert 0.2 <= d["aspect"] * d["w"] <= 0.6  # column height
        assert 5000 <= c.n_fluid <= 60000
        cp, _ = z.params_from_json(c.json)
        assert abs(cp.xmax - 2.5 * d["w"]) < 1e-6 and abs(cp.ymax - d["w"]) < 1e-6  # tank 2.5 w x w
    again, _ = cases.batch_scenes(256, seed=2026)
    assert all(np.array_equal(a.state.pos, b.state.pos) for a, b in zip(cs[:8], again[:8]))
    other, _ = cases.batch_scenes(8, seed=7)
    assert [c.n for c in other] != [c.n for c in cs[:8]]
