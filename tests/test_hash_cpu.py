"""The cell hash's division-free fast path (floor_quot in
zsph_b200/csrc/search_dev.cuh), restated in numpy FP32 and checked against
floor(RN(a / c)) (hash.cu:13-15) over many divisors and quotients, near cell
faces above all.  The GPU search tests check the kernel itself bit-exactly
against the oracle on a cloud placed on cell faces."""
import numpy as np

F = np.float32


def floor_quot(a, c):
    rc = F(1) / F(c)
    q = (a * rc).astype(F)
    f = np.floor(q)
    with np.errstate(invalid="ignore"):  # inf - inf for infinite quotients
        d = np.minimum(q - f, (f + F(1)) - q)
    fast = d > np.maximum(np.abs(q) * F(2.0 ** -20), F(2.0 ** -100))
    exact = np.floor((a / F(c)).astype(F))
    return np.where(fast, f, exact), fast


def test_floor_quot_matches_the_rounded_division():
    rng = np.random.default_rng(5)
    checked = fast_total = 0
    for c in np.concatenate([rng.uniform(1e-3, 1.0, 40), [0.052, 0.0104, 0.012, 0.024, 1.0, 0.1, 3.0]]).astype(F):
        m = rng.integers(-50, 2000, 40000).astype(F)
        face = (m * c).astype(F)
        near = [np.nextafter(face, np.where(rng.uniform(size=face.size) < 0.5, F(np.inf), F(-np.inf)))]
        for _ in range(6):
            near.append(np.nextafter(near[-1], np.where(rng.uniform(size=face.size) < 0.5, F(np.inf), F(-np.inf))))
        wide = (face * (F(1) + rng.uniform(-2e-6, 2e-6, face.size).astype(F))).astype(F)
        rand = rng.uniform(-5 * c, 2000 * c, 200000).astype(F)
        tiny = np.array([0, -0.0, 1e-45, -1e-45, 1e-38, -1e-38, 1e-30, -1e-30], F)
        a = np.concatenate([face, *near, wide, rand, tiny]).astype(F)
        got, fast = floor_quot(a, c)
        want = np.floor((a / c).astype(F))
        assert np.array_equal(got, want), c
        checked += a.size
        fast_total += int(fast.sum())
    assert fast_total > checked // 4  # the fast path carries the random quotients


def test_floor_quot_non_finite_take_the_division():
    a = np.array([np.nan, np.inf, -np.inf], F)
    got, fast = floor_quot(a, F(0.052))
    assert not fast.any()
    assert np.isnan(got[0]) and got[1] == np.inf and got[2] == -np.inf
