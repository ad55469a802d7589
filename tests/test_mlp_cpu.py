"""The learned-corrector network's CPU oracle pinned on its own: bf16
rounding known answers, the tile layout, and the backward pass against
finite differences of the float64 loss."""
import numpy as np

from oracle import mlp_oracle as mo


def test_bf16_rounding_known_answers():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, 1.0 + 2**-7, -2.5, 3.0e-3, 65504.0], np.float32)
    # ties go to even: 1 + 2^-8 -> 1, 1 + 3*2^-8 -> 1 + 2^-6
    want = np.array([1.0, 1.0, 1.0 + 2**-6, 1.0 + 2**-7, -2.5, 0.0030059814453125, 65536.0], np.float32)
    assert np.array_equal(mo.bf16(x), want)
    assert mo.bf16_bits(np.array([1.0], np.float32))[0] == 0x3F80


def test_tile_layout_positions():
    n = 300
    X = np.arange(n * 32, dtype=np.float32).reshape(n, 32) % 251
    t = mo.tile_layout(X)
    assert t.shape == (3, 4096)
    for (r, c) in [(0, 0), (1, 0), (0, 1), (7, 7), (8, 0), (0, 8), (127, 31), (45, 17)]:
        off = ((c // 8) * 16 + r // 8) * 64 + (r % 8) * 8 + c % 8
        for tile in range(3):
            row = tile * 128 + r
            want = mo.bf16_bits(X[row:row + 1, c])[0] if row < n else 0
            assert t[tile, off] == want


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.2, mo.NPARAM).astype(np.float32)
    X = rng.normal(size=(40, 32))
    Y = rng.normal(size=(40, 4))
    w = rng.uniform(0.5, 1.5, 40)
    g = mo.grad_fp64(p, X, Y, w, 1.0 / w.sum())
    idx = np.concatenate([rng.choice(np.arange(a, b), min(6, b - a), replace=False)
                          for a, b in [(0, 4096), (4096, 4224), (4224, 20608), (20608, 20736), (20736, 21248),
                                       (21248, 21252)]])
    h = 1e-6
    for k in idx:
        pp = p.astype(np.float64).copy()
        pm = pp.copy()
        pp[k] += h
        pm[k] -= h
        # the fp64 loss reads p through unpack (float32 view): go through a float64 path
        fp = _loss64(pp, X, Y, w)
        fm = _loss64(pm, X, Y, w)
        assert abs((fp - fm) / (2 * h) - g[k]) <= 1e-6 + 1e-5 * abs(g[k]), k


def _loss64(p, X, Y, w):
    o = mo.OFF
    W1 = p[o["W1"]:o["b1"]].reshape(128, 32)
    W2 = p[o["W2"]:o["b2"]].reshape(128, 128)
    W3 = p[o["W3"]:o["b3"]].reshape(4, 128)
    silu = lambda z: z / (1 + np.exp(-z))
    h1 = silu(X @ W1.T + p[o["b1"]:o["W2"]])
    h2 = silu(h1 @ W2.T + p[o["b2"]:o["W3"]])
    y = h2 @ W3.T + p[o["b3"]:mo.NPARAM]
    return float(np.sum(w[:, None] * (y - Y) ** 2) / w.sum())


def test_rounded_backward_close_to_exact():
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.15, mo.NPARAM).astype(np.float32)
    X = mo.bf16(rng.normal(size=(256, 32)).astype(np.float32))
    Y = rng.normal(size=(256, 4)).astype(np.float32)
    w = np.ones(256, np.float32)
    g, loss = mo.grad(p, X, Y, w, 1.0 / 256)
    g64 = mo.grad_fp64(p, X.astype(np.float64), Y, w, 1.0 / 256)
    assert np.linalg.norm(g - g64) / np.linalg.norm(g64) < 2e-2
    assert abs(loss / 256 - mo.loss_fp64(p, X, Y, w, 1.0 / 256)) < 2e-2 * loss / 256


def test_adam_first_step_is_signed_lr():
    p = np.zeros(mo.NPARAM, np.float32)
    part = np.zeros((2, mo.NPARTIAL), np.float32)
    part[0, :mo.NPARAM] = 0.5
    part[1, :mo.NPARAM] = -2.0
    z = np.zeros(mo.NPARAM, np.float32)
    p1, m1, m2 = mo.adam(p, z, z, part, 1, 1e-3, 0.9, 0.999, 1e-8)
    assert np.allclose(p1, 1e-3, rtol=1e-5)  # g = -1.5: first Adam step moves by +lr
    assert np.allclose(m1, -0.15) and np.allclose(m2, 0.001 * 2.25)
