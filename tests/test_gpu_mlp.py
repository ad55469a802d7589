"""Tensor-core network kernels (zsph_b200/csrc/mlp.cu) against the CPU
oracle: feature packing bit-exact, forward and backward within the bf16
tolerance, Adam bit-exact, and a training run that fits a target."""
import numpy as np
import pytest

import zsph_b200 as z
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu

FWD_TOL = 1e-2   # relative L2, forward outputs (MUFU SiLU vs exact, bf16 ties)
GRAD_TOL = 3e-2  # relative L2 per parameter block


def _params(seed, scale=0.25):
    rng = np.random.default_rng(seed)
    p = rng.uniform(-1, 1, mo.NPARAM).astype(np.float32)
    p[mo.OFF["W1"]:mo.OFF["b1"]] *= scale * 2
    p[mo.OFF["W2"]:mo.OFF["b2"]] *= scale
    p[mo.OFF["W3"]:mo.OFF["b3"]] *= scale
    p[mo.OFF["b1"]:mo.OFF["W2"]] *= 0.1
    p[mo.OFF["b2"]:mo.OFF["W3"]] *= 0.1
    return p


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 20011])
def test_pack_bit_exact(n):
    rng = np.random.default_rng(n)
    rows = rng.normal(3.0, 2.0, (n, 32)).astype(np.float32)
    mean = rng.normal(3.0, 0.1, 32).astype(np.float32)
    inv = rng.uniform(0.4, 0.6, 32).astype(np.float32)
    tiles = z.Mlp.pack(z.DeviceArray.from_host(rows), n, mean, inv).get()
    want = mo.tile_layout(mo.standardize(rows, mean, inv))
    assert np.array_equal(tiles, want)


@pytest.mark.parametrize("n", [5, 128, 4099, 70000])
def test_forward_matches_oracle(n):
    rng = np.random.default_rng(10 + n)
    net = z.Mlp(seed=1)
    p = _params(2)
    net.params = p
    X = rng.normal(size=(n, 32)).astype(np.float32)
    tiles = z.Mlp.pack(z.DeviceArray.from_host(X), n)
    y = net.forward(tiles, n)
    want = mo.forward(p, mo.standardize(X))
    assert _rel(y, want) < FWD_TOL, _rel(y, want)
    net.close()


@pytest.mark.parametrize("n,ntiles_sel", [(128, None), (3000, None), (40000, 37)])
def test_grad_matches_oracle(n, ntiles_sel):
    rng = np.random.default_rng(20 + n)
    net = z.Mlp(seed=3)
    p = _params(4)
    net.params = p
    X = rng.normal(size=(n, 32)).astype(np.float32)
    nt = (n + 127) // 128
    Y = np.zeros((nt * 128, 4), np.float32)
    Y[:n] = rng.normal(size=(n, 4))
    w = np.zeros(nt * 128, np.float32)
    w[:n] = rng.uniform(0.2, 1.0, n)
    tiles = z.Mlp.pack(z.DeviceArray.from_host(X), n)
    if ntiles_sel is None:
        ids = None
        sel = np.arange(nt)
    else:
        sel = rng.choice(nt, ntiles_sel, replace=False).astype(np.int32)
        ids = z.DeviceArray.from_host(sel)
    rows = (sel[:, None] * 128 + np.arange(128)[None, :]).ravel()
    inv_wsum = 1.0 / float(w[rows].sum())
    partial, nparts = net.grad(tiles, z.DeviceArray.from_host(Y), z.DeviceArray.from_host(w), len(sel), inv_wsum,
                               tile_ids=ids)
    P = partial.get()[:nparts]
    g = P[:, :mo.NPARAM].astype(np.float64).sum(0)
    loss = P[:, mo.NPARAM].sum()
    Xs = np.zeros((nt * 128, 32), np.float32)
    Xs[:n] = mo.standardize(X)
    gw, lw = mo.grad(p, Xs[rows], Y[rows], w[rows], inv_wsum)
    for name, a, b in [("W1", 0, 4096), ("b1", 4096, 4224), ("W2", 4224, 20608), ("b2", 20608, 20736),
                       ("W3", 20736, 21248), ("b3", 21248, 21252)]:
        assert _rel(g[a:b], gw[a:b]) < GRAD_TOL, (name, _rel(g[a:b], gw[a:b]))
    assert abs(loss - lw) < 1e-2 * lw
    assert np.all(P[:, mo.NPARAM + 1:] == 0)
    net.close()


def test_adam_bit_exact():
    rng = np.random.default_rng(7)
    net = z.Mlp(seed=5)
    p = _params(6)
    m1 = rng.normal(0, 1e-3, mo.NPARAM).astype(np.float32)
    m2 = rng.uniform(0, 1e-5, mo.NPARAM).astype(np.float32)
    net.params = p
    net.set_moments(m1, m2, 41)
    part = rng.normal(0, 1e-2, (3, mo.NPARTIAL)).astype(np.float32)
    net.adam(z.DeviceArray.from_host(part), 3, lr=3e-4, beta1=0.9, beta2=0.999, eps=1e-8)
    p1, a1, a2 = mo.adam(p, m1, m2, part, 42, 3e-4, 0.9, 0.999, 1e-8)
    g1, g2, step = net.moments()
    assert step == 42
    assert np.array_equal(net.params, p1)
    assert np.array_equal(g1, a1) and np.array_equal(g2, a2)
    net.close()


def test_training_fits_a_smooth_target():
    """Full-batch Adam on the tensor-core gradients fits a smooth map of a
    few inputs; the loss must fall by an order of magnitude."""
    rng = np.random.default_rng(8)
    n = 128 * 64
    X = rng.normal(size=(n, 32)).astype(np.float32)
    Y = np.stack([np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2], np.tanh(X[:, 3]), 0.5 * X[:, 4] ** 2 - 0.5,
                  X[:, 5] - X[:, 6]], 1).astype(np.float32)
    net = z.Mlp(seed=11)
    tiles = z.Mlp.pack(z.DeviceArray.from_host(X), n)
    yd, wd = z.DeviceArray.from_host(Y), z.DeviceArray.from_host(np.ones(n, np.float32))
    losses = []
    for it in range(400):
        partial, nparts = net.grad(tiles, yd, wd, n // 128, 1.0 / n)
        if it % 50 == 0 or it == 399:
            losses.append(float(partial.get()[:nparts, mo.NPARAM].sum()) / n)
        net.adam(partial, nparts, lr=2e-3)
    print("loss", losses)
    assert losses[-1] < 0.1 * losses[0]
    assert np.all(np.diff(losses[1:]) < 0.05 * losses[0])  # no divergence along the way
    net.close()
