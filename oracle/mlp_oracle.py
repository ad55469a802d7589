"""Learned-corrector network -- CPU ORACLE (test infrastructure only).

The network has no counterpart in the reference solver; this module restates
the arithmetic of the project's tensor-core kernels (zsph_b200/csrc/mlp.cu)
in numpy so that tests can check them:

* feature packing: standardize in float32, round to bf16 (nearest even),
  place rows in the 128-row tile layout of the tensor-core operands;
* forward: z = x W^T + b with bf16 operands and float32 results, SiLU,
  activations rounded to bf16 for the next layer;
* backward of  sum_r w_r |yhat_r - y_r|^2 * inv_wsum  with the kernel's
  rounding points (output gradient and hidden gradients rounded to bf16 as
  tensor-core operands, the b3 gradient summed unrounded);
* Adam in float32 with every operation rounded separately.

`grad_fp64` is the same backward without any rounding, used to pin the
formulas against finite differences.
"""
from __future__ import annotations

import numpy as np

NIN, NHID, NOUT, NOUT_PAD = 32, 128, 4, 16
OFF = dict(W1=0, b1=4096, W2=4224, b2=20608, W3=20736, b3=21248)
NPARAM = 21252
NPARTIAL = 21256
TILE = 128


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bf16 (nearest, ties to even), kept as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32)


def bf16_bits(x: np.ndarray) -> np.ndarray:
    return (bf16(x).view(np.uint32) >> 16).astype(np.uint16)


def unpack(p: np.ndarray) -> dict:
    p = np.asarray(p, np.float32)
    return dict(W1=p[OFF["W1"]:OFF["b1"]].reshape(NHID, NIN), b1=p[OFF["b1"]:OFF["W2"]],
                W2=p[OFF["W2"]:OFF["b2"]].reshape(NHID, NHID), b2=p[OFF["b2"]:OFF["W3"]],
                W3=p[OFF["W3"]:OFF["b3"]].reshape(NOUT, NHID), b3=p[OFF["b3"]:NPARAM])


def pack_vector(d: dict) -> np.ndarray:
    return np.concatenate([d["W1"].ravel(), d["b1"], d["W2"].ravel(), d["b2"], d["W3"].ravel(), d["b3"]]).astype(
        np.float32)


def standardize(rows: np.ndarray, mean=None, inv_std=None) -> np.ndarray:
    """bf16((x - mean) * inv_std), float32 arithmetic (the packing kernel)."""
    x = np.asarray(rows, np.float32)
    mean = np.zeros(NIN, np.float32) if mean is None else np.asarray(mean, np.float32)
    inv_std = np.ones(NIN, np.float32) if inv_std is None else np.asarray(inv_std, np.float32)
    return bf16((x - mean) * inv_std)


def tile_layout(X: np.ndarray) -> np.ndarray:
    """bf16 rows [n][32] -> uint16 tiles [ntiles][4096] in the operand layout:
    element (r, c) of a tile at ((c//8)*16 + r//8)*64 + (r%8)*8 + c%8 (in
    bf16 units)."""
    n = X.shape[0]
    nt = (n + TILE - 1) // TILE
    bits = np.zeros((nt * TILE, NIN), np.uint16)
    bits[:n] = bf16_bits(X)
    out = np.zeros((nt, 4096), np.uint16)
    r = np.arange(TILE)[:, None]
    c = np.arange(NIN)[None, :]
    off = ((c // 8) * 16 + r // 8) * 64 + (r % 8) * 8 + c % 8
    for t in range(nt):
        out[t, off.ravel()] = bits[t * TILE:(t + 1) * TILE].ravel()
    return out


def _silu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return z * s, s * (1.0 + z * (1.0 - s))


def _mm(a, b):
    """float32 result of a product of float32 (bf16-valued) operands."""
    return (a.astype(np.float64) @ b.astype(np.float64)).astype(np.float32)


def forward(p: np.ndarray, X: np.ndarray, keep: bool = False):
    d = unpack(p)
    W1, W2, W3 = bf16(d["W1"]), bf16(d["W2"]), bf16(d["W3"])
    z1 = _mm(X, W1.T) + d["b1"]
    h1, s1 = _silu(z1)
    H1, S1 = bf16(h1), bf16(s1)
    z2 = _mm(H1, W2.T) + d["b2"]
    h2, s2 = _silu(z2)
    H2, S2 = bf16(h2), bf16(s2)
    y = _mm(H2, W3.T) + d["b3"]
    if keep:
        return y, dict(H1=H1, S1=S1, H2=H2, S2=S2, W1=W1, W2=W2, W3=W3)
    return y


def grad(p: np.ndarray, X: np.ndarray, Y: np.ndarray, w: np.ndarray, inv_wsum: float):
    """Gradient vector (NPARAM) and the weighted loss sum (without inv_wsum)."""
    y, c = forward(p, X, keep=True)
    dlt = (y - Y).astype(np.float32)
    loss = float(np.sum(w[:, None].astype(np.float64) * dlt.astype(np.float64) ** 2))
    g3 = (2.0 * w[:, None] * dlt * np.float32(inv_wsum)).astype(np.float32)
    G3 = bf16(g3)
    dW3 = _mm(G3.T, c["H2"])
    db3 = g3.astype(np.float64).sum(0).astype(np.float32)
    G2 = bf16(_mm(G3, c["W3"]) * c["S2"])
    dW2 = _mm(G2.T, c["H1"])
    db2 = G2.astype(np.float64).sum(0).astype(np.float32)
    G1 = bf16(_mm(G2, c["W2"]) * c["S1"])
    dW1 = _mm(G1.T, X)
    db1 = G1.astype(np.float64).sum(0).astype(np.float32)
    return pack_vector(dict(W1=dW1, b1=db1, W2=dW2, b2=db2, W3=dW3, b3=db3)), loss


def loss_fp64(p: np.ndarray, X: np.ndarray, Y: np.ndarray, w: np.ndarray, inv_wsum: float) -> float:
    d = {k: v.astype(np.float64) for k, v in unpack(p).items()}
    h1 = _silu(X @ d["W1"].T + d["b1"])[0]
    h2 = _silu(h1 @ d["W2"].T + d["b2"])[0]
    y = h2 @ d["W3"].T + d["b3"]
    return float(np.sum(w[:, None] * (y - Y) ** 2) * inv_wsum)


def grad_fp64(p: np.ndarray, X: np.ndarray, Y: np.ndarray, w: np.ndarray, inv_wsum: float) -> np.ndarray:
    """The same backward pass in float64 with no rounding."""
    d = {k: v.astype(np.float64) for k, v in unpack(p).items()}
    X = X.astype(np.float64)
    z1 = X @ d["W1"].T + d["b1"]
    h1, s1 = _silu(z1)
    z2 = h1 @ d["W2"].T + d["b2"]
    h2, s2 = _silu(z2)
    y = h2 @ d["W3"].T + d["b3"]
    g3 = 2.0 * w[:, None] * (y - Y) * inv_wsum
    g2 = (g3 @ d["W3"]) * s2
    g1 = (g2 @ d["W2"]) * s1
    return np.concatenate([(g1.T @ X).ravel(), g1.sum(0), (g2.T @ h1).ravel(), g2.sum(0), (g3.T @ h2).ravel(),
                           g3.sum(0)])


def adam(p, m1, m2, partial, step, lr, b1, b2, eps):
    """One Adam step exactly as the kernel computes it.  `partial` has one
    row of NPARTIAL floats per CTA; rows are summed in order.  `step` is the
    step number after the increment (1 for the first step)."""
    f = np.float32
    g = np.zeros(NPARAM, f)
    for row in np.asarray(partial, f).reshape(-1, NPARTIAL):
        g = (g + row[:NPARAM]).astype(f)
    b1, b2, lr, eps = f(b1), f(b2), f(lr), f(eps)
    bc1 = f(1.0 - float(np.float64(b1)) ** step)
    bc2 = f(1.0 - float(np.float64(b2)) ** step)
    m = (b1 * m1).astype(f) + ((f(1) - b1) * g).astype(f)
    v = (b2 * m2).astype(f) + ((f(1) - b2) * (g * g).astype(f)).astype(f)
    m, v = m.astype(f), v.astype(f)
    upd = ((lr * (m / bc1).astype(f)).astype(f) / (np.sqrt((v / bc2).astype(f)).astype(f) + eps).astype(f)).astype(f)
    return (np.asarray(p, f) - upd).astype(f), m, v
