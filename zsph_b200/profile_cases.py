"""Small, fixed GPU workloads of the added forms' kernels, for profiling one
kernel family at a time (python -m zsph_b200.profile_cases CASE).

  mlp_predict  k_mlp inference mode on 3,456,000 rows (the fluid of the
               full-size dam break): pack, then three forward passes
  mlp_train    k_mlp training mode (forward + backward, one partial row per
               CTA) over the same rows, then k_adam, three iterations
  rigid        the floating cube (dx = 0.02 m, 362,408 particles) with
               contact on: two steps (k_rigid_contact, k_rigid_sum,
               k_rigid_step, k_rigid_place) and the FP64 sums (k_conserve)
  transfer     the dam break at dx = 0.0075 m (1,367,542 particles) with the
               list transfer on: three steps (skin-list build, k_xfer_classify,
               k_xfer_search, k_nblist_xfer, k_nblist_fallback)

Inputs are seeded and synthetic; the cases only launch kernels and print a
one-line summary, they check nothing (the parity tests do).
"""
from __future__ import annotations

import sys

import numpy as np

import zsph_b200 as z
from zsph_b200 import cases

ROWS = 3_456_000


def _rows(rng):
    return z.DeviceArray.from_host(rng.normal(size=(ROWS, 32)).astype(np.float32))


def mlp_predict():
    rng = np.random.default_rng(1)
    net = z.Mlp(seed=1)
    tiles = z.Mlp.pack(_rows(rng), ROWS)
    for _ in range(3):
        out = net.forward(tiles, ROWS)
    print(f"mlp_predict: {ROWS} rows, output mean {float(np.mean(out)):.4f}")
    net.close()


def mlp_train():
    rng = np.random.default_rng(2)
    net = z.Mlp(seed=2)
    tiles = z.Mlp.pack(_rows(rng), ROWS)
    y = z.DeviceArray.from_host(rng.normal(size=(ROWS, 4)).astype(np.float32))
    w = z.DeviceArray.from_host(np.ones(ROWS, np.float32))
    for _ in range(3):
        partial, nparts = net.grad(tiles, y, w, ROWS // z.MLP_TILE, 1.0 / ROWS)
        net.adam(partial, nparts, lr=1e-3)
    print(f"mlp_train: {ROWS} rows, {nparts} partial rows")
    net.close()


def rigid():
    dx = 0.02
    c = cases.floating_body(dx, end_step=10)
    s = z.Solver.from_case(c)
    b = c.body
    s.attach_body(b["first"], b["count"], b["mass"])
    s.set_contact(b["mass"] * 9.81 / (100 * 0.05 * dx), 1.0, dx)
    s.run(2)
    e = s.conservation()
    print(f"rigid: {c.n} particles, body z {s.body()['pos'][2]:.4f}, fluid mass {e['mass']:.3f}")
    s.close()


def transfer():
    c = cases.dam_break(0.0075)
    s = z.Solver.from_case(c)
    s.set_list_transfer(True)
    for _ in range(3):
        s.step()
    s.sync()
    print(f"transfer: {c.n} particles, {s.list_transfer_info()}")
    s.close()


CASES = {"mlp_predict": mlp_predict, "mlp_train": mlp_train, "rigid": rigid, "transfer": transfer}

if __name__ == "__main__":
    if len(sys.argv) != 2 or sys.argv[1] not in CASES:
        raise SystemExit(f"usage: python -m zsph_b200.profile_cases {{{','.join(CASES)}}}")
    CASES[sys.argv[1]]()
