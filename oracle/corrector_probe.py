"""Corrector-stage accuracy probe on the CPU oracle (test infrastructure):
what the learned form's corrector must see to reproduce the plain
corrector's accelerations.

At each checkpoint of a plain dam-break run (FP32 oracle) the plain
predictor sub-step is taken, then the plain corrector's accelerations
(single_gpu_sph_src/deltasph/main.cu:79-88) are compared (relative L2 over
fluid particles, x y z) with the governing pass (delta_ns.cu:179-267) run at
the predicted state on inputs of different freshness:

  predictor stage    the predictor-stage accelerations themselves
  lagged all         boundary data (grad rho, div v) and wall (rho, p) of the
                     predictor stage
  fresh walls        wall (rho, p) extrapolated at the predicted state
  + own div v        also the particle's own div v fresh (neighbours' lagged;
                     by linearity of the viscous term in div v_i)
  + all div v        every div v fresh, grad rho still lagged
  all fresh          the plain corrector (zero by construction)

and the half-step change of div v is regressed (least squares, one held-out
checkpoint at a time) on per-particle aggregates a network corrector could
see (pressure and density Laplacians, Shepard sums, div v, p, rho,
predictor-stage drho/dt): whether particle-local information predicts it.

    python -m oracle.corrector_probe [dx] [checkpoints]   e.g. 0.03 200,700,1000
"""
from __future__ import annotations

import sys

import numpy as np

from oracle import pyoracle as po
from zsph_b200 import cases


def rel(a, b):
    d = (a - b).astype(np.float64)
    r = b.astype(np.float64)
    return float(np.sqrt((d * d).sum() / (r * r).sum()))


def local_aggregates(p, st, dofv, acc):
    """Per-particle aggregates of the predictor stage over neighbours within 2h."""
    from scipy.spatial import cKDTree
    n = len(st["type"])
    x = st["pos"].astype(np.float64)
    rho = st["rhop"][:, 0].astype(np.float64)
    pr = st["rhop"][:, 1].astype(np.float64)
    fl = st["type"] == 1
    pairs = cKDTree(x).query_pairs(2 * p.h, output_type="ndarray")
    I = np.concatenate([pairs[:, 0], pairs[:, 1]])
    J = np.concatenate([pairs[:, 1], pairs[:, 0]])
    q = np.sqrt(((x[I] - x[J]) ** 2).sum(1)) / p.h
    f = (1 - q / 2) ** 3
    F = -5 * p.adh * f / p.h ** 2
    W = f * (1 - q / 2) * (2 * q + 1) * p.adh
    m = p.m
    ff = fl[I] & fl[J]

    def S(val, sel=None):
        out = np.zeros(n)
        s = np.ones(len(I), bool) if sel is None else sel
        np.add.at(out, I[s], val[s])
        return out

    return np.stack([S(2 * m / rho[J] * (pr[I] - pr[J]) * F), S(2 * m / rho[J] * (pr[I] - pr[J]) * F, ff),
                     S(2 * m / rho[J] * (rho[I] - rho[J]) * F), S(m / rho[J] * W), S(m / rho[J] * W, ~fl[J]),
                     dofv[:, 3].astype(np.float64), pr, rho - p.rho0, acc[:, 3].astype(np.float64), np.ones(n)], 1)


def main(dx: float, checkpoints: list[int]) -> None:
    c = cases.dam_break(dx)
    o = po.Oracle(c.json, c.state, np.float32)
    step = 0
    regress = []
    print(f"dam break dx = {dx}: {c.n} particles; acceleration relative L2 against the plain corrector")
    for cp in checkpoints:
        o.step(cp - step)
        step = cp
        snap = {k: v.copy() for k, v in o.old.items()}
        o.search("old", "new")
        o.boundary("new")
        o.governing("new")
        acc_n, dofv_n = o.tmp["acc_drhodt"].copy(), o.tmp["dofv_grandrho"].copy()
        pred = {k: v.copy() for k, v in o.new.items()}
        o.prediction("new")
        o.search("new", "old")
        idx = o.tmp["index"].copy()
        walls_lagged = o.old["rhop"].copy()
        o.boundary("old")
        dofv_c, walls_fresh = o.tmp["dofv_grandrho"].copy(), o.old["rhop"].copy()
        o.governing("old")
        acc_c = o.tmp["acc_drhodt"].copy()
        fluid = o.old["type"] == 1
        lag = dofv_n[idx]

        def gov(rhop, dofv):
            o.old["rhop"][:] = rhop
            o.tmp["dofv_grandrho"][:] = dofv
            o.governing("old")
            return o.tmp["acc_drhodt"][:, :3].copy()

        a_lag = gov(walls_lagged, lag)
        a_walls = gov(walls_fresh, lag)
        all_divv = lag.copy()
        all_divv[:, 3] = dofv_c[:, 3]
        a_divv = gov(walls_fresh, all_divv)
        plus1 = lag.copy()
        plus1[:, 3] += 1.0
        s1 = (gov(walls_fresh, plus1) - a_walls) / 2.0  # coefficient of div v_i in the viscous sum
        a_own = a_walls + (dofv_c[:, 3] - lag[:, 3])[:, None] * s1
        a_fresh = gov(walls_fresh, dofv_c)
        want = acc_c[fluid, :3]
        rows = [("predictor stage", acc_n[idx][:, :3]), ("lagged all", a_lag), ("fresh walls", a_walls),
                ("+ own div v", a_own), ("+ all div v", a_divv), ("all fresh", a_fresh)]
        print(f"step {cp}: " + ", ".join(f"{nm} {rel(a[fluid], want):.2e}" for nm, a in rows))
        fresh_divv = np.empty_like(dofv_c[:, 3])
        fresh_divv[idx] = dofv_c[:, 3]
        fl = pred["type"] == 1
        X = local_aggregates(o.p, pred, dofv_n, acc_n)[fl]
        regress.append((X, (fresh_divv - dofv_n[:, 3])[fl].astype(np.float64), fresh_divv[fl].astype(np.float64),
                        dofv_n[fl, 3].astype(np.float64)))
        for k in o.old:
            o.old[k][:] = snap[k]
    print("half-step change of div v against particle-local aggregates (least squares, held-out checkpoint):")
    for k, cp in enumerate(checkpoints):
        train = [r for j, r in enumerate(regress) if j != k] or regress
        X = np.concatenate([r[0] for r in train])
        Y = np.concatenate([r[1] for r in train])
        sc = np.abs(X).max(0) + 1e-30
        w = np.linalg.lstsq(X / sc, Y, rcond=None)[0] / sc
        Xk, _, fresh, lagged = regress[k]
        print(f"step {cp}: div v error lagged {rel(lagged, fresh):.2e}, fitted {rel(lagged + Xk @ w, fresh):.2e}")


if __name__ == "__main__":
    dx = float(sys.argv[1]) if len(sys.argv) > 1 else 0.03
    cps = [int(v) for v in (sys.argv[2] if len(sys.argv) > 2 else "200,700,1000").split(",")]
    main(dx, cps)
