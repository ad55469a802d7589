"""Generates the golden fixtures under tests/golden/ by running the
reference's OWN hot-path kernels (oracle/_ref/libzsph_ref.so, built from the
reference sources by oracle/build_ref.sh) on a GPU.

    python tests/golden/make_golden.py [output_dir]

Fixtures (numpy .npz, compressed):
  ref_params.npz      derived constants of three cases (reference host code)
  ref_search_*.npz    one neighbour search (hash, sort_by_key, cuda_sort_data)
                      of a case: sorted hash/index, cell bounds, gathered state,
                      and per-particle neighbour counts by the reference's test
  ref_kernels_*.npz   + cuda_boundary_ns + cuda_govering_ns outputs, on the
                      case with wall-consistent initial (rho, p) ("cond")
                      and on the raw case ("raw", where the reference's wall
                      density race decides part of the result)
  ref_steps_*.npz     N full reference steps of the conditioned case, run
                      twice (the race can still make runs differ)
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402
from tests.helpers import condition_walls  # noqa: E402
from zsph_b200 import cases  # noqa: E402

OUT = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))

GOLDEN_CASES = {
    "dam05": lambda: cases.dam_break(0.05, end_step=20),
    "cloud": lambda: cases.random_cloud(3000, 21, kill_frac=0.12),  # 12% killed: crowded cell 0
    "cloud_single_last": lambda: _single_last(),
}


def _single_last():
    c = cases.random_cloud(1500, 22)
    c.state.pos[-1] = [0.2, 0.15, 0.36]
    return c


def _params_record(c):
    gp, G = po.ref_params(c.json)
    rec = {f: getattr(gp, f) for f, _ in gp._fields_}
    rec["grid_num"] = G
    return rec


def main():
    assert po.ref_available(), "build oracle/_ref first (oracle/build_ref.sh)"
    prm = {}
    for name, mk in [("config0", cases.config0), ("config1", cases.config1), ("dam05", GOLDEN_CASES["dam05"])]:
        c = mk()
        for k, v in _params_record(c).items():
            prm[f"{name}.{k}"] = np.array(v)
    np.savez_compressed(os.path.join(OUT, "ref_params.npz"), **prm)

    for name, mk in GOLDEN_CASES.items():
        c = mk()
        out, tmp = po.ref_substep(c.json, c.state, 3)
        np.savez_compressed(os.path.join(OUT, f"ref_search_{name}.npz"),
                            **{f"new.{k}": v for k, v in out.items()},
                            **{k: tmp[k] for k in ("hash", "index", "grid_start", "grid_end", "nb_boundary",
                                                   "nb_governing")})
    raw = GOLDEN_CASES["dam05"]()
    c = condition_walls(raw)
    for tag, cc in (("cond", c), ("raw", raw)):
        out, tmp = po.ref_substep(cc.json, cc.state, 5)
        np.savez_compressed(os.path.join(OUT, f"ref_kernels_dam05_{tag}.npz"), rhop=out["rhop"], type=out["type"],
                            acc_drhodt=tmp["acc_drhodt"], dofv_grandrho=tmp["dofv_grandrho"])
    runs = {}
    for r in range(2):
        out, tmp, _ = po.ref_run(c.json, c.state, 20)
        for k in ("pos", "vel", "rhop", "table", "type"):
            runs[f"run{r}.{k}"] = out[k]
    np.savez_compressed(os.path.join(OUT, "ref_steps_dam05.npz"), nsteps=np.array(20), **runs)
    # simplesph build (equation/simple_ns.cu): one sub-step's kernels and 20 steps of the raw case
    if po.ref_available(simple=True):
        out, tmp = po.ref_substep(raw.json, raw.state, 5, simple=True)
        np.savez_compressed(os.path.join(OUT, "ref_simple_kernels_dam05.npz"), rhop=out["rhop"],
                            acc_drhodt=tmp["acc_drhodt"], dofv=tmp["dofv"])
        out, _, _ = po.ref_run(raw.json, raw.state, 20, simple=True)
        np.savez_compressed(os.path.join(OUT, "ref_simple_steps_dam05.npz"), nsteps=np.array(20),
                            **{k: out[k] for k in ("pos", "vel", "rhop", "table")})
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
