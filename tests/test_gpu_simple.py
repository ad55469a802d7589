"""The simple-SPH equations (the reference's simplesph target,
single_gpu_sph_src/equation/simple_ns.cu) on the GPU: kernels against the FP32
oracle, whole steps against the FP64 oracle, and kernels and steps against the
reference's own simplesph CUDA build (which has no wall-density race: walls
read only fluid densities there)."""
import numpy as np
import pytest

import zsph_b200 as z
from oracle import pyoracle as po
from tests.helpers import err_norms
from zsph_b200 import cases

pytestmark = pytest.mark.gpu


def _solver(c):
    s = z.Solver.from_case(c)
    s.set_equations(z.EQ_SIMPLE)
    return s


def _close(gpu, ref, what, rtol=1e-4):
    scale = max(float(np.abs(ref).max()), 1e-30)
    d = float(np.abs(gpu.astype(np.float64) - ref.astype(np.float64)).max())
    assert d <= rtol * scale, f"{what}: max diff {d:.3e}, scale {scale:.3e}"


@pytest.mark.parametrize("mk", [lambda: cases.small(0.04), cases.config0])
def test_simple_kernels_match_oracle(mk):
    c = mk()
    sol = _solver(c)
    sol.neighbor_search("old", "new")
    o = po.Oracle(c.json, c.state, np.float32)
    o.search()
    sol.boundary("new")
    o.boundary_simple("new")
    _close(sol.download_dofv(), o.dofv, "dofv")
    _close(sol.download("new").rhop, o.new["rhop"], "wall rhop")
    sol.governing("new")
    o.governing_simple("new")
    t = sol.download_tmp()
    for a in range(4):
        _close(t["acc_drhodt"][:, a], o.tmp["acc_drhodt"][:, a], f"acc[{a}]")
    sol.close()


def _by_id(arr, table):
    out = np.empty_like(arr)
    out[table + np.arange(len(table), dtype=np.int32)] = arr
    return out


def test_simple_steps_match_fp64_oracle():
    c = cases.small(0.04)
    n = 20
    sol = _solver(c)
    sol.run(n)
    g = sol.download("old")
    assert sol.status() & z.FLAG_NAN == 0
    o32 = po.Oracle(c.json, c.state, np.float32)
    o32.step_simple(n)
    o64 = po.Oracle(c.json, c.state, np.float64)
    o64.step_simple(n)
    for k in ("pos", "vel"):
        gv, v32, v64 = (_by_id(x, t) for x, t in ((getattr(g, k), g.table), (o32.old[k], o32.old["table"]),
                                                   (o64.old[k], o64.old["table"])))
        e_gpu, e_32 = err_norms(gv, v64), err_norms(v32, v64)
        scale = float(np.abs(v64).max())
        assert e_gpu[0] <= 4 * e_32[0] + 1e-6 * scale, (k, e_gpu, e_32)
    sol.close()


@pytest.mark.skipif(not po.ref_available(simple=True), reason="oracle/_ref simplesph build missing")
def test_simple_kernels_and_steps_match_reference_simplesph_build():
    c = cases.small(0.04)
    out, tmp = po.ref_substep(c.json, c.state, 5, simple=True)
    sol = _solver(c)
    sol.neighbor_search("old", "new")
    sol.boundary("new")
    sol.governing("new")
    t = sol.download_tmp()
    _close(sol.download_dofv(), tmp["dofv"], "dofv vs reference")
    for a in range(4):
        _close(t["acc_drhodt"][:, a], tmp["acc_drhodt"][:, a], f"acc[{a}] vs reference")
    sol.close()
    n = 20
    r0, _, _ = po.ref_run(c.json, c.state, n, simple=True)
    sol = _solver(c)
    sol.run(n)
    g = sol.download("old")
    o64 = po.Oracle(c.json, c.state, np.float64)
    o64.step_simple(n)
    for k in ("pos", "vel"):
        a = _by_id(getattr(g, k), g.table)
        b = _by_id(r0[k], r0["table"])
        c64 = _by_id(o64.old[k], o64.old["table"])
        ours, ref = np.abs(a - c64).max(), np.abs(b - c64).max()
        print(f"simple {k}: |ours-fp64| {ours:.3e} |ref-fp64| {ref:.3e} |ours-ref| {np.abs(a - b).max():.3e}")
        assert ours <= 2 * ref + 1e-6
    sol.close()
