"""Host-side logic on the CPU: the C ABI library loads and exports every
declared symbol, case constants match the reference derivation, JSON case
files parse like the reference's read_json, dt is checked like check_dt."""
import ctypes
import json
import math
import os
import re

import numpy as np
import pytest

import zsph_b200 as z
from zsph_b200 import cases
from oracle import pyoracle as po

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "zsph.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zsph_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(z.lib, s)]
    assert not missing, missing


def test_case_generator_does_not_map_the_library():
    # the reference arm of bench.py builds its case with zsph_b200.cases; that
    # must leave libzsph_b200.so unmapped (a fresh process, so nothing earlier loaded it)
    import subprocess
    import sys
    code = ("import zsph_b200 as z\nfrom zsph_b200 import cases\ncases.config0(); cases.batch_scenes(4, seed=1)\n"
            "maps = open('/proc/self/maps').read()\n"
            "print(int(z.lib.loaded()), int('libzsph_b200' in maps))\n")
    out = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, check=True)
    assert out.stdout.split() == ["0", "0"], out.stdout + out.stderr


def test_no_cpu_fallback_path():
    # the package binds only the CUDA library; no oracle import on the product path
    src = open(os.path.join(ROOT, "zsph_b200", "__init__.py")).read()
    assert "oracle" not in src.replace("no CPU fallback", "")


@pytest.mark.parametrize("case_fn,expect", [
    (cases.config0, dict(n=105048, nf=54000, nw=51048, G=13770, dims=(34, 15, 27))),
    (cases.config1, dict(n=4221468, nf=3456000, nw=765468, G=609600, dims=(127, 50, 96))),
])
def test_case_shapes_and_grid(case_fn, expect):
    c = case_fn()
    assert (c.n, c.n_fluid, c.n_wall) == (expect["n"], expect["nf"], expect["nw"])
    cp, gp = z.params_from_json(c.json)
    assert cp.grid_num == expect["G"]
    assert (cp.grid_xdim, cp.grid_ydim, cp.grid_zdim) == expect["dims"]
    # every particle lies inside the covered grid (x overflow would alias rows)
    for a, lo, d in zip(range(3), (cp.grid_xmin, cp.grid_ymin, cp.grid_zmin), expect["dims"]):
        assert c.state.pos[:, a].min() > lo
        assert c.state.pos[:, a].max() < lo + d * cp.grid_size


def test_params_match_oracle_derivation_bit_exact():
    for c in (cases.config0(), cases.config1(), cases.small(0.04)):
        cp, gp = z.params_from_json(c.json)
        rc, op = po.params(c.json)
        assert rc == 0
        for f in ("half_dt", "h", "g", "m", "rho0", "adh", "h2", "eta2", "cs2", "alpha", "delta_h_cs",
                  "h_cs_rho_m", "grid_size", "grid_xmin", "grid_ymin", "grid_zmin"):
            assert np.float32(getattr(gp, f)).tobytes() == np.float32(getattr(op, f)).tobytes(), f
        for f in ("grid_factor", "grid_xdim", "grid_ydim", "grid_zdim", "grid_hash_min", "grid_hash_max",
                  "ptc_num"):
            assert getattr(gp, f) == getattr(op, f), f
        assert cp.grid_num == op.grid_num


def test_config0_constants():
    # values of the configuration table: h, c0, m, adh, dt, dt_max
    c = cases.config0()
    cp, gp = z.params_from_json(c.json)
    assert cp.h == pytest.approx(0.026, rel=1e-6)
    assert cp.cs == pytest.approx(34.310349, rel=1e-6)
    assert cp.m == pytest.approx(0.008, rel=1e-6)
    assert cp.adh == pytest.approx(23770, rel=1e-4)
    assert cp.dt == pytest.approx(1.5156e-4, rel=1e-3)
    dtmax = ctypes.c_float()
    assert z.lib.zsph_check_dt(ctypes.byref(cp), ctypes.byref(dtmax)) == z.ZSPH_OK
    assert dtmax.value == pytest.approx(1.894e-3, rel=1e-3)


def test_check_dt_rejects_large_dt():
    c = cases.config0()
    c.json.dt = 0.01
    with pytest.raises(z.ZsphError) as e:
        z.params_from_json(c.json)
    assert e.value.code == z.ZSPH_EINVAL


REQUIRED_KEYS = ["g", "rho0", "dx", "h_factor", "r_factor", "eta_factor", "cs_factor", "delta", "alpha", "xmin",
                 "xmax", "ymin", "ymax", "zmin", "zmax", "grid_layer_factor", "grid_size_factor", "dt",
                 "start_step", "current_step", "end_step", "output_step", "ptc_num", "water_ptc_num",
                 "air_ptc_num", "wall_ptc_num", "rigid_ptc_num", "thread_num", "gpu_id", "input_path",
                 "output_path", "git_hash"]


def case_dict(c):
    d = {}
    for k in REQUIRED_KEYS:
        v = getattr(c.json, k)
        d[k] = v.decode() if isinstance(v, bytes) else v
    return d


def test_read_json_roundtrip(tmp_path):
    c = cases.config0()
    d = case_dict(c)
    d["unused_extra_key"] = {"nested": [1, 2, {"a": "b"}]}
    p = tmp_path / "input.json"
    p.write_text(json.dumps(d, indent=2))
    j = z.read_json(str(p))
    for k in REQUIRED_KEYS:
        a, b = getattr(j, k), getattr(c.json, k)
        if isinstance(a, float):
            assert np.float32(a) == np.float32(b), k
        else:
            assert a == b, k
    cp1, gp1 = z.params_from_json(j)
    cp2, gp2 = z.params_from_json(c.json)
    assert bytes(gp1) == bytes(gp2)


def test_read_json_int_keys_accept_float_numbers(tmp_path):
    d = case_dict(cases.config0())
    d["end_step"] = 2000.0
    p = tmp_path / "input.json"
    p.write_text(json.dumps(d))
    assert z.read_json(str(p)).end_step == 2000


@pytest.mark.parametrize("key", ["dt", "ptc_num", "git_hash", "grid_size_factor"])
def test_read_json_missing_key_is_an_error(tmp_path, key):
    d = case_dict(cases.config0())
    del d[key]
    p = tmp_path / "input.json"
    p.write_text(json.dumps(d))
    with pytest.raises(z.ZsphError) as e:
        z.read_json(str(p))
    assert e.value.code == z.ZSPH_EIO and key in str(e.value)


def test_read_json_type_and_syntax_errors(tmp_path):
    d = case_dict(cases.config0())
    d["dx"] = "0.02"
    p = tmp_path / "a.json"
    p.write_text(json.dumps(d))
    with pytest.raises(z.ZsphError):
        z.read_json(str(p))
    p.write_text("{ \"g\": -9.81, ")
    with pytest.raises(z.ZsphError):
        z.read_json(str(p))
    with pytest.raises(z.ZsphError):
        z.read_json(str(tmp_path / "missing.json"))


@pytest.mark.parametrize("value", [1e20, -3e9, float("inf")])
def test_read_json_int_key_out_of_range_is_an_error(tmp_path, value):
    # a number outside the int range cannot become an int key: an error code,
    # not an undefined conversion
    d = case_dict(cases.config0())
    d["ptc_num"] = value
    p = tmp_path / "input.json"
    p.write_text(json.dumps(d))
    with pytest.raises(z.ZsphError) as e:
        z.read_json(str(p))
    assert e.value.code == z.ZSPH_EIO and "ptc_num" in str(e.value)


def test_create_rejects_bad_grid_and_factor():
    c = cases.small(0.04)
    cp, gp = z.params_from_json(c.json)
    h = ctypes.c_void_p()
    assert z.lib.zsph_create(ctypes.byref(gp), cp.grid_num + 1, ctypes.byref(h)) == z.ZSPH_EINVAL
    gp.grid_factor = 3
    assert z.lib.zsph_create(ctypes.byref(gp), cp.grid_num, ctypes.byref(h)) == z.ZSPH_EINVAL
    assert "grid_factor" in z.last_error()


def test_set_launch_shapes_rejects_a_null_handle_or_shapes():
    # argument checks come before any CUDA call, so they run without a GPU
    t = z.TuneResult(list_cells_per_cta=2, governing_min_ctas=1, steps_per_graph=1)
    assert z.lib.zsph_set_launch_shapes(None, ctypes.byref(t)) == z.ZSPH_EINVAL
    assert "null handle" in z.last_error()


def test_case_options_defaults_and_values(tmp_path):
    d = case_dict(cases.config0())
    p = tmp_path / "input.json"
    p.write_text(json.dumps(d))
    o = z.read_case_options(str(p))
    assert (o.equations, o.snapshot_every, o.resume) == (z.EQ_DELTA, 0, b"")
    d.update(equations="simple", eos="linear", snapshot_every=100, resume="/runs/snapshot300.zsnap")
    p.write_text(json.dumps(d))
    o = z.read_case_options(str(p))
    assert (o.equations, o.snapshot_every, o.resume) == (z.EQ_SIMPLE, 100, b"/runs/snapshot300.zsnap")
    # the reference's keys still read as before next to the optional ones
    assert z.read_json(str(p)).ptc_num == d["ptc_num"]


@pytest.mark.parametrize("key,value", [("equations", "sph"), ("equations", 1), ("eos", "tait"),
                                       ("snapshot_every", -1), ("snapshot_every", 2.5), ("resume", 3),
                                       ("resume", "x" * 300)])
def test_case_options_errors(tmp_path, key, value):
    d = case_dict(cases.config0())
    d[key] = value
    p = tmp_path / "input.json"
    p.write_text(json.dumps(d))
    with pytest.raises(z.ZsphError) as e:
        z.read_case_options(str(p))
    assert e.value.code == z.ZSPH_EINVAL and key in str(e.value)
