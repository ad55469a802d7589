"""zsph_compat_run's host-side failures, which it reports before any CUDA
call (so these run without a GPU): a null path, an unknown mode, a missing
case JSON and a missing input.vtk each return a ZSPH_* status with the
failing step in zsph_last_error, and no step is run."""
import ctypes
import json
import os

import zsph_b200 as z
from zsph_b200 import cases

_KEYS_F = ("g", "rho0", "dx", "h_factor", "r_factor", "eta_factor", "cs_factor", "delta", "alpha", "xmin", "xmax",
           "ymin", "ymax", "zmin", "zmax", "grid_layer_factor", "grid_size_factor", "dt")
_KEYS_I = ("start_step", "current_step", "end_step", "output_step", "ptc_num", "water_ptc_num", "air_ptc_num",
           "wall_ptc_num", "rigid_ptc_num", "thread_num", "gpu_id")


def _run(path, mode):
    steps = ctypes.c_int(-1)
    rc = z.lib.zsph_compat_run(path.encode() if path is not None else None, mode, ctypes.byref(steps))
    return rc, steps.value


def _case_json_without_input(root):
    """input.json of a small dam break whose input directory holds no input.vtk."""
    c = cases.small(0.04)
    inp, out = os.path.join(root, "input"), os.path.join(root, "output")
    os.makedirs(inp)
    os.makedirs(out)
    j = {k: float(getattr(c.json, k)) for k in _KEYS_F}
    j.update({k: int(getattr(c.json, k)) for k in _KEYS_I})
    j.update(start_step=0, current_step=0, end_step=2, output_step=1, thread_num=1, gpu_id=0, input_path=inp,
             output_path=out, git_hash="test")
    path = os.path.join(root, "input.json")
    with open(path, "w") as f:
        json.dump(j, f)
    return path


def test_null_path_and_unknown_mode_are_rejected(tmp_path):
    assert _run(None, z.COMPAT_SEPARATE) == (z.ZSPH_EINVAL, 0)
    assert "null json path" in z.last_error()
    path = _case_json_without_input(str(tmp_path))
    assert _run(path, 4) == (z.ZSPH_EINVAL, 0)
    assert "unknown mode" in z.last_error()


def test_missing_case_json_is_an_io_error(tmp_path):
    rc, steps = _run(os.path.join(str(tmp_path), "no_such.json"), z.COMPAT_FUSED)
    assert rc == z.ZSPH_EIO and steps == 0
    assert "read_json" in z.last_error()


def test_missing_input_vtk_is_reported_before_any_step(tmp_path):
    path = _case_json_without_input(str(tmp_path))
    for mode in (z.COMPAT_SEPARATE, z.COMPAT_FUSED | z.COMPAT_SIMPLE):
        rc, steps = _run(path, mode)
        assert rc != z.ZSPH_OK and steps == 0
        assert "read_vtk" in z.last_error()


def test_negative_particle_count_is_rejected(tmp_path):
    path = _case_json_without_input(str(tmp_path))
    with open(path) as f:
        j = json.load(f)
    j["ptc_num"] = -1
    with open(path, "w") as f:
        json.dump(j, f)
    assert _run(path, z.COMPAT_FUSED) == (z.ZSPH_EINVAL, 0)
    assert "negative ptc_num" in z.last_error()


def test_an_unwritable_metrics_log_is_reported_before_any_step(tmp_path, monkeypatch):
    path = _case_json_without_input(str(tmp_path))
    monkeypatch.setenv("ZSPH_METRICS", str(tmp_path / "no_such_dir" / "metrics.jsonl"))
    assert _run(path, z.COMPAT_FUSED) == (z.ZSPH_EIO, 0)
    assert "metrics log" in z.last_error()


def test_bad_case_options_are_rejected_before_any_step(tmp_path):
    path = _case_json_without_input(str(tmp_path))
    with open(path) as f:
        j = json.load(f)
    j["eos"] = "tait"
    with open(path, "w") as f:
        json.dump(j, f)
    assert _run(path, z.COMPAT_FUSED) == (z.ZSPH_EINVAL, 0)
    assert "case options" in z.last_error() and "eos" in z.last_error()
