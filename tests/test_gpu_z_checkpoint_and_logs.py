"""Checkpoint and resume, the driver program's run log, and trace ranges,
on the GPU:
- a run resumed from a snapshot of old_ and tmp (zsph_snapshot_save /
  zsph_snapshot_load) continues bit for bit as the saved run does, and the
  file holds exactly the device arrays;
- zsph_compat_run's optional case-file keys: periodic snapshots and a resumed
  run that writes the same output file as the run that never stopped, and the
  JSONL run log (ZSPH_METRICS);
- a step pushes its NVTX range and those of its kernel groups (probe tool
  tests/nvtx_probe.c through NVTX_INJECTION64_PATH).
These tests are collected after the other GPU tests (and before the
allocation-free sort's own file, which comes last)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

import zsph_b200 as z
from zsph_b200 import cases
from tests.test_gpu_compat import _write_case
from tests.test_nvtx_cpu import ROOT, probe  # noqa: F401  (the probe fixture)

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


def _assert_same(sa, ta, sb, tb):
    for k in ("pos", "vel", "rhop", "type", "table"):
        assert np.array_equal(_bits(getattr(sa, k)), _bits(getattr(sb, k))), k
    for k in ("hash", "index", "grid_start", "grid_end", "acc_drhodt"):
        assert np.array_equal(_bits(ta[k]), _bits(tb[k])), k


@pytest.mark.parametrize("mk,equations", [(lambda: cases.small(0.04), z.EQ_DELTA), (cases.config0, z.EQ_DELTA),
                                          (lambda: cases.small(0.04), z.EQ_SIMPLE)])
def test_resume_from_a_snapshot_is_bit_exact(tmp_path, mk, equations):
    c = mk()
    path = str(tmp_path / "run.zsnap")
    a = z.Solver.from_case(c)
    a.set_equations(equations)
    a.run(5)
    a.save_snapshot(path, step=5)
    a.run(5)
    want, want_tmp = a.download("old"), a.download_tmp()
    a.close()
    b = z.Solver.from_case(c)  # the case's initial state, replaced by the load
    b.set_equations(equations)
    assert b.load_snapshot(path) == 5
    b.run(5)
    got, got_tmp = b.download("old"), b.download_tmp()
    b.close()
    _assert_same(want, want_tmp, got, got_tmp)


def test_device_snapshot_holds_the_device_arrays(tmp_path):
    c = cases.small(0.04)
    s = z.Solver.from_case(c)
    s.run(3)
    path = str(tmp_path / "s.zsnap")
    s.save_snapshot(path, step=3)
    st, tmp = s.download("old"), s.download_tmp()
    arrays, step = z.snapshot_load_host(path, s.n, s.G, names=["pos", "vel", "rhop", "type", "table", "hash",
                                                                 "index", "grid_start", "grid_end", "acc_drhodt"])
    assert step == 3
    for k in ("pos", "vel", "rhop", "type", "table"):
        assert np.array_equal(_bits(arrays[k]), _bits(getattr(st, k))), k
    for k in ("hash", "index", "grid_start", "grid_end", "acc_drhodt"):
        assert np.array_equal(_bits(arrays[k]), _bits(tmp[k])), k
    # a snapshot of another size is refused without touching the buffers
    other = z.Solver.from_case(cases.small(0.05))
    before = other.download("old")
    with pytest.raises(z.ZsphError) as e:
        other.load_snapshot(path)
    assert e.value.code == z.ZSPH_EINVAL
    after = other.download("old")
    assert np.array_equal(_bits(before.pos), _bits(after.pos))
    other.close()
    s.close()


def test_compat_run_metrics_log(tmp_path, monkeypatch):
    # ZSPH_METRICS: one JSON line per output step with the steps since the
    # previous line, their wall time and the FP64 conservation sums
    c = cases.small(0.04)
    path, out = _write_case(str(tmp_path), c, 12, 5)
    log = tmp_path / "metrics.jsonl"
    monkeypatch.setenv("ZSPH_METRICS", str(log))
    assert z.compat_run(path, z.COMPAT_FUSED) == 12
    lines = [json.loads(l) for l in log.read_text().splitlines()]
    assert [l["step"] for l in lines] == [0, 5, 10]
    assert [l["steps"] for l in lines] == [1, 5, 5]
    assert all(l["seconds"] > 0 and l["particle_steps_per_s"] > 0 and (l["flags"] & z.FLAG_NAN) == 0 for l in lines)
    mass = c.n_fluid * float(c.json.rho0) * float(c.json.dx) ** 3
    assert all(abs(l["mass"] - mass) < 1e-6 * mass for l in lines)  # no fluid particle leaves the tank
    assert sorted(os.listdir(out)) == sorted(f"zsph{i}.vtk" for i in (0, 5, 10))


@pytest.mark.parametrize("mode", [z.COMPAT_SEPARATE, z.COMPAT_FUSED])
def test_compat_run_resumes_from_its_snapshot(tmp_path, mode):
    # "snapshot_every": 6 writes output/snapshot6.zsnap (the state before step
    # 6); a second run with "resume" pointing at it runs steps 6..11 and writes
    # the same zsph10.vtk, byte for byte, as the run that never stopped
    c = cases.small(0.04)
    full = tmp_path / "full"
    full.mkdir()
    path, out = _write_case(str(full), c, 12, 5)
    with open(path) as f:
        j = json.load(f)
    j["snapshot_every"] = 6
    with open(path, "w") as f:
        json.dump(j, f)
    assert z.compat_run(path, mode) == 12
    assert sorted(n for n in os.listdir(out) if n.endswith(".zsnap")) == ["snapshot12.zsnap", "snapshot6.zsnap"]
    part = tmp_path / "resumed"
    part.mkdir()
    path2, out2 = _write_case(str(part), c, 12, 5)
    with open(path2) as f:
        j2 = json.load(f)
    j2["resume"] = os.path.join(out, "snapshot6.zsnap")
    with open(path2, "w") as f:
        json.dump(j2, f)
    assert z.compat_run(path2, mode) == 6
    assert sorted(os.listdir(out2)) == ["zsph10.vtk"]
    a = open(os.path.join(out, "zsph10.vtk"), "rb").read()
    b = open(os.path.join(out2, "zsph10.vtk"), "rb").read()
    assert a == b


CHILD = r"""
import zsph_b200 as z
from zsph_b200 import cases
s = z.Solver.from_case(cases.small(0.04))
s.step()
s.sync()
s.close()
print("child ok")
"""


def test_step_pushes_entry_and_group_ranges(probe, tmp_path):  # noqa: F811
    log = tmp_path / "nvtx.log"
    env = dict(os.environ, NVTX_INJECTION64_PATH=probe, ZSPH_NVTX_LOG=str(log),
               PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=tmp_path, env=env, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0 and "child ok" in r.stdout, r.stdout + r.stderr
    lines = log.read_text().split("\n")
    pushes = [l[5:] for l in lines if l.startswith("push ")]
    i = pushes.index("zsph_step")
    assert pushes[i + 1:i + 7] == ["search", "boundary", "governing"] * 2
    assert sum(1 if l.startswith("push ") else -1 if l == "pop" else 0 for l in lines) == 0
