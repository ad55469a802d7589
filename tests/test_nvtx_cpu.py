"""Trace ranges on the CPU: with an NVTX tool attached (here a probe that
logs each range, tests/nvtx_probe.c, loaded through NVTX_INJECTION64_PATH),
entry points of libzsph_b200.so push a range named after themselves and pop
it on every return path, errors included.  The entry points run here are the
host-only ones; the handle entry points use the same range (through their
common argument checks) and, inside a step, ranges per kernel group."""
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, numpy as np, zsph_b200 as z
from zsph_b200 import cases
c = cases.config0()
d = {k: (v.decode() if isinstance(v, bytes) else v) for k, v in ((k, getattr(c.json, k)) for k, _ in z.JsonCase._fields_) if k != "m"}
open("case.json", "w").write(json.dumps(d))
z.read_json("case.json")
n, G = 16, 4
a = {"pos": np.zeros((n, 3), np.float32), "vel": np.zeros((n, 3), np.float32), "rhop": np.zeros((n, 2), np.float32),
     "type": np.ones(n, np.int32), "table": np.zeros(n, np.int32), "grid_start": np.zeros(G, np.int32),
     "grid_end": np.zeros(G, np.int32)}
z.snapshot_save_host("s.zsnap", a, n, G, step=1)
try:
    z.snapshot_load_host("missing.zsnap", n, G)
except z.ZsphError:
    pass
try:
    z.read_vtk("missing.vtk", n)
except z.ZsphError:
    pass
print("child ok")
"""


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    out = str(tmp_path_factory.mktemp("nvtx") / "libnvtx_probe.so")
    subprocess.run(["gcc", "-shared", "-fPIC", "-O2", "-Wall", "-Werror", "-I/usr/local/cuda/include",
                    os.path.join(ROOT, "tests", "nvtx_probe.c"), "-o", out], check=True, capture_output=True,
                   text=True)
    return out


def test_entry_points_push_and_pop_named_ranges(probe, tmp_path):
    log = tmp_path / "nvtx.log"
    env = dict(os.environ, NVTX_INJECTION64_PATH=probe, ZSPH_NVTX_LOG=str(log),
               PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", CHILD], cwd=tmp_path, env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0 and "child ok" in r.stdout, r.stdout + r.stderr
    lines = log.read_text().split("\n")
    pushes = [l[5:] for l in lines if l.startswith("push ")]
    assert pushes == ["zsph_read_json", "zsph_snapshot_save_host", "zsph_snapshot_load_host", "zsph_read_vtk"]
    # every range is closed, on the error returns too
    depth = 0
    for l in lines:
        depth += 1 if l.startswith("push ") else -1 if l == "pop" else 0
        assert depth >= 0
    assert depth == 0
