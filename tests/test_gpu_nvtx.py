"""Trace ranges of a step on the GPU: with the probe tool attached
(tests/nvtx_probe.c through NVTX_INJECTION64_PATH), zsph_step pushes its own
range and, per sub-step, the search, boundary and governing groups."""
import os
import subprocess
import sys

import pytest

from tests.test_nvtx_cpu import ROOT, probe  # noqa: F401  (the probe fixture)

pytestmark = pytest.mark.gpu

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
