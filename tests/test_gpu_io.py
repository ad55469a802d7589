"""The output thread pool (io/mul_thread.cu, deltasph/main.cu:101-142): device
arrays copied into pinned buffers on the caller's stream, VTK files written by
worker threads, one file per submitted step."""
import ctypes
import os

import numpy as np
import pytest

import zsph_b200 as z
from zsph_b200 import cases

pytestmark = pytest.mark.gpu


def test_writer_pool_writes_each_submitted_step(tmp_path):
    c = cases.small(0.04)
    sol = z.Solver.from_case(c)
    w = ctypes.c_void_p()
    flags = z.OUT_REFERENCE | z.OUT_RHO | z.OUT_TABLE
    z.check(z.lib.zsph_writer_create(str(tmp_path).encode(), sol.n, flags, 2, ctypes.byref(w)))
    snapshots = {}
    for step in range(5):
        sol.step()
        z.check(z.lib.zsph_writer_submit(w, ctypes.byref(sol.old), ctypes.byref(sol.tmp), step, None))
        snapshots[step] = sol.download("old")
    z.check(z.lib.zsph_writer_destroy(w))
    for step, st in snapshots.items():
        path = os.path.join(str(tmp_path), f"zsph{step}.vtk")
        got, acc = z.read_vtk(path, sol.n, accept_float=True)
        for k in ("pos", "vel", "rhop", "type", "table"):
            assert np.array_equal(getattr(got, k), getattr(st, k)), (step, k)
    sol.close()
