"""The reference's driver program (deltasph/main.cu) on this library:
zsph_compat_run reads a reference-style case directory (input.json and
input/input.vtk with double arrays), runs the step loop through the drop-in
entry points or the fused step, and writes output/zsph<i>.vtk every
output_step.  Checked against the Solver API run from the same state."""
import json
import os

import numpy as np
import pytest

import zsph_b200 as z
from zsph_b200 import cases

pytestmark = pytest.mark.gpu

_KEYS_F = ("g", "rho0", "dx", "h_factor", "r_factor", "eta_factor", "cs_factor", "delta", "alpha", "xmin", "xmax",
           "ymin", "ymax", "zmin", "zmax", "grid_layer_factor", "grid_size_factor", "dt")
_KEYS_I = ("start_step", "current_step", "end_step", "output_step", "ptc_num", "water_ptc_num", "air_ptc_num",
           "wall_ptc_num", "rigid_ptc_num", "thread_num", "gpu_id")


def _write_case(root, c, end_step, output_step):
    """A reference case directory: input.json, input/input.vtk (ASCII legacy
    VTK with double arrays, which the reference reader requires) and output/."""
    inp, out = os.path.join(root, "input"), os.path.join(root, "output")
    os.makedirs(inp)
    os.makedirs(out)
    st, n = c.state, c.n
    dbl = lambda a: " ".join(repr(float(v)) for v in np.asarray(a, np.float64).ravel())
    lines = ["# vtk DataFile Version 3.0", "zsph case", "ASCII", "DATASET UNSTRUCTURED_GRID",
             f"POINTS {n} double", dbl(st.pos), "CELLS 0 0", "CELL_TYPES 0", f"POINT_DATA {n}",
             "SCALARS p double 1", "LOOKUP_TABLE default", dbl(st.rhop[:, 1]),
             "SCALARS rho double 1", "LOOKUP_TABLE default", dbl(st.rhop[:, 0]),
             "SCALARS type int 1", "LOOKUP_TABLE default", " ".join(str(int(v)) for v in st.type),
             "VECTORS vel double", dbl(st.vel)]
    with open(os.path.join(inp, "input.vtk"), "w") as f:
        f.write("\n".join(lines) + "\n")
    j = {k: float(getattr(c.json, k)) for k in _KEYS_F}
    j.update({k: int(getattr(c.json, k)) for k in _KEYS_I})
    j.update(start_step=0, current_step=0, end_step=end_step, output_step=output_step, thread_num=2, gpu_id=0,
             input_path=inp, output_path=out, git_hash="test")
    path = os.path.join(root, "input.json")
    with open(path, "w") as f:
        json.dump(j, f)
    return path, out


@pytest.mark.parametrize("mode", [z.COMPAT_SEPARATE, z.COMPAT_FUSED, z.COMPAT_SEPARATE | z.COMPAT_SIMPLE,
                                  z.COMPAT_FUSED | z.COMPAT_SIMPLE])
def test_compat_run_matches_solver(tmp_path, mode):
    c = cases.small(0.04)
    nsteps, every = 12, 5
    path, out = _write_case(str(tmp_path), c, nsteps, every)
    assert z.compat_run(path, mode) == nsteps
    names = sorted(os.listdir(out))
    assert names == sorted(f"zsph{i}.vtk" for i in range(0, nsteps, every)), names
    # output at i = 10 holds the state after 11 steps
    sol = z.Solver.from_case(c)
    if mode & z.COMPAT_SIMPLE:
        sol.set_equations(z.EQ_SIMPLE)
    sol.run(11)
    want = sol.download("old")
    sol.close()
    got, acc = z.read_vtk(os.path.join(out, "zsph10.vtk"), c.n, rho0=float(c.json.rho0), accept_float=True)
    assert np.array_equal(got.pos, want.pos)
    assert np.array_equal(got.vel, want.vel)
    assert np.array_equal(got.type, want.type)


def test_compat_run_reports_a_missing_input(tmp_path):
    c = cases.small(0.04)
    path, _ = _write_case(str(tmp_path), c, 2, 1)
    os.remove(os.path.join(str(tmp_path), "input", "input.vtk"))
    with pytest.raises(z.ZsphError):
        z.compat_run(path)
