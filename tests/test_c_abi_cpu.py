"""The C ABI from a plain C99 caller (tests/c_abi_check.c), on the CPU: the
header compiles as C, the entry points link with C linkage against
libzsph_b200.so, the public structs have the same sizes under the C compiler
as in the Python mirror, and the host-only set-up calls give, byte for byte,
the GPU parameters the Python binding gets for the same case file."""
import ctypes
import json
import os
import shutil
import subprocess

import pytest

import zsph_b200 as z
from zsph_b200 import cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

MIRRORS = {
    "zsph_json_t": z.JsonCase, "zsph_cpu_param_t": z.CpuParam, "zsph_gpu_param_t": z.GpuParam,
    "zsph_ptc_t": z.Ptc, "zsph_tmp_t": z.Tmp, "zsph_learn_train_stats_t": z.LearnTrainStats,
    "zsph_learn_run_stats_t": z.LearnRunStats, "zsph_tune_t": z.TuneResult,
    "zsph_conservation_t": z.Conservation, "zsph_rigid_t": z.RigidBody, "zsph_case_options_t": z.CaseOptions,
}


@pytest.fixture(scope="module")
def c_caller(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    libdir = os.path.join(ROOT, "zsph_b200")
    assert os.path.exists(os.path.join(libdir, "libzsph_b200.so")), "build the library first"
    exe = str(tmp_path_factory.mktemp("cabi") / "c_abi_check")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-Werror", "-pedantic", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "c_abi_check.c"), "-L", libdir, "-lzsph_b200",
                    f"-Wl,-rpath,{libdir}", "-o", exe], check=True, capture_output=True, text=True)
    return exe


def _run(exe, *args):
    out = subprocess.run([exe, *args], capture_output=True, text=True, timeout=60)
    lines = {}
    for line in out.stdout.splitlines():
        key, _, val = line.rpartition(" ")
        lines[key] = val
    return out.returncode, lines


def test_struct_sizes_match_the_python_mirror(c_caller):
    rc, out = _run(c_caller)
    assert rc == 0
    for name, cls in MIRRORS.items():
        assert int(out[f"sizeof {name}"]) == ctypes.sizeof(cls), name


@pytest.mark.parametrize("case_fn", [cases.config0, cases.config1])
def test_c_caller_derives_the_same_gpu_parameters(c_caller, tmp_path, case_fn):
    c = case_fn()
    d = {}
    for k, _ in z.JsonCase._fields_:
        if k == "m":
            continue  # not a key of the reference's case file
        v = getattr(c.json, k)
        d[k] = v.decode() if isinstance(v, bytes) else v
    p = tmp_path / "input.json"
    p.write_text(json.dumps(d))
    rc, out = _run(c_caller, str(p))
    assert rc == 0, out
    assert out["set_cpu_param"] == "0" and out["check_dt"] == "0" and out["set_gpu_param"] == "0"
    cp, gp = z.params_from_json(z.read_json(str(p)))
    assert int(out["grid_num"]) == cp.grid_num
    assert bytes.fromhex(out["gparam"]) == bytes(gp)


def test_c_caller_gets_an_error_code_for_a_missing_file(c_caller, tmp_path):
    missing = str(tmp_path / "missing.json")
    out = subprocess.run([c_caller, missing], capture_output=True, text=True, timeout=60)
    assert out.returncode == 1
    assert out.stdout.strip().endswith(f"read_json {z.ZSPH_EIO} cannot open {missing}")
