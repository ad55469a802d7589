"""zsph_sort_index_noalloc: the stable sort for callers that cannot allocate
device memory (an application whose device memory belongs to another
allocator, or a loop that must not call cudaMalloc/cudaFree, which may
synchronise the device).  It keeps its scratch in a fixed static device array
instead of a handle's allocations.  Checked through the C ABI against the
existing entry point zsph_sort_index on two calls in a row (integer output:
bit-exact), the second one smaller so that it runs on what the first left in
the shared array.  This file is collected last on purpose."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import zsph_b200 as z
from zsph_b200 import cases

pytestmark = pytest.mark.gpu


def _inputs(n, G, seed):
    rng = np.random.default_rng(seed)
    keys = rng.integers(0, G, size=n).astype(np.int32)
    keys[::5] = keys[1]                      # many ties: stability matters
    keys[-300:] = rng.integers(0, 3, 300)    # and a crowded low cell
    vals = rng.integers(-(2**30), 2**30, size=n).astype(np.int32)
    return keys, vals


def _sort_with(sol, keys, vals, noalloc):
    sol.upload_tmp(hash=keys, index=vals)
    if noalloc:
        rc = z.lib.zsph_sort_index_noalloc(ctypes.byref(sol.gp), sol.G, ctypes.byref(sol.tmp), None)
        assert rc == z.ZSPH_OK, z.last_error()
    else:
        sol.sort_index()
    sol.sync()
    t = sol.download_tmp()
    return t["hash"], t["index"]


def test_noalloc_sort_matches_zsph_sort_index_on_two_calls():
    for call, (mk, seed) in enumerate([(lambda: cases.random_cloud(60000, 31), 1),
                                       (lambda: cases.random_cloud(7001, 32), 2)]):
        c = mk()
        cp, gp = z.params_from_json(c.json)
        sol = z.Solver(gp, cp.grid_num)
        keys, vals = _inputs(c.n, cp.grid_num, seed)
        ref_h, ref_i = _sort_with(sol, keys, vals, noalloc=False)
        got_h, got_i = _sort_with(sol, keys, vals, noalloc=True)
        assert np.array_equal(got_h, ref_h), f"call {call}: sorted keys differ"
        assert np.array_equal(got_i, ref_i), f"call {call}: carried values differ"
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(got_i, vals[order])
        sol.close()


def test_noalloc_rejects_sizes_beyond_its_fixed_scratch():
    c = cases.small(0.04)
    cp, gp = z.params_from_json(c.json)
    gp.ptc_num = 131073
    tmp = z.Tmp()
    rc = z.lib.zsph_sort_index_noalloc(ctypes.byref(gp), cp.grid_num, ctypes.byref(tmp), None)
    assert rc == z.ZSPH_EINVAL
    assert "131072" in z.last_error()
    gp.ptc_num = 10
    rc = z.lib.zsph_sort_index_noalloc(ctypes.byref(gp), 131073, ctypes.byref(tmp), None)
    assert rc == z.ZSPH_EINVAL


def test_noalloc_clamps_keys_outside_the_grid():
    # keys must lie in [0, grid_num); one below and one above are sorted and
    # written back as 0 and grid_num - 1, and the call still succeeds
    c = cases.random_cloud(5000, 33)
    cp, gp = z.params_from_json(c.json)
    G = cp.grid_num
    sol = z.Solver(gp, G)
    keys, vals = _inputs(c.n, G, 3)
    keys[17] = -5
    keys[4000] = G + 7
    got_h, got_i = _sort_with(sol, keys, vals, noalloc=True)
    clamped = np.clip(keys, 0, G - 1)
    order = np.argsort(clamped, kind="stable")
    assert np.array_equal(got_h, clamped[order])
    assert np.array_equal(got_i, vals[order])
    sol.close()


_CONTEXT_SCRIPT = r"""
import ctypes, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import zsph_b200 as z
from zsph_b200 import cases

c = cases.random_cloud(20000, 34)
cp, gp = z.params_from_json(c.json)
G, n = cp.grid_num, c.n
rng = np.random.default_rng(5)
keys = rng.integers(0, G, size=n).astype(np.int32)
keys[::3] = keys[2]
vals = np.arange(n, dtype=np.int32)[::-1].copy()
order = np.argsort(keys, kind="stable")

def sort_once():
    tmp = z.Tmp()
    hp, ip = ctypes.c_void_p(), ctypes.c_void_p()
    z.check(z.lib.zsph_device_malloc(ctypes.byref(hp), 4 * n))
    z.check(z.lib.zsph_device_malloc(ctypes.byref(ip), 4 * n))
    tmp.hash, tmp.index = hp, ip
    z.check(z.lib.zsph_memcpy(hp, keys.ctypes.data, 4 * n, 1, None))
    z.check(z.lib.zsph_memcpy(ip, vals.ctypes.data, 4 * n, 1, None))
    z.check(z.lib.zsph_sort_index_noalloc(ctypes.byref(gp), G, ctypes.byref(tmp), None))
    z.check(z.lib.zsph_device_synchronize())
    h, i = np.empty(n, np.int32), np.empty(n, np.int32)
    z.check(z.lib.zsph_memcpy(h.ctypes.data, hp, 4 * n, 2, None))
    z.check(z.lib.zsph_memcpy(i.ctypes.data, ip, 4 * n, 2, None))
    z.check(z.lib.zsph_device_free(hp))
    z.check(z.lib.zsph_device_free(ip))
    return np.array_equal(h, keys[order]) and np.array_equal(i, vals[order])

cu = ctypes.CDLL("libcuda.so.1")
ok = [sort_once()]                       # primary context: set-up call
ctx = ctypes.c_void_p()
assert cu.cuCtxCreate_v2(ctypes.byref(ctx), 0, 0) == 0
ok.append(sort_once())                   # a second context of the same device
assert cu.cuCtxDestroy_v2(ctx) == 0
prim = ctypes.c_void_p()
assert cu.cuDevicePrimaryCtxRetain(ctypes.byref(prim), 0) == 0
assert cu.cuCtxSetCurrent(prim) == 0
ok.append(sort_once())                   # back in the primary context
print("results", " ".join(str(int(v)) for v in ok))
"""


def test_noalloc_looks_the_scratch_up_again_in_a_new_context():
    # the scratch address belongs to a context: a call made in another context
    # of the same device (here one made with cuCtxCreate; cudaDeviceReset gives
    # the same situation) must look it up again rather than reuse the first
    # context's address.  A fresh process, so that this test's contexts touch
    # nothing else.
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", _CONTEXT_SCRIPT, root], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "results 1 1 1" in r.stdout, r.stdout + r.stderr
