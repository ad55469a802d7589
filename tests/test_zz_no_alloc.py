"""zsph_sort_index_noalloc: the stable sort for callers that cannot allocate
device memory (an application whose device memory belongs to another
allocator, or a loop that must not call cudaMalloc/cudaFree, which may
synchronise the device).  It keeps its scratch in a fixed static device array
instead of a handle's allocations.  Checked through the C ABI against the
existing entry point zsph_sort_index on two calls in a row (integer output:
bit-exact), the second one smaller so that it runs on what the first left in
the shared array.  This file is collected last on purpose."""
import ctypes

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
