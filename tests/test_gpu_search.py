"""GPU parity of the neighbour search (hash, stable sort, cell bounds,
reorder) and of the neighbour counts: bit-exact against the FP32 oracle,
through the C ABI, on lattices, random clouds and edge cases."""
import numpy as np
import pytest

import zsph_b200 as z
from oracle import pyoracle as po
from zsph_b200 import cases

pytestmark = pytest.mark.gpu


def _on_cell_faces(n, seed):
    """Random cloud with most coordinates on a cell face (including the grid's
    far faces, which kill the particle) or a few ulps to either side of it:
    the inputs where the hash's quotient is within rounding of an integer."""
    c = cases.random_cloud(n, seed)
    p = po.Oracle(c.json, c.state, np.float32).p
    rng = np.random.default_rng(seed)
    pos = c.state.pos
    size = np.float32(p.grid_size)
    for ax, (lo, dim) in enumerate(((p.grid_xmin, p.grid_xdim), (p.grid_ymin, p.grid_ydim),
                                    (p.grid_zmin, p.grid_zdim))):
        pick = rng.uniform(size=n) < 0.8
        m = rng.integers(0, dim + 1, size=n).astype(np.float32)
        v = (np.float32(lo) + m * size).astype(np.float32)
        ulps = rng.choice([-64, -16, -3, -2, -1, 0, 0, 0, 1, 2, 3, 16, 64], size=n)
        for k in range(64):
            more = np.abs(ulps) > k
            v[more] = np.nextafter(v[more], np.where(ulps[more] > 0, np.float32(np.inf), np.float32(-np.inf)))
        pos[pick, ax] = v[pick]
    c.state.tmp_pos[:] = pos
    return c


def _cases():
    return {
        "cloud_on_cell_faces": lambda: _on_cell_faces(6000, 31),
        "small_dam": lambda: cases.small(0.04),
        "config0_dam": cases.config0,
        "cloud_killed": lambda: cases.random_cloud(5000, 1, kill_frac=0.02),
        "cloud_crowded_cell0": lambda: cases.random_cloud(6000, 3, kill_frac=0.3),  # >256 in cell 0
        "cloud_257": lambda: cases.random_cloud(257, 4),
        "cloud_1": lambda: cases.random_cloud(1, 5),
        "cloud_2": lambda: cases.random_cloud(2, 6),
    }


def _oracle_search(c):
    o = po.Oracle(c.json, c.state, np.float32)
    o.search()
    return o


def _assert_same(sol, o, tag=""):
    tmp = sol.download_tmp()
    for k in ("hash", "index", "grid_start", "grid_end"):
        assert np.array_equal(tmp[k], o.tmp[k]), f"{tag}{k}"
    new = sol.download("new")
    for k in ("pos", "vel", "rhop", "tmp_pos", "tmp_vel", "tmp_rhop", "type", "table"):
        assert np.array_equal(getattr(new, k), o.new[k].reshape(getattr(new, k).shape)), f"{tag}new.{k}"
    old = sol.download("old")  # out-of-grid particles are killed in place in the source buffer
    for k in ("pos", "vel", "rhop", "type"):
        assert np.array_equal(getattr(old, k), o.old[k].reshape(getattr(old, k).shape)), f"{tag}old.{k}"


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_fused_search_bit_exact(name):
    c = _cases()[name]()
    sol = z.Solver.from_case(c)
    sol.neighbor_search("old", "new")
    sol.sync()
    _assert_same(sol, _oracle_search(c), "fused ")
    sol.close()


@pytest.mark.parametrize("name", ["small_dam", "cloud_killed", "cloud_crowded_cell0", "cloud_1", "cloud_on_cell_faces"])
def test_dropin_hash_sort_index_sort_data_bit_exact(name):
    c = _cases()[name]()
    sol = z.Solver.from_case(c)
    sol.hash("old")
    sol.sort_index()
    sol.sort_data("old", "new")
    sol.sync()
    _assert_same(sol, _oracle_search(c), "drop-in ")
    sol.close()


def test_sort_index_carries_arbitrary_values_stably():
    c = cases.random_cloud(20000, 9)
    sol = z.Solver.from_case(c)
    rng = np.random.default_rng(0)
    keys = rng.integers(0, sol.G, size=c.n).astype(np.int32)
    keys[::7] = keys[0]  # many ties
    vals = rng.integers(-10**6, 10**6, size=c.n).astype(np.int32)
    sol.upload_tmp(hash=keys, index=vals)
    sol.sort_index()
    t = sol.download_tmp()
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(t["hash"], keys[order])
    assert np.array_equal(t["index"], vals[order])
    assert sol.status() & z.FLAG_BAD_KEY == 0
    sol.close()


def test_singleton_last_cell_keeps_stale_bounds():
    c = cases.random_cloud(3000, 7)
    c.state.pos[-1] = [0.2, 0.15, 0.36]
    sol = z.Solver.from_case(c)
    G = sol.G
    sol.upload_tmp(grid_start=np.full(G, -7, np.int32), grid_end=np.full(G, -9, np.int32))
    sol.neighbor_search("old", "new")
    o = po.Oracle(c.json, c.state, np.float32)
    o.tmp["grid_start"][:] = -7
    o.tmp["grid_end"][:] = -9
    o.search()
    t = sol.download_tmp()
    assert np.array_equal(t["grid_start"], o.tmp["grid_start"])
    assert np.array_equal(t["grid_end"], o.tmp["grid_end"])
    k = t["hash"][-1]
    assert t["grid_end"][k] == -9
    sol.close()


def test_killed_flag_and_type100():
    c = cases.random_cloud(4000, 11, kill_frac=0.05)
    sol = z.Solver.from_case(c)
    sol.neighbor_search("old", "new")
    f = sol.status()
    assert f & z.FLAG_KILLED
    assert (sol.download("new").type == 100).sum() > 0
    sol.close()


@pytest.mark.parametrize("name", ["small_dam", "config0_dam", "cloud_killed"])
def test_neighbor_counts_bit_exact(name):
    c = _cases()[name]()
    sol = z.Solver.from_case(c)
    sol.neighbor_search("old", "new")
    nb_b, nb_g = sol.neighbor_counts("new")
    o = _oracle_search(c)
    assert np.array_equal(nb_b, o.neighbor_count("new", "boundary"))
    assert np.array_equal(nb_g, o.neighbor_count("new", "governing"))
    sol.close()


def test_search_twice_reuses_scratch():
    # the counting-sort buckets must be left zeroed between searches
    c = cases.small(0.04)
    sol = z.Solver.from_case(c)
    for _ in range(3):
        sol.neighbor_search("old", "new")
        sol.neighbor_search("new", "old")
    o = po.Oracle(c.json, c.state, np.float32)
    for _ in range(3):
        o.search("old", "new")
        o.search("new", "old")
    t = sol.download_tmp()
    assert np.array_equal(t["index"], o.tmp["index"])
    assert np.array_equal(t["grid_end"], o.tmp["grid_end"])
    assert np.array_equal(sol.download("old").pos, o.old["pos"])
    sol.close()


def test_fused_search_many_scan_tiles():
    # dx = 0.0075: 190,060 cells = 47 one-pass scan tiles, so the look-back
    # crosses more than one 32-tile window
    c = cases.dam_break(0.0075, end_step=500)
    sol = z.Solver.from_case(c)
    sol.neighbor_search("old", "new")
    sol.sync()
    _assert_same(sol, _oracle_search(c), "medium ")
    sol.close()


def test_dropin_sort_between_fused_searches():
    # the drop-in sort and the fused search share the counting-sort scratch
    c = cases.random_cloud(5000, 21, kill_frac=0.01)
    sol = z.Solver.from_case(c)
    o = po.Oracle(c.json, c.state, np.float32)
    sol.neighbor_search("old", "new")
    o.search("old", "new")
    sol.hash("new")
    sol.sort_index()
    o.hash("new")
    o.sort_index()
    t = sol.download_tmp()
    assert np.array_equal(t["index"], o.tmp["index"])
    sol.neighbor_search("new", "old")
    o.search("new", "old")
    t = sol.download_tmp()
    for k in ("hash", "index", "grid_start", "grid_end"):
        assert np.array_equal(t[k], o.tmp[k]), k
    sol.close()


def test_profiled_steps_report_every_launch_and_group():
    c = cases.small(0.04)
    a = z.Solver.from_case(c)
    b = z.Solver.from_case(c)
    per = a.step_profiled()
    names = [k for k, _ in per]
    search = ["hash_count", "scan", "scatter", "rank_gather"]
    sub = search + ["nblist", "walls", "boundary", "governing"]
    assert names == sub + sub
    assert len(names) == a.launches_per_step() == 16
    # the corrector's lists by the list transfer (opt-in)
    a.set_list_transfer(True)
    corr = search + ["xfer_classify", "xfer_search", "nblist_xfer", "nblist_fallback", "walls", "boundary",
                     "governing"]
    assert [k for k, _ in a.step_profiled()] == sub + corr
    assert a.launches_per_step() == 19
    a.set_list_transfer(False)
    b.step()
    grp = a.step_profiled(groups=True)
    assert [k for k, _ in grp] == ["search", "pair", "search", "pair"]
    assert all(t > 0 for _, t in per + grp)
    b.step()
    b.step()
    sa, sb = a.download("old"), b.download("old")
    assert np.array_equal(sa.pos, sb.pos) and np.array_equal(sa.table, sb.table)
    a.close()
    b.close()


def test_misaligned_particle_buffer_is_refused_before_any_launch():
    # the kernels move the float2 arrays with 8-byte accesses; a buffer
    # whose float arrays do not start on an 8-byte boundary is rejected on the
    # host (a view 4 bytes into the pos array, still inside its allocation)
    import ctypes
    c = cases.small(0.04)
    sol = z.Solver.from_case(c)
    bad = z.Ptc()
    ctypes.memmove(ctypes.byref(bad), ctypes.byref(sol.old), ctypes.sizeof(z.Ptc))
    bad.pos = sol.old.pos + 4
    before = sol.download("new").pos.copy()
    with pytest.raises(z.ZsphError) as e:
        lib = z.lib
        z.check(lib.zsph_neighbor_search(sol.h, ctypes.byref(bad), ctypes.byref(sol.new), ctypes.byref(sol.tmp), None),
                sol.h)
    assert e.value.code == z.ZSPH_EINVAL and "8-byte" in str(e.value)
    assert np.array_equal(sol.download("new").pos, before)  # nothing ran
    sol.close()
