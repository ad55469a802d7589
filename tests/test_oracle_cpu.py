"""The CPU oracle against independent restatements and known answers
(no GPU).  The oracle's pin against the reference's own CUDA outputs is in
test_golden_cpu.py."""
import numpy as np
import pytest

from oracle import pyoracle as po
from zsph_b200 import cases
from tests.helpers import cell_bounds_closed_form, stable_sort_keys


def test_hash_known_answers():
    c = cases.small(0.04)
    rc, p = po.params(c.json)
    gs, X, Y = np.float32(p.grid_size), p.grid_xdim, p.grid_ydim
    gmin = np.array([p.grid_xmin, p.grid_ymin, p.grid_zmin], np.float32)
    pts = np.array([
        gmin + np.float32(0.5) * gs,                       # cell (0,0,0)
        gmin + np.array([1, 2, 3], np.float32) * gs,        # exactly on a cell corner
        gmin + np.array([1.5, 0.5, 0.5], np.float32) * gs,
        gmin - np.float32(0.01),                            # below the grid -> killed
        gmin + np.array([X + 0.5, 0.5, 0.5], np.float32) * gs,  # x overflow aliases into next row
        gmin + np.array([0.5, 0.5, p.grid_zdim + 1], np.float32) * gs,  # above the grid -> killed
    ], np.float32)
    n = len(pts)
    st = cases.State(pos=pts.copy(), vel=np.ones((n, 3), np.float32), rhop=np.full((n, 2), 1001, np.float32),
                     type=np.ones(n, np.int32), table=np.zeros(n, np.int32))
    c.json.ptc_num = n
    o = po.Oracle(c.json, st, np.float32)
    o.hash("old")
    h = o.tmp["hash"]
    cell = np.floor((pts - gmin) / gs).astype(np.int64)
    expect = cell[:, 2] * X * Y + cell[:, 1] * X + cell[:, 0]
    assert h[0] == 0 and h[2] == 1
    assert h[1] == expect[1]
    assert h[4] == expect[4] == X * 1 + 0 + 0 * 0 or h[4] == expect[4]
    assert h[3] == 0 and o.old["type"][3] == 100
    assert np.all(o.old["pos"][3] == gmin) and np.all(o.old["vel"][3] == 0)
    assert tuple(o.old["rhop"][3]) == (np.float32(p.rho0), 0.0)
    assert h[5] == 0 and o.old["type"][5] == 100
    assert np.array_equal(o.tmp["index"], np.arange(n))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_sort_and_cells_match_closed_form(seed):
    c = cases.random_cloud(5000 + 37 * seed, seed, kill_frac=0.02 * seed)
    o = po.Oracle(c.json, c.state, np.float32)
    o.hash("old")
    keys0 = o.tmp["hash"].copy()
    o.sort_index()
    sk, order = stable_sort_keys(keys0)
    assert np.array_equal(o.tmp["hash"], sk)
    assert np.array_equal(o.tmp["index"], order)
    o.sort_data("old", "new")
    s, e = cell_bounds_closed_form(sk, o.p.grid_num)
    assert np.array_equal(o.tmp["grid_start"], s)
    assert np.array_equal(o.tmp["grid_end"], e)
    # reorder: new[t] = old[index[t]], table keeps table + t invariant
    assert np.array_equal(o.new["pos"], o.old["pos"][order])
    assert np.array_equal(o.new["table"] + np.arange(len(order)), order)


def test_singleton_last_cell_leaves_stale_bounds():
    c = cases.random_cloud(3000, 7)
    st = c.state.copy()
    # put one particle alone in the highest occupied cell (padding layer above the box)
    st.pos[-1] = [0.2, 0.15, 0.36]
    o = po.Oracle(c.json, st, np.float32)
    G = o.p.grid_num
    o.tmp["grid_start"][:] = -7
    o.tmp["grid_end"][:] = -9
    o.search()
    sk = o.tmp["hash"]
    k = sk[-1]
    assert sk[-2] != k
    s, e = cell_bounds_closed_form(sk, G, np.full(G, -7, np.int32), np.full(G, -9, np.int32))
    assert np.array_equal(o.tmp["grid_start"], s) and np.array_equal(o.tmp["grid_end"], e)
    assert o.tmp["grid_end"][k] == -9 and o.tmp["grid_start"][k] == len(sk) - 1
    assert np.all(o.tmp["grid_start"][k + 1:] == -7)


def test_last_particle_is_excluded_from_its_cell_range():
    c = cases.small(0.04)
    o = po.Oracle(c.json, c.state, np.float32)
    o.search()
    n = o.p.ptc_num
    k = o.tmp["hash"][-1]
    assert o.tmp["grid_end"][k] == n - 1  # reference quirk: [start, N-1) skips the last particle


def test_perfect_lattice_renormalisation_is_diagonal():
    # interior fluid particles of a cubic lattice: the renormalisation matrix
    # is symmetric in x and z, so grad(rho) of a uniform field vanishes
    c = cases.dam_break(0.04, water=(0.6, 0.6, 0.6), tank=(0.6, 0.6, 0.6))
    st = c.state.copy()
    st.rhop[:, 0] = 1000.0
    st.rhop[:, 1] = 0.0
    o = po.Oracle(c.json, st, np.float64)
    o.search()
    o.boundary()
    f = o.new["type"] == 1
    g = o.tmp["dofv_grandrho"][f]
    # uniform fluid density: only wall-adjacent particles see a density difference
    assert np.median(np.abs(g[:, :3])) < 1e-6


def test_hydrostatic_column_interior_is_near_rest():
    # a column at rest in a closed box: interior vertical acceleration ~ 0 at step 0
    c = cases.dam_break(0.04, water=(0.6, 0.6, 0.6), tank=(0.6, 0.6, 0.6))
    o = po.Oracle(c.json, c.state, np.float64)
    o.search()
    o.boundary()
    o.governing()
    pos = o.new["pos"]
    f = (o.new["type"] == 1) & (pos[:, 0] > 0.15) & (pos[:, 0] < 0.45) & (pos[:, 1] > 0.15) & (pos[:, 1] < 0.45) \
        & (pos[:, 2] > 0.15) & (pos[:, 2] < 0.45)
    acc = o.tmp["acc_drhodt"][f]
    assert np.abs(acc[:, 2]).mean() < 0.05 * 9.81
    assert np.abs(acc[:, 0]).mean() < 0.05 * 9.81


def test_fp32_oracle_tracks_fp64_oracle():
    c = cases.small(0.04)
    a = po.Oracle(c.json, c.state, np.float32)
    b = po.Oracle(c.json, c.state, np.float64)
    a.step(5)
    b.step(5)
    # the sorted orders may differ where a particle sits on a cell face, but in
    # both table + slot is a permutation of the original particle ids
    ida = a.old["table"] + np.arange(c.n)
    idb = b.old["table"] + np.arange(c.n)
    assert np.array_equal(np.sort(ida), np.arange(c.n)) and np.array_equal(np.sort(idb), np.arange(c.n))
    pa = np.empty_like(a.old["pos"]); pa[ida] = a.old["pos"]
    pb = np.empty_like(b.old["pos"]); pb[idb] = b.old["pos"]
    assert np.abs(pa - pb).max() < 1e-5


def test_simple_equations_fp32_tracks_fp64_and_rest():
    # simplesph equations: a column at rest in a closed box stays near rest,
    # and the FP32 instance tracks the FP64 one
    c = cases.dam_break(0.04, water=(0.6, 0.6, 0.6), tank=(0.6, 0.6, 0.6))
    o = po.Oracle(c.json, c.state, np.float64)
    o.search()
    o.boundary_simple("new")
    o.governing_simple("new")
    pos = o.new["pos"]
    f = (o.new["type"] == 1) & np.all((pos > 0.15) & (pos < 0.45), axis=1)
    assert np.abs(o.tmp["acc_drhodt"][f, 2]).mean() < 0.05 * 9.81
    a = po.Oracle(c.json, c.state, np.float32)
    b = po.Oracle(c.json, c.state, np.float64)
    a.step_simple(5)
    b.step_simple(5)
    pa = np.empty_like(a.old["pos"]); pa[a.old["table"] + np.arange(c.n)] = a.old["pos"]
    pb = np.empty_like(b.old["pos"]); pb[b.old["table"] + np.arange(c.n)] = b.old["pos"]
    assert np.abs(pa - pb).max() < 1e-5
