"""Precision form (cell + FP32 offset positions), FP64 global sums and the
FP64 6DOF floating body, against the FP64 oracle run of the same equations."""
import dataclasses

import numpy as np
import pytest

import zsph_b200 as z
from oracle import pyoracle as po
from zsph_b200 import cases

pytestmark = pytest.mark.gpu


def _solver(c, precise):
    s = z.Solver.from_case(c)
    if precise:
        s.set_precision(True, c.pos64 if c.pos64 is not None else c.state.pos.astype(np.float64))
    return s


def _exact_state(c):
    pos = c.pos64 if c.pos64 is not None else c.state.pos.astype(np.float64)
    return dataclasses.replace(c.state, pos=pos)


def _by_id(sol_or_state, n, pos):
    """Rows in original particle order (table[i] + i)."""
    ids = sol_or_state.table + np.arange(n)
    out = np.empty_like(pos)
    out[ids] = pos
    return out


def test_load_and_positions_round_trip():
    c = cases.floating_body(0.04, end_step=10)
    s = _solver(c, True)
    x = s.positions64()
    assert np.max(np.abs(x - c.pos64)) < 1e-8  # FP32 offsets of at most one cell
    s.close()


def test_precision_form_tracks_fp64_oracle():
    c = cases.dam_break(0.04, end_step=100)
    nsteps = 60
    o = po.Oracle(c.json, _exact_state(c), dtype=np.float64)
    o.step(nsteps)
    want = {k: _by_id(type("S", (), {"table": o.old["table"]}), c.n, o.old[k]) for k in ("pos", "vel")}
    err = {}
    for precise in (False, True):
        s = _solver(c, precise)
        s.run(nsteps)
        st = s.download("old")
        x = s.positions64()
        got_pos = _by_id(st, c.n, x)
        got_vel = _by_id(st, c.n, st.vel.astype(np.float64))
        err[precise] = (np.max(np.abs(got_pos - want["pos"])), np.max(np.abs(got_vel - want["vel"])))
        s.close()
    print("max |err| vs FP64 (pos, vel): plain", err[False], "precision", err[True])
    assert err[True][0] < 1e-5 and err[True][1] < 1e-3
    assert err[True][0] <= 1.5 * err[False][0] + 1e-7


def test_conservation_sums():
    c = cases.dam_break(0.04, end_step=100)
    s = _solver(c, True)
    a = s.conservation()
    assert a["mass"] == pytest.approx(c.n_fluid * float(s.gp.m), rel=1e-12)
    assert a["kinetic"] == 0.0 and np.all(a["momentum"] == 0.0)
    s.run(40)
    b = s.conservation()
    assert b["mass"] == a["mass"]  # particles carry fixed mass; none left the grid
    assert b["kinetic"] > 0 and b["potential"] < a["potential"]  # the column starts to fall
    e0 = a["kinetic"] + a["potential"] + a["internal"]
    e1 = b["kinetic"] + b["potential"] + b["internal"]
    print("energy", e0, "->", e1, "released potential", a["potential"] - b["potential"])
    assert e1 <= e0 * (1 + 1e-9)  # artificial viscosity and density diffusion only dissipate
    s.close()


@pytest.mark.parametrize("precise", [False, True])
def test_floating_body_matches_fp64_oracle(precise):
    c = cases.floating_body(0.04, end_step=1000)
    nsteps = 400  # free fall onto the water (about 0.1 s), then entry
    o = po.Oracle(c.json, _exact_state(c), dtype=np.float64)
    o.attach_rigid(c.body["first"], c.body["count"], c.body["mass"])
    s = _solver(c, precise)
    b0 = s.attach_body(c.body["first"], c.body["count"], c.body["mass"])
    assert np.allclose(b0["pos"], o.rigid_state()["x"], atol=1e-6)
    n_cube = round(0.2 / 0.04)
    i_want = c.body["mass"] * 0.04 ** 2 * (n_cube ** 2 - 1) / 6  # lattice cube about its centroid
    assert np.allclose(np.diag(b0["inertia"].reshape(3, 3)), i_want, rtol=1e-9)
    heave, ref = [], []
    for k in range(nsteps // 50):
        o.step_rigid(50)
        s.run(50)
        heave.append(s.body()["pos"][2])
        ref.append(o.rigid_state()["x"][2])
    heave, ref = np.array(heave), np.array(ref)
    b = s.body()
    print("heave", heave.round(5), "oracle", ref.round(5), "force", b["force"])
    assert b["force"][2] > 0  # the water pushes up
    assert np.max(np.abs(heave - ref)) < 2e-3
    assert np.all(np.isfinite(s.download("old").vel))
    s.close()


# ---- the FP64 GPU checker and the config[2] floating-body comparison --------

def _state_of(d):
    return {k: d[k] for k in ("pos", "vel", "rhop", "type", "table")}


@pytest.mark.parametrize("body", [False, True])
def test_gpu_fp64_checker_matches_cpu_fp64_oracle(body):
    # the GPU instance of the FP64 oracle repeats the CPU oracle's arithmetic
    c = cases.floating_body(0.04, end_step=1000) if body else cases.dam_break(0.04, end_step=100)
    nsteps = 20
    cpu = po.Oracle(c.json, _exact_state(c), dtype=np.float64)
    gpu = po.GpuOracle64(c.json, _exact_state(c))
    if body:
        cpu.attach_rigid(c.body["first"], c.body["count"], c.body["mass"])
        gpu.attach_rigid(c.body["first"], c.body["count"], c.body["mass"])
        cpu.step_rigid(nsteps)
    else:
        cpu.step(nsteps)
    gpu.step(nsteps)
    g = gpu.download()
    for k in ("type", "table"):
        assert np.array_equal(g[k], cpu.old[k]), k
    for k in ("pos", "vel", "rhop"):
        d = float(np.max(np.abs(g[k] - cpu.old[k])))
        assert d == 0.0, f"{k}: max |gpu - cpu| = {d}"
    if body:
        rc, rg = cpu.rigid_state(), gpu.rigid_state()
        for k in ("x", "v", "w", "q"):
            assert np.array_equal(rc[k], rg[k]), k
    gpu.close()


def _pitch(q):
    """Rotation of the body about the y axis (rad) from its quaternion (w, x, y, z)."""
    w, x, y, z = q
    return float(np.arcsin(np.clip(2.0 * (w * y - z * x), -1.0, 1.0)))


def _floating_body_comparison(dx, nsteps, every):
    """The floating cube of config[2] (same tank, cube and drop) run by the
    FP64 GPU checker and by the product in the plain FP32 form and in the
    precision form; returns the final max and RMS errors against FP64 and the
    heave and pitch trajectories."""
    c = cases.floating_body(dx, end_step=nsteps)
    first, count, mass = c.body["first"], c.body["count"], c.body["mass"]
    ref = po.GpuOracle64(c.json, _exact_state(c))
    ref.attach_rigid(first, count, mass)
    runs = {"fp64": ref}
    for precise in (False, True):
        s = _solver(c, precise)
        s.attach_body(first, count, mass)
        runs["precision" if precise else "plain"] = s
    traj = {k: {"heave": [], "pitch": []} for k in runs}
    for _ in range(nsteps // every):
        for k, r in runs.items():
            if k == "fp64":
                r.step(every)
                b = r.rigid_state()
                traj[k]["heave"].append(float(b["x"][2]))
                traj[k]["pitch"].append(_pitch(b["q"]))
            else:
                r.run(every)
                b = r.body()
                traj[k]["heave"].append(float(b["pos"][2]))
                traj[k]["pitch"].append(_pitch(b["q"]))
    want = ref.download()
    ids_w = want["table"] + np.arange(c.n)
    out = {"particles": c.n, "steps": nsteps, "dx": dx}
    for k in ("plain", "precision"):
        s = runs[k]
        st = s.download("old")
        ids = st.table + np.arange(c.n)
        got = {"pos": s.positions64() if k == "precision" else st.pos.astype(np.float64),
               "vel": st.vel.astype(np.float64), "rho": st.rhop[:, 0].astype(np.float64)}
        ref_by_id = {"pos": np.empty((c.n, 3)), "vel": np.empty((c.n, 3)), "rho": np.empty(c.n)}
        ref_by_id["pos"][ids_w] = want["pos"]
        ref_by_id["vel"][ids_w] = want["vel"]
        ref_by_id["rho"][ids_w] = want["rhop"][:, 0]
        fluid = np.zeros(c.n, bool)
        fluid[ids[st.type == 1]] = True
        e = {}
        for q in ("pos", "vel", "rho"):
            g = np.empty_like(ref_by_id[q])
            g[ids] = got[q]
            d = np.abs(g - ref_by_id[q])[fluid]
            d = d.reshape(len(d), -1)
            e[q] = {"max": float(d.max()), "rms": float(np.sqrt(np.mean(d * d)))}
        e["heave_max_diff"] = float(np.max(np.abs(np.array(traj[k]["heave"]) - np.array(traj["fp64"]["heave"]))))
        e["pitch_max_diff"] = float(np.max(np.abs(np.array(traj[k]["pitch"]) - np.array(traj["fp64"]["pitch"]))))
        out[k] = e
        s.close()
    out["heave_fp64"] = traj["fp64"]["heave"]
    out["pitch_fp64"] = traj["fp64"]["pitch"]
    ref.close()
    return out


def test_floating_body_against_fp64_checker():
    # config[2] at its full size (dx = 0.01, 2,440,708 particles) over its
    # first 500 steps (the cube still falling toward the water); the whole
    # 5000-step case (entry, splash, floating) runs with ZSPH_FULL_CONFIG2=1
    import json
    import os
    full = os.environ.get("ZSPH_FULL_CONFIG2") == "1"
    r = _floating_body_comparison(0.01, 5000, 100) if full else _floating_body_comparison(0.01, 500, 50)
    print("config2 comparison", json.dumps(r))
    assert r["precision"]["pos"]["rms"] <= r["plain"]["pos"]["rms"]
    assert r["precision"]["heave_max_diff"] < 2e-3 and r["plain"]["heave_max_diff"] < 2e-3


# ---- several bodies and contact ---------------------------------------------

def _contact_for(body, dx, n_bottom, sag=0.05, zeta=0.5, g=9.81):
    """Spring-dashpot constants: the body's weight carried by n_bottom pairs at
    a static penetration of sag * dx, damped at zeta of critical."""
    kn = body["mass"] * g / (n_bottom * sag * dx)
    cn = zeta * 2.0 * np.sqrt(kn * n_bottom * body["mass"]) / n_bottom
    return kn, cn


@pytest.mark.parametrize("precise", [False, True])
def test_two_floating_bodies_match_fp64_oracle(precise):
    """Two cubes of different densities dropped from different heights into
    the same tank: each body's heave follows the FP64 oracle run of the same
    equations (per-body FP64 force and torque sums, one update per body)."""
    dx = 0.04
    c = cases.floating_bodies(dx, cubes=[dict(x=1.0, size=0.2, rho=500.0, bottom=0.55),
                                         dict(x=2.6, size=0.2, rho=800.0, bottom=0.62)], end_step=1000)
    o = po.Oracle(c.json, _exact_state(c), dtype=np.float64)
    o.attach_bodies(c.bodies)
    s = _solver(c, precise)
    for b in c.bodies:
        s.attach_body(b["first"], b["count"], b["mass"])
    assert s.body_count() == 2
    got, want = [[], []], [[], []]
    for _ in range(8):
        o.step_bodies(50)
        s.run(50)
        for k in range(2):
            got[k].append(s.body(k)["pos"][2])
            want[k].append(o.rigid_state(k)["x"][2])
    got, want = np.array(got), np.array(want)
    print("heave", got.round(5), "oracle", want.round(5))
    assert np.max(np.abs(got - want)) < 2e-3
    assert s.body(1)["pos"][2] < s.body(0)["pos"][2] + 0.07  # the denser cube sits deeper
    assert all(s.body(k)["force"][2] > 0 for k in range(2))
    s.close()


def test_stacked_bodies_rest_on_the_floor_with_contact():
    """Empty tank, two cubes dropped one above the other, contact on: the
    lower cube lands on the floor, the upper one on the lower, and both come
    to rest; the trajectories follow the FP64 oracle and the resting heights
    are those of the springs' static penetration (the lower contact carries
    both weights)."""
    dx = 0.04
    c = cases.floating_bodies(dx, tank=(0.6, 0.6, 0.6), depth=0.0,
                              cubes=[dict(x=0.3, size=0.2, rho=500.0, bottom=0.08),
                                     dict(x=0.3, size=0.2, rho=500.0, bottom=0.36)], end_step=10)
    kn, cn = _contact_for(c.bodies[0], dx, 25)
    o = po.Oracle(c.json, c.state, dtype=np.float64)
    o.attach_bodies(c.bodies, contact=(kn, cn, dx))
    s = z.Solver.from_case(c)
    for b in c.bodies:
        s.attach_body(b["first"], b["count"], b["mass"])
    s.set_contact(kn, cn, dx)
    diff = 0.0
    for _ in range(20):
        o.step_bodies(100)
        s.run(100)
        for k in range(2):
            diff = max(diff, abs(s.body(k)["pos"][2] - o.rigid_state(k)["x"][2]))
    lo, hi = s.body(0), s.body(1)
    print("resting", lo["pos"], hi["pos"], "max |gpu - oracle| heave", diff)
    sag = dx * 0.05
    want_lo = -dx / 2 + dx - 2 * sag + (0.2 - dx) / 2  # the floor contact carries both cubes
    want_hi = want_lo + 0.2 - sag                        # one cube's weight on the contact between them
    assert abs(lo["pos"][2] - want_lo) < 0.1 * dx and abs(hi["pos"][2] - want_hi) < 0.1 * dx
    assert np.linalg.norm(lo["vel"]) < 0.02 and np.linalg.norm(hi["vel"]) < 0.02
    assert diff < 2e-3
    s.close()


def test_body_api_rejects_overlap_and_bad_contact():
    dx = 0.04
    c = cases.floating_bodies(dx, tank=(0.6, 0.6, 0.6), depth=0.0,
                              cubes=[dict(x=0.3, size=0.2, rho=500.0, bottom=0.1)], end_step=10)
    s = z.Solver.from_case(c)
    b = c.bodies[0]
    with pytest.raises(z.ZsphError):
        s.set_contact(1.0, 0.0, dx)  # no body yet
    s.attach_body(b["first"], b["count"], b["mass"])
    with pytest.raises(z.ZsphError):
        s.attach_body(b["first"] + 3, 10, 1.0)  # overlaps the first body
    with pytest.raises(z.ZsphError):
        s.set_contact(1.0, 0.0, 3 * dx)  # beyond the 2h support
    s.attach_body(b["first"], b["count"], 2 * b["mass"])  # same first index: replaces
    assert s.body_count() == 1 and s.body(0)["mass"] == 2 * b["mass"]
    s.close()


def test_overflowed_lists_in_the_precision_form():
    # a block of fluid compressed to 0.7 of its spacing: its particles have
    # more than 128 neighbours within 2h, so the pair walks re-filter their
    # stencil rows (with the candidates moved into the particle's cell frame
    # in the precision form); both forms must then agree to FP32 rounding
    dx = 0.04
    c = cases.dam_break(dx, end_step=20)
    pos = c.state.pos
    fl = c.state.type == 1
    ctr = np.median(pos[fl], axis=0).astype(np.float32)
    box = fl & np.all(np.abs(pos - ctr) < 3.5 * dx, axis=1)
    pos[box] = (ctr + np.float32(0.7) * (pos[box] - ctr)).astype(np.float32)
    c.state.tmp_pos[:] = pos
    c = dataclasses.replace(c, pos64=pos.astype(np.float64))
    got = {}
    for precise in (False, True):
        s = _solver(c, precise)
        s.run(2)
        f = s.status()
        assert f & z.FLAG_NB_OVERFLOW and not f & z.FLAG_NAN
        st = s.download("old")
        got[precise] = _by_id(st, c.n, st.vel.astype(np.float64))
        s.close()
    dv = np.abs(got[True] - got[False]).max()
    scale = np.abs(got[False]).max()
    assert dv < 1e-3 * scale, f"max |dv| {dv:.3e} of {scale:.3e}"
