"""The rigid-body oracle on known answers: free fall under gravity is exact
for the predictor-corrector (constant acceleration), a torque-free cube
keeps its angular velocity and turns by |w| t, and the floating-body case
has the stated particle counts."""
import numpy as np

from oracle import pyoracle as po
from zsph_b200 import cases


def test_floating_body_case_counts():
    c = cases.floating_body(0.04, end_step=10)
    nf = int(round(4.0 / 0.04)) * int(round(1.0 / 0.04)) * int(round(0.5 / 0.04))
    assert c.n_fluid == nf and c.body["count"] == 5 ** 3
    assert c.body["first"] == c.n_fluid + c.n_wall
    assert np.all(c.state.type[c.body["first"]:] == 2)
    assert abs(c.body["mass"] - 4.0) < 1e-12
    # cube bottom 0.05 m above the 0.5 m surface
    zb = c.pos64[c.body["first"]:, 2]
    assert abs(zb.min() - 0.04 / 2 - 0.55) < 1e-12


def test_free_fall_is_exact():
    c = cases.floating_body(0.04, end_step=10)
    o = po.Oracle(c.json, c.state, dtype=np.float64)
    o.attach_rigid(c.body["first"], c.body["count"], c.body["mass"], vel=(0.1, 0, 0.2))
    x0 = o.rigid_state()["x"].copy()
    n = 20
    o.step_rigid(n)
    t = n * 2 * o.p.half_dt
    r = o.rigid_state()
    assert np.allclose(r["F"], 0.0)  # still in the air
    want = x0 + np.array([0.1, 0.0, 0.2]) * t + np.array([0, 0, 0.5 * o.p.g]) * t * t
    assert np.allclose(r["x"], want, rtol=0, atol=1e-12)
    assert np.allclose(r["v"], [0.1, 0.0, 0.2 + o.p.g * t], rtol=0, atol=1e-12)


def test_torque_free_cube_spins_uniformly():
    c = cases.floating_body(0.04, end_step=10)
    o = po.Oracle(c.json, c.state, dtype=np.float64)
    w = np.array([0.0, 0.0, 2.0])
    o.attach_rigid(c.body["first"], c.body["count"], c.body["mass"], omega=w)
    n = 30
    o.step_rigid(n)
    t = n * 2 * o.p.half_dt
    r = o.rigid_state()
    assert np.allclose(r["w"], w, atol=1e-12)  # isotropic inertia: no gyroscopic term
    angle = 2 * np.arctan2(np.linalg.norm(r["q"][1:]), r["q"][0])
    assert abs(angle - np.linalg.norm(w) * t) < 1e-6


def _contact_for(body, dx, n_bottom, sag=0.05, zeta=0.5, g=9.81):
    """Spring-dashpot constants: the body's weight carried by n_bottom pairs at
    a static penetration of sag * dx, damped at zeta of critical."""
    kn = body["mass"] * g / (n_bottom * sag * dx)
    cn = zeta * 2.0 * np.sqrt(kn * n_bottom * body["mass"]) / n_bottom
    return kn, cn


def test_cube_settles_on_the_floor_with_contact():
    """Empty tank, one cube dropped 0.1 m: with contact it comes to rest on
    the floor at the spring's static penetration (each of the 25 bottom
    particles carries 1/25 of the weight against the wall particle right
    below it); without contact it falls through."""
    dx = 0.04
    c = cases.floating_bodies(dx, tank=(0.6, 0.6, 0.6), depth=0.0,
                              cubes=[dict(x=0.3, size=0.2, rho=500.0, bottom=0.1)], end_step=10)
    b = c.bodies[0]
    kn, cn = _contact_for(b, dx, 25)
    o = po.Oracle(c.json, c.state, dtype=np.float64)
    o.attach_bodies([b], contact=(kn, cn, dx))
    o.step_bodies(1500)
    r = o.rigid_state(0)
    # bottom particles at z = -dx/2 + dx - sag*dx, centre (0.2 - dx)/2 above them
    want = -dx / 2 + dx * (1 - 0.05) + (0.2 - dx) / 2
    print("resting centre", r["x"], "expected z", want, "v", r["v"])
    assert abs(r["x"][2] - want) < 0.1 * dx
    assert np.linalg.norm(r["v"]) < 0.02
    assert abs(r["F"][2] - b["mass"] * 9.81) < 0.05 * b["mass"] * 9.81  # the floor carries the weight
    o2 = po.Oracle(c.json, c.state, dtype=np.float64)
    o2.attach_bodies([b])
    o2.step_bodies(700)
    assert o2.rigid_state(0)["x"][2] < 0.0  # no contact: through the floor
