"""Synthetic case generator: 3-D dam break in the reference's JSON schema and
particle layout.

The reference ships no input cases (its driver reads input/input.json and
input/input.vtk, single_gpu_sph_src/deltasph/main.cu:13,17); these cases are
seeded-free, lattice-built stand-ins with the shapes of the workloads the
solver is measured on:

* water column wx x wy x wz at the x = 0 end of a tank lx x wy x lz, fluid on
  the cubic lattice ((i+1/2)dx, (j+1/2)dx, (k+1/2)dx), type 1, zero velocity;
* ``layers`` layers of dummy wall particles (type 0) outside the tank's floor
  and four sides, up to the tank top (open top);
* hydrostatic initial pressure p = rho0*|g|*(H - z) with the reference's
  linear equation of state rho = rho0 + p/c0^2 (time_int.cu:39-40), for
  walls below the water level too (p = 0, rho = rho0 above it);
* dt = cfl * h / c0.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import JsonCase, State


@dataclass
class Case:
    json: JsonCase
    state: State
    n_fluid: int
    n_wall: int
    name: str
    pos64: np.ndarray | None = None  # exact (FP64) positions, for the precision form
    body: dict | None = None         # rigid body: first, count, mass (floating-body case)
    bodies: list | None = None       # every rigid body of the case (floating_bodies)

    @property
    def n(self) -> int:
        return self.state.n


def _json(dx, xmax, ymax, zmax, dt, n, nf, nw, end_step, g=-9.81, rho0=1000.0, h_factor=1.3, r_factor=2.0,
          eta_factor=0.1, cs_factor=10.0, delta=0.1, alpha=0.02, grid_layer_factor=2.0, grid_size_factor=1.0):
    j = JsonCase()
    j.g, j.rho0, j.dx = g, rho0, dx
    j.h_factor, j.r_factor, j.eta_factor, j.cs_factor = h_factor, r_factor, eta_factor, cs_factor
    j.delta, j.alpha = delta, alpha
    j.xmin, j.xmax, j.ymin, j.ymax, j.zmin, j.zmax = 0.0, xmax, 0.0, ymax, 0.0, zmax
    j.grid_layer_factor, j.grid_size_factor = grid_layer_factor, grid_size_factor
    j.dt = dt
    j.start_step, j.current_step, j.end_step, j.output_step = 0, 0, end_step, max(end_step, 1)
    j.ptc_num, j.water_ptc_num, j.air_ptc_num, j.wall_ptc_num, j.rigid_ptc_num = n, nf, 0, nw, 0
    j.thread_num, j.gpu_id = 1, 0
    j.input_path, j.output_path, j.git_hash = b"input", b"output", b"zsph-b200"
    return j


def dam_break(dx: float = 0.02, water=(0.6, 0.6, 1.2), tank=(1.6, 0.6, 1.2), layers: int = 3, cfl: float = 0.2,
              end_step: int = 2000, order: str = "fluid_first", **phys) -> Case:
    """Dam break of the measured workloads: dx = 0.02 gives 54,000 fluid +
    51,048 wall particles, dx = 0.005 gives 3,456,000 + 765,468."""
    g = phys.get("g", -9.81)
    rho0 = phys.get("rho0", 1000.0)
    cs_factor = phys.get("cs_factor", 10.0)
    h_factor = phys.get("h_factor", 1.3)
    lx, ly, lz = tank
    wx, wy, wz = water
    nx, ny, nz = (int(round(v / dx)) for v in (wx, wy, wz))
    tx, ty, tz = (int(round(v / dx)) for v in (lx, ly, lz))
    # fluid lattice
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    fl = np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1)
    # wall lattice: the extended box minus the tank interior, up to the tank top
    ii, jj, kk = np.meshgrid(np.arange(-layers, tx + layers), np.arange(-layers, ty + layers),
                             np.arange(-layers, tz), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    outside = (ii < 0) | (ii >= tx) | (jj < 0) | (jj >= ty) | (kk < 0)
    wl = np.stack([ii[outside], jj[outside], kk[outside]], axis=1)
    pos_f = ((fl.astype(np.float64) + 0.5) * dx)
    pos_w = ((wl.astype(np.float64) + 0.5) * dx)
    c0 = cs_factor * math.sqrt(abs(g) * lz)
    H = nz * dx

    def hydro(z):
        p = rho0 * abs(g) * np.clip(H - z, 0.0, None)
        return rho0 + p / (c0 * c0), p

    rf, pf = hydro(pos_f[:, 2])
    rw, pw = hydro(pos_w[:, 2])
    if order == "fluid_first":
        parts = [(pos_f, rf, pf, 1), (pos_w, rw, pw, 0)]
    else:
        parts = [(pos_w, rw, pw, 0), (pos_f, rf, pf, 1)]
    pos = np.concatenate([p[0] for p in parts]).astype(np.float32)
    rho = np.concatenate([p[1] for p in parts]).astype(np.float32)
    prs = np.concatenate([p[2] for p in parts]).astype(np.float32)
    typ = np.concatenate([np.full(len(p[0]), p[3], np.int32) for p in parts])
    n = len(typ)
    st = State(pos=pos, vel=np.zeros((n, 3), np.float32), rhop=np.stack([rho, prs], axis=1).astype(np.float32),
               type=typ, table=np.zeros(n, np.int32), tmp_pos=np.zeros((n, 3), np.float32),
               tmp_vel=np.zeros((n, 3), np.float32), tmp_rhop=np.zeros((n, 2), np.float32))
    h = h_factor * dx
    dt = cfl * h / c0
    js = _json(dx, lx, ly, lz, dt, n, len(pos_f), len(pos_w), end_step, **phys)
    return Case(js, st, len(pos_f), len(pos_w), f"dam_break_dx{dx:g}")


def floating_body(dx: float = 0.01, tank=(4.0, 1.0, 1.0), depth: float = 0.5, cube: float = 0.2,
                  body_rho: float = 500.0, drop: float = 0.05, cube_x: float = 1.0, layers: int = 3,
                  cfl: float = 0.2, end_step: int = 5000, **phys) -> Case:
    """Still water of the given depth in a tank, walls as in dam_break, and a
    cube of side `cube` (type 2 particles on the same lattice) centred at
    (cube_x, tank_y/2) with its bottom `drop` above the surface.  dx = 0.01
    gives 2,000,000 fluid, 432,708 wall and 8,000 body particles.  Order:
    fluid, walls, body; case.body = {first, count, mass}."""
    c = floating_bodies(dx, tank, depth, [dict(x=cube_x, size=cube, rho=body_rho, bottom=depth + drop)],
                        layers, cfl, end_step, **phys)
    c.name = f"floating_body_dx{dx:g}"
    return c


def floating_bodies(dx: float, tank=(4.0, 1.0, 1.0), depth: float = 0.5, cubes=(), layers: int = 3,
                    cfl: float = 0.2, end_step: int = 5000, **phys) -> Case:
    """Still water of the given depth (0: an empty tank) and several cubes of
    type 2 particles on the fluid's lattice.  Each cube is a dict with its
    centre x (and optionally y, default the tank's middle), side `size`,
    density `rho` and the height of its bottom face `bottom`.  Order: fluid,
    walls, then the cubes one after another; case.bodies lists each cube's
    {first, count, mass} and case.body is the first one."""
    g = phys.get("g", -9.81)
    rho0 = phys.get("rho0", 1000.0)
    cs_factor = phys.get("cs_factor", 10.0)
    h_factor = phys.get("h_factor", 1.3)
    lx, ly, lz = tank
    nx, ny, nz = (int(round(v / dx)) for v in (lx, ly, depth))
    tx, ty, tz = (int(round(v / dx)) for v in (lx, ly, lz))
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    pos_f = (np.stack([i.ravel(), j.ravel(), k.ravel()], axis=1).astype(np.float64) + 0.5) * dx
    ii, jj, kk = np.meshgrid(np.arange(-layers, tx + layers), np.arange(-layers, ty + layers),
                             np.arange(-layers, tz), indexing="ij")
    ii, jj, kk = ii.ravel(), jj.ravel(), kk.ravel()
    outside = (ii < 0) | (ii >= tx) | (jj < 0) | (jj >= ty) | (kk < 0)
    pos_w = (np.stack([ii[outside], jj[outside], kk[outside]], axis=1).astype(np.float64) + 0.5) * dx
    blocks, bodies = [], []
    first = len(pos_f) + len(pos_w)
    for cb in cubes:
        side = cb["size"]
        nc = int(round(side / dx))
        a, b, c = np.meshgrid(np.arange(nc), np.arange(nc), np.arange(nc), indexing="ij")
        corner = np.array([cb["x"] - side / 2, cb.get("y", ly / 2) - side / 2, cb["bottom"]])
        blocks.append(corner + (np.stack([a.ravel(), b.ravel(), c.ravel()], axis=1).astype(np.float64) + 0.5) * dx)
        bodies.append({"first": first, "count": nc ** 3, "mass": cb["rho"] * side ** 3})
        first += nc ** 3
    pos_b = np.concatenate(blocks) if blocks else np.zeros((0, 3))
    c0 = cs_factor * math.sqrt(abs(g) * lz)
    H = nz * dx

    def hydro(z):
        p = rho0 * abs(g) * np.clip(H - z, 0.0, None)
        return rho0 + p / (c0 * c0), p

    rf, pf = hydro(pos_f[:, 2])
    rw, pw = hydro(pos_w[:, 2])
    rb, pb = np.full(len(pos_b), rho0), np.zeros(len(pos_b))
    pos64 = np.concatenate([pos_f, pos_w, pos_b])
    rho = np.concatenate([rf, rw, rb]).astype(np.float32)
    prs = np.concatenate([pf, pw, pb]).astype(np.float32)
    typ = np.concatenate([np.ones(len(pos_f), np.int32), np.zeros(len(pos_w), np.int32),
                          np.full(len(pos_b), 2, np.int32)])
    n = len(typ)
    st = State(pos=pos64.astype(np.float32), vel=np.zeros((n, 3), np.float32),
               rhop=np.stack([rho, prs], axis=1).astype(np.float32), type=typ, table=np.zeros(n, np.int32),
               tmp_pos=np.zeros((n, 3), np.float32), tmp_vel=np.zeros((n, 3), np.float32),
               tmp_rhop=np.zeros((n, 2), np.float32))
    h = h_factor * dx
    dt = cfl * h / c0
    js = _json(dx, lx, ly, lz, dt, n, len(pos_f), len(pos_w), end_step, **phys)
    js.rigid_ptc_num = len(pos_b)
    c = Case(js, st, len(pos_f), len(pos_w), f"floating_bodies_dx{dx:g}", pos64=pos64,
             body=bodies[0] if bodies else None)
    c.bodies = bodies
    return c


def config2() -> Case:
    """Floating body at dx = 0.01 m: 2,000,000 fluid + 432,708 wall + 8,000 body particles, 5000 steps."""
    return floating_body(0.01)


def batch_scenes(nscenes: int = 256, seed: int = 2026, fluid_range=(5000, 60000), max_tries: int = 1_000_000):
    """Seeded dam-break scenes of uneven sizes: column width w ~ U[0.2, 0.6] m,
    aspect a = height / width ~ U[0.5, 2], dx ~ U[0.01, 0.02] m, column depth
    = w, height a w; a draw is kept when the height lies in [0.2, 0.6] m and
    the fluid count in fluid_range.  Tank 2.5 w x w x 1.2 a w, same physics
    and walls as dam_break.  Returns (cases, draws)."""
    rng = np.random.default_rng(seed)
    out, draws = [], []
    tries = 0
    while len(out) < nscenes and tries < max_tries:
        tries += 1
        w, a, dx = rng.uniform(0.2, 0.6), rng.uniform(0.5, 2.0), rng.uniform(0.01, 0.02)
        hgt = a * w
        if not (0.2 <= hgt <= 0.6):
            continue
        n = round(w / dx) * round(w / dx) * round(hgt / dx)
        if not (fluid_range[0] <= n <= fluid_range[1]):
            continue
        c = dam_break(dx, water=(w, w, hgt), tank=(2.5 * w, w, 1.2 * hgt), end_step=1000)
        if not (fluid_range[0] <= c.n_fluid <= fluid_range[1]):
            continue
        out.append(c)
        draws.append({"w": w, "aspect": a, "dx": dx})
    if len(out) < nscenes:
        raise ValueError("not enough scenes within the ranges")
    return out, draws


def config0() -> Case:
    """Plain dam break, dx = 0.02 m: 54,000 fluid + 51,048 wall particles, 2000 steps."""
    return dam_break(0.02, end_step=2000)


def config1() -> Case:
    """Dam break at scale, dx = 0.005 m: 3,456,000 fluid + 765,468 wall particles, 500 steps."""
    return dam_break(0.005, end_step=500)


def small(dx: float = 0.04) -> Case:
    """A small dam break of the same geometry for fast parity tests."""
    return dam_break(dx, end_step=100)


def random_cloud(n: int, seed: int, dx: float = 0.02, box=(0.4, 0.3, 0.3), kill_frac: float = 0.0) -> Case:
    """Seeded random particle cloud in a closed box (every particle type 1
    except a wall shell fraction), for hash / sort / neighbour edge cases.
    With kill_frac > 0 some particles are placed outside the grid."""
    rng = np.random.default_rng(seed)
    lx, ly, lz = box
    pos = rng.uniform([0, 0, 0], [lx, ly, lz], size=(n, 3)).astype(np.float32)
    typ = (rng.uniform(size=n) < 0.8).astype(np.int32)
    if kill_frac > 0:
        m = rng.uniform(size=n) < kill_frac
        pos[m] = (pos[m] + np.float32(10.0)).astype(np.float32)
    rho = (1000.0 + rng.uniform(0, 5, size=n)).astype(np.float32)
    prs = ((rho - 1000.0) * 34.310349 ** 2).astype(np.float32)
    vel = rng.normal(0, 0.1, size=(n, 3)).astype(np.float32)
    st = State(pos=pos, vel=vel, rhop=np.stack([rho, prs], 1).astype(np.float32), type=typ,
               table=np.zeros(n, np.int32), tmp_pos=pos.copy(), tmp_vel=vel.copy(),
               tmp_rhop=np.stack([rho, prs], 1).astype(np.float32))
    c0 = 10.0 * math.sqrt(9.81 * lz)
    dt = 0.2 * 1.3 * dx / c0
    js = _json(dx, lx, ly, lz, dt, n, int(typ.sum()), int(n - typ.sum()), 10)
    return Case(js, st, int(typ.sum()), int(n - typ.sum()), f"cloud_{n}_{seed}")
