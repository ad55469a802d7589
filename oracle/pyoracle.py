"""ctypes wrapper over the CPU oracle (liboracle.so) and the reference-build
checker (_ref/libzsph_ref.so).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the product package.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libzsph_ref.so")
REF_SIMPLE_SO = os.path.join(HERE, "_ref", "libzsph_ref_simple.so")

WALLS_FIRST, WALLS_OLD, WALLS_SPLIT = 0, 1, 2
_F, _I, _VP = ctypes.c_float, ctypes.c_int, ctypes.c_void_p


class OCase(ctypes.Structure):
    _fields_ = [(n, _F) for n in ("g", "rho0", "dx", "h_factor", "r_factor", "eta_factor", "cs_factor", "delta",
                                  "alpha", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax", "grid_layer_factor",
                                  "grid_size_factor", "dt")] + [("ptc_num", _I)]


class OParams(ctypes.Structure):
    _fields_ = [(n, _F) for n in ("half_dt", "h", "g", "m", "rho0", "adh", "h2", "eta2", "cs2", "alpha",
                                  "delta_h_cs", "h_cs_rho_m", "grid_size")] + \
               [("grid_factor", _I)] + [(n, _F) for n in ("grid_xmin", "grid_ymin", "grid_zmin")] + \
               [(n, _I) for n in ("grid_xdim", "grid_ydim", "grid_zdim", "grid_hash_min", "grid_hash_max",
                                  "ptc_num", "grid_num")] + \
               [(n, _F) for n in ("dt", "dt_max", "cs", "eta", "r")]


class OState(ctypes.Structure):
    _fields_ = [(n, _VP) for n in ("pos", "vel", "rhop", "tmp_pos", "tmp_vel", "tmp_rhop", "type", "table")]


class OTmp(ctypes.Structure):
    _fields_ = [(n, _VP) for n in ("acc_drhodt", "dofv_grandrho", "index", "hash", "grid_start", "grid_end")]


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        _lib = ctypes.CDLL(ORACLE_SO)
        _lib.oracle_params.argtypes = [ctypes.POINTER(OCase), ctypes.POINTER(OParams)]
        _lib.oracle_params.restype = _I
        _lib.oracle_sizeof_params.restype = _I
        _lib.oracle_set_threads.argtypes = [_I]
        _lib.oracle_max_threads.restype = _I
        assert _lib.oracle_sizeof_params() == ctypes.sizeof(OParams), "oracle Params layout mismatch"
    return _lib


def case_of(json) -> OCase:
    """OCase from a zsph_b200.JsonCase (or any object with the same fields)."""
    c = OCase()
    for name, _ in OCase._fields_:
        setattr(c, name, getattr(json, name))
    return c


def params(json) -> tuple[int, OParams]:
    p = OParams()
    rc = lib().oracle_params(ctypes.byref(case_of(json)), ctypes.byref(p))
    return rc, p


def _p(a):
    return None if a is None else a.ctypes.data_as(_VP)


class ORigid(ctypes.Structure):
    """zsph_oracle::Rigid."""
    _fields_ = [(n, ctypes.c_double * k) for n, k in (("x", 3), ("v", 3), ("w", 3), ("q", 4), ("xn", 3), ("vn", 3),
                                                       ("wn", 3), ("qn", 4), ("F", 3), ("T", 3), ("I", 9),
                                                       ("Iinv", 9))] + \
               [("M", ctypes.c_double), ("g", ctypes.c_double), ("first", ctypes.c_int), ("count", ctypes.c_int),
                ("r0", ctypes.POINTER(ctypes.c_double))]


class OContact(ctypes.Structure):
    """zsph_oracle::Contact."""
    _fields_ = [("kn", ctypes.c_double), ("cn", ctypes.c_double), ("dist", ctypes.c_double)]


class Oracle:
    """One oracle run (FP32 or FP64) on host arrays in the reference layout."""

    def __init__(self, json, state, dtype=np.float32):
        self.dtype = np.dtype(dtype)
        self.suf = "f32" if self.dtype == np.float32 else "f64"
        rc, self.p = params(json)
        if rc != 0:
            raise ValueError("dt > dt_max")
        n, G = self.p.ptc_num, self.p.grid_num
        # always a private copy: the oracle steps in place, and a caller's
        # float32 arrays would otherwise be shared with (and mutated by) it
        cv = lambda a, shape: (np.zeros(shape, self.dtype) if a is None else np.array(a, self.dtype, order="C"))
        self.old = dict(pos=cv(state.pos, (n, 3)), vel=cv(state.vel, (n, 3)), rhop=cv(state.rhop, (n, 2)),
                        tmp_pos=cv(state.tmp_pos, (n, 3)), tmp_vel=cv(state.tmp_vel, (n, 3)),
                        tmp_rhop=cv(state.tmp_rhop, (n, 2)),
                        type=np.ascontiguousarray(state.type, np.int32).copy(),
                        table=np.ascontiguousarray(state.table, np.int32).copy())
        self.new = {k: np.zeros_like(v) for k, v in self.old.items()}
        self.tmp = dict(acc_drhodt=np.zeros((n, 4), self.dtype), dofv_grandrho=np.zeros((n, 4), self.dtype),
                        index=np.zeros(n, np.int32), hash=np.zeros(n, np.int32),
                        grid_start=np.zeros(G, np.int32), grid_end=np.zeros(G, np.int32))
        self._mk()

    def _mk(self):
        self._so = OState(*[_p(self.old[k]) for k, _ in OState._fields_])
        self._sn = OState(*[_p(self.new[k]) for k, _ in OState._fields_])
        self._t = OTmp(*[_p(self.tmp[k]) for k, _ in OTmp._fields_])

    def _s(self, which):
        return self._so if which == "old" else self._sn

    def _fn(self, name):
        f = getattr(lib(), f"oracle_{name}_{self.suf}")
        f.restype = None
        return f

    def hash(self, which="old"):
        self._fn("hash")(ctypes.byref(self.p), ctypes.byref(self._s(which)), ctypes.byref(self._t))

    def sort_index(self):
        self._fn("sort_index")(ctypes.byref(self.p), ctypes.byref(self._t))

    def sort_data(self, src="old", dst="new"):
        self._fn("sort_data")(ctypes.byref(self.p), ctypes.byref(self._s(src)), ctypes.byref(self._s(dst)),
                              ctypes.byref(self._t))

    def search(self, src="old", dst="new"):
        self.hash(src)
        self.sort_index()
        self.sort_data(src, dst)

    def boundary(self, which="new", wall_mode=WALLS_FIRST):
        self._fn("boundary")(ctypes.byref(self.p), ctypes.byref(self._s(which)), ctypes.byref(self._t),
                             _I(wall_mode))

    def governing(self, which="new"):
        self._fn("governing")(ctypes.byref(self.p), ctypes.byref(self._s(which)), ctypes.byref(self._t))

    def prediction(self, which="new"):
        self._fn("prediction")(ctypes.byref(self.p), ctypes.byref(self._s(which)), ctypes.byref(self._t))

    def correction(self, which="old"):
        self._fn("correction")(ctypes.byref(self.p), ctypes.byref(self._s(which)), ctypes.byref(self._t))

    def step(self, nsteps=1, wall_mode=WALLS_FIRST):
        self._fn("step")(ctypes.byref(self.p), ctypes.byref(self._so), ctypes.byref(self._sn),
                         ctypes.byref(self._t), _I(nsteps), _I(wall_mode))

    def features(self, scale, which="new", acc_prev=None) -> np.ndarray:
        """Learned-corrector inputs of `which` (after search, boundary and
        governing); acc_prev: previous corrector-stage (acc, drho/dt) in the
        order before the search (None: those four features are zero)."""
        out = np.zeros((self.p.ptc_num, 32), self.dtype)
        sc = np.ascontiguousarray(scale, np.float32)
        ap = None if acc_prev is None else np.ascontiguousarray(acc_prev, self.dtype)
        self._fn("features")(ctypes.byref(self.p), ctypes.byref(self._s(which)), ctypes.byref(self._t),
                             _p(sc), _p(ap), _p(out))
        return out

    # ---- rigid body (the product's FP64 6DOF coupling, restated) ----------
    def attach_rigid(self, first, count, mass, vel=(0, 0, 0), omega=(0, 0, 0), q=(1, 0, 0, 0)):
        """Centroid, inertia (Test_6DOF/equation/rigid_info.cpp:3-39) and
        body-frame offsets from the current positions of `old`."""
        b, self._r0 = rigid_from(self.p, self.old, first, count, mass, vel, omega, q)
        self.rigid = b
        f = self._fn("rigid_place")
        f(ctypes.byref(self.p), ctypes.byref(self._so), ctypes.byref(self.rigid))
        return b

    def step_rigid(self, nsteps=1, wall_mode=WALLS_FIRST):
        self._fn("step_rigid")(ctypes.byref(self.p), ctypes.byref(self._so), ctypes.byref(self._sn),
                               ctypes.byref(self._t), ctypes.byref(self.rigid), _I(nsteps), _I(wall_mode))

    def rigid_state(self, body: int = 0) -> dict:
        b = self.rigid if body == 0 and not hasattr(self, "_bodies") else self._bodies[body]
        return {k: np.array(getattr(b, k)[:]) for k in ("x", "v", "w", "q", "F", "T")}

    def attach_bodies(self, bodies, contact=(0.0, 0.0, 0.0)):
        """Several bodies (each a dict with first, count, mass and optionally
        vel, omega, q) and the wall/body contact (kn N/m, cn N s/m, distance m;
        kn = 0: off), for step_bodies."""
        n = len(bodies)
        self._bodies = (ORigid * n)()
        self._r0s = []
        for k, bd in enumerate(bodies):
            b, r0 = rigid_from(self.p, self.old, bd["first"], bd["count"], bd["mass"], bd.get("vel", (0, 0, 0)),
                               bd.get("omega", (0, 0, 0)), bd.get("q", (1, 0, 0, 0)))
            self._r0s.append(r0)
            self._bodies[k] = b
            self._bodies[k].r0 = r0.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            self._fn("rigid_place")(ctypes.byref(self.p), ctypes.byref(self._so), ctypes.byref(self._bodies[k]))
        self._contact = OContact(*[float(v) for v in contact])
        return self._bodies

    def step_bodies(self, nsteps=1, wall_mode=WALLS_FIRST):
        self._fn("step_rigid_bodies")(ctypes.byref(self.p), ctypes.byref(self._so), ctypes.byref(self._sn),
                                      ctypes.byref(self._t), self._bodies, _I(len(self._bodies)),
                                      ctypes.byref(self._contact), _I(nsteps), _I(wall_mode))

    # simple-SPH equations (the reference's simplesph target); div(v) is the
    # scalar array self.dofv
    def _dofv(self):
        if not hasattr(self, "dofv"):
            self.dofv = np.zeros(self.p.ptc_num, self.dtype)
        return self.dofv

    def boundary_simple(self, which="new"):
        self._fn("boundary_simple")(ctypes.byref(self.p), ctypes.byref(self._s(which)), ctypes.byref(self._t),
                                    _p(self._dofv()))

    def governing_simple(self, which="new"):
        self._fn("governing_simple")(ctypes.byref(self.p), ctypes.byref(self._s(which)), ctypes.byref(self._t),
                                     _p(self._dofv()))

    def step_simple(self, nsteps=1):
        self._fn("step_simple")(ctypes.byref(self.p), ctypes.byref(self._so), ctypes.byref(self._sn),
                                ctypes.byref(self._t), _p(self._dofv()), _I(nsteps))

    def neighbor_count(self, which="new", stencil="governing") -> np.ndarray:
        out = np.zeros(self.p.ptc_num, np.int32)
        ylast = self.p.grid_factor if stencil == "governing" else self.p.grid_factor - 1
        self._fn("neighbor_count")(ctypes.byref(self.p), ctypes.byref(self._s(which)), ctypes.byref(self._t),
                                   _I(ylast), _p(out))
        return out


def rigid_from(p, st, first, count, mass, vel=(0, 0, 0), omega=(0, 0, 0), q=(1, 0, 0, 0)):
    """The oracle's body (ORigid) and its body-frame offsets r0[count][3] from
    the positions of the state dict st: centroid, inertia about it
    (Test_6DOF/equation/rigid_info.cpp:3-39) and the pose q."""
    ids = st["table"] + np.arange(p.ptc_num)
    sel = (st["type"] == 2) & (ids >= first) & (ids < first + count)
    x = np.zeros((count, 3))
    x[ids[sel] - first] = st["pos"][sel].astype(np.float64)
    c = x.mean(0)
    r = x - c
    I = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            I[a, b] = -(r[:, a] * r[:, b]).sum()
    I += np.eye(3) * (r * r).sum()
    I *= mass / count
    qq = np.asarray(q, np.float64) / np.linalg.norm(q)
    w, xx, yy, zz = qq
    R = np.array([[1 - 2 * (yy * yy + zz * zz), 2 * (xx * yy - w * zz), 2 * (xx * zz + w * yy)],
                  [2 * (xx * yy + w * zz), 1 - 2 * (xx * xx + zz * zz), 2 * (yy * zz - w * xx)],
                  [2 * (xx * zz - w * yy), 2 * (yy * zz + w * xx), 1 - 2 * (xx * xx + yy * yy)]])
    r0 = np.ascontiguousarray(r @ R)  # R^T r per row
    Ib = R.T @ I @ R
    b = ORigid()
    for name, v in (("x", c), ("xn", c), ("v", vel), ("vn", vel), ("w", omega), ("wn", omega), ("q", qq),
                    ("qn", qq), ("I", Ib.ravel()), ("Iinv", np.linalg.inv(Ib).ravel())):
        getattr(b, name)[:] = list(np.asarray(v, np.float64))
    b.M, b.g, b.first, b.count = mass, p.g, first, count
    b.r0 = r0.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return b, r0


GPU_ORACLE_SO = os.path.join(HERE, "libgpu_oracle.so")
_gpu = None


def gpu_lib() -> ctypes.CDLL:
    global _gpu
    if _gpu is None:
        _gpu = ctypes.CDLL(GPU_ORACLE_SO)
        _gpu.gor_create.restype = _VP
        _gpu.gor_create.argtypes = [ctypes.POINTER(OParams)] + [_VP] * 8
        _gpu.gor_error.restype = ctypes.c_char_p
        _gpu.gor_error.argtypes = [_VP]
        for f in ("gor_attach_rigid", "gor_step", "gor_download"):
            getattr(_gpu, f).restype = _I
        _gpu.gor_attach_rigid.argtypes = [_VP, ctypes.POINTER(ORigid)]
        _gpu.gor_step.argtypes = [_VP, _I]
        _gpu.gor_download.argtypes = [_VP] * 6
        _gpu.gor_rigid.argtypes = [_VP, ctypes.POINTER(ORigid)]
        _gpu.gor_destroy.argtypes = [_VP]
    return _gpu


class GpuOracle64:
    """The FP64 oracle run on the GPU (oracle/gpu_oracle.cu, test
    infrastructure): the T = double instance of the same restatement with the
    same arithmetic and visit order, for cases too large for the CPU oracle.
    Steps use the WALLS_FIRST order; with a body attached, every step is the
    oracle's step_rigid."""

    def __init__(self, json, state):
        rc, self.p = params(json)
        if rc != 0:
            raise ValueError("dt > dt_max")
        n = self.p.ptc_num
        cv = lambda a, shape: (np.zeros(shape) if a is None else np.ascontiguousarray(a, np.float64))
        self._host = dict(pos=cv(state.pos, (n, 3)), vel=cv(state.vel, (n, 3)), rhop=cv(state.rhop, (n, 2)),
                          tmp_pos=cv(state.tmp_pos, (n, 3)), tmp_vel=cv(state.tmp_vel, (n, 3)),
                          tmp_rhop=cv(state.tmp_rhop, (n, 2)),
                          type=np.ascontiguousarray(state.type, np.int32), table=np.ascontiguousarray(state.table, np.int32))
        L = gpu_lib()
        h = self._host
        self.h = L.gor_create(ctypes.byref(self.p), *[_p(h[k]) for k in ("pos", "vel", "rhop", "tmp_pos", "tmp_vel",
                                                                          "tmp_rhop", "type", "table")])
        if not self.h:
            raise RuntimeError("gor_create failed")
        self.rigid = None

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(gpu_lib().gor_error(self.h).decode())

    def attach_rigid(self, first, count, mass, vel=(0, 0, 0), omega=(0, 0, 0), q=(1, 0, 0, 0)):
        b, self._r0 = rigid_from(self.p, self._host, first, count, mass, vel, omega, q)
        self._check(gpu_lib().gor_attach_rigid(self.h, ctypes.byref(b)))
        self.rigid = b
        return b

    def step(self, nsteps=1):
        self._check(gpu_lib().gor_step(self.h, int(nsteps)))

    def download(self) -> dict:
        n = self.p.ptc_num
        out = dict(pos=np.empty((n, 3)), vel=np.empty((n, 3)), rhop=np.empty((n, 2)),
                   type=np.empty(n, np.int32), table=np.empty(n, np.int32))
        self._check(gpu_lib().gor_download(self.h, *[_p(out[k]) for k in ("pos", "vel", "rhop", "type", "table")]))
        return out

    def rigid_state(self) -> dict:
        b = ORigid()
        gpu_lib().gor_rigid(self.h, ctypes.byref(b))
        return {k: np.array(getattr(b, k)[:]) for k in ("x", "v", "w", "q", "F", "T")}

    def close(self):
        if self.h:
            gpu_lib().gor_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def max_threads() -> int:
    return int(lib().oracle_max_threads())


# ---- the reference's own CUDA kernels (checker build in _ref/) ---------------

class RState(ctypes.Structure):
    _fields_ = [(n, _VP) for n in ("pos", "vel", "rhop", "tmp_pos", "tmp_vel", "tmp_rhop", "type", "table")]


class RTmp(ctypes.Structure):
    _fields_ = [(n, _VP) for n in ("acc_drhodt", "dofv_grandrho", "index", "hash", "grid_start", "grid_end",
                                   "nb_boundary", "nb_governing", "dofv")]


_ref = {}


def ref_available(simple: bool = False) -> bool:
    return os.path.exists(REF_SIMPLE_SO if simple else REF_SO)


def ref_lib(simple: bool = False) -> ctypes.CDLL:
    """The reference build: deltasph (default) or simplesph (simple=True)."""
    if simple not in _ref:
        lib_ = ctypes.CDLL(REF_SIMPLE_SO if simple else REF_SO)
        lib_.ref_substep.restype = _I
        lib_.ref_run.restype = _I
        lib_.ref_run_profiled.restype = _I
        lib_.ref_params.restype = _I
        lib_.ref_last_error.restype = ctypes.c_char_p
        _ref[simple] = lib_
    return _ref[simple]


def ref_params(json, simple: bool = False):
    from zsph_b200 import GpuParam  # same field layout as the reference's gpu_param_t
    gp = GpuParam()
    G = _I(0)
    ref_lib(simple).ref_params(ctypes.byref(case_of(json)), ctypes.byref(gp), ctypes.byref(G))
    return gp, G.value


def _rstate(st, n):
    f = lambda a, s: np.ascontiguousarray(a if a is not None else np.zeros(s, np.float32), np.float32)
    arrs = dict(pos=f(st.pos, (n, 3)), vel=f(st.vel, (n, 3)), rhop=f(st.rhop, (n, 2)),
                tmp_pos=f(st.tmp_pos, (n, 3)), tmp_vel=f(st.tmp_vel, (n, 3)), tmp_rhop=f(st.tmp_rhop, (n, 2)),
                type=np.ascontiguousarray(st.type, np.int32), table=np.ascontiguousarray(st.table, np.int32))
    return arrs, RState(*[_p(arrs[k]) for k, _ in RState._fields_])


def _rout(n, G):
    out = dict(pos=np.zeros((n, 3), np.float32), vel=np.zeros((n, 3), np.float32), rhop=np.zeros((n, 2), np.float32),
               tmp_pos=np.zeros((n, 3), np.float32), tmp_vel=np.zeros((n, 3), np.float32),
               tmp_rhop=np.zeros((n, 2), np.float32), type=np.zeros(n, np.int32), table=np.zeros(n, np.int32))
    tmp = dict(acc_drhodt=np.zeros((n, 4), np.float32), dofv_grandrho=np.zeros((n, 4), np.float32),
               index=np.zeros(n, np.int32), hash=np.zeros(n, np.int32), grid_start=np.zeros(G, np.int32),
               grid_end=np.zeros(G, np.int32), nb_boundary=np.zeros(n, np.int32),
               nb_governing=np.zeros(n, np.int32), dofv=np.zeros(n, np.float32))
    return out, tmp, RState(*[_p(out[k]) for k, _ in RState._fields_]), RTmp(*[_p(tmp[k]) for k, _ in RTmp._fields_])


def ref_substep(json, state, stage: int, simple: bool = False):
    """Runs the reference's kernels of one predictor sub-step up to `stage`
    (1 hash, 2 sort_index, 3 sort_data, 4 boundary, 5 governing, 6 prediction)."""
    _, G = ref_params(json, simple)
    n = int(json.ptc_num)
    arrs, rin = _rstate(state, n)
    out, tmp, rout, rtmp = _rout(n, G)
    c = case_of(json)
    lib_ = ref_lib(simple)
    rc = lib_.ref_substep(ctypes.byref(c), ctypes.byref(rin), _I(stage), ctypes.byref(rout), ctypes.byref(rtmp))
    if rc:
        raise RuntimeError(lib_.ref_last_error().decode())
    return out, tmp


def ref_run(json, state, nsteps: int, warmup: int = 0, simple: bool = False):
    """Runs `warmup + nsteps` full reference steps; returns (OLD state, tmp, ms/step of the last nsteps)."""
    _, G = ref_params(json, simple)
    n = int(json.ptc_num)
    arrs, rin = _rstate(state, n)
    out, tmp, rout, rtmp = _rout(n, G)
    ms = ctypes.c_float(0.0)
    lib_ = ref_lib(simple)
    rc = lib_.ref_run(ctypes.byref(case_of(json)), ctypes.byref(rin), _I(warmup), _I(nsteps), ctypes.byref(rout),
                      ctypes.byref(rtmp), ctypes.byref(ms))
    if rc:
        raise RuntimeError(lib_.ref_last_error().decode())
    return out, tmp, float(ms.value)


REF_SLOTS = ("hash", "sort_index", "sort_data", "boundary", "governing", "prediction",
             "hash_2", "sort_index_2", "sort_data_2", "boundary_2", "governing_2", "correction")


def ref_run_profiled(json, state, nsteps: int, warmup: int = 0, simple: bool = False) -> dict:
    """`warmup + nsteps` reference steps with a CUDA event after each of the
    step's twelve launch slots (main.cu:63-88) and the host time of each
    Thrust sort call; returns per-step means in ms."""
    n = int(json.ptc_num)
    arrs, rin = _rstate(state, n)
    ms = ctypes.c_float(0.0)
    slots = (ctypes.c_float * 12)()
    host = (ctypes.c_float * 2)()
    lib_ = ref_lib(simple)
    rc = lib_.ref_run_profiled(ctypes.byref(case_of(json)), ctypes.byref(rin), _I(warmup), _I(nsteps),
                               ctypes.byref(ms), slots, host)
    if rc:
        raise RuntimeError(lib_.ref_last_error().decode())
    return {"ms_per_step": float(ms.value), "slot_ms": dict(zip(REF_SLOTS, (float(v) for v in slots))),
            "host_sort_ms": [float(host[0]), float(host[1])]}
