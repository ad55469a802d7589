"""Python host bindings for the B200-native delta-SPH step (C ABI: include/zsph.h).

The product is the CUDA library ``libzsph_b200.so`` built in this directory;
this module only binds its C entry points with ctypes and offers a thin
``Solver`` that owns device buffers in the reference solver's particle layout
(single_gpu_sph_src/header/data_structure.cuh:158-182).  The library is
loaded on the first call that needs it (so that the case generator and the
ctypes struct types can be used without mapping it); that first call fails
loudly if the library has not been built: there is no fallback.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "ZsphError", "lib", "JsonCase", "CpuParam", "GpuParam", "Ptc", "Tmp", "Solver", "State",
    "params_from_json", "LIB_PATH",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libzsph_b200.so")

ZSPH_OK, ZSPH_EINVAL, ZSPH_ECUDA, ZSPH_ENAN, ZSPH_ETIMEOUT, ZSPH_EIO, ZSPH_ENOMEM = range(7)
EQ_DELTA, EQ_SIMPLE = 0, 1
CORR_NETWORK, CORR_REUSE_LAGGED, CORR_REUSE_FRESH = 0, 1, 2
FLAG_NAN, FLAG_KILLED, FLAG_NB_OVERFLOW, FLAG_BAD_KEY = 1, 2, 4, 8
_CODES = {0: "ZSPH_OK", 1: "ZSPH_EINVAL", 2: "ZSPH_ECUDA", 3: "ZSPH_ENAN", 4: "ZSPH_ETIMEOUT", 5: "ZSPH_EIO",
          6: "ZSPH_ENOMEM"}


class ZsphError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_CODES.get(code, code)}: {msg}")
        self.code = code


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C zsph_b200` or __graft_entry__.build(); "
            "zsph_b200 has no CPU fallback")
    cdll = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _sig.items():
        fn = getattr(cdll, name)
        fn.restype = res
        fn.argtypes = args
    return cdll


class _LazyLib:
    """Stands for the ctypes handle of libzsph_b200.so: the first attribute
    lookup loads the library (raising ImportError if it is missing) and
    binds every entry point's signature; later lookups go straight to it."""

    def __init__(self):
        self._cdll = None

    def loaded(self) -> bool:
        return self._cdll is not None

    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        if self._cdll is None:
            self._cdll = _load()
        return getattr(self._cdll, name)


lib = _LazyLib()

_F = ctypes.c_float
_I = ctypes.c_int
_FP = ctypes.POINTER(ctypes.c_float)
_IP = ctypes.POINTER(ctypes.c_int)
_VP = ctypes.c_void_p


class JsonCase(ctypes.Structure):
    """zsph_json_t: the reference's cpu_json_t (data_structure.cuh:6-51)."""
    _fields_ = [(n, _F) for n in ("g", "m", "rho0", "dx", "h_factor", "r_factor", "eta_factor", "cs_factor",
                                  "delta", "alpha", "xmin", "xmax", "ymin", "ymax", "zmin", "zmax",
                                  "grid_layer_factor", "grid_size_factor", "dt")] + \
              [(n, _I) for n in ("start_step", "current_step", "end_step", "output_step", "ptc_num",
                                 "water_ptc_num", "air_ptc_num", "wall_ptc_num", "rigid_ptc_num", "thread_num",
                                 "gpu_id")] + \
              [("input_path", ctypes.c_char * 256), ("output_path", ctypes.c_char * 256),
               ("git_hash", ctypes.c_char * 64)]


class CaseOptions(ctypes.Structure):
    """zsph_case_options_t: the optional keys of a case file (no reference counterpart)."""
    _fields_ = [("equations", _I), ("snapshot_every", _I), ("resume", ctypes.c_char * 256)]


class CpuParam(ctypes.Structure):
    """zsph_cpu_param_t: the reference's cpu_param_t (data_structure.cuh:53-105)."""
    _fields_ = [(n, _F) for n in ("g", "m", "rho0", "dx", "h", "r", "eta", "cs", "adh", "delta", "alpha", "dt")] + \
              [(n, _I) for n in ("start_step", "current_step", "end_step", "output_step")] + \
              [(n, _F) for n in ("xmin", "xmax", "ymin", "ymax", "zmin", "zmax")] + \
              [("grid_factor", _I), ("grid_size", _F)] + \
              [(n, _F) for n in ("grid_xmin", "grid_ymin", "grid_zmin", "grid_xmax", "grid_ymax", "grid_zmax")] + \
              [(n, _I) for n in ("grid_xdim", "grid_ydim", "grid_zdim", "grid_num", "grid_hash_min",
                                 "grid_hash_max", "ptc_num", "water_ptc_num", "air_ptc_num", "wall_ptc_num",
                                 "rigid_ptc_num", "thread_num", "gpu_id")] + \
              [("input_path", ctypes.c_char * 256), ("output_path", ctypes.c_char * 256),
               ("git_hash", ctypes.c_char * 64)]


class GpuParam(ctypes.Structure):
    """zsph_gpu_param_t: the reference's gpu_param_t (data_structure.cuh:107-134)."""
    _fields_ = [(n, _F) for n in ("half_dt", "h", "g", "m", "rho0", "adh", "h2", "eta2", "cs2", "alpha",
                                  "delta_h_cs", "h_cs_rho_m", "grid_size")] + \
              [("grid_factor", _I)] + [(n, _F) for n in ("grid_xmin", "grid_ymin", "grid_zmin")] + \
              [(n, _I) for n in ("grid_xdim", "grid_ydim", "grid_zdim", "grid_hash_min", "grid_hash_max",
                                 "ptc_num")]


class Ptc(ctypes.Structure):
    """zsph_ptc_t: the reference's gpu_ptc_t (data_structure.cuh:158-168)."""
    _fields_ = [(n, _VP) for n in ("pos", "vel", "rhop", "tmp_pos", "tmp_vel", "tmp_rhop", "type", "table")]


class Tmp(ctypes.Structure):
    """zsph_tmp_t: the reference's gpu_tmp_t (data_structure.cuh:170-182)."""
    _fields_ = [(n, _VP) for n in ("acc_drhodt", "dofv_grandrho", "dofv", "index", "hash", "grid_start",
                                   "grid_end")]


class LearnTrainStats(ctypes.Structure):
    """zsph_learn_train_stats_t."""
    _fields_ = [("snapshots_train", ctypes.c_int), ("snapshots_val", ctypes.c_int), ("rows_train", ctypes.c_longlong),
                ("epochs", ctypes.c_int), ("iterations", ctypes.c_int)] + \
               [(n, ctypes.c_float) for n in ("loss_first", "loss_last", "val_acc_rel_l2", "val_acc_rel_l2_base",
                                              "val_acc_rel_l2_extrap", "val_drho_rel_l2", "val_drho_rel_l2_base",
                                              "val_drho_rel_l2_extrap", "seconds")]


class LearnRunStats(ctypes.Structure):
    """zsph_learn_run_stats_t."""
    _fields_ = [(n, ctypes.c_int) for n in ("steps", "learned", "plain", "judged", "fallbacks")] + \
               [(n, ctypes.c_float) for n in ("err_max", "err_mean", "err_last")]


class RigidBody(ctypes.Structure):
    """zsph_rigid_t."""
    _fields_ = [("first", ctypes.c_int), ("count", ctypes.c_int), ("mass", ctypes.c_double)] + \
               [(n, ctypes.c_double * k) for n, k in (("pos", 3), ("vel", 3), ("omega", 3), ("q", 4), ("force", 3),
                                                       ("torque", 3), ("inertia", 9))]


class Conservation(ctypes.Structure):
    """zsph_conservation_t."""
    _fields_ = [("mass", ctypes.c_double), ("volume", ctypes.c_double), ("momentum", ctypes.c_double * 3)] + \
               [(n, ctypes.c_double) for n in ("kinetic", "potential", "internal", "body_kinetic",
                                               "body_potential")]


class TuneResult(ctypes.Structure):
    """zsph_tune_t."""
    _fields_ = [("list_cells_per_cta", ctypes.c_int), ("governing_min_ctas", ctypes.c_int),
                ("steps_per_graph", ctypes.c_int), ("ms_per_step", ctypes.c_float), ("ms_default", ctypes.c_float),
                ("candidates", ctypes.c_int), ("list_segments", ctypes.c_int)]


def _as_dict(s: ctypes.Structure) -> dict:
    out = {}
    for k, _ in s._fields_:
        v = getattr(s, k)
        out[k] = np.array(v[:]) if isinstance(v, ctypes.Array) else v
    return out


_HP = ctypes.c_void_p
_sig = {
    "zsph_read_json": (_I, [ctypes.c_char_p, ctypes.POINTER(JsonCase), ctypes.c_char_p, _I]),
    "zsph_compat_run": (_I, [ctypes.c_char_p, _I, _IP]),
    "zsph_read_case_options": (_I, [ctypes.c_char_p, ctypes.POINTER(CaseOptions), ctypes.c_char_p, _I]),
    "zsph_set_cpu_param": (_I, [ctypes.POINTER(CpuParam), ctypes.POINTER(JsonCase)]),
    "zsph_set_gpu_param": (_I, [ctypes.POINTER(GpuParam), ctypes.POINTER(CpuParam)]),
    "zsph_check_dt": (_I, [ctypes.POINTER(CpuParam), _FP]),
    "zsph_alloc_ptc": (_I, [ctypes.POINTER(Ptc), _I]),
    "zsph_free_ptc": (_I, [ctypes.POINTER(Ptc)]),
    "zsph_alloc_tmp": (_I, [ctypes.POINTER(Tmp), _I, _I]),
    "zsph_free_tmp": (_I, [ctypes.POINTER(Tmp)]),
    "zsph_cpu_to_gpu": (_I, [ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP, _VP, _VP, _VP, _VP, _VP, _I, _VP]),
    "zsph_gpu_to_cpu": (_I, [ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP, _VP, _VP, _VP, _VP, _VP, _VP, _I, _VP]),
    "zsph_create": (_I, [ctypes.POINTER(GpuParam), _I, ctypes.POINTER(_HP)]),
    "zsph_destroy": (None, [_HP]),
    "zsph_set_params": (_I, [_HP, ctypes.POINTER(GpuParam)]),
    "zsph_set_equations": (_I, [_HP, _I]),
    "zsph_hash": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP]),
    "zsph_sort_index": (_I, [_HP, ctypes.POINTER(Tmp), _VP]),
    "zsph_sort_index_noalloc": (_I, [ctypes.POINTER(GpuParam), _I, ctypes.POINTER(Tmp), _VP]),
    "zsph_sort_data": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP]),
    "zsph_neighbor_search": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP]),
    "zsph_boundary": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP]),
    "zsph_governing": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP]),
    "zsph_prediction": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP]),
    "zsph_correction": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP]),
    "zsph_step": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP]),
    "zsph_run": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _I, _VP]),
    "zsph_status": (_I, [_HP, _IP, _I]),
    "zsph_neighbor_counts": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP, _VP, _VP]),
    "zsph_launches_per_step": (_I, [_HP]),
    "zsph_step_profiled": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP, _FP, _I,
                                _IP, ctypes.c_char_p, _I]),
    "zsph_step_profiled_groups": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP, _FP, _I,
                                _IP, ctypes.c_char_p, _I]),
    "zsph_last_error": (_I, [_HP, ctypes.c_char_p, _I]),
    "zsph_version": (ctypes.c_char_p, []),
    "zsph_memcpy": (_I, [_VP, _VP, ctypes.c_size_t, _I, _VP]),
    "zsph_device_malloc": (_I, [ctypes.POINTER(_VP), ctypes.c_size_t]),
    "zsph_device_free": (_I, [_VP]),
    "zsph_device_synchronize": (_I, []),
    "zsph_write_vtk": (_I, [ctypes.c_char_p, _I, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _I]),
    "zsph_read_vtk": (_I, [ctypes.c_char_p, _I, _F, _I, _VP, _VP, _VP, _VP, _VP, _VP]),
    "zsph_writer_create": (_I, [ctypes.c_char_p, _I, _I, _I, ctypes.POINTER(_VP)]),
    "zsph_writer_submit": (_I, [_VP, ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _I, _VP]),
    "zsph_writer_destroy": (_I, [_VP]),
    "zsph_mlp_create": (_I, [ctypes.c_ulonglong, ctypes.POINTER(_VP)]),
    "zsph_mlp_destroy": (_I, [_VP]),
    "zsph_mlp_set_params": (_I, [_VP, _VP]),
    "zsph_mlp_get_params": (_I, [_VP, _VP]),
    "zsph_mlp_set_moments": (_I, [_VP, _VP, _VP, _I]),
    "zsph_mlp_get_moments": (_I, [_VP, _VP, _VP, _IP]),
    "zsph_mlp_pack": (_I, [_VP, _I, _VP, _VP, _VP, _VP]),
    "zsph_mlp_forward": (_I, [_VP, _VP, _I, _VP, _VP]),
    "zsph_mlp_grad": (_I, [_VP, _VP, _VP, _VP, _VP, _I, _F, _VP, _IP, _VP]),
    "zsph_mlp_adam": (_I, [_VP, _VP, _I, _F, _F, _F, _F, _VP]),
    "zsph_mlp_set_norm": (_I, [_VP, _VP, _VP, _VP, _VP]),
    "zsph_mlp_get_norm": (_I, [_VP, _VP, _VP, _VP, _VP]),
    "zsph_learn_feature_scales": (_I, [_HP, _VP]),
    "zsph_learn_features": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _VP, _VP]),
    "zsph_learn_collect": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _I, _I, _I, _IP,
                                _VP]),
    "zsph_learn_clear": (_I, [_HP]),
    "zsph_learn_train": (_I, [_HP, _VP, _I, _I, _F, ctypes.c_ulonglong, _F, ctypes.POINTER(LearnTrainStats), _VP]),
    "zsph_run_learned": (_I, [_HP, _VP, ctypes.POINTER(Ptc), ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _I, _I, _F,
                              ctypes.POINTER(LearnRunStats), _VP]),
    "zsph_run_learned_ex": (_I, [_HP, _VP, ctypes.POINTER(Ptc), ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _I, _I, _F,
                                 _I, _VP, _I, ctypes.POINTER(LearnRunStats), _VP]),
    "zsph_set_precision": (_I, [_HP, _I]),
    "zsph_precise_load": (_I, [_HP, ctypes.POINTER(Ptc), _VP, _VP]),
    "zsph_precise_positions": (_I, [_HP, ctypes.POINTER(Ptc), _VP, _VP]),
    "zsph_conservation": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Conservation), _VP]),
    "zsph_rigid_attach": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(RigidBody), _VP]),
    "zsph_rigid_get": (_I, [_HP, ctypes.POINTER(RigidBody)]),
    "zsph_rigid_count": (_I, [_HP, _IP]),
    "zsph_rigid_get_body": (_I, [_HP, _I, ctypes.POINTER(RigidBody)]),
    "zsph_rigid_contact": (_I, [_HP, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    "zsph_create_batch": (_I, [ctypes.POINTER(GpuParam), _IP, _I, ctypes.POINTER(_HP)]),
    "zsph_autotune": (_I, [_HP, ctypes.POINTER(Ptc), ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _I,
                           ctypes.POINTER(TuneResult), _VP]),
    "zsph_set_launch_shapes": (_I, [_HP, ctypes.POINTER(TuneResult)]),
    "zsph_set_batch_persistent": (_I, [_HP, _I]),
    "zsph_set_list_transfer": (_I, [_HP, _I, _F]),
    "zsph_list_transfer_info": (_I, [_HP, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                     ctypes.POINTER(ctypes.c_longlong)]),
    "zsph_persistent_info": (_I, [_HP, _IP, _IP]),
    "zsph_persistent_barrier_test": (_I, [_HP, _I, _VP]),
    "zsph_snapshot_save": (_I, [ctypes.c_char_p, ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _I, _I, _I, _VP]),
    "zsph_snapshot_load": (_I, [ctypes.c_char_p, ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _I, _I, _IP, _VP]),
    "zsph_snapshot_save_host": (_I, [ctypes.c_char_p, ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _I, _I, _I]),
    "zsph_snapshot_load_host": (_I, [ctypes.c_char_p, ctypes.POINTER(Ptc), ctypes.POINTER(Tmp), _I, _I, _IP]),
}

OUT_P, OUT_TYPE, OUT_VEL, OUT_ACC, OUT_RHO, OUT_HASH, OUT_TABLE = 1, 2, 4, 8, 16, 32, 64
OUT_REFERENCE = OUT_P | OUT_TYPE | OUT_VEL | OUT_ACC


def write_vtk(path: str, st, acc=None, hash=None, flags: int = OUT_REFERENCE) -> None:
    """zsph_write_vtk of a host State (io/write_vtk.cu:29-130)."""
    f = lambda a, dt: None if a is None else np.ascontiguousarray(a, dtype=dt)
    pos, vel, rhop = f(st.pos, np.float32), f(st.vel, np.float32), f(st.rhop, np.float32)
    typ, tab, a4, hs = f(st.type, np.int32), f(st.table, np.int32), f(acc, np.float32), f(hash, np.int32)
    check(lib.zsph_write_vtk(path.encode(), len(st.type), _ptr(pos), _ptr(vel), _ptr(rhop), _ptr(typ), _ptr(a4),
                             _ptr(hs), _ptr(tab), int(flags)))


def read_vtk(path: str, n: int, rho0: float = 1000.0, accept_float: bool = False):
    """zsph_read_vtk (io/read_vkt.cu:3-92): returns (State, acc_drhodt)."""
    st = State(np.empty((n, 3), np.float32), np.empty((n, 3), np.float32), np.empty((n, 2), np.float32),
               np.empty(n, np.int32), np.empty(n, np.int32))
    acc = np.empty((n, 4), np.float32)
    check(lib.zsph_read_vtk(path.encode(), n, float(rho0), 1 if accept_float else 0, _ptr(st.pos), _ptr(st.vel),
                            _ptr(st.rhop), _ptr(acc), _ptr(st.type), _ptr(st.table)))
    return st, acc
SNAPSHOT_PTC = {"pos": (3, np.float32), "vel": (3, np.float32), "rhop": (2, np.float32),
                "tmp_pos": (3, np.float32), "tmp_vel": (3, np.float32), "tmp_rhop": (2, np.float32),
                "type": (1, np.int32), "table": (1, np.int32)}
SNAPSHOT_TMP = {"acc_drhodt": (4, np.float32), "dofv_grandrho": (4, np.float32), "dofv": (1, np.float32),
                "index": (1, np.int32), "hash": (1, np.int32), "grid_start": (1, np.int32),
                "grid_end": (1, np.int32)}


def _host_structs(arrays: dict):
    """Ptc/Tmp structs pointing at the host arrays of `arrays` (absent: NULL)."""
    p, t = Ptc(), Tmp()
    for k in SNAPSHOT_PTC:
        if arrays.get(k) is not None:
            setattr(p, k, arrays[k].ctypes.data)
    for k in SNAPSHOT_TMP:
        if arrays.get(k) is not None:
            setattr(t, k, arrays[k].ctypes.data)
    return p, t


def snapshot_save_host(path: str, arrays: dict, n: int, grid_num: int, step: int = 0) -> None:
    """zsph_snapshot_save_host of host arrays keyed by their zsph_ptc_t /
    zsph_tmp_t member names (missing keys are NULL arrays)."""
    arrays = {k: np.ascontiguousarray(v, dtype={**SNAPSHOT_PTC, **SNAPSHOT_TMP}[k][1])
              for k, v in arrays.items() if v is not None}
    p, t = _host_structs(arrays)
    check(lib.zsph_snapshot_save_host(path.encode(), ctypes.byref(p), ctypes.byref(t), int(n), int(grid_num),
                                      int(step)))


def snapshot_load_host(path: str, n: int, grid_num: int, names=None) -> tuple[dict, int]:
    """zsph_snapshot_load_host into fresh host arrays for `names` (default:
    every array); returns (arrays, step)."""
    spec = {**SNAPSHOT_PTC, **SNAPSHOT_TMP}
    names = list(spec) if names is None else list(names)
    out = {}
    for k in names:
        w, dt = spec[k]
        rows = grid_num if k in ("grid_start", "grid_end") else n
        out[k] = np.empty((rows, w) if w > 1 else rows, dt)
    p, t = _host_structs(out)
    step = ctypes.c_int(-1)
    check(lib.zsph_snapshot_load_host(path.encode(), ctypes.byref(p), ctypes.byref(t), int(n), int(grid_num),
                                      ctypes.byref(step)))
    return out, step.value


def last_error(handle=None) -> str:
    buf = ctypes.create_string_buffer(1024)
    lib.zsph_last_error(handle, buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int, handle=None) -> None:
    if rc != ZSPH_OK:
        raise ZsphError(rc, last_error(handle))


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


COMPAT_SEPARATE, COMPAT_FUSED, COMPAT_SIMPLE = 0, 1, 2


def compat_run(json_path: str, mode: int = COMPAT_SEPARATE) -> int:
    """zsph_compat_run: the reference's driver program (deltasph/main.cu) on
    this library; returns the number of steps run."""
    steps = ctypes.c_int(0)
    check(lib.zsph_compat_run(json_path.encode(), int(mode), ctypes.byref(steps)))
    return steps.value


def read_json(path: str) -> JsonCase:
    """zsph_read_json (io/read_json.cu:5-51)."""
    j = JsonCase()
    err = ctypes.create_string_buffer(512)
    rc = lib.zsph_read_json(path.encode(), ctypes.byref(j), err, len(err))
    if rc != ZSPH_OK:
        raise ZsphError(rc, err.value.decode())
    return j


def read_case_options(path: str) -> CaseOptions:
    """zsph_read_case_options: the optional keys of a case file."""
    o = CaseOptions()
    err = ctypes.create_string_buffer(256)
    rc = lib.zsph_read_case_options(path.encode(), ctypes.byref(o), err, len(err))
    if rc != ZSPH_OK:
        raise ZsphError(rc, err.value.decode(errors="replace"))
    return o


def params_from_json(j: JsonCase) -> tuple[CpuParam, GpuParam]:
    """set_cpu_param + set_gpu_param (lib/init.cu:153-251); raises on dt > dt_max."""
    cp, gp = CpuParam(), GpuParam()
    check(lib.zsph_set_cpu_param(ctypes.byref(cp), ctypes.byref(j)))
    check(lib.zsph_set_gpu_param(ctypes.byref(gp), ctypes.byref(cp)))
    return cp, gp


@dataclass
class State:
    """Host copy of one particle buffer set in the reference layout."""
    pos: np.ndarray
    vel: np.ndarray
    rhop: np.ndarray
    type: np.ndarray
    table: np.ndarray
    tmp_pos: np.ndarray | None = None
    tmp_vel: np.ndarray | None = None
    tmp_rhop: np.ndarray | None = None
    extra: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.type.shape[0])

    def copy(self) -> "State":
        c = lambda a: None if a is None else a.copy()
        return State(c(self.pos), c(self.vel), c(self.rhop), c(self.type), c(self.table), c(self.tmp_pos),
                     c(self.tmp_vel), c(self.tmp_rhop), dict(self.extra))


class Solver:
    """Owns a solver handle and two particle buffer sets plus tmp arrays on
    the current CUDA device, in the reference's layout (the OLD/NEW/tmp
    buffers of single_gpu_sph_src/deltasph/main.cu:32-45)."""

    def __init__(self, gparam: GpuParam, grid_num: int):
        self.gp = gparam
        self.n = int(gparam.ptc_num)
        self.G = int(grid_num)
        self.old, self.new, self.tmp = Ptc(), Ptc(), Tmp()
        check(lib.zsph_alloc_ptc(ctypes.byref(self.old), self.n))
        check(lib.zsph_alloc_ptc(ctypes.byref(self.new), self.n))
        check(lib.zsph_alloc_tmp(ctypes.byref(self.tmp), self.n, self.G))
        h = _HP()
        check(lib.zsph_create(ctypes.byref(gparam), self.G, ctypes.byref(h)))
        self.h = h

    @classmethod
    def from_case(cls, case) -> "Solver":
        _, gp = params_from_json(case.json)
        cp, _ = params_from_json(case.json)
        s = cls(gp, cp.grid_num)
        s.upload(case.state)
        return s

    @classmethod
    def from_batch(cls, case_list) -> "Solver":
        """Batched form (zsph_create_batch) over independent cases, stored
        one after another; `scene_ptc` holds each scene's particle count."""
        gps, gnums = [], []
        for c in case_list:
            cp, gp = params_from_json(c.json)
            gps.append(gp)
            gnums.append(int(cp.grid_num))
        arr = (GpuParam * len(gps))(*gps)
        gn = (ctypes.c_int * len(gnums))(*gnums)
        s = cls.__new__(cls)
        s.n = int(sum(int(g.ptc_num) for g in gps))
        s.G = int(sum(gnums))
        s.gp = gps[0]
        s.scene_ptc = [int(g.ptc_num) for g in gps]
        s.old, s.new, s.tmp = Ptc(), Ptc(), Tmp()
        check(lib.zsph_alloc_ptc(ctypes.byref(s.old), s.n))
        check(lib.zsph_alloc_ptc(ctypes.byref(s.new), s.n))
        check(lib.zsph_alloc_tmp(ctypes.byref(s.tmp), s.n, s.G))
        h = _HP()
        check(lib.zsph_create_batch(arr, gn, len(gps), ctypes.byref(h)))
        s.h = h
        cat = lambda k: np.concatenate([np.asarray(getattr(c.state, k)) for c in case_list])
        s.upload(State(pos=cat("pos"), vel=cat("vel"), rhop=cat("rhop"), type=cat("type"), table=cat("table"),
                       tmp_pos=cat("tmp_pos"), tmp_vel=cat("tmp_vel"), tmp_rhop=cat("tmp_rhop")))
        return s

    def autotune(self, trial_steps: int = 3, stream=None) -> dict:
        r = TuneResult()
        self._call(lib.zsph_autotune, ctypes.byref(self.old), ctypes.byref(self.new), ctypes.byref(self.tmp),
                   int(trial_steps), ctypes.byref(r), stream)
        return _as_dict(r)

    def set_launch_shapes(self, list_cells_per_cta: int = 0, governing_min_ctas: int = 0,
                          steps_per_graph: int = 0, list_segments: int = 0) -> None:
        """Applies launch shapes from an earlier autotune() result (0 = default) without timing."""
        r = TuneResult(list_cells_per_cta=int(list_cells_per_cta), governing_min_ctas=int(governing_min_ctas),
                       steps_per_graph=int(steps_per_graph), list_segments=int(list_segments))
        self._call(lib.zsph_set_launch_shapes, ctypes.byref(r))

    def close(self) -> None:
        if getattr(self, "h", None):
            lib.zsph_destroy(self.h)
            self.h = None
            lib.zsph_free_ptc(ctypes.byref(self.old))
            lib.zsph_free_ptc(ctypes.byref(self.new))
            lib.zsph_free_tmp(ctypes.byref(self.tmp))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _buf(self, which: str) -> Ptc:
        return self.old if which == "old" else self.new

    # -- host <-> device -------------------------------------------------
    def upload(self, st: State, which: str = "old", acc: np.ndarray | None = None, stream=None) -> None:
        b = self._buf(which)
        f = lambda a: np.ascontiguousarray(a, dtype=np.float32)
        i = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        pos, vel, rhop, typ, tab = f(st.pos), f(st.vel), f(st.rhop), i(st.type), i(st.table)
        a = None if acc is None else f(acc)
        check(lib.zsph_cpu_to_gpu(ctypes.byref(b), ctypes.byref(self.tmp), _ptr(pos), _ptr(vel), _ptr(rhop),
                                  _ptr(typ), _ptr(tab), _ptr(a), self.n, stream))
        for name in ("tmp_pos", "tmp_vel", "tmp_rhop"):
            arr = getattr(st, name)
            if arr is not None:
                self.copy_to_device(getattr(b, name), f(arr))

    def copy_to_device(self, dptr, host: np.ndarray) -> None:
        _cudart_memcpy(dptr, host.ctypes.data, host.nbytes, 1)

    def copy_from_device(self, dptr, host: np.ndarray) -> np.ndarray:
        _cudart_memcpy(host.ctypes.data, dptr, host.nbytes, 2)
        return host

    def download(self, which: str = "old") -> State:
        b = self._buf(which)
        n = self.n
        st = State(np.empty((n, 3), np.float32), np.empty((n, 3), np.float32), np.empty((n, 2), np.float32),
                   np.empty(n, np.int32), np.empty(n, np.int32), np.empty((n, 3), np.float32),
                   np.empty((n, 3), np.float32), np.empty((n, 2), np.float32))
        check(lib.zsph_gpu_to_cpu(ctypes.byref(b), ctypes.byref(self.tmp), _ptr(st.pos), _ptr(st.vel),
                                  _ptr(st.rhop), _ptr(st.type), _ptr(st.table), None, None, n, None))
        self.copy_from_device(b.tmp_pos, st.tmp_pos)
        self.copy_from_device(b.tmp_vel, st.tmp_vel)
        self.copy_from_device(b.tmp_rhop, st.tmp_rhop)
        return st

    def download_tmp(self) -> dict:
        n, G = self.n, self.G
        out = {
            "acc_drhodt": np.empty((n, 4), np.float32), "dofv_grandrho": np.empty((n, 4), np.float32),
            "index": np.empty(n, np.int32), "hash": np.empty(n, np.int32),
            "grid_start": np.empty(G, np.int32), "grid_end": np.empty(G, np.int32),
        }
        for k, v in out.items():
            self.copy_from_device(getattr(self.tmp, k), v)
        return out

    def upload_tmp(self, **arrays) -> None:
        for k, v in arrays.items():
            dt = np.int32 if k in ("index", "hash", "grid_start", "grid_end") else np.float32
            self.copy_to_device(getattr(self.tmp, k), np.ascontiguousarray(v, dtype=dt))

    def save_snapshot(self, path: str, step: int = 0, which: str = "old", stream=None) -> None:
        """zsph_snapshot_save of one buffer set and tmp (checkpoint)."""
        check(lib.zsph_snapshot_save(path.encode(), ctypes.byref(self._buf(which)), ctypes.byref(self.tmp), self.n,
                                     self.G, int(step), stream))

    def load_snapshot(self, path: str, which: str = "old", stream=None) -> int:
        """zsph_snapshot_load into one buffer set and tmp (resume); returns the saved step."""
        step = ctypes.c_int(-1)
        check(lib.zsph_snapshot_load(path.encode(), ctypes.byref(self._buf(which)), ctypes.byref(self.tmp), self.n,
                                     self.G, ctypes.byref(step), stream))
        return step.value

    # -- entry points ----------------------------------------------------
    def _call(self, fn, *args):
        check(fn(self.h, *args), self.h)

    def hash(self, which="old", stream=None):
        self._call(lib.zsph_hash, ctypes.byref(self._buf(which)), ctypes.byref(self.tmp), stream)

    def sort_index(self, stream=None):
        self._call(lib.zsph_sort_index, ctypes.byref(self.tmp), stream)

    def sort_data(self, src="old", dst="new", stream=None):
        self._call(lib.zsph_sort_data, ctypes.byref(self._buf(src)), ctypes.byref(self._buf(dst)),
                   ctypes.byref(self.tmp), stream)

    def neighbor_search(self, src="old", dst="new", stream=None):
        self._call(lib.zsph_neighbor_search, ctypes.byref(self._buf(src)), ctypes.byref(self._buf(dst)),
                   ctypes.byref(self.tmp), stream)

    def boundary(self, which="new", stream=None):
        self._call(lib.zsph_boundary, ctypes.byref(self._buf(which)), ctypes.byref(self.tmp), stream)

    def governing(self, which="new", stream=None):
        self._call(lib.zsph_governing, ctypes.byref(self._buf(which)), ctypes.byref(self.tmp), stream)

    def prediction(self, which="new", stream=None):
        self._call(lib.zsph_prediction, ctypes.byref(self._buf(which)), ctypes.byref(self.tmp), stream)

    def correction(self, which="old", stream=None):
        self._call(lib.zsph_correction, ctypes.byref(self._buf(which)), ctypes.byref(self.tmp), stream)

    def step(self, stream=None):
        self._call(lib.zsph_step, ctypes.byref(self.old), ctypes.byref(self.new), ctypes.byref(self.tmp), stream)

    def run(self, nsteps: int, stream=None):
        self._call(lib.zsph_run, ctypes.byref(self.old), ctypes.byref(self.new), ctypes.byref(self.tmp),
                   int(nsteps), stream)

    def status(self, clear: bool = True) -> int:
        f = ctypes.c_int(0)
        rc = lib.zsph_status(self.h, ctypes.byref(f), 1 if clear else 0)
        if rc not in (ZSPH_OK, ZSPH_ENAN, ZSPH_EINVAL):
            check(rc, self.h)
        return f.value

    def sync(self) -> None:
        _cudart_sync()

    def neighbor_counts(self, which="new") -> tuple[np.ndarray, np.ndarray]:
        nb_b = _DeviceInts(self.n)
        nb_g = _DeviceInts(self.n)
        self._call(lib.zsph_neighbor_counts, ctypes.byref(self._buf(which)), ctypes.byref(self.tmp), nb_b.ptr,
                   nb_g.ptr, None)
        return nb_b.get(), nb_g.get()

    def step_profiled(self, stream=None, groups: bool = False) -> list[tuple[str, float]]:
        """One step with CUDA-event timing: [(kernel, ms), ...] per launch, or,
        with groups=True, [(group, ms), ...] per sub-step's search and pair kernels."""
        cap = 64
        ms = (ctypes.c_float * cap)()
        cnt = ctypes.c_int(0)
        names = ctypes.create_string_buffer(4096)
        fn = lib.zsph_step_profiled_groups if groups else lib.zsph_step_profiled
        self._call(fn, ctypes.byref(self.old), ctypes.byref(self.new), ctypes.byref(self.tmp),
                   stream, ms, cap, ctypes.byref(cnt), names, len(names))
        nm = names.value.decode().split(",")
        return [(nm[k], float(ms[k])) for k in range(cnt.value)]

    def set_equations(self, which: int) -> None:
        """EQ_DELTA (deltasph, default) or EQ_SIMPLE (simplesph)."""
        self._call(lib.zsph_set_equations, int(which))

    def download_dofv(self) -> np.ndarray:
        return self.copy_from_device(self.tmp.dofv, np.empty(self.n, np.float32))

    def launches_per_step(self) -> int:
        return int(lib.zsph_launches_per_step(self.h))

    # ---- precision form, FP64 sums, rigid body ------------------------------
    def set_precision(self, on: bool = True, pos64=None) -> None:
        """Switch the precision form on (cell + offset positions); pos64:
        exact absolute positions of old_ to load (default: the FP32 ones)."""
        self._call(lib.zsph_set_precision, 1 if on else 0)
        if on:
            if pos64 is None:
                pos64 = self.download("old").pos
            p = np.ascontiguousarray(pos64, np.float64)
            self._call(lib.zsph_precise_load, ctypes.byref(self.old), p.ctypes.data, None)

    def positions64(self, which: str = "old") -> np.ndarray:
        out = np.empty((self.n, 3), np.float64)
        self._call(lib.zsph_precise_positions, ctypes.byref(self._buf(which)), out.ctypes.data, None)
        return out

    def conservation(self) -> dict:
        c = Conservation()
        self._call(lib.zsph_conservation, ctypes.byref(self.old), ctypes.byref(c), None)
        return _as_dict(c)

    def attach_body(self, first: int, count: int, mass: float, vel=(0, 0, 0), omega=(0, 0, 0),
                    q=(1, 0, 0, 0)) -> dict:
        b = RigidBody()
        b.first, b.count, b.mass = int(first), int(count), float(mass)
        b.vel[:], b.omega[:], b.q[:] = list(map(float, vel)), list(map(float, omega)), list(map(float, q))
        self._call(lib.zsph_rigid_attach, ctypes.byref(self.old), ctypes.byref(b), None)
        return self.body(self.body_count() - 1 if self.body_count() else 0)

    def body(self, index: int = 0) -> dict:
        b = RigidBody()
        self._call(lib.zsph_rigid_get_body, int(index), ctypes.byref(b))
        return _as_dict(b)

    def set_list_transfer(self, on: bool = True, skin: float = 0.05) -> None:
        """zsph_set_list_transfer: the corrector's lists made from the predictor's
        (bit-identical results; skin is a multiple of h, 0 = always build in full)."""
        self._call(lib.zsph_set_list_transfer, 1 if on else 0, float(skin))

    def list_transfer_info(self) -> dict:
        """zsph_list_transfer_info: steps that transferred, steps that built in full,
        particles that got a full search in the transferred steps."""
        a, b, c = ctypes.c_longlong(0), ctypes.c_longlong(0), ctypes.c_longlong(0)
        self._call(lib.zsph_list_transfer_info, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c))
        return {"transferred": a.value, "full_builds": b.value, "full_searches": c.value}

    def set_persistent(self, on: bool = True) -> None:
        """zsph_set_batch_persistent (batched handles)."""
        self._call(lib.zsph_set_batch_persistent, 1 if on else 0)

    def persistent_info(self) -> dict:
        c, g = ctypes.c_int(0), ctypes.c_int(0)
        self._call(lib.zsph_persistent_info, ctypes.byref(c), ctypes.byref(g))
        return {"ctas": c.value, "graph": g.value}

    def body_count(self) -> int:
        n = ctypes.c_int(0)
        self._call(lib.zsph_rigid_count, ctypes.byref(n))
        return n.value

    def set_contact(self, stiffness: float, damping: float, distance: float) -> None:
        """zsph_rigid_contact: body-wall and body-body contact (stiffness 0: off)."""
        self._call(lib.zsph_rigid_contact, float(stiffness), float(damping), float(distance))

    # ---- learned-corrector form (zsph_learn_*, zsph_run_learned) ----------
    def feature_scales(self) -> np.ndarray:
        s = np.empty(32, np.float32)
        self._call(lib.zsph_learn_feature_scales, s.ctypes.data)
        return s

    def learn_features(self, stream=None) -> np.ndarray:
        """Predictor sub-step that also returns the raw features of the
        sorted (new_) order."""
        buf = DeviceArray((self.n, 32), np.float32)
        self._call(lib.zsph_learn_features, ctypes.byref(self.old), ctypes.byref(self.new), ctypes.byref(self.tmp),
                   buf.ptr, stream)
        _cudart_sync()
        return buf.get()

    def collect(self, nsteps: int, every: int, capacity: int, stream=None) -> int:
        c = ctypes.c_int(0)
        self._call(lib.zsph_learn_collect, ctypes.byref(self.old), ctypes.byref(self.new), ctypes.byref(self.tmp),
                   int(nsteps), int(every), int(capacity), ctypes.byref(c), stream)
        return c.value

    def clear_snapshots(self) -> None:
        self._call(lib.zsph_learn_clear)

    def train(self, net: "Mlp", epochs: int = 10, batch_tiles: int = 148, lr: float = 2e-3, seed: int = 0,
              val_frac: float = 0.1, stream=None) -> dict:
        st = LearnTrainStats()
        self._call(lib.zsph_learn_train, net.h, int(epochs), int(batch_tiles), float(lr), int(seed), float(val_frac),
                   ctypes.byref(st), stream)
        return _as_dict(st)

    def run_learned(self, net: "Mlp | None", nsteps: int, judge_every: int = 10, tol: float = 1e-2, stream=None,
                    corrector: int = None, series: int = 0) -> dict:
        """zsph_run_learned (network corrector), or zsph_run_learned_ex with
        `corrector` (CORR_*); with series > 0 the result also holds the first
        `series` judged errors under "err_series"."""
        st = LearnRunStats()
        if corrector is None and not series:
            self._call(lib.zsph_run_learned, net.h, ctypes.byref(self.old), ctypes.byref(self.new),
                       ctypes.byref(self.tmp), int(nsteps), int(judge_every), float(tol), ctypes.byref(st), stream)
            return _as_dict(st)
        errs = np.zeros(max(int(series), 1), np.float32)
        self._call(lib.zsph_run_learned_ex, net.h if net is not None else None, ctypes.byref(self.old),
                   ctypes.byref(self.new), ctypes.byref(self.tmp), int(nsteps), int(judge_every), float(tol),
                   CORR_NETWORK if corrector is None else int(corrector), _ptr(errs) if series else None,
                   int(series), ctypes.byref(st), stream)
        out = _as_dict(st)
        if series:
            out["err_series"] = errs[:min(out["judged"], int(series))].tolist()
        return out


# ---- device-memory helpers through the library's own C ABI ----------------
def _cudart_memcpy(dst, src, nbytes, kind):
    check(lib.zsph_memcpy(dst, src, nbytes, kind, None))


def _cudart_sync():
    check(lib.zsph_device_synchronize())


class _DeviceInts:
    def __init__(self, n: int):
        self.n = n
        p = _VP()
        check(lib.zsph_device_malloc(ctypes.byref(p), max(n, 1) * 4))
        self.ptr = p

    def get(self) -> np.ndarray:
        out = np.empty(self.n, np.int32)
        _cudart_memcpy(out.ctypes.data, self.ptr, out.nbytes, 2)
        return out

    def __del__(self):
        try:
            lib.zsph_device_free(self.ptr)
        except Exception:
            pass


class DeviceArray:
    """A device buffer with a fixed numpy shape/dtype (library allocator)."""

    def __init__(self, shape, dtype=np.float32):
        self.shape = tuple(np.atleast_1d(shape)) if not isinstance(shape, tuple) else shape
        self.dtype = np.dtype(dtype)
        self.nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        p = _VP()
        check(lib.zsph_device_malloc(ctypes.byref(p), max(self.nbytes, 16)))
        self.ptr = p

    @classmethod
    def from_host(cls, a: np.ndarray) -> "DeviceArray":
        a = np.ascontiguousarray(a)
        d = cls(a.shape, a.dtype)
        d.set(a)
        return d

    def set(self, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, self.dtype)
        assert a.nbytes == self.nbytes
        if self.nbytes:
            _cudart_memcpy(self.ptr, a.ctypes.data, self.nbytes, 1)

    def zero(self) -> None:
        self.set(np.zeros(self.shape, self.dtype))

    def get(self) -> np.ndarray:
        out = np.empty(self.shape, self.dtype)
        if self.nbytes:
            _cudart_memcpy(out.ctypes.data, self.ptr, self.nbytes, 2)
        return out

    def __del__(self):
        try:
            lib.zsph_device_free(self.ptr)
        except Exception:
            pass


MLP_IN, MLP_HID, MLP_OUT, MLP_NPARAM, MLP_NPARTIAL, MLP_TILE = 32, 128, 4, 21252, 21256, 128


class Mlp:
    """The learned-corrector network (zsph_mlp_*): tensor-core forward,
    backward and Adam on the current device."""

    def __init__(self, seed: int = 0):
        self.h = _VP()
        check(lib.zsph_mlp_create(int(seed), ctypes.byref(self.h)))

    def close(self) -> None:
        if self.h:
            lib.zsph_mlp_destroy(self.h)
            self.h = _VP()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def params(self) -> np.ndarray:
        out = np.empty(MLP_NPARAM, np.float32)
        check(lib.zsph_mlp_get_params(self.h, out.ctypes.data))
        return out

    @params.setter
    def params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == MLP_NPARAM
        check(lib.zsph_mlp_set_params(self.h, p.ctypes.data))

    def moments(self):
        m1, m2, st = np.empty(MLP_NPARAM, np.float32), np.empty(MLP_NPARAM, np.float32), ctypes.c_int(0)
        check(lib.zsph_mlp_get_moments(self.h, m1.ctypes.data, m2.ctypes.data, ctypes.byref(st)))
        return m1, m2, st.value

    @property
    def norm(self) -> dict:
        v = {k: np.zeros(n, np.float32) for k, n in (("in_mean", 32), ("in_inv_std", 32), ("out_mean", 4),
                                                       ("out_std", 4))}
        check(lib.zsph_mlp_get_norm(self.h, v["in_mean"].ctypes.data, v["in_inv_std"].ctypes.data,
                                    v["out_mean"].ctypes.data, v["out_std"].ctypes.data))
        return v

    @norm.setter
    def norm(self, v: dict) -> None:
        a = {k: np.ascontiguousarray(v[k], np.float32) for k in ("in_mean", "in_inv_std", "out_mean", "out_std")}
        check(lib.zsph_mlp_set_norm(self.h, a["in_mean"].ctypes.data, a["in_inv_std"].ctypes.data,
                                    a["out_mean"].ctypes.data, a["out_std"].ctypes.data))

    def set_moments(self, m1, m2, step: int) -> None:
        m1, m2 = np.ascontiguousarray(m1, np.float32), np.ascontiguousarray(m2, np.float32)
        check(lib.zsph_mlp_set_moments(self.h, m1.ctypes.data, m2.ctypes.data, int(step)))

    @staticmethod
    def pack(rows: DeviceArray, n: int, mean=None, inv_std=None) -> DeviceArray:
        tiles = DeviceArray(((n + MLP_TILE - 1) // MLP_TILE, 4096), np.uint16)
        mv = None if mean is None else np.ascontiguousarray(mean, np.float32)
        sv = None if inv_std is None else np.ascontiguousarray(inv_std, np.float32)
        check(lib.zsph_mlp_pack(rows.ptr, int(n), None if mv is None else mv.ctypes.data,
                                None if sv is None else sv.ctypes.data, tiles.ptr, None))
        _cudart_sync()
        return tiles

    def forward(self, tiles: DeviceArray, n: int) -> np.ndarray:
        out = DeviceArray((n, 4), np.float32)
        check(lib.zsph_mlp_forward(self.h, tiles.ptr, int(n), out.ptr, None))
        return out.get()

    def grad(self, tiles: DeviceArray, y: DeviceArray, w: DeviceArray, ntiles: int, inv_wsum: float,
             tile_ids: DeviceArray | None = None):
        """Returns (partial rows as a DeviceArray, number of rows)."""
        partial = DeviceArray((max(ntiles, 1) if ntiles < 512 else 512, MLP_NPARTIAL), np.float32)
        nparts = ctypes.c_int(0)
        check(lib.zsph_mlp_grad(self.h, tiles.ptr, y.ptr, w.ptr, None if tile_ids is None else tile_ids.ptr,
                                int(ntiles), float(inv_wsum), partial.ptr, ctypes.byref(nparts), None))
        return partial, nparts.value

    def adam(self, partial: DeviceArray, nparts: int, lr: float = 1e-3, beta1: float = 0.9, beta2: float = 0.999,
             eps: float = 1e-8) -> None:
        check(lib.zsph_mlp_adam(self.h, partial.ptr, int(nparts), float(lr), float(beta1), float(beta2), float(eps),
                                None))
        _cudart_sync()
