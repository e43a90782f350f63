"""ctypes binding of the C ABI in include/dsmc_gpu.h.

This is how the tests, the smoke check and the bench drive the CUDA library:
every call goes through the same extern "C" entry points a C or C++ host
(the reference's ProcessDSMC callers) would use. There is no Python or CPU
fallback: if ``libdsmcgpu.so`` is missing or cannot be loaded, loading fails
with an error.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .case import MESH_MESSAGE_DTYPE
from .mesh import DSMC_CELL_DTYPE, DSMC_EDGE_DTYPE, DsmcMesh

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libdsmcgpu.so")

PRECISION_FP64 = 0
PRECISION_MIXED = 1

ROLE_NONE, ROLE_INTERFACE, ROLE_INLET, ROLE_OUTLET, ROLE_WALL, ROLE_SPECULAR = range(6)

STAGE_INJECT, STAGE_MOVE, STAGE_SORT, STAGE_COLLIDE, STAGE_SAMPLE = 1, 2, 4, 8, 16
STAGE_ALL = 31

MACRO_LOCAL, MACRO_RECORD, MACRO_FINAL_RECORD = 0, 1, 2

MAX_ZONES = 16
NOALLOC_MAX_TRACE = 32768


class CaseParams(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("nss", C.c_int32), ("nscheme", C.c_int32), ("nevery", C.c_int32),
        ("nrepeat", C.c_int32), ("wall_stats", C.c_int32), ("inflow_dir", C.c_double * 2),
        ("nzones", C.c_int32), ("zone_tag", C.c_int32 * MAX_ZONES), ("zone_role", C.c_int32 * MAX_ZONES),
        ("zone_inject", C.c_int32 * MAX_ZONES), ("capacity", C.c_int64), ("seed", C.c_uint64),
        ("max_crossings", C.c_int32), ("keep_step_moments", C.c_int32),
    ]


class MeshDesc(C.Structure):
    _fields_ = [
        ("ncell", C.c_int32), ("nface", C.c_int32), ("npoint", C.c_int32),
        ("cells", C.c_void_p), ("edges", C.c_void_p), ("localPointXY", C.c_void_p), ("faceSplitTag", C.c_void_p),
    ]


COUNTER_NAMES = ["steps", "injected", "removed", "dropped", "lost", "wall_hits", "crossings",
                 "candidate_pairs", "collisions", "fp64_fallbacks", "overflow", "big_cells"]


class Counters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in COUNTER_NAMES]


class GsisReport(C.Structure):
    _fields_ = [("nan_cell", C.c_int32), ("cells_updated", C.c_int32), ("cells_skipped", C.c_int32),
                ("pad", C.c_int32), ("added", C.c_int64), ("removed", C.c_int64), ("particles", C.c_int64)]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_ if n != "pad"}


class LaunchShape(C.Structure):
    _fields_ = [("move_threads", C.c_int32), ("move_blocks_per_sm", C.c_int32),
                ("sort_blocks_per_sm", C.c_int32), ("collide_blocks_per_sm", C.c_int32),
                ("stay_per_thread", C.c_int32)]

    def as_dict(self):
        return {n: int(getattr(self, n)) for n, _ in self._fields_}


_lib = None

# (name, restype, argtypes) for every entry point of include/dsmc_gpu.h
_P = C.c_void_p
_SIGS = [
    ("dsmc_default_params", None, [_P]),
    ("dsmc_create", C.c_int, [_P, _P, _P, C.c_int, C.POINTER(C.c_void_p)]),
    ("dsmc_destroy", None, [_P]),
    ("dsmc_last_error", C.c_char_p, [_P]),
    ("dsmc_upload_particles", C.c_int, [_P, C.c_int64] + [_P] * 8),
    ("dsmc_particle_count", C.c_int, [_P, C.POINTER(C.c_int64)]),
    ("dsmc_fill_initial", C.c_int, [_P, C.c_double, C.c_uint64]),
    ("dsmc_fill_freestream", C.c_int, [_P, C.c_double, C.c_uint64]),
    ("dsmc_molecular_velocity_change", C.c_int, [_P, _P, _P, _P]),
    ("dsmc_download_particles", C.c_int, [_P, C.c_int64] + [_P] * 9),
    ("dsmc_step", C.c_int, [_P, C.c_int32, C.c_uint32]),
    ("dsmc_preprocesseffquad", C.c_int, [_P, C.c_int32]),
    ("dsmc_advection", C.c_int, [_P, C.c_int32]),
    ("dsmc_cache2chain", C.c_int, [_P]),
    ("dsmc_collisionDSMC", C.c_int, [_P]),
    ("dsmc_statistic_macro", C.c_int, [_P, C.c_int32]),
    ("dsmc_statistic_macroPre", C.c_int, [_P]),
    ("dsmc_download_macro", C.c_int, [_P, C.c_int32, _P]),
    ("dsmc_download_counts", C.c_int, [_P] + [_P] * 6),
    ("dsmc_download_step_moments", C.c_int, [_P, _P]),
    ("dsmc_download_wall", C.c_int, [_P, _P]),
    ("dsmc_download_cell_state", C.c_int, [_P, _P, _P, _P]),
    ("dsmc_upload_cell_state", C.c_int, [_P, _P, _P, _P]),
    ("dsmc_upload_sparse_state", C.c_int, [_P, _P]),
    ("dsmc_get_counters", C.c_int, [_P, _P]),
    ("dsmc_trace", C.c_int, [_P, C.c_int64] + [_P] * 8 + [C.c_int32] + [_P] * 12),
    ("dsmc_trace_noalloc", C.c_int, [_P, C.c_int64] + [_P] * 8 + [C.c_int32] + [_P] * 12),
    ("dsmc_set_timing", C.c_int, [_P, C.c_int32]),
    ("dsmc_stage_ms", C.c_int, [_P, _P, C.POINTER(C.c_int64), C.c_int32]),
    ("dsmc_stream", C.c_void_p, [_P]),
    ("dsmc_sync", C.c_int, [_P]),
    ("dsmc_get_launch_shape", C.c_int, [_P, _P]),
    ("dsmc_set_launch_shape", C.c_int, [_P, _P]),
    ("dsmc_autotune", C.c_int, [_P, C.c_int32, C.c_int32, C.POINTER(C.c_int32), _P]),
    ("dsmc_batch_create", C.c_int, [_P, C.c_int32, C.POINTER(C.c_void_p)]),
    ("dsmc_batch_destroy", None, [_P]),
    ("dsmc_batch_last_error", C.c_char_p, [_P]),
    ("dsmc_batch_step", C.c_int, [_P, C.c_int32]),
    ("dsmc_batch_stream", C.c_void_p, [_P]),
    ("dsmc_batch_sync", C.c_int, [_P]),
]
EXPORTED = [s[0] for s in _SIGS]


def lib_path() -> str:
    return LIB_PATH


def load(path: str | None = None):
    """Load libdsmcgpu.so, LIB_PATH unless a path is given (raises OSError if
    it is not built). The library of the default path is loaded once."""
    global _lib
    p = os.path.abspath(path or LIB_PATH)
    if _lib is not None and path is None and p == os.path.abspath(LIB_PATH):
        return _lib
    if not os.path.exists(p):
        raise OSError(f"{p} not built: run __graft_entry__.build()")
    lib = C.CDLL(p)
    for name, res, args in _SIGS:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def default_params(**over) -> CaseParams:
    lib = load()
    p = CaseParams()
    lib.dsmc_default_params(C.byref(p))
    zones = over.pop("zones", None)
    for k, v in over.items():
        if k == "inflow_dir":
            p.inflow_dir[0], p.inflow_dir[1] = v
        else:
            setattr(p, k, v)
    if zones is not None:
        # zones: list of (tag, role, inject)
        p.nzones = len(zones)
        for i, (tag, role, inj) in enumerate(zones):
            p.zone_tag[i] = tag
            p.zone_role[i] = role
            p.zone_inject[i] = int(inj)
    return p


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class DsmcError(RuntimeError):
    pass


class Case:
    """One DSMC case resident on a GPU, driven through the C ABI."""

    def __init__(self, mesh: DsmcMesh, mess: np.ndarray, params: CaseParams | None = None, device: int = 0):
        self.lib = load()
        self.mesh = mesh
        self._cells = np.ascontiguousarray(mesh.cells, dtype=DSMC_CELL_DTYPE)
        self._edges = np.ascontiguousarray(mesh.edges, dtype=DSMC_EDGE_DTYPE)
        self._pts = np.ascontiguousarray(mesh.points, dtype=np.float64)
        self._split = np.ascontiguousarray(mesh.split, dtype=np.uint8)
        self.mess = np.ascontiguousarray(np.asarray(mess, dtype=MESH_MESSAGE_DTYPE).reshape(()))
        self.params = params if params is not None else default_params()
        desc = MeshDesc(mesh.ncell, mesh.nface, mesh.npoint, _ptr(self._cells), _ptr(self._edges),
                        _ptr(self._pts), _ptr(self._split))
        h = C.c_void_p()
        rc = self.lib.dsmc_create(C.byref(desc), self.mess.ctypes.data_as(C.c_void_p), C.byref(self.params),
                                  device, C.byref(h))
        if rc != 0:
            raise DsmcError(f"dsmc_create failed ({rc}): {self.lib.dsmc_last_error(None).decode()}")
        self.h = h
        self.ncell = mesh.ncell
        self.nface = mesh.nface

    # -- plumbing -----------------------------------------------------------
    def _check(self, rc: int, what: str):
        if rc != 0:
            msg = self.lib.dsmc_last_error(self.h).decode()
            raise DsmcError(f"{what} failed ({rc}): {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.dsmc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- particles ------------------------------------------------------------
    def upload_particles(self, x, v, ir, cell):
        x = np.ascontiguousarray(x, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        ir = np.ascontiguousarray(ir, dtype=np.float64)
        cell = np.ascontiguousarray(cell, dtype=np.int32)
        n = cell.shape[0]
        cols = [np.ascontiguousarray(x[:, k]) for k in range(3)] + [np.ascontiguousarray(v[:, k]) for k in range(3)]
        self._check(self.lib.dsmc_upload_particles(self.h, n, *[_ptr(c) for c in cols], _ptr(ir), _ptr(cell)),
                    "dsmc_upload_particles")

    def upload_columns(self, px, py, pz, vx, vy, vz, ir, cell):
        """upload_particles with positions and velocities as the C ABI's
        separate columns: no copy is made of a column that is already a
        contiguous float64 array (cell: int32)."""
        cols = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in (px, py, pz, vx, vy, vz, ir)]
        cell = np.ascontiguousarray(cell, dtype=np.int32).reshape(-1)
        n = cell.shape[0]
        if any(c.shape[0] != n for c in cols):
            raise ValueError("every column needs one value per particle")
        self._check(self.lib.dsmc_upload_particles(self.h, n, *[_ptr(c) for c in cols], _ptr(cell)),
                    "dsmc_upload_particles")

    def particle_count(self) -> int:
        n = C.c_int64()
        self._check(self.lib.dsmc_particle_count(self.h, C.byref(n)), "dsmc_particle_count")
        return int(n.value)

    def download_particles(self):
        n = self.particle_count()
        arrs = [np.empty(n) for _ in range(7)]
        cell = np.empty(n, dtype=np.int32)
        pid = np.empty(n, dtype=np.uint32)
        self._check(self.lib.dsmc_download_particles(self.h, n, *[_ptr(a) for a in arrs], _ptr(cell), _ptr(pid)),
                    "dsmc_download_particles")
        return (np.stack(arrs[:3], 1), np.stack(arrs[3:6], 1), arrs[6], cell)

    # -- stages -----------------------------------------------------------------
    def step(self, istep: int, stages: int = STAGE_ALL):
        self._check(self.lib.dsmc_step(self.h, istep, stages), "dsmc_step")

    def preprocesseffquad(self, istep):
        self._check(self.lib.dsmc_preprocesseffquad(self.h, istep), "dsmc_preprocesseffquad")

    def advection(self, istep):
        self._check(self.lib.dsmc_advection(self.h, istep), "dsmc_advection")

    def cache2chain(self):
        self._check(self.lib.dsmc_cache2chain(self.h), "dsmc_cache2chain")

    def collisionDSMC(self):
        self._check(self.lib.dsmc_collisionDSMC(self.h), "dsmc_collisionDSMC")

    def statistic_macro(self, istep):
        self._check(self.lib.dsmc_statistic_macro(self.h, istep), "dsmc_statistic_macro")

    def statistic_macroPre(self):
        self._check(self.lib.dsmc_statistic_macroPre(self.h), "dsmc_statistic_macroPre")

    def sync(self):
        self._check(self.lib.dsmc_sync(self.h), "dsmc_sync")

    # -- outputs ----------------------------------------------------------------
    def macro(self, which: int) -> np.ndarray:
        out = np.empty((self.ncell, 18))
        self._check(self.lib.dsmc_download_macro(self.h, which, _ptr(out)), "dsmc_download_macro")
        return out

    def counts(self) -> dict:
        nc = self.ncell
        ppc = np.empty(nc, dtype=np.int32)
        ws = np.empty(nc)
        wv = np.empty(nc, dtype=np.int8)
        ss = np.empty(nc, dtype=np.uint8)
        sr = np.empty(nc)
        st = np.empty(nc)
        self._check(self.lib.dsmc_download_counts(self.h, _ptr(ppc), _ptr(ws), _ptr(wv), _ptr(ss), _ptr(sr), _ptr(st)),
                    "dsmc_download_counts")
        return {"ppc": ppc, "window_samples": ws, "window_valid": wv, "sparse_state": ss,
                "stepinter_rho": sr, "steady_rho": st}

    def step_moments(self) -> np.ndarray:
        out = np.empty((self.ncell, 18))
        self._check(self.lib.dsmc_download_step_moments(self.h, _ptr(out)), "dsmc_download_step_moments")
        return out

    def wall(self) -> np.ndarray:
        out = np.empty((self.nface, 6))
        self._check(self.lib.dsmc_download_wall(self.h, _ptr(out)), "dsmc_download_wall")
        return out

    def cell_state(self):
        cr, rc, ri = np.empty(self.ncell), np.empty(self.ncell), np.empty(self.ncell)
        self._check(self.lib.dsmc_download_cell_state(self.h, _ptr(cr), _ptr(rc), _ptr(ri)), "dsmc_download_cell_state")
        return cr, rc, ri

    def set_cell_state(self, crmax=None, rem_coll=None, rem_inj=None):
        f = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        crmax, rem_coll, rem_inj = f(crmax), f(rem_coll), f(rem_inj)
        self._check(self.lib.dsmc_upload_cell_state(self.h, _ptr(crmax), _ptr(rem_coll), _ptr(rem_inj)),
                    "dsmc_upload_cell_state")

    def set_sparse_state(self, sparse_state):
        """Write back the per-cell sparse-sample states (0 normal, 1
        accumulating, 2 released) the host's GSIS exchange decided."""
        ss = np.ascontiguousarray(sparse_state, dtype=np.uint8).reshape(-1)
        if ss.shape[0] != self.ncell:
            raise ValueError("one sparse state per cell")
        self._check(self.lib.dsmc_upload_sparse_state(self.h, _ptr(ss)), "dsmc_upload_sparse_state")

    def counters(self) -> dict:
        c = Counters()
        self._check(self.lib.dsmc_get_counters(self.h, C.byref(c)), "dsmc_get_counters")
        return {n: int(getattr(c, n)) for n in COUNTER_NAMES}

    def set_timing(self, on: bool):
        self._check(self.lib.dsmc_set_timing(self.h, int(on)), "dsmc_set_timing")

    def stage_ms(self, reset: bool = False):
        ms = np.zeros(5)
        n = C.c_int64()
        self._check(self.lib.dsmc_stage_ms(self.h, _ptr(ms), C.byref(n), int(reset)), "dsmc_stage_ms")
        return ms, int(n.value)

    def trace(self, x, v, dt, cell, stop_at_wall: bool = True, noalloc: bool = False):
        """The move kernel's trace on given particles (dsmc_trace, or
        dsmc_trace_noalloc with noalloc=True)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        v = np.ascontiguousarray(v, dtype=np.float64)
        dt = np.ascontiguousarray(dt, dtype=np.float64)
        cell = np.ascontiguousarray(cell, dtype=np.int32)
        n = cell.shape[0]
        cols = [np.ascontiguousarray(x[:, k]) for k in range(3)] + [np.ascontiguousarray(v[:, k]) for k in range(3)]
        oi = [np.empty(n, dtype=np.int32) for _ in range(5)]
        of = [np.empty(n) for _ in range(7)]
        fn = self.lib.dsmc_trace_noalloc if noalloc else self.lib.dsmc_trace
        self._check(fn(self.h, n, *[_ptr(c) for c in cols], _ptr(dt), _ptr(cell), int(stop_at_wall),
                       *[_ptr(a) for a in oi], *[_ptr(a) for a in of]),
                    "dsmc_trace_noalloc" if noalloc else "dsmc_trace")
        return {"cell": oi[0], "ifout": oi[1], "face": oi[2], "tri": oi[3], "ncross": oi[4],
                "x": np.stack(of[:3], 1), "v": np.stack(of[3:6], 1), "dt": of[6]}

    def fill_initial(self, ppc_mean: float, seed: int = 0):
        """The reference's initial fill on the device (dsmc_fill_initial)."""
        self._check(self.lib.dsmc_fill_initial(self.h, float(ppc_mean), int(seed)), "dsmc_fill_initial")

    def fill_freestream(self, ppc_mean: float, seed: int = 0):
        """The initial fill with the case's freestream (dsmc_fill_freestream)."""
        self._check(self.lib.dsmc_fill_freestream(self.h, float(ppc_mean), int(seed)), "dsmc_fill_freestream")

    def molecular_velocity_change(self, nsresult, accepted=None) -> dict:
        """GSIS particle update (dsmc_molecular_velocity_change); nsresult
        [ncell, 6], accepted [ncell] or None."""
        ns = np.ascontiguousarray(nsresult, dtype=np.float64).reshape(-1, 6)
        acc = None if accepted is None else np.ascontiguousarray(accepted, dtype=np.int8)
        rep = GsisReport()
        self._check(self.lib.dsmc_molecular_velocity_change(self.h, _ptr(ns), None if acc is None else _ptr(acc),
                                                            C.byref(rep)), "dsmc_molecular_velocity_change")
        return rep.as_dict()

    # -- launch shapes ----------------------------------------------------------
    def launch_shape(self) -> dict:
        sh = LaunchShape()
        self._check(self.lib.dsmc_get_launch_shape(self.h, C.byref(sh)), "dsmc_get_launch_shape")
        return sh.as_dict()

    def set_launch_shape(self, **kw):
        sh = LaunchShape()
        self._check(self.lib.dsmc_get_launch_shape(self.h, C.byref(sh)), "dsmc_get_launch_shape")
        for k, v in kw.items():
            setattr(sh, k, v)
        self._check(self.lib.dsmc_set_launch_shape(self.h, C.byref(sh)), "dsmc_set_launch_shape")

    def autotune(self, first_istep: int, trial_steps: int = 2):
        """Run steps first_istep, ... while timing launch shapes; returns
        (next step to run, shape kept)."""
        nxt = C.c_int32()
        sh = LaunchShape()
        self._check(self.lib.dsmc_autotune(self.h, first_istep, trial_steps, C.byref(nxt), C.byref(sh)),
                    "dsmc_autotune")
        return int(nxt.value), sh.as_dict()


class Batch:
    """Independent cases on one device stepped together: each batch step is
    one CUDA graph whose branches are the cases' steps (dsmc_batch_*)."""

    def __init__(self, cases):
        self.lib = load()
        self.cases = list(cases)
        arr = (C.c_void_p * len(self.cases))(*[c.h for c in self.cases])
        b = C.c_void_p()
        rc = self.lib.dsmc_batch_create(arr, len(self.cases), C.byref(b))
        if rc != 0:
            raise DsmcError(f"dsmc_batch_create failed ({rc}): {self.lib.dsmc_batch_last_error(None).decode()}")
        self.b = b

    def _check(self, rc, what):
        if rc != 0:
            raise DsmcError(f"{what} failed ({rc}): {self.lib.dsmc_batch_last_error(self.b).decode()}")

    def step(self, nsteps: int = 1):
        self._check(self.lib.dsmc_batch_step(self.b, nsteps), "dsmc_batch_step")

    def sync(self):
        self._check(self.lib.dsmc_batch_sync(self.b), "dsmc_batch_sync")

    def stream(self):
        return self.lib.dsmc_batch_stream(self.b)

    def close(self):
        if getattr(self, "b", None):
            self.lib.dsmc_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
