"""ctypes binding of the C restatement oracle (oracle/dsmc_oracle.c).
ORACLE TEST INFRASTRUCTURE: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg only."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libdsmc_oracle.so")
_lib = None
_P = C.c_void_p


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise OSError(f"{LIB} not built: make -C oracle")
        lib = C.CDLL(LIB)
        lib.oracle_create.restype = _P
        lib.oracle_create.argtypes = [C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P, C.c_int, _P, _P, _P,
                                      C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_uint64, C.c_int]
        lib.oracle_destroy.argtypes = [_P]
        lib.oracle_philox.argtypes = [_P, _P, _P]
        lib.oracle_trace.argtypes = [_P, C.c_int64] + [_P] * 8 + [C.c_int] + [_P] * 12
        lib.oracle_set_particles.restype = C.c_int
        lib.oracle_set_particles.argtypes = [_P, C.c_int64] + [_P] * 8
        lib.oracle_count.restype = C.c_int64
        lib.oracle_count.argtypes = [_P]
        lib.oracle_get_particles.argtypes = [_P] + [_P] * 8
        lib.oracle_step.restype = C.c_int
        lib.oracle_step.argtypes = [_P, C.c_int, C.c_uint]
        lib.oracle_macro_pre.argtypes = [_P]
        lib.oracle_get_macro.argtypes = [_P, C.c_int, _P]
        lib.oracle_get_step_moments.argtypes = [_P, _P]
        lib.oracle_get_acc.argtypes = [_P, _P]
        lib.oracle_get_cell_state.argtypes = [_P, _P, _P, _P]
        lib.oracle_set_cell_state.argtypes = [_P, _P, _P, _P]
        lib.oracle_set_sparse_state.restype = C.c_int
        lib.oracle_set_sparse_state.argtypes = [_P, _P]
        lib.oracle_get_counts.argtypes = [_P, _P, _P, _P, _P]
        lib.oracle_get_wall.argtypes = [_P, _P]
        lib.oracle_counters.argtypes = [_P, _P]
        lib.oracle_placement.restype = C.c_int
        lib.oracle_placement.argtypes = [_P, _P, _P, _P]
        lib.oracle_fill.restype = C.c_int
        lib.oracle_fill.argtypes = [_P, C.c_double, C.c_uint64, C.c_int]
        lib.oracle_molecular_velocity_change.restype = C.c_int
        lib.oracle_molecular_velocity_change.argtypes = [_P, _P, _P, _P]
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def philox(ctr, key) -> np.ndarray:
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    load().oracle_philox(_p(c), _p(k), _p(out))
    return out


class Oracle:
    """The FP64 CPU restatement of the DSMC step on one mesh."""

    def __init__(self, dm, mess, params):
        """params: a pydsmc.gpu.CaseParams-like object (zone table, controls,
        seed) so the oracle and the GPU case run the same configuration."""
        self.lib = load()
        self.dm = dm
        self._keep = [np.ascontiguousarray(dm.cells), np.ascontiguousarray(dm.edges),
                      np.ascontiguousarray(dm.points, dtype=np.float64), np.ascontiguousarray(dm.split, dtype=np.uint8),
                      np.ascontiguousarray(np.asarray(mess).reshape(()))]
        nz = int(params.nzones)
        zt = np.array([params.zone_tag[i] for i in range(nz)], dtype=np.int32)
        zr = np.array([params.zone_role[i] for i in range(nz)], dtype=np.int32)
        zi = np.array([params.zone_inject[i] for i in range(nz)], dtype=np.int32)
        self._keep += [zt, zr, zi]
        self.h = self.lib.oracle_create(dm.ncell, dm.nface, dm.npoint, *[_p(a) for a in self._keep[:5]], nz,
                                        _p(zt), _p(zr), _p(zi), float(params.inflow_dir[0]),
                                        float(params.inflow_dir[1]), int(params.nss), int(params.nscheme),
                                        int(params.nevery), int(params.nrepeat), int(params.wall_stats),
                                        int(params.seed), int(params.max_crossings))
        if not self.h:
            raise RuntimeError("oracle_create failed")
        self.ncell, self.nface = dm.ncell, dm.nface

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_destroy(self.h)
            self.h = None

    def trace(self, x, v, dt, cell, stop_at_wall=True):
        n = int(np.asarray(cell).shape[0])
        cols = [np.ascontiguousarray(x[:, k], dtype=np.float64) for k in range(3)] + \
               [np.ascontiguousarray(v[:, k], dtype=np.float64) for k in range(3)]
        dt = np.ascontiguousarray(dt, dtype=np.float64)
        cell = np.ascontiguousarray(cell, dtype=np.int32)
        oi = [np.empty(n, dtype=np.int32) for _ in range(5)]
        of = [np.empty(n) for _ in range(7)]
        self.lib.oracle_trace(self.h, n, *[_p(c) for c in cols], _p(dt), _p(cell), int(stop_at_wall),
                              *[_p(a) for a in oi], *[_p(a) for a in of])
        return {"cell": oi[0], "ifout": oi[1], "face": oi[2], "tri": oi[3], "ncross": oi[4],
                "x": np.stack(of[:3], 1), "v": np.stack(of[3:6], 1), "dt": of[6]}

    def set_particles(self, x, v, ir, cell):
        cols = [np.ascontiguousarray(x[:, k], dtype=np.float64) for k in range(3)] + \
               [np.ascontiguousarray(v[:, k], dtype=np.float64) for k in range(3)]
        ir = np.ascontiguousarray(ir, dtype=np.float64)
        cell = np.ascontiguousarray(cell, dtype=np.int32)
        rc = self.lib.oracle_set_particles(self.h, cell.shape[0], *[_p(c) for c in cols], _p(ir), _p(cell))
        if rc:
            raise RuntimeError(f"oracle_set_particles failed {rc}")

    def particles(self):
        n = int(self.lib.oracle_count(self.h))
        a = [np.empty(n) for _ in range(7)]
        c = np.empty(n, dtype=np.int32)
        self.lib.oracle_get_particles(self.h, *[_p(x) for x in a], _p(c))
        return np.stack(a[:3], 1), np.stack(a[3:6], 1), a[6], c

    def step(self, istep, stages=31):
        rc = self.lib.oracle_step(self.h, int(istep), int(stages))
        if rc:
            raise RuntimeError(f"oracle_step failed {rc}")

    def macro_pre(self):
        self.lib.oracle_macro_pre(self.h)

    def macro(self, which):
        out = np.empty((self.ncell, 18))
        self.lib.oracle_get_macro(self.h, int(which), _p(out))
        return out

    def step_moments(self):
        out = np.empty((self.ncell, 18))
        self.lib.oracle_get_step_moments(self.h, _p(out))
        return out

    def acc(self):
        out = np.empty((self.ncell, 54))
        self.lib.oracle_get_acc(self.h, _p(out))
        return out

    def cell_state(self):
        a, b, c = np.empty(self.ncell), np.empty(self.ncell), np.empty(self.ncell)
        self.lib.oracle_get_cell_state(self.h, _p(a), _p(b), _p(c))
        return a, b, c

    def counts(self):
        ppc = np.empty(self.ncell, dtype=np.int32)
        ws = np.empty(self.ncell)
        wv = np.empty(self.ncell, dtype=np.int8)
        ss = np.empty(self.ncell, dtype=np.uint8)
        self.lib.oracle_get_counts(self.h, _p(ppc), _p(ws), _p(wv), _p(ss))
        return {"ppc": ppc, "window_samples": ws, "window_valid": wv, "sparse_state": ss}

    def wall(self):
        out = np.empty((self.nface, 6))
        self.lib.oracle_get_wall(self.h, _p(out))
        return out

    def set_sparse_state(self, sparse_state):
        ss = np.ascontiguousarray(sparse_state, dtype=np.uint8)
        if self.lib.oracle_set_sparse_state(self.h, _p(ss)):
            raise ValueError("sparse state outside 0..2")

    def counters(self):
        out = np.zeros(8, dtype=np.uint64)
        self.lib.oracle_counters(self.h, _p(out))
        names = ["injected", "removed", "dropped", "lost", "wall_hits", "crossings", "candidate_pairs", "collisions"]
        return {k: int(v) for k, v in zip(names, out)}

    def placement(self):
        """Placement tetrahedra: offsets [ncell+1], vertices [nplace, 4, 3], volumes."""
        off = np.empty(self.ncell + 1, dtype=np.int32)
        n = int(self.lib.oracle_placement(self.h, _p(off), None, None))
        V = np.empty((n, 4, 3))
        vol = np.empty(n)
        self.lib.oracle_placement(self.h, _p(off), _p(V), _p(vol))
        return off, V, vol

    def fill(self, ppc_mean, seed, at_rest=True):
        rc = self.lib.oracle_fill(self.h, float(ppc_mean), int(seed), 1 if at_rest else 0)
        if rc:
            raise RuntimeError(f"oracle_fill failed {rc}")

    def molecular_velocity_change(self, ns, accepted=None):
        ns = np.ascontiguousarray(ns, dtype=np.float64).reshape(self.ncell, 6)
        acc = None if accepted is None else np.ascontiguousarray(accepted, dtype=np.int8)
        rep = np.zeros(6, dtype=np.int64)
        rc = self.lib.oracle_molecular_velocity_change(self.h, _p(ns), None if acc is None else _p(acc), _p(rep))
        if rc:
            raise RuntimeError(f"oracle_molecular_velocity_change failed {rc}")
        names = ["nan_cell", "cells_updated", "cells_skipped", "added", "removed", "particles"]
        return {k: int(v) for k, v in zip(names, rep)}
