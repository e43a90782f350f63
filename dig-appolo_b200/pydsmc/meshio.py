"""Binding of include/dsmc_meshio.h: the native Fluent case reader and DSMC
topology builder, the case constants, and the Fluent field writers of
libdsmcgpu.so (host code; no GPU needed)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import case as CS
from . import gpu
from . import mesh as M

_P = C.c_void_p


class Zone(C.Structure):
    _fields_ = [("section", C.c_int32), ("id", C.c_int32), ("first", C.c_int32), ("last", C.c_int32)]


class MeshDesc(C.Structure):
    _fields_ = [("ncell", C.c_int32), ("nface", C.c_int32), ("npoint", C.c_int32), ("cells", _P), ("edges", _P),
                ("localPointXY", _P), ("faceSplitTag", _P)]


ZONE_DTYPE = np.dtype([("section", "<i4"), ("id", "<i4"), ("first", "<i4"), ("last", "<i4")])

# (name, restype, argtypes) for every entry point of include/dsmc_meshio.h
_SIGS = [
    ("dsmc_mesh_read_cas", C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    ("dsmc_mesh_free", None, [_P]),
    ("dsmc_meshio_last_error", C.c_char_p, []),
    ("dsmc_mesh_get_desc", C.c_int, [_P, _P]),
    ("dsmc_mesh_get_zones", C.c_int, [_P, _P, C.c_int32, C.POINTER(C.c_int32)]),
    ("dsmc_mesh_get_stats", C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    ("dsmc_mesh_message", C.c_int, [_P, C.c_double, C.c_double, C.c_int32, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, _P]),
    ("dsmc_write_fluent_cells", C.c_int, [C.c_char_p, _P, _P, C.c_int32, _P, C.c_int32]),
    ("dsmc_write_fluent_wall", C.c_int, [C.c_char_p, _P, _P, _P, C.c_int32, _P, C.c_int32, _P, C.c_int32]),
    ("dsmc_out2dat", C.c_int, [_P, C.c_int32, _P, C.c_int32, C.c_char_p]),
    ("dsmc_out_boundary_stress_heat", C.c_int, [_P, C.c_int32, _P, C.c_int32, C.c_char_p]),
]
EXPORTED = [s[0] for s in _SIGS]

_lib = None


def load():
    global _lib
    if _lib is None:
        lib = gpu.load()
        for name, res, args in _SIGS:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class MeshIOError(RuntimeError):
    pass


def _check(rc, what):
    if rc != 0:
        raise MeshIOError(f"{what} failed ({rc}): {load().dsmc_meshio_last_error().decode()}")


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def zones_array(zones) -> np.ndarray:
    """Zone declarations as a ZONE_DTYPE array (from MeshFile.zones() or
    (section, id, first, last) tuples)."""
    if isinstance(zones, np.ndarray) and zones.dtype == ZONE_DTYPE:
        return np.ascontiguousarray(zones)
    return np.array([tuple(z) for z in zones], dtype=ZONE_DTYPE)


class MeshFile:
    """A mesh read from a Fluent ASCII case by the library (dsmc_mesh_read_cas)."""

    def __init__(self, path: str):
        lib = load()
        h = C.c_void_p()
        _check(lib.dsmc_mesh_read_cas(str(path).encode(), C.byref(h)), "dsmc_mesh_read_cas")
        self.h = h
        self.lib = lib

    def close(self):
        if getattr(self, "h", None):
            self.lib.dsmc_mesh_free(self.h)
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

    def dsmc_mesh(self) -> M.DsmcMesh:
        """Copies of the arrays as a pydsmc.mesh.DsmcMesh (what gpu.Case takes)."""
        d = MeshDesc()
        _check(self.lib.dsmc_mesh_get_desc(self.h, C.byref(d)), "dsmc_mesh_get_desc")
        cells = np.frombuffer((C.c_char * (d.ncell * M.DSMC_CELL_DTYPE.itemsize)).from_address(d.cells),
                              dtype=M.DSMC_CELL_DTYPE).copy()
        edges = np.frombuffer((C.c_char * (d.nface * M.DSMC_EDGE_DTYPE.itemsize)).from_address(d.edges),
                              dtype=M.DSMC_EDGE_DTYPE).copy()
        pts = np.frombuffer((C.c_double * (3 * d.npoint)).from_address(d.localPointXY), dtype=np.float64).copy()
        split = np.frombuffer((C.c_ubyte * d.nface).from_address(d.faceSplitTag), dtype=np.uint8).copy()
        area, me, bc = self.stats()
        return M.DsmcMesh(cells, edges, pts, split, area, me, bc)

    def zones(self) -> np.ndarray:
        n = C.c_int32()
        _check(self.lib.dsmc_mesh_get_zones(self.h, None, 0, C.byref(n)), "dsmc_mesh_get_zones")
        z = np.zeros(n.value, dtype=ZONE_DTYPE)
        _check(self.lib.dsmc_mesh_get_zones(self.h, _ptr(z), n.value, C.byref(n)), "dsmc_mesh_get_zones")
        return z

    def stats(self):
        a, m, b = C.c_double(), C.c_double(), C.c_int32()
        _check(self.lib.dsmc_mesh_get_stats(self.h, C.byref(a), C.byref(m), C.byref(b)), "dsmc_mesh_get_stats")
        return a.value, m.value, b.value

    def message(self, Ma: float, Kn: float, ppc: int = CS.REFERENCE_PPC, L0: float = CS.REFERENCE_L0,
                T_in: float = CS.REFERENCE_T_IN, T_wall: float = CS.REFERENCE_T_WALL, cfl: float = 1e2,
                cfl_ns: float = 5.0) -> np.ndarray:
        out = np.zeros((), dtype=CS.MESH_MESSAGE_DTYPE)
        _check(self.lib.dsmc_mesh_message(self.h, Ma, Kn, int(ppc), L0, T_in, T_wall, cfl, cfl_ns, _ptr(out)),
               "dsmc_mesh_message")
        return out


def write_fluent_cells(path: str, mess, zones, w) -> None:
    lib = load()
    m = np.ascontiguousarray(np.asarray(mess).reshape(()))
    z = zones_array(zones)
    w = np.ascontiguousarray(w, dtype=np.float64).reshape(-1, 18)
    _check(lib.dsmc_write_fluent_cells(str(path).encode(), _ptr(m), _ptr(z), len(z), _ptr(w), w.shape[0]),
           "dsmc_write_fluent_cells")


def write_fluent_wall(path: str, mess, params, zones, edges, tally, istep: int) -> None:
    lib = load()
    m = np.ascontiguousarray(np.asarray(mess).reshape(()))
    z = zones_array(zones)
    e = np.ascontiguousarray(edges)
    t = np.ascontiguousarray(tally, dtype=np.float64).reshape(-1, 6)
    _check(lib.dsmc_write_fluent_wall(str(path).encode(), _ptr(m), C.byref(params), _ptr(z), len(z), _ptr(e),
                                      e.shape[0], _ptr(t), int(istep)), "dsmc_write_fluent_wall")


def out2dat(case: "gpu.Case", istep: int, zones, path: str) -> None:
    """ProcessDSMC::out2dat for a case on the device (dsmc_out2dat)."""
    lib = load()
    z = zones_array(zones)
    case._check(lib.dsmc_out2dat(case.h, int(istep), _ptr(z), len(z), str(path).encode()), "dsmc_out2dat")


def out_boundary_stress_heat(case: "gpu.Case", istep: int, zones, path: str) -> None:
    """ProcessDSMC::outBoundaryStressHeat for a case on the device."""
    lib = load()
    z = zones_array(zones)
    case._check(lib.dsmc_out_boundary_stress_heat(case.h, int(istep), _ptr(z), len(z), str(path).encode()),
                "dsmc_out_boundary_stress_heat")
