"""Case constants in the reference's ``meshMessage`` layout.

``mesh_message`` restates ``meshImport::setMeshMessage`` and
``setParticleMessage`` (src/meshImport.cpp:1273-1405) operation for
operation, with the constants the reference hard-codes (L0 = 3.912 m,
T_in = 142.2 K, T_w = 300 K at src/meshImport.cpp:1316-1318, 100 particles
per cell at src/meshImport.h:47) exposed as arguments.
"""
from __future__ import annotations

import math

import numpy as np

MESH_MESSAGE_DTYPE = np.dtype([
    ("Ncell", "<i4"), ("Nface", "<i4"), ("Npoint", "<i4"), ("Nk", "<i4"), ("bcnumber", "<i4"), ("Nghost", "<i4"),
    ("Area", "<f8"), ("Ma", "<f8"), ("Kn", "<f8"), ("cfl", "<f8"),
    ("gamma", "<f8"), ("dr", "<f8"), ("dv", "<f8"), ("zr", "<f8"), ("zv", "<f8"), ("omega", "<f8"),
    ("var", "<i4"), ("qn", "<i4"), ("f_tra", "<f8"), ("f_rot", "<f8"),
    ("delta_rp", "<f8"), ("delta_sm", "<f8"), ("omeag0", "<f8"), ("omeag1", "<f8"),
    ("cfl_ns", "<f8"), ("pr", "<f8"), ("cp", "<f8"), ("cv", "<f8"),
    ("kB", "<f8"), ("p_mass", "<f8"), ("p_mass_r", "<f8"), ("T_ref", "<f8"), ("n_ref", "<f8"),
    ("miu_ref", "<f8"), ("Twall_ref", "<f8"), ("p_ref", "<f8"), ("d_ref", "<f8"),
    ("alpha", "<f8"), ("v_rms", "<f8"), ("eta", "<f8"), ("P_relax", "<f8"), ("dt_ref", "<f8"),
    ("T_in", "<f8"), ("v_in", "<f8"), ("eNface", "<i4"), ("iNface", "<i4"), ("Neff", "<f8"), ("dtime", "<f8"),
], align=True)
assert MESH_MESSAGE_DTYPE.itemsize == 344

REFERENCE_L0 = 3.912
REFERENCE_T_IN = 142.2
REFERENCE_T_WALL = 300.0
REFERENCE_PPC = 100


def mesh_message(dm, Ma: float, Kn: float, ppc: int = REFERENCE_PPC, L0: float = REFERENCE_L0,
                 T_in: float = REFERENCE_T_IN, T_wall: float = REFERENCE_T_WALL,
                 cfl: float = 1e2, cfl_ns: float = 5.0) -> np.ndarray:
    """meshMessage for mesh ``dm`` (a pydsmc.mesh.DsmcMesh)."""
    m = np.zeros((), dtype=MESH_MESSAGE_DTYPE)
    pi = math.pi
    dr, dv, zr = 2.0, 1.626, 3.5
    zv = 2 * zr
    omega = 0.74
    f_tra, f_rot = 2.365, 1.435
    gamma = (5.0 + dr) / (3.0 + dr)
    delta_rp = math.pow(pi * 0.5, 0.5) / Kn
    delta_sm = 1.0 / 1.33
    omeag0 = 1.0 - 2.0 * zr * (2.5 / f_tra - 1.0)
    omeag1 = 1 - (1 / (f_rot * delta_sm) - 1) * (delta_sm / (1 - delta_sm)) * zr
    cv = 1 / (gamma - 1.0)
    cp = cv * gamma
    pr = (5.0 + dr) * 0.5 / (1.5 * f_tra + dr * 0.5 * f_rot)
    m["Ncell"] = dm.ncell
    m["Nface"] = dm.nface
    m["Npoint"] = dm.npoint
    m["Nk"] = 0
    m["bcnumber"] = dm.bcnumber
    m["Nghost"] = dm.ncell + dm.bcnumber
    m["Ma"] = Ma
    m["Kn"] = Kn
    m["cfl"] = cfl
    m["Area"] = dm.area_sum
    m["gamma"] = gamma
    m["omega"] = omega
    m["dr"] = dr
    m["dv"] = dv
    m["zr"] = zr
    m["zv"] = zv
    m["var"] = 6
    m["qn"] = 2
    m["cfl_ns"] = cfl_ns
    m["f_tra"] = f_tra
    m["f_rot"] = f_rot
    m["pr"] = pr
    m["delta_rp"] = delta_rp
    m["delta_sm"] = delta_sm
    m["omeag0"] = omeag0
    m["omeag1"] = omeag1
    m["cp"] = cp
    m["cv"] = cv
    m["eNface"] = dm.bcnumber
    m["iNface"] = dm.nface - dm.bcnumber
    kB, T_ref, p_mass = 1.3806e-23, 273.15, 4.65e-26
    p_mass_r = 0.5 * p_mass
    d_ref, alpha = 4.17e-10, 1.0
    Twall_ref = T_wall / T_ref
    eta = omega - 0.5
    v_rms = math.sqrt(2 * kB * T_ref / p_mass)
    v_in = math.sqrt(2 * kB * T_in / p_mass)
    d_ref2 = d_ref * d_ref
    miu_ref = (5.0 * (alpha + 1.0) * (alpha + 2.0) * math.sqrt(p_mass * kB * T_ref / pi)
               / 4.0 / alpha / (5.0 - 2.0 * omega) / (7.0 - 2.0 * omega) / d_ref2)
    miu_ref *= math.pow(T_in / T_ref, omega)
    p_ref = miu_ref / (Kn * L0) * math.sqrt(pi * kB / p_mass * T_in / 2.0)
    n_ref = p_ref / (kB * T_in)
    dt_ref = (1 / Kn) * math.sqrt(pi) / 2 * miu_ref / p_ref * math.sqrt(T_in / T_ref)
    m["kB"] = kB
    m["T_ref"] = T_ref
    m["T_in"] = T_in
    m["v_in"] = v_in
    m["n_ref"] = n_ref
    m["p_ref"] = p_ref
    m["d_ref"] = d_ref
    m["p_mass"] = p_mass
    m["p_mass_r"] = p_mass_r
    m["miu_ref"] = miu_ref
    m["v_rms"] = v_rms
    m["eta"] = eta
    m["Twall_ref"] = Twall_ref
    m["alpha"] = alpha
    m["P_relax"] = 0.18
    m["dt_ref"] = dt_ref
    nps = int(ppc) * dm.ncell
    m["Neff"] = dm.area_sum * n_ref / nps
    m["dtime"] = dm.min_edge * 0.2
    return m


def inflow_direction(aoa_deg: float) -> tuple[float, float]:
    """Unit drift direction (x, y) of the freestream inlet.

    The reference hard-codes a 30 degree angle of attack as the factors
    ``sqrt(3)/2`` and ``1/2`` (src/ProcessDSMC.cpp:2330-2331); for that angle
    the same two doubles are returned, so the drift velocity is bit-identical
    (multiplying by ``sqrt(3)/2`` equals multiplying by ``sqrt(3)`` and
    halving, as halving is exact)."""
    if aoa_deg == 30.0:
        return (math.sqrt(3.0) / 2.0, 0.5)
    a = math.radians(aoa_deg)
    return (math.cos(a), math.sin(a))
