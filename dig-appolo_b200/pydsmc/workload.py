"""Seeded synthetic inputs for the DSMC step: initial particle fills and the
tracing-check particle sets.

The reference fills cells from a macroscopic solution (NS2DSMC /
molecular_velocity_change, src/ProcessGSIS.cpp:2239-2354) with positions from
random barycentric points of sub-tetrahedra (velocityLocationGenerate,
src/MeshparticalInitial.cpp:688-721). The workloads here start from the
freestream Maxwellian instead, which is what the block and capsule cases
specify; positions are uniform in each cell.
"""
from __future__ import annotations

import math

import numpy as np

from .mesh import DsmcMesh


def freestream(mess, inflow_dir) -> tuple[np.ndarray, float, float]:
    """Drift velocity (normalised by v_rms), per-component thermal sigma and
    normalised temperature of the inlet gas (computeBoundaryGasState,
    src/ProcessDSMC.cpp:2318-2367)."""
    base = 1.0 * float(mess["Ma"]) * math.sqrt(float(mess["gamma"]) / 2.0) * float(mess["v_in"]) / float(mess["v_rms"])
    u = np.array([base * inflow_dir[0], base * inflow_dir[1], 0.0])
    tN = float(mess["T_in"]) / float(mess["T_ref"])
    return u, math.sqrt(tN / 2.0), tN


def uniform_positions(dm: DsmcMesh, cells: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    """Uniform points inside the given cells (tetrahedra, or axis-aligned
    hexahedra)."""
    P = dm.points.reshape(-1, 3)
    cells = np.asarray(cells, dtype=np.int64)
    out = np.empty((cells.shape[0], 3))
    num = dm.cells["num"][cells]
    tet = num == 4
    if tet.any():
        # the 4 distinct nodes of a tet from its faces
        c4 = cells[tet]
        f = dm.cells["cell2face"][c4, :2]
        fm = dm.edges["faceMap"]
        a = fm[f[:, 0], :3]
        b = fm[f[:, 1], :3]
        in_a = (b[:, :, None] == a[:, None, :]).any(-1)
        extra = np.where(~in_a, b, -1).max(axis=1)
        verts = np.concatenate([a, extra[:, None]], axis=1)
        w = rng.dirichlet(np.ones(4), size=c4.shape[0])
        out[tet] = np.einsum("nk,nkd->nd", w, P[verts])
    hexm = ~tet
    if hexm.any():
        lo, hi = cell_boxes(dm)
        ch = cells[hexm]
        out[hexm] = lo[ch] + (hi[ch] - lo[ch]) * rng.random((ch.shape[0], 3))
    return out


def cell_boxes(dm: DsmcMesh):
    """Axis-aligned bounding box of every cell (from its faces' nodes)."""
    P = dm.points.reshape(-1, 3)
    fm = dm.edges["faceMap"]
    ft = dm.edges["faceType"]
    lo = np.full((dm.ncell, 3), np.inf)
    hi = np.full((dm.ncell, 3), -np.inf)
    num = dm.cells["num"]
    for m in range(6):
        has = num > m
        f = dm.cells["cell2face"][has, m]
        for q in range(4):
            nq = np.where(ft[f] > q, fm[f, q], fm[f, 0])
            pts = P[nq]
            lo[has] = np.minimum(lo[has], pts)
            hi[has] = np.maximum(hi[has], pts)
    return lo, hi


def proportional_counts(dm: DsmcMesh, ppc: float, rng: np.random.Generator) -> np.ndarray:
    """A mean of ``ppc`` particles per cell in proportion to the cell volumes,
    each cell's count rounded up with probability equal to its fraction
    (setParticleMessage, src/meshImport.cpp:1399-1421)."""
    vol = dm.cells["area"].astype(float)
    ns = vol * (ppc * dm.ncell) / vol.sum()
    return (np.floor(ns).astype(np.int64) + (rng.random(dm.ncell) < ns - np.floor(ns))).astype(np.int32)


def initial_fill(dm: DsmcMesh, mess, ppc: int, seed: int, inflow_dir, proportional: bool = False) -> dict:
    """Particles from the freestream Maxwellian: ``ppc`` in every cell, or
    with ``proportional`` a mean of ``ppc`` per cell in proportion to the
    cell volumes, each cell's count rounded up with probability equal to its
    fraction (the reference's initial counts, src/meshImport.cpp:1399-1421)."""
    rng = np.random.default_rng(seed)
    if proportional:
        cells = np.repeat(np.arange(dm.ncell, dtype=np.int32), proportional_counts(dm, ppc, rng))
    else:
        cells = np.repeat(np.arange(dm.ncell, dtype=np.int32), ppc)
    x = uniform_positions(dm, cells, rng)
    u, sig, tN = freestream(mess, inflow_dir)
    v = u[None, :] + sig * rng.standard_normal((cells.shape[0], 3))
    ir = -np.log(1.0 - rng.random(cells.shape[0])) * tN * 0.5
    return {"x": x, "v": v, "ir": ir, "cell": cells}


def trace_particles(dm: DsmcMesh, mess, n: int, seed: int, inflow_dir, speed_factor: float = 3.0) -> dict:
    """Tracing-check set: uniform random cells, uniform positions, isotropic
    Maxwellian velocities whose mean speed is ``speed_factor`` times the
    freestream speed, one dt each."""
    rng = np.random.default_rng(seed)
    cells = rng.integers(0, dm.ncell, size=n).astype(np.int32)
    x = uniform_positions(dm, cells, rng)
    u, _, _ = freestream(mess, inflow_dir)
    sigma = speed_factor * float(np.linalg.norm(u)) / math.sqrt(8.0 / math.pi)
    v = sigma * rng.standard_normal((n, 3))
    dt = np.full(n, float(mess["dtime"]))
    return {"x": x, "v": v, "dt": dt, "cell": cells}
