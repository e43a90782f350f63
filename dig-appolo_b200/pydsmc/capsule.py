"""Apollo-shaped capsule case: an unstructured tetrahedral mesh around a
spherical-segment heat shield (nose radius 4.7 m, base diameter 3.912 m)
with a 33-degree half-angle conical afterbody.

The reference's own mesh (mesh/3dapollo372500.cas, 372,500 cells) is not
part of its repository; this generator stands in for it. Points come from a
seeded jittered lattice, finer around the body, in a box of
6 L0 x 4 L0 x 4 L0 (L0 = 3.912 m), plus points on the body surface; they are
tetrahedralised with scipy's Delaunay (Qhull) and the tetrahedra whose
centroid lies inside the body are removed. With ``target_cells`` the count is
then brought to exactly that number by splitting a few seeded far-field cells:
a tetrahedron at its centroid (one cell becomes four) and an interior face at
its centroid (its two cells become six); both keep the mesh conforming and
every cell's orientation. Faces between kept and removed
tetrahedra form the diffuse wall (zone 6); box faces whose outward normal
points against the freestream (or across it) are freestream inlets (zone 4),
the rest outlets (zone 5).
"""
from __future__ import annotations

import math

import numpy as np

from . import case as C
from .mesh import ZONE_INLET, ZONE_INTERIOR, ZONE_OUTLET, ZONE_WALL, RawMesh, _order_by_zone, build_dsmc_mesh, morton_order

L0 = 3.912
NOSE_RADIUS = 4.7
BASE_RADIUS = 3.912 / 2
CONE_HALF_ANGLE = math.radians(33.0)
TOP_RADIUS = 0.35


class CapsuleShape:
    """Axisymmetric body along +x; heat shield apex at x = x0 facing -x."""

    def __init__(self, x0: float, yc: float, zc: float):
        self.x0, self.yc, self.zc = x0, yc, zc
        self.cap_depth = NOSE_RADIUS - math.sqrt(NOSE_RADIUS ** 2 - BASE_RADIUS ** 2)
        self.cone_len = (BASE_RADIUS - TOP_RADIUS) / math.tan(CONE_HALF_ANGLE)
        self.x_base = x0 + self.cap_depth
        self.x_top = self.x_base + self.cone_len
        self.sphere_cx = x0 + NOSE_RADIUS

    def inside(self, p: np.ndarray) -> np.ndarray:
        x = p[:, 0]
        r = np.hypot(p[:, 1] - self.yc, p[:, 2] - self.zc)
        in_cap = (x >= self.x0) & (x <= self.x_base) & \
                 ((x - self.sphere_cx) ** 2 + r ** 2 <= NOSE_RADIUS ** 2)
        rc = BASE_RADIUS - (x - self.x_base) * math.tan(CONE_HALF_ANGLE)
        in_cone = (x > self.x_base) & (x <= self.x_top) & (r <= rc)
        return in_cap | in_cone

    def surface_points(self, h: float, rng: np.random.Generator) -> np.ndarray:
        pts = []
        # spherical cap: rings of constant polar angle about the sphere centre
        th_max = math.asin(BASE_RADIUS / NOSE_RADIUS)
        nth = max(2, int(math.ceil(NOSE_RADIUS * th_max / h)))
        for i in range(nth + 1):
            th = th_max * i / nth
            r = NOSE_RADIUS * math.sin(th)
            x = self.sphere_cx - NOSE_RADIUS * math.cos(th)
            nphi = max(1, int(math.ceil(2 * math.pi * r / h)))
            phi = 2 * math.pi * (np.arange(nphi) + rng.random()) / nphi
            pts.append(np.column_stack([np.full(nphi, x), self.yc + r * np.cos(phi), self.zc + r * np.sin(phi)]))
        # cone: rings along x
        nx = max(2, int(math.ceil(self.cone_len / math.cos(CONE_HALF_ANGLE) / h)))
        for i in range(1, nx + 1):
            x = self.x_base + self.cone_len * i / nx
            r = BASE_RADIUS - (x - self.x_base) * math.tan(CONE_HALF_ANGLE)
            nphi = max(3, int(math.ceil(2 * math.pi * r / h)))
            phi = 2 * math.pi * (np.arange(nphi) + rng.random()) / nphi
            pts.append(np.column_stack([np.full(nphi, x), self.yc + r * np.cos(phi), self.zc + r * np.sin(phi)]))
        # flat top disc
        nr = max(1, int(math.ceil(TOP_RADIUS / h)))
        for i in range(nr):
            r = TOP_RADIUS * i / nr
            nphi = max(1, int(math.ceil(2 * math.pi * r / h)))
            phi = 2 * math.pi * (np.arange(nphi) + rng.random()) / nphi
            pts.append(np.column_stack([np.full(nphi, self.x_top), self.yc + r * np.cos(phi), self.zc + r * np.sin(phi)]))
        return np.concatenate(pts)


def _lattice(lo, hi, h, rng, jitter=0.2):
    n = np.maximum(1, np.round((np.asarray(hi) - np.asarray(lo)) / h).astype(int))
    axes = [np.linspace(lo[d], hi[d], n[d] + 1) for d in range(3)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    P = np.column_stack([X.ravel(), Y.ravel(), Z.ravel()])
    step = (np.asarray(hi) - np.asarray(lo)) / n
    interior = np.all((P > np.asarray(lo) + 1e-9) & (P < np.asarray(hi) - 1e-9), axis=1)
    P[interior] += (rng.random((int(interior.sum()), 3)) - 0.5) * 2 * jitter * step
    return P


# the reference's Apollo mesh (mesh/3dapollo372500.cas) has 372,500 cells
CAP_CELLS = 372500


def _split_to_count(pts, tets, target, far, rng):
    """Split cells of the mask `far` until there are `target` cells: `a`
    tetrahedra at their centroid (+3 cells each) and `b` interior faces at
    their centroid (+4 each), 3a + 4b = target - len(tets), on distinct
    cells. Each new cell is its parent with one vertex moved to the new
    point, so it keeps the parent's orientation."""
    extra = target - tets.shape[0]
    if extra == 0:
        return pts, tets
    sol = [(a, (extra - 3 * a) // 4) for a in range(4) if extra - 3 * a >= 0 and (extra - 3 * a) % 4 == 0]
    if extra < 0 or not sol:
        raise ValueError(f"cannot reach {target} cells from {tets.shape[0]} by splitting")
    a, b = sol[0]
    cand = np.nonzero(far)[0]
    # interior faces between two candidate cells, in a seeded order
    fl = np.concatenate([tets[cand][:, [1, 2, 3]], tets[cand][:, [0, 3, 2]],
                         tets[cand][:, [0, 1, 3]], tets[cand][:, [0, 2, 1]]])
    own = np.tile(cand, 4)
    key = np.sort(fl, axis=1)
    order = np.lexsort((key[:, 2], key[:, 1], key[:, 0]))
    ks = key[order]
    dup = np.nonzero(np.all(ks[1:] == ks[:-1], axis=1))[0]
    pairs = np.column_stack([own[order][dup], own[order][dup + 1]])
    tris = ks[dup]
    used = np.zeros(tets.shape[0], dtype=bool)
    new_pts, new_tets, drop = [], [], []
    npts = pts.shape[0]
    for i in rng.permutation(len(pairs)):
        if b == 0:
            break
        c0, c1 = pairs[i]
        if used[c0] or used[c1]:
            continue
        used[c0] = used[c1] = True
        m = npts + len(new_pts)
        new_pts.append(pts[tris[i]].mean(axis=0))
        for c in (c0, c1):
            t = tets[c]
            for v in tris[i]:
                tt = t.copy()
                tt[tt == v] = m
                new_tets.append(tt)
            drop.append(c)
        b -= 1
    for c in rng.permutation(cand):
        if a == 0:
            break
        if used[c]:
            continue
        used[c] = True
        g = npts + len(new_pts)
        new_pts.append(pts[tets[c]].mean(axis=0))
        for k in range(4):
            tt = tets[c].copy()
            tt[k] = g
            new_tets.append(tt)
        drop.append(c)
        a -= 1
    if a or b:
        raise ValueError("not enough far-field cells to split")
    keep = np.ones(tets.shape[0], dtype=bool)
    keep[np.asarray(drop)] = False
    tets = np.concatenate([tets[keep], np.asarray(new_tets, dtype=tets.dtype)])
    return np.concatenate([pts, np.asarray(new_pts)]), tets


def capsule_mesh(h_fine: float = 0.215, h_coarse: float = 0.60, seed: int = 0, aoa_deg: float = 30.0,
                 r_fine: float = 4.2, target_cells: int | None = None, morton: bool = False) -> RawMesh:
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    box_lo = np.array([0.0, 0.0, 0.0])
    box_hi = np.array([6 * L0, 4 * L0, 4 * L0])
    shape = CapsuleShape(x0=2.0 * L0, yc=2.0 * L0, zc=2.0 * L0)
    body_c = np.array([shape.x0 + 0.5 * (shape.cap_depth + shape.cone_len), shape.yc, shape.zc])
    coarse = _lattice(box_lo, box_hi, h_coarse, rng)
    flo = np.maximum(box_lo, body_c - r_fine)
    fhi = np.minimum(box_hi, body_c + r_fine)
    fine = _lattice(flo, fhi, h_fine, rng)
    fine = fine[np.linalg.norm(fine - body_c, axis=1) <= r_fine]
    # drop coarse points inside the fine ball (plus a margin) and any point
    # inside or too near the body surface
    coarse = coarse[np.linalg.norm(coarse - body_c, axis=1) > r_fine + 0.5 * h_coarse]
    surf = shape.surface_points(h_fine, rng)
    vol = np.concatenate([coarse, fine])
    keep = ~shape.inside(vol)
    vol = vol[keep]
    # keep lattice points off the surface by at least ~0.3 h
    from scipy.spatial import cKDTree
    d, _ = cKDTree(surf).query(vol)
    vol = vol[d > 0.3 * h_fine]
    pts = np.concatenate([vol, surf])
    tri = Delaunay(pts, qhull_options="Qbb Qc Qz Q12")
    tets = tri.simplices.astype(np.int64)
    cent = pts[tets].mean(axis=1)
    tets = tets[~shape.inside(cent)]
    # drop degenerate tetrahedra (zero volume)
    a, b, c_, d_ = (pts[tets[:, k]] for k in range(4))
    v6 = np.einsum("ij,ij->i", b - a, np.cross(c_ - a, d_ - a))
    tets = tets[np.abs(v6) > 1e-12]
    if target_cells is not None:
        cent = pts[tets].mean(axis=1)
        far = np.linalg.norm(cent - body_c, axis=1) > r_fine + 2.0 * h_coarse
        pts, tets = _split_to_count(pts, tets, int(target_cells), far, np.random.default_rng(seed + 7919))
    if morton:
        # cells numbered along a Morton curve of their centroids (the
        # triangulator's order scatters neighbours across the numbering)
        tets = tets[morton_order(pts[tets].mean(axis=1))]
    ncell = tets.shape[0]

    # faces: 4 per tet, matched by sorted node triple
    fl = np.concatenate([tets[:, [1, 2, 3]], tets[:, [0, 3, 2]], tets[:, [0, 1, 3]], tets[:, [0, 2, 1]]])
    owner = np.tile(np.arange(ncell), 4)
    key = np.sort(fl, axis=1)
    order = np.lexsort((key[:, 2], key[:, 1], key[:, 0]))
    ks = key[order]
    same = np.all(ks[1:] == ks[:-1], axis=1)
    first = np.ones(ks.shape[0], dtype=bool)
    first[1:] = ~same
    grp = np.cumsum(first) - 1
    nfaces = int(grp[-1]) + 1
    cnt = np.bincount(grp, minlength=nfaces)
    if cnt.max() > 2:
        raise RuntimeError("non-manifold tetrahedralisation")
    idx_first = np.nonzero(first)[0]
    f_nodes = fl[order][idx_first]
    c0 = owner[order][idx_first]
    c1 = -np.ones(nfaces, dtype=np.int64)
    second = np.nonzero(~first)[0]
    c1[grp[second]] = owner[order][second]

    # boundary classification
    bnd = c1 < 0
    fc = pts[f_nodes].mean(axis=1)
    on_box = bnd & (np.any(np.abs(fc - box_lo) < 1e-6, axis=1) | np.any(np.abs(fc - box_hi) < 1e-6, axis=1))
    # outward normal of a box face
    nrm = np.zeros((nfaces, 3))
    for d in range(3):
        nrm[np.abs(fc[:, d] - box_lo[d]) < 1e-6, d] = -1.0
        nrm[np.abs(fc[:, d] - box_hi[d]) < 1e-6, d] = 1.0
    dirx, diry = C.inflow_direction(aoa_deg)
    udot = nrm[:, 0] * dirx + nrm[:, 1] * diry
    zone = np.full(nfaces, ZONE_INTERIOR, dtype=np.int32)
    zone[bnd & ~on_box] = ZONE_WALL
    zone[on_box & (udot <= 1e-12)] = ZONE_INLET
    zone[on_box & (udot > 1e-12)] = ZONE_OUTLET

    faces = -np.ones((nfaces, 4), dtype=np.int32)
    faces[:, :3] = f_nodes
    ftype = np.full(nfaces, 3, dtype=np.int32)
    faces, ftype, c0, c1, zone = _order_by_zone(faces, ftype, c0.astype(np.int32), c1.astype(np.int32), zone)
    used = np.zeros(pts.shape[0], dtype=bool)
    used[faces[:, :3].ravel()] = True
    remap = -np.ones(pts.shape[0], dtype=np.int64)
    remap[used] = np.arange(int(used.sum()))
    f2 = faces.copy()
    f2[:, :3] = remap[faces[:, :3]]
    return RawMesh(pts[used], f2, ftype, c0, c1, zone, ncell, 2,
                   meta={"kind": "capsule", "seed": seed, "h_fine": h_fine, "h_coarse": h_coarse,
                         "aoa_deg": aoa_deg, "target_cells": target_cells})


def capsule_workload(ppc: int = 100, seed: int = 0):
    """CAP: 372,500 tetrahedra; Ma 5, Kn 0.01 on L0, AoA 30 deg, T_in 142.2 K,
    T_w 300 K diffuse."""
    raw = capsule_mesh(seed=seed, target_cells=CAP_CELLS, morton=True)
    dm = build_dsmc_mesh(raw)
    mess = C.mesh_message(dm, 5.0, 0.01, ppc=ppc, L0=L0)
    zones = [(3, 1, 0), (4, 2, 1), (5, 3, 0), (6, 4, 0)]
    return {"name": "capsule", "dm": dm, "mess": mess, "zones": zones, "inflow_dir": C.inflow_direction(30.0),
            "desc": {"workload": f"capsule-{dm.ncell}", "cells": dm.ncell, "ppc": ppc,
                     "mesh": "tet Delaunay fill of 6L0x4L0x4L0 around spherical-segment shield + 33 deg cone",
                     "Ma": 5.0, "Kn": 0.01, "aoa_deg": 30.0}}
