"""Synthetic meshes in the reference's DSMC mesh format.

The reference reads a Fluent ASCII CAS file (``meshImport::readCAS``,
src/meshImport.cpp:177-195), derives face normals, face centres and cell
volumes (``setFaceCellNew``, src/meshImport.cpp:590-736; ``preprocess``,
src/meshImport.cpp:742-849), picks a diagonal for every quad face
(``choose_face_level_quad_split_tag``, src/meshImportDsmcTopology.cpp:126-147)
and hands the DSMC step the compact arrays ``DsmcCell[]``, ``DsmcEdge[]``,
``localPointXY`` and ``faceSplitTag`` (src/meshImport.h:168-189,
src/meshImportDsmcTopology.cpp:175-228).

This module generates the synthetic meshes the workloads use, writes them as
CAS files the reference parser accepts, and rebuilds the same compact arrays
with the same floating-point operation order, so the device mesh built from
them is bit-identical to the one the reference traces through.

Zone ids follow the reference's boundary table (src/BoundaryCondition.h:79-117):
3 interior (interface), 4 inlet, 5 outlet, 6 diffuse wall; 7 marks the
specular side planes of the block case, which the reference table leaves
unmapped.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

ZONE_CELLS = 2
ZONE_INTERIOR = 3
ZONE_INLET = 4
ZONE_OUTLET = 5
ZONE_WALL = 6
ZONE_SIDE = 7

# Fluent boundary-condition type codes written in the face zone headers.
_FLUENT_BC = {ZONE_INTERIOR: 2, ZONE_INLET: 4, ZONE_OUTLET: 5, ZONE_WALL: 3, ZONE_SIDE: 7}

FACE_SPLIT_02 = 0
FACE_SPLIT_13 = 1
FACE_SPLIT_INVALID = 255

# Byte layouts of DsmcCell / DsmcEdge / meshMessage (src/meshImport.h:168-208).
DSMC_CELL_DTYPE = np.dtype([
    ("num", "<i4"), ("fluentCellType", "<i4"),
    ("cell2face", "<i4", (6,)), ("cell2cell", "<i4", (6,)), ("cell2face_sgn", "<i4", (6,)),
    ("area", "<f8"), ("no", "<i4"), ("cellXY", "<f8", (3,)),
], align=True)
DSMC_EDGE_DTYPE = np.dtype([
    ("faceTag", "<i4"), ("faceType", "<i4"), ("length", "<f8"),
    ("faceMap", "<i4", (6,)), ("edgeNormal", "<f8", (3,)), ("edgeCenter", "<f8", (3,)),
], align=True)
assert DSMC_CELL_DTYPE.itemsize == 120 and DSMC_EDGE_DTYPE.itemsize == 88


@dataclass
class RawMesh:
    """A mesh as a CAS file describes it: nodes, faces with two cells, zones.

    ``faces`` rows are node ids (4 columns, -1 in the last one for
    triangles); ``c0``/``c1`` are the cells on either side (``c1 = -1`` on a
    boundary face, where ``c0`` is the fluid cell). Faces are ordered by zone.
    """
    points: np.ndarray            # (npoint, 3) float64
    faces: np.ndarray             # (nface, 4) int32
    ftype: np.ndarray             # (nface,) int32: 3 or 4 nodes
    c0: np.ndarray                # (nface,) int32
    c1: np.ndarray                # (nface,) int32, -1 on boundaries
    zone: np.ndarray              # (nface,) int32 zone id
    ncell: int
    cell_type: int                # Fluent element type: 2 tet, 4 hex
    meta: dict = field(default_factory=dict)

    @property
    def nface(self) -> int:
        return int(self.faces.shape[0])

    @property
    def npoint(self) -> int:
        return int(self.points.shape[0])


def morton_order(points: np.ndarray, bits: int = 21) -> np.ndarray:
    """Order of `points` (n x 3) along a Morton (Z-order) curve of their
    bounding box, 2^bits cells per axis: the permutation that numbers
    nearby points nearby, as mesh tools renumber cells for locality."""
    p = np.asarray(points, dtype=np.float64)
    if len(p) == 0:
        return np.zeros(0, dtype=np.int64)
    lo, hi = p.min(axis=0), p.max(axis=0)
    span = np.where(hi > lo, hi - lo, 1.0)
    q = np.minimum(((p - lo) / span * (1 << bits)).astype(np.uint64), np.uint64((1 << bits) - 1))
    key = np.zeros(len(p), dtype=np.uint64)
    for b in range(bits):
        for a in range(3):
            key |= ((q[:, a] >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b + a)
    return np.argsort(key, kind="stable")


def _order_by_zone(faces, ftype, c0, c1, zone, order=(ZONE_INTERIOR, ZONE_INLET, ZONE_OUTLET, ZONE_WALL, ZONE_SIDE)):
    idx = np.concatenate([np.nonzero(zone == z)[0] for z in order])
    assert idx.size == zone.size
    return faces[idx], ftype[idx], c0[idx], c1[idx], zone[idx]


def hex_box(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float,
            hole: tuple | None = None) -> RawMesh:
    """Uniform hex box ``[0,lx]x[0,ly]x[0,lz]`` of ``nx*ny*nz`` cells.

    ``hole = (i0, i1, j0, j1, k0, k1)`` removes the cells with
    ``i0 <= i < i1`` etc.; the faces between the fluid and the removed block
    form the wall zone. x-min is the inlet, x-max the outlet, the other four
    sides are zone 7.
    """
    solid = np.zeros((nx, ny, nz), dtype=bool)
    if hole is not None:
        i0, i1, j0, j1, k0, k1 = hole
        solid[i0:i1, j0:j1, k0:k1] = True
    fluid = ~solid
    cid = -np.ones((nx, ny, nz), dtype=np.int64)
    cid[fluid] = np.arange(int(fluid.sum()))
    ncell = int(fluid.sum())

    gx = np.linspace(0.0, lx, nx + 1)
    gy = np.linspace(0.0, ly, ny + 1)
    gz = np.linspace(0.0, lz, nz + 1)
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    points = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    faces, c0s, c1s, zones = [], [], [], []

    def add_plane(axis):
        # faces normal to `axis` at integer plane index p in [0, n_axis]
        n = (nx, ny, nz)
        shape = list(n)
        shape[axis] = n[axis] + 1
        P = np.indices(shape).reshape(3, -1).T          # (i,j,k) of the face's "upper" cell
        i, j, k = P[:, 0], P[:, 1], P[:, 2]
        if axis == 0:
            quad = np.stack([nid(i, j, k), nid(i, j + 1, k), nid(i, j + 1, k + 1), nid(i, j, k + 1)], 1)
        elif axis == 1:
            quad = np.stack([nid(i, j, k), nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j, k)], 1)
        else:
            quad = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k)], 1)
        lo = P.copy()
        lo[:, axis] -= 1
        hi = P
        def cell_at(q):
            inside = (q[:, axis] >= 0) & (q[:, axis] < n[axis])
            out = -np.ones(q.shape[0], dtype=np.int64)
            qq = q[inside]
            out[inside] = cid[qq[:, 0], qq[:, 1], qq[:, 2]]
            return out, inside
        clo, in_lo = cell_at(lo)
        chi, in_hi = cell_at(hi)
        for m in range(P.shape[0]):
            a, b = clo[m], chi[m]
            if a < 0 and b < 0:
                continue
            if a >= 0 and b >= 0:
                faces.append(quad[m]); c0s.append(a); c1s.append(b); zones.append(ZONE_INTERIOR)
                continue
            fcell = a if a >= 0 else b
            # boundary face: the fluid cell is c0
            if (a >= 0 and in_hi[m]) or (b >= 0 and in_lo[m]):
                z = ZONE_WALL                      # neighbour is a removed (solid) cell
            elif axis == 0:
                z = ZONE_INLET if b >= 0 else ZONE_OUTLET
            else:
                z = ZONE_SIDE
            faces.append(quad[m]); c0s.append(fcell); c1s.append(-1); zones.append(z)

    for ax in range(3):
        add_plane(ax)
    faces = np.asarray(faces, dtype=np.int32)
    ftype = np.full(faces.shape[0], 4, dtype=np.int32)
    c0 = np.asarray(c0s, dtype=np.int32)
    c1 = np.asarray(c1s, dtype=np.int32)
    zone = np.asarray(zones, dtype=np.int32)
    faces, ftype, c0, c1, zone = _order_by_zone(faces, ftype, c0, c1, zone)
    used = np.zeros(points.shape[0], dtype=bool)
    used[faces.ravel()] = True
    remap = -np.ones(points.shape[0], dtype=np.int64)
    remap[used] = np.arange(int(used.sum()))
    faces = remap[faces].astype(np.int32)
    points = points[used]
    return RawMesh(points, faces, ftype, c0, c1, zone, ncell, 4,
                   meta={"kind": "hex_box", "n": (nx, ny, nz), "L": (lx, ly, lz), "hole": hole})


def pyramid_box(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float) -> RawMesh:
    """Box ``[0,lx]x[0,ly]x[0,lz]`` of ``nx*ny*nz`` cubes, each split into six
    pyramids (Fluent element type 5) with the cube's centre as apex and a
    cube face as base: cell ``6 q + d`` is the pyramid of cube ``q`` on face
    ``d`` (-x, +x, -y, +y, -z, +z). Base quads are shared with the
    neighbouring cube's pyramid or lie on the boundary (x-min inlet, x-max
    outlet, the other sides zone 7); the triangles from each cube edge to the
    centre are shared by the two pyramids of that edge."""
    gx = np.linspace(0.0, lx, nx + 1)
    gy = np.linspace(0.0, ly, ny + 1)
    gz = np.linspace(0.0, lz, nz + 1)
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    grid = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    cx = 0.5 * (gx[:-1] + gx[1:])
    cy = 0.5 * (gy[:-1] + gy[1:])
    cz = 0.5 * (gz[:-1] + gz[1:])
    CX, CY, CZ = np.meshgrid(cx, cy, cz, indexing="ij")
    centres = np.stack([CX.ravel(), CY.ravel(), CZ.ravel()], axis=1)
    points = np.concatenate([grid, centres])
    G = grid.shape[0]
    n = (nx, ny, nz)

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    def qid(i, j, k):
        return (i * ny + j) * nz + k

    faces, ftype, c0s, c1s, zones = [], [], [], [], []
    # base quads, plane by plane as in hex_box
    for axis in range(3):
        shape = list(n)
        shape[axis] += 1
        for i, j, k in np.ndindex(*shape):
            if axis == 0:
                quad = [nid(i, j, k), nid(i, j + 1, k), nid(i, j + 1, k + 1), nid(i, j, k + 1)]
            elif axis == 1:
                quad = [nid(i, j, k), nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j, k)]
            else:
                quad = [nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k)]
            p = (i, j, k)
            lo = list(p)
            lo[axis] -= 1
            has_lo = lo[axis] >= 0
            has_hi = p[axis] < n[axis]
            a = qid(*lo) * 6 + 2 * axis + 1 if has_lo else -1     # the lower cube's +face pyramid
            b = qid(*p) * 6 + 2 * axis if has_hi else -1          # the upper cube's -face pyramid
            if a >= 0 and b >= 0:
                faces.append(quad); ftype.append(4); c0s.append(a); c1s.append(b); zones.append(ZONE_INTERIOR)
            else:
                z = (ZONE_INLET if b >= 0 else ZONE_OUTLET) if axis == 0 else ZONE_SIDE
                faces.append(quad); ftype.append(4); c0s.append(a if a >= 0 else b); c1s.append(-1); zones.append(z)
    # edge triangles inside every cube
    for i, j, k in np.ndindex(nx, ny, nz):
        q = qid(i, j, k)
        ctr = G + q
        for o1 in (0, 1):
            for o2 in (0, 1):
                # along z at x-offset o1, y-offset o2: pyramids -/+x and -/+y
                tri = [nid(i + o1, j + o2, k), nid(i + o1, j + o2, k + 1), ctr, -1]
                faces.append(tri); ftype.append(3); c0s.append(q * 6 + o1); c1s.append(q * 6 + 2 + o2)
                zones.append(ZONE_INTERIOR)
                # along x at y-offset o1, z-offset o2: pyramids -/+y and -/+z
                tri = [nid(i, j + o1, k + o2), nid(i + 1, j + o1, k + o2), ctr, -1]
                faces.append(tri); ftype.append(3); c0s.append(q * 6 + 2 + o1); c1s.append(q * 6 + 4 + o2)
                zones.append(ZONE_INTERIOR)
                # along y at x-offset o1, z-offset o2: pyramids -/+x and -/+z
                tri = [nid(i + o1, j, k + o2), nid(i + o1, j + 1, k + o2), ctr, -1]
                faces.append(tri); ftype.append(3); c0s.append(q * 6 + o1); c1s.append(q * 6 + 4 + o2)
                zones.append(ZONE_INTERIOR)
    faces = np.asarray(faces, dtype=np.int32)
    ftype = np.asarray(ftype, dtype=np.int32)
    c0 = np.asarray(c0s, dtype=np.int32)
    c1 = np.asarray(c1s, dtype=np.int32)
    zone = np.asarray(zones, dtype=np.int32)
    faces, ftype, c0, c1, zone = _order_by_zone(faces, ftype, c0, c1, zone)
    return RawMesh(points, faces, ftype, c0, c1, zone, 6 * nx * ny * nz, 5,
                   meta={"kind": "pyramid_box", "n": (nx, ny, nz), "L": (lx, ly, lz)})


def prism_box(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float) -> RawMesh:
    """Box ``[0,lx]x[0,ly]x[0,lz]`` of ``nx*ny*nz`` cubes, each split into two
    wedges (Fluent element type 6) by the vertical plane through its xy
    diagonal from (i, j) to (i+1, j+1): cell ``2 q`` has the triangle
    (i,j), (i+1,j), (i+1,j+1) as cross-section (it owns the cube's -y and +x
    faces), cell ``2 q + 1`` the triangle (i,j), (i+1,j+1), (i,j+1) (the +y
    and -x faces). Triangles lie on the z planes, quads on the x and y planes
    and on the diagonals. x-min is the inlet, x-max the outlet, the other
    sides zone 7."""
    gx = np.linspace(0.0, lx, nx + 1)
    gy = np.linspace(0.0, ly, ny + 1)
    gz = np.linspace(0.0, lz, nz + 1)
    X, Y, Z = np.meshgrid(gx, gy, gz, indexing="ij")
    points = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    def qid(i, j, k):
        return (i * ny + j) * nz + k

    faces, ftype, c0s, c1s, zones = [], [], [], [], []

    def add(nodes, a, b, zone):
        faces.append(list(nodes) + [-1] * (4 - len(nodes)))
        ftype.append(len(nodes))
        c0s.append(a)
        c1s.append(b)
        zones.append(zone)

    # x planes: the +x face of a cube is wedge 0's, the -x face wedge 1's
    for i, j, k in np.ndindex(nx + 1, ny, nz):
        quad = [nid(i, j, k), nid(i, j + 1, k), nid(i, j + 1, k + 1), nid(i, j, k + 1)]
        a = 2 * qid(i - 1, j, k) if i > 0 else -1
        b = 2 * qid(i, j, k) + 1 if i < nx else -1
        if a >= 0 and b >= 0:
            add(quad, a, b, ZONE_INTERIOR)
        else:
            add(quad, a if a >= 0 else b, -1, ZONE_INLET if b >= 0 else ZONE_OUTLET)
    # y planes: the -y face is wedge 0's, the +y face wedge 1's
    for i, j, k in np.ndindex(nx, ny + 1, nz):
        quad = [nid(i, j, k), nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j, k)]
        a = 2 * qid(i, j - 1, k) + 1 if j > 0 else -1
        b = 2 * qid(i, j, k) if j < ny else -1
        if a >= 0 and b >= 0:
            add(quad, a, b, ZONE_INTERIOR)
        else:
            add(quad, a if a >= 0 else b, -1, ZONE_SIDE)
    # z planes: two triangles per cube column, shared with the wedge above
    for i, j, k in np.ndindex(nx, ny, nz + 1):
        tris = ([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k)],
                [nid(i, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k)])
        for t, tri in enumerate(tris):
            a = 2 * qid(i, j, k - 1) + t if k > 0 else -1
            b = 2 * qid(i, j, k) + t if k < nz else -1
            if a >= 0 and b >= 0:
                add(tri, a, b, ZONE_INTERIOR)
            else:
                add(tri, a if a >= 0 else b, -1, ZONE_SIDE)
    # the diagonal quad inside every cube
    for i, j, k in np.ndindex(nx, ny, nz):
        q = qid(i, j, k)
        add([nid(i, j, k), nid(i + 1, j + 1, k), nid(i + 1, j + 1, k + 1), nid(i, j, k + 1)], 2 * q, 2 * q + 1,
            ZONE_INTERIOR)
    faces = np.asarray(faces, dtype=np.int32)
    ftype = np.asarray(ftype, dtype=np.int32)
    c0 = np.asarray(c0s, dtype=np.int32)
    c1 = np.asarray(c1s, dtype=np.int32)
    zone = np.asarray(zones, dtype=np.int32)
    faces, ftype, c0, c1, zone = _order_by_zone(faces, ftype, c0, c1, zone)
    return RawMesh(points, faces, ftype, c0, c1, zone, 2 * nx * ny * nz, 6,
                   meta={"kind": "prism_box", "n": (nx, ny, nz), "L": (lx, ly, lz)})


def block_case_mesh(scale: int = 1) -> RawMesh:
    """The block case: 1.0 x 0.5 x 0.5 m box of 48x32x32 hexes with the
    central 8x8x8-cell block removed (48,640 cells). ``scale`` > 1 divides
    every cell count by ``scale`` (a geometrically similar, coarser mesh for
    CPU-sized tests)."""
    nx, ny, nz = 48 // scale, 32 // scale, 32 // scale
    h = 8 // scale
    i0, j0, k0 = (nx - h) // 2, (ny - h) // 2, (nz - h) // 2
    return hex_box(nx, ny, nz, 1.0, 0.5, 0.5, (i0, i0 + h, j0, j0 + h, k0, k0 + h))


# ---------------------------------------------------------------------------
# CAS writer (the subset of the Fluent ASCII format that readCAS parses)
# ---------------------------------------------------------------------------

def write_cas(path: str, raw: RawMesh) -> None:
    """Write ``raw`` as a Fluent ASCII case the reference's ``readCAS``
    (src/meshImport.cpp:177-405) reads back to the same nodes, faces, cells
    and zone tags. Coordinates use 17 significant digits, so they parse back
    to the identical doubles."""
    hx = lambda v: format(int(v), "x")
    lines = ['(0 "dig-appolo_b200 synthetic mesh")', "(2 3)"]
    npt, ncell, nface = raw.npoint, raw.ncell, raw.nface
    lines.append(f"(10 (0 1 {hx(npt)} 0 3))")
    lines.append(f"(10 (1 1 {hx(npt)} 1 3)(")
    for p in raw.points:
        lines.append(f"{p[0]:.17g} {p[1]:.17g} {p[2]:.17g}")
    lines.append("))")
    lines.append(f"(12 (0 1 {hx(ncell)} 0))")
    lines.append(f"(12 ({ZONE_CELLS:x} 1 {hx(ncell)} 1 {raw.cell_type}))")
    lines.append(f"(13 (0 1 {hx(nface)} 0))")
    start = 0
    zones = []
    for z in (ZONE_INTERIOR, ZONE_INLET, ZONE_OUTLET, ZONE_WALL, ZONE_SIDE):
        n = int((raw.zone == z).sum())
        if n:
            zones.append((z, start, start + n))
            start += n
    assert start == nface
    for z, a, b in zones:
        lines.append(f"(13 ({z:x} {hx(a + 1)} {hx(b)} {_FLUENT_BC[z]:x} 0)(")
        for f in range(a, b):
            t = int(raw.ftype[f])
            nodes = [hx(raw.faces[f, q] + 1) for q in range(t)]
            cc1 = hx(raw.c1[f] + 1) if raw.c1[f] >= 0 else "0"
            lines.append(f"{t} " + " ".join(nodes) + f" {hx(raw.c0[f] + 1)} {cc1}")
        lines.append("))")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


# ---------------------------------------------------------------------------
# Compact DSMC arrays, restating the reference's preprocessing op for op
# ---------------------------------------------------------------------------

@dataclass
class DsmcMesh:
    cells: np.ndarray           # DSMC_CELL_DTYPE (ncell,)
    edges: np.ndarray           # DSMC_EDGE_DTYPE (nface,)
    points: np.ndarray          # (npoint*3,) float64, localPointXY
    split: np.ndarray           # (nface,) uint8, faceSplitTag
    area_sum: float             # meshImport::Area, the summed cell volumes
    min_edge: float             # meshImport::miniLength
    bcnumber: int               # number of boundary faces
    raw: RawMesh | None = None

    @property
    def ncell(self) -> int:
        return int(self.cells.shape[0])

    @property
    def nface(self) -> int:
        return int(self.edges.shape[0])

    @property
    def npoint(self) -> int:
        return int(self.points.shape[0] // 3)


def _face_geometry(P, faces, ftype):
    """Face centroid, area and unit normal, in the operation order of
    setFaceCellNew (src/meshImport.cpp:596-668)."""
    nf = faces.shape[0]
    t = ftype.astype(np.float64)
    centre = np.zeros((nf, 3))
    for q in range(4):
        m = ftype > q
        centre[m] += P[faces[m, q]] / t[m, None]
    centroid = np.zeros((nf, 3))
    SF = np.zeros((nf, 3))
    area = np.zeros(nf)
    for q in range(4):
        m = ftype > q
        idx = np.nonzero(m)[0]
        p1 = faces[idx, q]
        nxt = np.where(q < ftype[idx] - 1, (q + 1), 0)
        p2 = faces[idx, nxt]
        x0 = centre[idx]
        X1 = P[p1]
        X2 = P[p2]
        lc = (X1 + X2 + x0) / 3
        l = X1 - x0
        r = X2 - x0
        vx = r[:, 1] * l[:, 2] - r[:, 2] * l[:, 1]
        vy = r[:, 2] * l[:, 0] - l[:, 2] * r[:, 0]
        vz = r[:, 0] * l[:, 1] - l[:, 0] * r[:, 1]
        vx = vx * 0.5
        vy = vy * 0.5
        vz = vz * 0.5
        la = np.sqrt(vx * vx + vy * vy + vz * vz)
        centroid[idx] += la[:, None] * lc
        SF[idx, 0] += vx
        SF[idx, 1] += vy
        SF[idx, 2] += vz
        area[idx] += la
    centroid = centroid / area[:, None]
    dS = np.sqrt(SF[:, 0] * SF[:, 0] + SF[:, 1] * SF[:, 1] + SF[:, 2] * SF[:, 2])
    normal = SF / dS[:, None]
    return centroid, area, normal


def _quad_split_tags(P, faces, ftype):
    """choose_face_level_quad_split_tag (src/meshImportDsmcTopology.cpp:85-147)."""
    tags = np.full(faces.shape[0], FACE_SPLIT_INVALID, dtype=np.uint8)
    q = np.nonzero(ftype == 4)[0]
    if q.size == 0:
        return tags
    Q = P[faces[q]]                                           # (nq, 4, 3)

    def tri_normal(a, b, c):
        e1 = Q[:, b] - Q[:, a]
        e2 = Q[:, c] - Q[:, a]
        n = np.stack([e1[:, 1] * e2[:, 2] - e1[:, 2] * e2[:, 1],
                      e1[:, 2] * e2[:, 0] - e1[:, 0] * e2[:, 2],
                      e1[:, 0] * e2[:, 1] - e1[:, 1] * e2[:, 0]], 1)
        ln = np.sqrt(n[:, 0] * n[:, 0] + n[:, 1] * n[:, 1] + n[:, 2] * n[:, 2])
        ok = np.isfinite(ln) & (ln > 1.0e-30)
        return n, ln, ok

    def score(ta, tb):
        n0, l0, ok0 = tri_normal(*ta)
        n1, l1, ok1 = tri_normal(*tb)
        with np.errstate(divide="ignore", invalid="ignore"):
            cosang = (n0[:, 0] * n1[:, 0] + n0[:, 1] * n1[:, 1] + n0[:, 2] * n1[:, 2]) / (l0 * l1)
            cosang = np.clip(cosang, -1.0, 1.0)
            s = (1.0 - cosang) * 16.0 + np.abs(l0 - l1) / (l0 + l1)
        return np.where(ok0 & ok1, s, np.finfo(np.float64).max)

    s02 = score((0, 1, 2), (0, 2, 3))
    s13 = score((0, 1, 3), (1, 2, 3))
    big = np.finfo(np.float64).max * 0.5
    v02 = s02 < big
    v13 = s13 < big
    use13 = (~v02) | (v13 & (s13 + 1.0e-12 < s02))
    t = np.where(use13, FACE_SPLIT_13, FACE_SPLIT_02).astype(np.uint8)
    t[~v02 & ~v13] = FACE_SPLIT_02
    tags[q] = t
    return tags


def build_dsmc_mesh(raw: RawMesh) -> DsmcMesh:
    """DsmcCell/DsmcEdge/localPointXY/faceSplitTag as the reference builds
    them from the same CAS input for a single partition."""
    P = raw.points.astype(np.float64)
    nf, ncell = raw.nface, raw.ncell
    centroid, farea, normal = _face_geometry(P, raw.faces, raw.ftype)

    # boundary faces get ghost ids Ncell, Ncell+1, ... in file order (readFaces)
    c0 = raw.c0.astype(np.int64)
    c1 = raw.c1.astype(np.int64).copy()
    bmask = c1 < 0
    c1[bmask] = ncell + np.arange(int(bmask.sum()))
    bc_faces = np.nonzero(bmask)[0]

    # cell2face / cell2cell / sgn in face order (setFaceCellNew, :671-687):
    # each cell lists its faces in ascending face index
    f_all = np.arange(nf, dtype=np.int64)
    inner = c1 < ncell
    cell_k = np.concatenate([c0, c1[inner]])
    face_k = np.concatenate([f_all, f_all[inner]])
    other = np.concatenate([c1, c0[inner]])
    sg = np.concatenate([np.ones(nf, dtype=np.int64), -np.ones(int(inner.sum()), dtype=np.int64)])
    order = np.lexsort((face_k, cell_k))
    cell_k, face_k, other, sg = cell_k[order], face_k[order], other[order], sg[order]
    tag = np.bincount(cell_k, minlength=ncell).astype(np.int64)
    first = np.concatenate([[0], np.cumsum(tag)[:-1]])
    slot = np.arange(cell_k.shape[0]) - first[cell_k]
    if slot.max(initial=0) >= 6:
        raise ValueError("a cell has more than 6 faces")
    cell2face = -np.ones((ncell, 6), dtype=np.int32)
    cell2cell = -np.ones((ncell, 6), dtype=np.int32)
    sgn = -np.ones((ncell, 6), dtype=np.int32)
    cell2face[cell_k, slot] = face_k
    cell2cell[cell_k, slot] = other
    sgn[cell_k, slot] = sg

    # cell volumes and centroids (:688-723)
    T = tag.astype(np.float64)
    cc = np.zeros((ncell, 3))
    for j in range(6):
        m = tag > j
        cc[m] += centroid[cell2face[m, j]] / T[m, None]
    vsum = np.zeros(ncell)
    vcs = np.zeros((ncell, 3))
    for j in range(6):
        m = tag > j
        fidx = cell2face[m, j]
        Cf = centroid[fidx] - cc[m]
        n = normal[fidx]
        lv = np.abs(n[:, 0] * Cf[:, 0] + n[:, 1] * Cf[:, 1] + n[:, 2] * Cf[:, 2]) * farea[fidx] / 3
        lc = 0.75 * centroid[fidx] + 0.25 * cc[m]
        vcs[m] += lc * lv[:, None]
        vsum[m] += lv
    cellXY = vcs / vsum[:, None]

    # orient normals from c0 to c1 using ghost centroids (preprocess, :756-783)
    ghost = 2 * centroid[bc_faces] - cellXY[c0[bc_faces]]
    allc = np.concatenate([cellXY, ghost], 0)
    xl = allc[c0]
    xr = allc[c1]
    d = xl - xr
    dist = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    rij = (xr - xl) / dist[:, None]
    vn = normal[:, 0] * rij[:, 0] + normal[:, 1] * rij[:, 1] + normal[:, 2] * rij[:, 2]
    normal = np.where((vn < 0)[:, None], -normal, normal)

    area_sum = float(np.cumsum(vsum)[-1])

    # min edge length over all face edges (setParticleMessage, :1362-1390)
    mins = []
    for q in range(4):
        m = raw.ftype > q
        idx = np.nonzero(m)[0]
        p1 = raw.faces[idx, q]
        nxt = np.where(q < raw.ftype[idx] - 1, q + 1, 0)
        p2 = raw.faces[idx, nxt]
        a, b = P[p1], P[p2]
        dd = np.sqrt((a[:, 0] - b[:, 0]) * (a[:, 0] - b[:, 0]) + (a[:, 1] - b[:, 1]) * (a[:, 1] - b[:, 1])
                     + (a[:, 2] - b[:, 2]) * (a[:, 2] - b[:, 2]))
        if dd.size:
            mins.append(dd.min())
    min_edge = float(min(mins))

    cells = np.zeros(ncell, dtype=DSMC_CELL_DTYPE)
    cells["num"] = tag
    cells["fluentCellType"] = raw.cell_type
    cells["cell2face"] = cell2face
    cells["cell2cell"] = cell2cell
    cells["cell2face_sgn"] = sgn
    cells["area"] = vsum
    cells["no"] = 0
    cells["cellXY"] = cellXY

    edges = np.zeros(nf, dtype=DSMC_EDGE_DTYPE)
    edges["faceTag"] = raw.zone
    edges["faceType"] = raw.ftype
    edges["length"] = farea
    fm = -np.ones((nf, 6), dtype=np.int32)
    fm[:, :4] = raw.faces
    fm[raw.ftype == 3, 3] = -1
    fm[:, 4] = c0
    fm[:, 5] = c1
    edges["faceMap"] = fm
    edges["edgeNormal"] = normal
    edges["edgeCenter"] = centroid

    split = _quad_split_tags(P, raw.faces, raw.ftype)
    return DsmcMesh(cells, edges, P.reshape(-1).copy(), split, area_sum, min_edge,
                    int(bmask.sum()), raw)
