"""Deterministic inputs shared by the golden-fixture generator and the tests.

Inputs are rebuilt from seeds with numpy's legacy RandomState (MT19937),
whose streams numpy keeps fixed across versions, so the fixtures only need
to store the reference's outputs.
"""
from __future__ import annotations

import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "dig-appolo_b200"))

from pydsmc import case as C  # noqa: E402
from pydsmc import mesh as M  # noqa: E402

# the block case, 1/4 resolution: 12x8x8 hexes minus the central 2x2x2 block
BLOCK_SCALE = 4
BLOCK_MA = 5.0
BLOCK_KN = 0.1
BLOCK_L0 = 0.125          # edge of the removed block in y/z (8 cells of 0.5/32 m)
AOA_DEG = 30.0            # the reference's hard-coded angle of attack
# reference boundary table (src/BoundaryCondition.h:79-117); tag 7 unmapped
REF_ZONES = [(3, 1, 0), (4, 2, 1), (5, 3, 0), (6, 4, 0)]
# the same with the wall zone as an outlet: advection without random draws
NOWALL_ZONES = [(3, 1, 0), (4, 2, 1), (5, 3, 0), (6, 3, 0)]


def block_mesh(scale: int = BLOCK_SCALE):
    raw = M.block_case_mesh(scale=scale)
    return raw, M.build_dsmc_mesh(raw)


def block_mess(dm, ppc: int):
    return C.mesh_message(dm, BLOCK_MA, BLOCK_KN, ppc=ppc, L0=BLOCK_L0)


def inflow_dir():
    return C.inflow_direction(AOA_DEG)


def cell_boxes(dm):
    P = dm.points.reshape(-1, 3)
    fm = dm.edges["faceMap"]
    lo = np.full((dm.ncell, 3), np.inf)
    hi = np.full((dm.ncell, 3), -np.inf)
    for m in range(6):
        f = dm.cells["cell2face"][:, m]
        for q in range(4):
            pts = P[fm[f, q]]
            lo = np.minimum(lo, pts)
            hi = np.maximum(hi, pts)
    return lo, hi


def freestream(mess):
    d = inflow_dir()
    base = 1.0 * float(mess["Ma"]) * math.sqrt(float(mess["gamma"]) / 2.0) * float(mess["v_in"]) / float(mess["v_rms"])
    u = np.array([base * d[0], base * d[1], 0.0])
    tN = float(mess["T_in"]) / float(mess["T_ref"])
    return u, math.sqrt(tN / 2.0), tN


def trace_inputs(dm, mess, n: int, seed: int):
    """Uniform random hex cells, uniform positions, isotropic velocities with
    mean speed 3x the freestream speed, one dt."""
    rs = np.random.RandomState(seed)
    cells = rs.randint(0, dm.ncell, size=n).astype(np.int32)
    lo, hi = cell_boxes(dm)
    x = lo[cells] + (hi[cells] - lo[cells]) * rs.random_sample((n, 3))
    u, _, _ = freestream(mess)
    sigma = 3.0 * float(np.linalg.norm(u)) / math.sqrt(8.0 / math.pi)
    v = sigma * rs.standard_normal((n, 3))
    dt = np.full(n, float(mess["dtime"]))
    return x, v, dt, cells


TRACE_FULL_N = 1_000_000   # the TRACE configuration: 10^6 particles on the full block mesh, one dt
TRACE_FULL_SEED = 1


def fp32_state(dm, x, v, cell):
    """The state the mixed path stores for FP64 positions and velocities:
    FP32 offsets from the cell centre and FP32 velocities, widened back to
    FP64 the way the trace widens them (centre + offset)."""
    cc = dm.cells["cellXY"][cell]
    x32 = cc + (x - cc).astype(np.float32).astype(np.float64)
    return x32, v.astype(np.float32).astype(np.float64)


def fp32_positions(dm, x, cell):
    """FP64 positions as the mixed path stores and returns them: the FP32
    rounding of the offset from the centre of `cell`, widened again."""
    cc = dm.cells["cellXY"][cell]
    return cc + (x - cc).astype(np.float32).astype(np.float64)


def digest(a) -> str:
    """SHA-256 of an array's bytes (C order), for bit-exact comparisons of
    outputs too large to store."""
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def split_box_trace_inputs(raw, mess, n: int, seed: int):
    """Uniform random points in the cubes of a ``pydsmc.mesh.pyramid_box`` or
    ``prism_box`` mesh, each with the cell of its cube that holds it (the
    pyramid of the nearest cube face, or the wedge on its side of the
    diagonal), isotropic velocities with mean speed 3x the freestream speed,
    dt uniform in [0, dtime]."""
    nx, ny, nz = raw.meta["n"]
    h = np.array(raw.meta["L"], dtype=float) / np.array([nx, ny, nz])
    rs = np.random.RandomState(seed)
    q = rs.randint(0, nx * ny * nz, size=n)
    ijk = np.stack([q // (ny * nz), (q // nz) % ny, q % nz], 1)
    r = rs.random_sample((n, 3))
    x = (ijk + r) * h
    if raw.meta["kind"] == "pyramid_box":
        axis = np.abs(r - 0.5).argmax(1)
        side = (r[np.arange(n), axis] > 0.5).astype(np.int64)
        cells = (6 * q + 2 * axis + side).astype(np.int32)
    elif raw.meta["kind"] == "prism_box":
        cells = (2 * q + (r[:, 1] > r[:, 0])).astype(np.int32)
    else:
        raise ValueError(raw.meta["kind"])
    u, _, _ = freestream(mess)
    sigma = 3.0 * float(np.linalg.norm(u)) / math.sqrt(8.0 / math.pi)
    v = sigma * rs.standard_normal((n, 3))
    dt = float(mess["dtime"]) * rs.random_sample(n)
    return x, v, dt, cells


def degenerate_trace_inputs(dm, mess, ncells: int, seed: int):
    """Exact, degenerate paths in hexahedral cells: from the centre, a
    corner, the opposite corner, two face centres, an edge midpoint and a
    top-face centre of each of ncells random cells, along each of the 26
    directions (+-1, 0) x 3 at 3x the freestream speed, so that paths meet
    faces at their centres (on a quad's split diagonal), along edges and
    through vertices; then, per cell, a particle at rest, one with dt = 0,
    one with a denormal-small speed and one starting on a face and moving
    along it. dt = dtime."""
    lo, hi = cell_boxes(dm)
    ctr = 0.5 * (lo + hi)
    rs = np.random.RandomState(seed)
    cells = rs.choice(dm.ncell, ncells, replace=False)
    dirs = [d for d in ((a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)) if d != (0, 0, 0)]
    u, _, _ = freestream(mess)
    sp = 3.0 * float(np.linalg.norm(u))
    dtime = float(mess["dtime"])
    X, V, C, T = [], [], [], []
    for c in cells:
        L, H, M = lo[c], hi[c], ctr[c]
        starts = [M, L, H, np.array([L[0], M[1], M[2]]), np.array([H[0], M[1], M[2]]),
                  np.array([L[0], L[1], M[2]]), np.array([M[0], M[1], H[2]])]
        for s0 in starts:
            for d in dirs:
                X.append(s0); V.append(np.array(d, float) * sp); C.append(c); T.append(dtime)
        for x0, v0, t0 in ((M, np.zeros(3), dtime), (M, np.array([sp, 0.0, 0.0]), 0.0),
                           (M, np.array([1e-300, 0.0, 0.0]), dtime),
                           (np.array([L[0], M[1], M[2]]), np.array([0.0, sp, 0.3 * sp]), dtime)):
            X.append(x0); V.append(v0); C.append(c); T.append(t0)
    return np.array(X), np.array(V), np.array(T), np.array(C, dtype=np.int32)


def degenerate_tet_trace_inputs(dm, mess, ncells: int, seed: int):
    """Exact, degenerate paths in tetrahedral cells: from the centroid, the
    4 vertices, the 6 edge midpoints and the 4 face centroids of each of
    ncells random cells, towards and away from each other of those 15
    points at 3x the freestream speed, so that paths run along edges and
    faces and through vertices. dt = dtime."""
    P = dm.points.reshape(-1, 3)
    rs = np.random.RandomState(seed)
    cells = rs.choice(dm.ncell, ncells, replace=False)
    u, _, _ = freestream(mess)
    sp = 3.0 * float(np.linalg.norm(u))
    dtime = float(mess["dtime"])
    X, V, C = [], [], []
    for c, A in zip(cells, P[tet_vertices(dm, cells)]):
        pts = ([A.mean(0)] + [A[i] for i in range(4)] +
               [(A[i] + A[j]) / 2 for i in range(4) for j in range(i + 1, 4)] +
               [(A.sum(0) - A[i]) / 3 for i in range(4)])
        for s0 in pts:
            for t0 in pts:
                d = t0 - s0
                n = np.linalg.norm(d)
                if n == 0:
                    continue
                for sgn in (1.0, -1.0):
                    X.append(s0); V.append(sgn * d / n * sp); C.append(c)
    return np.array(X), np.array(V), np.full(len(C), dtime), np.array(C, dtype=np.int32)


def sampled_at(k: int, cell, ppc: int):
    """The particles (a mask over fill_inputs' cell-major order, ppc per
    cell) sampled at step k of the harness's "sample" command, and the
    velocity scale s (Ir scales by s * s): cells c % 5 == 0 hold one
    particle on two steps of every 100, cells c % 5 == 1 lose a third of
    theirs in turn."""
    i = np.arange(len(cell))
    c = np.asarray(cell)
    keep = np.ones(len(c), dtype=bool)
    a = c % 5 == 0
    keep[a] = (k % 50 == 0) & (i[a] % ppc == 0)
    b = c % 5 == 1
    keep[b] = (k + i[b]) % 3 != 0
    return keep, 1.0 + (k % 8) / 16.0


def ragged(parts, ncell: int, ppc: int, seed: int):
    """Thin particles given ppc per cell in cell-major order: each cell keeps
    a share drawn uniformly in [0, 1), so counts run from 0 to ppc."""
    rs = np.random.RandomState(seed)
    x, v, ir, cell = parts
    keep = rs.random_sample(len(cell)) < np.repeat(rs.random_sample(ncell), ppc)
    return x[keep], v[keep], ir[keep], cell[keep]


def wall_trace_inputs(dm, mess, n: int, seed: int, wall_tag: int = 6, tets: bool = False):
    """Uniform random points in the hexahedra (or tetrahedra) that touch the
    wall zone, isotropic velocities with mean speed 3x the freestream speed,
    one dt."""
    e = dm.edges
    cells = np.unique(e["faceMap"][e["faceTag"] == wall_tag, 4])
    rs = np.random.RandomState(seed)
    c = rs.choice(cells, n).astype(np.int32)
    if tets:
        w = -np.log(rs.random_sample((n, 4)))
        w /= w.sum(1, keepdims=True)
        x = np.einsum("nk,nkd->nd", w, dm.points.reshape(-1, 3)[tet_vertices(dm, c)])
    else:
        lo, hi = cell_boxes(dm)
        x = lo[c] + (hi[c] - lo[c]) * rs.random_sample((n, 3))
    u, _, _ = freestream(mess)
    sigma = 3.0 * float(np.linalg.norm(u)) / math.sqrt(8.0 / math.pi)
    v = sigma * rs.standard_normal((n, 3))
    return x, v, np.full(n, float(mess["dtime"])), c


def host_sparse_rule(states, k: int):
    """The harness's hostRule: the sparse-state decisions the GSIS exchange
    writes back after exchange step k (k % 100 == 0), j = k // 100: normal
    cells c % 7 == 3 become accumulating (1) when j is odd, accumulating
    cells c % 3 == 0 are released (2) when j is even."""
    st = np.array(states, dtype=np.uint8)
    c = np.arange(len(st))
    j = k // 100
    acc = (st == 0) & (c % 7 == 3) & (j % 2 == 1)
    rel = (st == 1) & (c % 3 == 0) & (j % 2 == 0)
    st[acc] = 1
    st[rel] = 2
    return st


def fill_inputs(dm, mess, ppc: int, seed: int):
    """ppc particles per cell from the freestream Maxwellian."""
    rs = np.random.RandomState(seed)
    cells = np.repeat(np.arange(dm.ncell, dtype=np.int32), ppc)
    lo, hi = cell_boxes(dm)
    x = lo[cells] + (hi[cells] - lo[cells]) * rs.random_sample((cells.shape[0], 3))
    u, sig, tN = freestream(mess)
    v = u[None, :] + sig * rs.standard_normal((cells.shape[0], 3))
    ir = -np.log(1.0 - rs.random_sample(cells.shape[0])) * tN * 0.5
    return x, v, ir, cells


# the capsule case, coarse: a tetrahedral test mesh (10,729 tets)
CAPSULE_SMALL = dict(h_fine=0.7, h_coarse=2.0, r_fine=4.2, seed=0)


def capsule_small():
    from pydsmc import capsule
    raw = capsule.capsule_mesh(**CAPSULE_SMALL)
    dm = M.build_dsmc_mesh(raw)
    mess = C.mesh_message(dm, 5.0, 0.01, ppc=20, L0=capsule.L0)
    return raw, dm, mess


def tet_trace_inputs(dm, mess, n: int, seed: int):
    """Uniform random tetrahedra, uniform barycentric positions, isotropic
    velocities with mean speed 3x the freestream speed, one dt."""
    rs = np.random.RandomState(seed)
    cells = rs.randint(0, dm.ncell, size=n).astype(np.int32)
    P = dm.points.reshape(-1, 3)
    fm = dm.edges["faceMap"]
    f = dm.cells["cell2face"][cells, :2]
    a = fm[f[:, 0], :3]
    b = fm[f[:, 1], :3]
    in_a = (b[:, :, None] == a[:, None, :]).any(-1)
    extra = np.where(~in_a, b, -1).max(axis=1)
    verts = np.concatenate([a, extra[:, None]], axis=1)
    w = -np.log(rs.random_sample((n, 4)))
    w /= w.sum(1, keepdims=True)
    x = np.einsum("nk,nkd->nd", w, P[verts])
    u, _, _ = freestream(mess)
    sigma = 3.0 * float(np.linalg.norm(u)) / math.sqrt(8.0 / math.pi)
    v = sigma * rs.standard_normal((n, 3))
    dt = np.full(n, float(mess["dtime"]))
    return x, v, dt, cells


def tet_vertices(dm, cells):
    """The 4 distinct nodes of each tetrahedral cell, from its first two faces."""
    fm = dm.edges["faceMap"]
    f = dm.cells["cell2face"][cells, :2]
    a = fm[f[:, 0], :3]
    b = fm[f[:, 1], :3]
    in_a = (b[:, :, None] == a[:, None, :]).any(-1)
    extra = np.where(~in_a, b, -1).max(axis=1)
    return np.concatenate([a, extra[:, None]], axis=1)


def fill_inputs_any(dm, mess, ppc: int, seed: int):
    """fill_inputs for meshes of tetrahedra: uniform barycentric positions."""
    rs = np.random.RandomState(seed)
    cells = np.repeat(np.arange(dm.ncell, dtype=np.int32), ppc)
    P = dm.points.reshape(-1, 3)
    w = -np.log(rs.random_sample((cells.shape[0], 4)))
    w /= w.sum(1, keepdims=True)
    x = np.einsum("nk,nkd->nd", w, P[tet_vertices(dm, cells)])
    u, sig, tN = freestream(mess)
    v = u[None, :] + sig * rs.standard_normal((cells.shape[0], 3))
    ir = -np.log(1.0 - rs.random_sample(cells.shape[0])) * tN * 0.5
    return x, v, ir, cells


def gsis_inputs(dm, mess, ppc: int, seed: int, gate: bool = True, nan: bool = True):
    """An NS solution for the GSIS particle update: densities of 0.5x..1.6x
    the given particles per cell, drift perturbed around the freestream,
    T and Tr of 0.7x..1.4x T_in; with ``gate`` a 10% gated-out set, with
    ``nan`` a NaN velocity 37 cells before the end (gated in)."""
    rs = np.random.RandomState(seed)
    nc = dm.ncell
    vol = dm.cells["area"].astype(float)
    u0, sig, tN = freestream(mess)
    ns = np.zeros((nc, 6))
    ns[:, 0] = rs.uniform(0.5, 1.6, nc) * ppc * float(mess["Neff"]) / (vol * float(mess["n_ref"]))
    ns[:, 1:4] = u0 + 0.3 * rs.standard_normal((nc, 3))
    ns[:, 4] = tN * rs.uniform(0.7, 1.4, nc)
    ns[:, 5] = tN * rs.uniform(0.7, 1.4, nc)
    acc = (rs.random_sample(nc) > 0.1).astype(np.int8) if gate else None
    nan_cell = None
    if nan:
        nan_cell = nc - 37
        ns[nan_cell, 2] = np.nan
        if acc is not None:
            acc[nan_cell] = 1
    return ns, acc, nan_cell


def gsis_edge_inputs(dm, mess, ppc: int, seed: int, tets: bool = False):
    """Particles (fill_inputs, or fill_inputs_any on tetrahedra) with 40
    cells emptied, and an NS solution (gsis_inputs, gate on, NaN cell) in
    which 5 of the empty cells have T < 0 and 10 occupied cells a negative
    density."""
    x, v, ir, cell = (fill_inputs_any if tets else fill_inputs)(dm, mess, ppc, seed)
    rs = np.random.RandomState(seed + 1)
    empty = rs.choice(dm.ncell - 40, 40, replace=False)
    keep = ~np.isin(cell, empty)
    ns, acc, nan_cell = gsis_inputs(dm, mess, ppc, seed + 2)
    ns[empty[:5], 4] = -1.0
    acc[empty] = 1
    neg = rs.choice(np.setdiff1d(np.arange(dm.ncell - 40), empty), 10, replace=False)
    ns[neg, 0] = -ns[neg, 0]
    acc[neg] = 1
    return (x[keep], v[keep], ir[keep], cell[keep]), ns, acc, nan_cell, empty, neg


def macro_from_moments(mom_sum: np.ndarray, nsteps: int, dm, mess) -> np.ndarray:
    """The 18 macro fields of writeAveragedMacro (src/ProcessDSMC.cpp:
    3158-3179) from raw moment sums over nsteps steps: rho, u (3), T, the
    deviatoric stress (xx, xy, yy, yz, zz, zx), the heat flux (3), Tr and
    the rotational heat flux (3). Cells the reference zeroes
    (guardInvalidMacro, :3194-3211: no particles, rho, T or Tr not positive,
    a non-finite field) give NaN."""
    m = mom_sum.T
    N = m[0]
    out = np.full((mom_sum.shape[0], 18), np.nan)
    with np.errstate(divide="ignore", invalid="ignore"):
        rho = float(mess["Neff"]) / dm.cells["area"] * N / nsteps / float(mess["n_ref"])
        u = m[1:4] / N
        ux, uy, uz = u
        u2 = (u * u).sum(0)
        T = 2.0 / 3.0 / N * (m[4] - N * u2)
        c = 2.0 * rho / N
        dev = lambda a, b, d, ua, ub, ud: c * (2.0 / 3.0 * a - b / 3.0 - d / 3.0 - 2.0 / 3.0 * N * ua * ua +
                                              N * ub * ub / 3.0 + N * ud * ud / 3.0)
        out[:, 0] = rho
        out[:, 1:4] = u.T
        out[:, 4] = T
        out[:, 5] = dev(m[5], m[7], m[9], ux, uy, uz)
        out[:, 6] = c * (m[6] - N * ux * uy)
        out[:, 7] = dev(m[7], m[5], m[9], uy, ux, uz)
        out[:, 8] = c * (m[8] - N * uy * uz)
        out[:, 9] = dev(m[9], m[5], m[7], uz, ux, uy)
        out[:, 10] = c * (m[10] - N * uz * ux)
        out[:, 11] = rho / N * (m[11] - 2 * ux * m[5] - 2 * uy * m[6] - 2 * uz * m[10] + u2 * m[1]) - ux * 1.5 * T * rho
        out[:, 12] = rho / N * (m[12] - 2 * ux * m[6] - 2 * uy * m[7] - 2 * uz * m[8] + u2 * m[2]) - uy * 1.5 * T * rho
        out[:, 13] = rho / N * (m[13] - 2 * ux * m[10] - 2 * uy * m[8] - 2 * uz * m[9] + u2 * m[3]) - uz * 1.5 * T * rho
        out[:, 14] = 4.0 / float(mess["dr"]) / N * m[14]
        out[:, 15] = c * (m[15] - ux * m[14])
        out[:, 16] = c * (m[16] - uy * m[14])
        out[:, 17] = c * (m[17] - uz * m[14])
    valid = (N > 1e-12) & (out[:, 0] > 0) & (out[:, 4] > 0) & (out[:, 14] > 0) & np.isfinite(out).all(1)
    out[~valid] = np.nan
    return out


def fields_from_moments(mom_sum: np.ndarray, nsteps: int, dm, mess) -> np.ndarray:
    """Time-averaged rho (per step), u (3), T and Tr from summed raw moments."""
    N = mom_sum[:, 0]
    with np.errstate(divide="ignore", invalid="ignore"):
        rho = float(mess["Neff"]) / dm.cells["area"] * N / nsteps / float(mess["n_ref"])
        u = mom_sum[:, 1:4] / N[:, None]
        T = 2.0 / 3.0 * (mom_sum[:, 4] / N - (u * u).sum(1))
        Tr = 4.0 / float(mess["dr"]) * mom_sum[:, 14] / N
    return np.column_stack([rho, u, T, Tr])
