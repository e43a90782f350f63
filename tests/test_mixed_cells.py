"""Pyramid and wedge cells with mixed triangle / quad faces, on the CPU,
against the reference's own code (tests/golden/pyramid_pin.npz,
pyramid_trace_pin.npz and prism_pin.npz, made by gen_golden.py from
oracle/_ref/ref_harness): a box of cubes, each split into six pyramids
around its centre (Fluent element type 5) or into two wedges by a diagonal
plane (type 6).

- The Python mesh builder and the native CAS reader (dsmc_mesh_read_cas)
  give the reference's DsmcCell / DsmcEdge / points / split-tag arrays bit
  for bit.
- Placement: a pyramid is split into its two base triangles with the apex
  (appendPyramidCellTets); a wedge takes the centre-face tetrahedra
  (appendCenterFaceTets: one per triangle, two per quad, eight per wedge).
  The tetrahedra fill the cell.
- The oracle's initial fill follows the reference's on these cells: the
  per-tetrahedron counts have the same rounding offsets, the positions the
  same distribution in each cube, and the unit Maxwellian the same moments.
- The oracle's tracing check is bit-exact with the reference's on these
  cells: crossings through triangles and split quads, exits through the
  inlet, outlet and side zones.
"""

import numpy as np
import pytest
from scipy import stats

import inputs as I
from conftest import OracleParams, golden
from pydsmc import mesh as M
from pydsmc import meshio as IO

KINDS = {
    # case builder, cells per cube, fill seed, pin files, trace seed, cell type, tetrahedra per cell
    "pyramid": ("pyramid_case", 6, "PYR_SEED", ("pyramid_pin.npz", "pyramid_trace_pin.npz", ""), 6, 5, 2),
    "prism": ("prism_case", 2, "PRISM_SEED", ("prism_pin.npz", "prism_pin.npz", "trace_"), 7, 6, 8),
}


@pytest.fixture(scope="module", params=sorted(KINDS))
def kind(request):
    import gen_golden as G
    name = request.param
    case, per_cube, seed, files, tseed, ctype, ntet = KINDS[name]
    raw, dm, mess = getattr(G, case)()
    return {"name": name, "raw": raw, "dm": dm, "mess": mess, "per_cube": per_cube, "seed": getattr(G, seed),
            "fill": golden(files[0]), "trace": golden(files[1]), "prefix": files[2], "trace_seed": tseed,
            "cell_type": ctype, "ntet": ntet}


def _same(a, g):
    for f in M.DSMC_CELL_DTYPE.names:
        if f == "no":
            continue
        assert np.array_equal(a.cells[f], g["cells"][f]), f
    for f in M.DSMC_EDGE_DTYPE.names:
        assert np.array_equal(a.edges[f], g["edges"][f]), f
    assert np.array_equal(a.points, g["points"])
    assert np.array_equal(a.split, g["split"])


def _oracle(oracle_lib, k):
    return oracle_lib.Oracle(k["dm"], k["mess"], OracleParams(I.REF_ZONES, I.inflow_dir()))


def test_builder_and_native_reader_match_the_reference(kind, tmp_path):
    raw, dm, g = kind["raw"], kind["dm"], kind["fill"]
    assert raw.cell_type == kind["cell_type"]
    assert set(np.unique(dm.cells["num"]).tolist()) == {5}
    assert set(np.unique(dm.edges["faceType"]).tolist()) == {3, 4}
    _same(dm, g)
    cas = str(tmp_path / "m.cas")
    M.write_cas(cas, raw)
    with IO.MeshFile(cas) as mf:
        _same(mf.dsmc_mesh(), g)


def test_placement_tetrahedra(kind, oracle_lib):
    dm = kind["dm"]
    off, V, vol = _oracle(oracle_lib, kind).placement()
    assert np.all(np.diff(off) == kind["ntet"])
    assert np.abs(np.add.reduceat(vol, off[:-1]) / dm.cells["area"] - 1.0).max() < 1e-12
    if kind["name"] == "pyramid":
        # both tetrahedra share the apex (the cube centre) as their last vertex
        assert np.array_equal(V[0::2, 3], V[1::2, 3])
    else:
        # every tetrahedron has the cell centre as its first vertex
        cell_of = np.repeat(np.arange(dm.ncell), kind["ntet"])
        assert np.array_equal(V[:, 0], dm.cells["cellXY"][cell_of])


def test_fill_follows_the_reference(kind, oracle_lib):
    from gen_golden import PYR_PPC, cube_relative
    dm, g = kind["dm"], kind["fill"]
    o = _oracle(oracle_lib, kind)
    o.fill(float(PYR_PPC), kind["seed"], at_rest=True)
    x, v, ir, cell = o.particles()
    mine_count = np.bincount(cell, minlength=dm.ncell)
    counts = g["counts"]
    off, V, vol = o.placement()
    ref_tri = g["np_tri"].astype(np.int64)
    assert len(ref_tri) == off[-1]
    assert np.array_equal(np.add.reduceat(ref_tri, off[:-1]), g["cell_count"])
    assert (mine_count - counts).min() >= 0 and (g["cell_count"] - counts).min() >= 0
    # per-tetrahedron offsets from Np V_t / V_cell: the same distribution
    cell_of = np.repeat(np.arange(dm.ncell), np.diff(off))
    share = counts[cell_of] * vol / np.add.reduceat(vol, off[:-1])[cell_of]
    first = np.concatenate([[0], np.cumsum(mine_count)])
    mine_tri = np.zeros(off[-1], np.int64)
    for c in range(dm.ncell):
        P = x[first[c]:first[c + 1]]
        for t in range(off[c], off[c + 1]):
            A = V[t]
            T = np.stack([A[1] - A[0], A[2] - A[0], A[3] - A[0]], 1)
            lam = np.linalg.solve(T, (P - A[0]).T).T
            mine_tri[t] = int(((lam >= -1e-12).all(1) & (lam.sum(1) <= 1 + 1e-12)).sum())
    assert np.array_equal(np.add.reduceat(mine_tri, off[:-1]), mine_count)
    da, db = ref_tri - np.floor(share), mine_tri - np.floor(share)
    vals = np.union1d(np.unique(da), np.unique(db))
    assert set(vals.tolist()) <= {-1, 0, 1, 2}
    tab = np.array([[(da == k).sum() for k in vals], [(db == k).sum() for k in vals]])
    keep = tab.sum(0) > 0
    assert stats.chi2_contingency(tab[:, keep]).pvalue > 1e-3
    rel = cube_relative(x, cell, kind["per_cube"])
    assert rel.min() >= -1e-12 and rel.max() <= 1 + 1e-12
    for k in range(3):
        assert stats.ks_2samp(g["rel"][:, k], rel[:, k]).pvalue > 1e-3
    ra = ((g["rel"] - 0.5) ** 2).sum(1)
    rb = ((rel - 0.5) ** 2).sum(1)
    assert stats.ks_2samp(ra, rb).pvalue > 1e-3
    n = int(g["n_v"])
    assert np.all(np.abs(v.mean(0) - g["v_mean"]) < 5 * np.sqrt(1.0 / len(v) + 1.0 / n))
    assert np.all(np.abs(v.var(0) - g["v_var"]) < 5 * np.sqrt(2.0 / len(v) + 2.0 / n))
    assert abs(ir.mean() - float(g["ir_mean"])) < 5 * np.sqrt(0.25 / len(v) + 0.25 / n)


def test_trace_is_bit_exact_vs_reference(kind, oracle_lib):
    dm, g, p = kind["dm"], kind["trace"], kind["prefix"]
    assert dm.ncell == int(g[p + "ncell"])
    x, v, dt, cell = I.split_box_trace_inputs(kind["raw"], kind["mess"], len(g[p + "cell"]), seed=kind["trace_seed"])
    r = _oracle(oracle_lib, kind).trace(x, v, dt, cell, stop_at_wall=True)
    for k in ("cell", "ifout", "face", "tri", "ncross", "x", "dt"):
        assert np.array_equal(r[k], g[p + k]), k
    # every outcome, and both halves of the split boundary quads
    assert {-1, 0, 1} <= set(np.unique(g[p + "ifout"]).tolist())
    assert g[p + "ncross"].max() >= 6
    hit = g[p + "face"] >= 0
    assert len(set(g[p + "tri"][hit & (dm.edges["faceType"][np.maximum(g[p + "face"], 0)] == 4)].tolist())) == 2
