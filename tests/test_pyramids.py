"""Pyramid cells and mixed triangle / quad faces, on the CPU, against the
reference's own code (tests/golden/pyramid_pin.npz, made by gen_golden.py
from oracle/_ref/ref_harness): a box of cubes, each split into six pyramids
around its centre.

- The Python mesh builder and the native CAS reader (dsmc_mesh_read_cas)
  give the reference's DsmcCell / DsmcEdge / points / split-tag arrays bit
  for bit.
- Placement: a pyramid is split into its two base triangles with the apex
  (appendPyramidCellTets), and the two tetrahedra fill the cell.
- The oracle's initial fill follows the reference's on these cells: two
  per-tetrahedron counts per cell with the same rounding offsets, the same
  distribution of positions in each cube, and the unit Maxwellian moments.
- The oracle's tracing check is bit-exact with the reference's on these
  cells (tests/golden/pyramid_trace_pin.npz): crossings through triangles
  and split quads, exits through the inlet, outlet and side zones.
"""

import numpy as np
import pytest
from scipy import stats

import inputs as I
from conftest import OracleParams, golden
from pydsmc import mesh as M
from pydsmc import meshio as IO


@pytest.fixture(scope="module")
def pyr():
    from gen_golden import pyramid_case
    return pyramid_case()


def _same(a, g):
    for f in M.DSMC_CELL_DTYPE.names:
        if f == "no":
            continue
        assert np.array_equal(a.cells[f], g["cells"][f]), f
    for f in M.DSMC_EDGE_DTYPE.names:
        assert np.array_equal(a.edges[f], g["edges"][f]), f
    assert np.array_equal(a.points, g["points"])
    assert np.array_equal(a.split, g["split"])


def test_builder_and_native_reader_match_the_reference(pyr, tmp_path):
    raw, dm, mess = pyr
    g = golden("pyramid_pin.npz")
    assert set(np.unique(dm.cells["num"]).tolist()) == {5}
    assert set(np.unique(dm.edges["faceType"]).tolist()) == {3, 4}
    _same(dm, g)
    cas = str(tmp_path / "p.cas")
    M.write_cas(cas, raw)
    with IO.MeshFile(cas) as mf:
        _same(mf.dsmc_mesh(), g)


def test_pyramid_placement_is_two_tetrahedra(pyr, oracle_lib):
    raw, dm, mess = pyr
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir()))
    off, V, vol = o.placement()
    assert np.all(np.diff(off) == 2)
    assert np.abs(np.add.reduceat(vol, off[:-1]) / dm.cells["area"] - 1.0).max() < 1e-12
    # both tetrahedra share the apex (the cube centre) as their last vertex
    assert np.array_equal(V[0::2, 3], V[1::2, 3])


def test_fill_on_pyramids_follows_the_reference(pyr, oracle_lib):
    from gen_golden import PYR_PPC, PYR_SEED, cube_relative
    raw, dm, mess = pyr
    g = golden("pyramid_pin.npz")
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir()))
    o.fill(float(PYR_PPC), PYR_SEED, at_rest=True)
    x, v, ir, cell = o.particles()
    mine_count = np.bincount(cell, minlength=dm.ncell)
    counts = g["counts"]
    # two tetrahedra per cell in the reference too; its counts sum to the cell's
    ref_tri = g["np_tri"].astype(np.int64)
    assert len(ref_tri) == 2 * dm.ncell
    assert np.array_equal(ref_tri[0::2] + ref_tri[1::2], g["cell_count"])
    assert (mine_count - counts).min() >= 0 and (g["cell_count"] - counts).min() >= 0
    # per-tetrahedron offsets from Np V_t / V_cell: the same distribution
    off, V, vol = o.placement()
    share = np.repeat(counts, 2) * vol / np.repeat(np.add.reduceat(vol, off[:-1]), 2)
    first = np.concatenate([[0], np.cumsum(mine_count)])
    mine_tri = np.zeros(2 * dm.ncell, np.int64)
    for c in range(dm.ncell):
        P = x[first[c]:first[c + 1]]
        for t in (2 * c, 2 * c + 1):
            A = V[t]
            T = np.stack([A[1] - A[0], A[2] - A[0], A[3] - A[0]], 1)
            lam = np.linalg.solve(T, (P - A[0]).T).T
            mine_tri[t] = int(((lam >= -1e-12).all(1) & (lam.sum(1) <= 1 + 1e-12)).sum())
    assert np.array_equal(mine_tri[0::2] + mine_tri[1::2], mine_count)
    da, db = ref_tri - np.floor(share), mine_tri - np.floor(share)
    vals = np.union1d(np.unique(da), np.unique(db))
    assert set(vals.tolist()) <= {-1, 0, 1, 2}
    tab = np.array([[(da == k).sum() for k in vals], [(db == k).sum() for k in vals]])
    keep = tab.sum(0) > 0
    assert stats.chi2_contingency(tab[:, keep]).pvalue > 1e-3
    rel = cube_relative(x, cell)
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


def test_trace_on_pyramids_is_bit_exact_vs_reference(pyr, oracle_lib):
    raw, dm, mess = pyr
    g = golden("pyramid_trace_pin.npz")
    assert dm.ncell == int(g["ncell"])
    x, v, dt, cell = I.pyramid_trace_inputs(raw, mess, len(g["cell"]), seed=6)
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir()))
    r = o.trace(x, v, dt, cell, stop_at_wall=True)
    for k in ("cell", "ifout", "face", "tri", "ncross", "x", "dt"):
        assert np.array_equal(r[k], g[k]), k
    # every outcome, both face kinds and both halves of the split quads
    assert {-1, 0, 1} <= set(np.unique(g["ifout"]).tolist())
    assert g["ncross"].max() >= 6
    hit = g["face"] >= 0
    kinds = set(dm.edges["faceType"][g["face"][hit]].tolist())
    assert kinds == {4}                      # only the box's quads are boundary faces
    assert len(set(g["tri"][hit].tolist())) == 2
