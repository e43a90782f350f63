"""The oracle's initial fill and GSIS particle update, pinned against the
reference's own code (tests/golden/gsis_pin.npz, gsis_tet_pin.npz and
fill_pin.npz, made by gen_golden.py from oracle/_ref/ref_harness on the same
inputs).

The reference draws from mt19937 and rand(), the oracle (and the CUDA
library) from Philox, so the pins are the properties that do not depend on
the draws, compared exactly, and the distributions, compared by tests:

- update (hexahedra of the block, and the capsule tets): every updated cell
  holds floor or ceil of its NS count (the ceil as often as the fractional
  parts say), empty cells with T < 0 stay empty,
  negative densities keep the count, gated-out cells and cells from the NaN
  cell on are untouched; the particles that kept their position number
  min(before, after); every moved particle carries a kept particle's
  velocity (copies); after the update the moments equal the NS values; the
  moved particles' positions in the cell have the same distribution;
- fill: per-tetrahedron counts have the same rounding offsets, cells hold
  their counts, positions have the same distribution in the hexahedra
  (centre-face tetrahedra) and the same barycentric weights in the
  tetrahedra (four uniforms over their sum: not uniform), and the unit
  Maxwellian at rest has the same moments.
"""
import numpy as np
import pytest
from scipy import stats

import inputs as I
from conftest import OracleParams, golden


def _oracle(oracle_lib, dm, mess, seed=0):
    return oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir(), seed=seed))


def _summary(dm, before, after):
    from gen_golden import gsis_summary
    return gsis_summary(dm, before, after)


@pytest.fixture(scope="module")
def gsis_case(block, oracle_lib):
    raw, dm, mess = block
    g = golden("gsis_pin.npz")
    parts, ns, acc, nan_cell, empty, neg = I.gsis_edge_inputs(dm, mess, int(g["ppc"]), int(g["seed"]))
    o = _oracle(oracle_lib, dm, mess, seed=21)
    o.set_particles(*parts)
    rep = o.molecular_velocity_change(ns, acc)
    mine = _summary(dm, parts, o.particles())
    return dm, mess, parts, ns, acc, nan_cell, empty, neg, g, mine, rep


def test_update_counts_follow_the_reference(gsis_case):
    dm, mess, parts, ns, acc, nan_cell, empty, neg, g, mine, rep = gsis_case
    nc = dm.ncell
    n0 = np.bincount(parts[3], minlength=nc)
    upd = acc.astype(bool)
    upd[nan_cell:] = False
    x = ns[:, 0] * dm.cells["area"] * float(mess["n_ref"]) / float(mess["Neff"])
    fl = np.floor(x)
    regular = upd & ~np.isin(np.arange(nc), empty[:5]) & ~np.isin(np.arange(nc), neg)
    for res in (g, mine):
        n = res["counts"]
        assert np.array_equal(n[~upd], n0[~upd])                      # gate, NaN stop
        assert np.all(n[empty[:5]] == 0)                               # T < 0: no samples
        assert np.array_equal(n[neg], n0[neg])                         # deletion refused
        assert np.all((n[regular] == fl[regular]) | (n[regular] == fl[regular] + 1))
    # the ceiling as often as the fractional parts say, in both
    frac = (x - fl)[regular]
    for res in (g, mine):
        k = (res["counts"][regular] == fl[regular] + 1).sum()
        assert abs(k - frac.sum()) < 5 * np.sqrt((frac * (1 - frac)).sum())
    assert rep["nan_cell"] == nan_cell and rep["cells_updated"] == int(upd.sum())


def test_update_structure_and_moments_follow_the_reference(gsis_case):
    dm, mess, parts, ns, acc, nan_cell, empty, neg, g, mine, rep = gsis_case
    nc = dm.ncell
    n0 = np.bincount(parts[3], minlength=nc)
    upd = acc.astype(bool)
    upd[nan_cell:] = False
    dr = float(mess["dr"])
    for res in (g, mine):
        n = res["counts"].astype(float)
        assert np.array_equal(res["kept"], np.minimum(n0, res["counts"]))
        assert res["dup_ok"].all()
        live = upd & (n > 1)
        m = np.maximum(n, 1)
        T = 2.0 / (3.0 * m) * (res["sums"][:, 0] - n * (res["u"] ** 2).sum(1))
        Tr = 4.0 / dr / m * res["sums"][:, 1]
        ok = live & (T > 0)
        assert ok.sum() > 0.8 * live.sum()
        assert np.abs(res["u"][ok] - ns[ok, 1:4]).max() < 1e-12 * np.abs(ns[ok, 1:4]).max()
        assert np.abs(T[ok] / ns[ok, 4] - 1).max() < 1e-11
        assert np.abs(Tr[ok] / ns[ok, 5] - 1).max() < 1e-11


def test_update_positions_follow_the_reference(gsis_case):
    *_, g, mine, rep = gsis_case
    a, b = g["rel"], mine["rel"]
    assert len(a) > 500 and len(b) > 500
    assert a.min() >= 0 and a.max() <= 1 and b.min() >= 0 and b.max() <= 1
    for k in range(3):
        assert stats.ks_2samp(a[:, k], b[:, k]).pvalue > 1e-3
    ra = ((a - 0.5) ** 2).sum(1)
    rb = ((b - 0.5) ** 2).sum(1)
    assert stats.ks_2samp(ra, rb).pvalue > 1e-3


def test_fill_follows_the_reference(block, oracle_lib):
    raw, dm, mess = block
    g = golden("fill_pin.npz")
    ppc, seed = float(g["ppc"]), int(g["seed"])
    o = _oracle(oracle_lib, dm, mess)
    o.fill(ppc, seed, at_rest=True)
    x, v, ir, cell = o.particles()
    counts = g["counts"]
    mine_count = np.bincount(cell, minlength=dm.ncell)
    # adjust_particles clamps at zero, so a cell can end above Np: the same
    # excess distribution in both
    ea, eb = g["cell_count"] - counts, mine_count - counts
    assert ea.min() >= 0 and eb.min() >= 0
    vals = np.union1d(np.unique(ea), np.unique(eb))
    tab = np.array([[(ea == k).sum() for k in vals], [(eb == k).sum() for k in vals]])
    assert stats.chi2_contingency(tab).pvalue > 1e-3
    # per-tetrahedron counts: the same offsets from Np V_t / V_cell
    off, V, vol = o.placement()
    ref_tri = g["np_tri"].astype(np.int64)
    assert len(ref_tri) == off[-1]
    cell_of = np.repeat(np.arange(dm.ncell), np.diff(off))
    share = counts[cell_of] * vol / np.add.reduceat(vol, off[:-1])[cell_of]
    mine_tri = np.zeros(off[-1], np.int64)
    first = np.concatenate([[0], np.cumsum(np.bincount(cell, minlength=dm.ncell))])
    lo, hi = I.cell_boxes(dm)
    rel = (x - lo[cell]) / (hi[cell] - lo[cell])
    # the oracle places tetrahedron by tetrahedron: recover counts from positions
    for c in range(dm.ncell):
        P = x[first[c]:first[c + 1]]
        for t in range(off[c], off[c + 1]):
            A = V[t]
            T = np.stack([A[1] - A[0], A[2] - A[0], A[3] - A[0]], 1)
            lam = np.linalg.solve(T, (P - A[0]).T).T
            inside = (lam >= -1e-12).all(1) & (lam.sum(1) <= 1 + 1e-12)
            mine_tri[t] = int(inside.sum())
    assert np.array_equal(np.add.reduceat(mine_tri, off[:-1]), mine_count)
    assert np.array_equal(np.add.reduceat(ref_tri, off[:-1]), g["cell_count"])
    da = ref_tri - np.floor(share)
    db = mine_tri - np.floor(share)
    assert set(np.unique(da)) <= {-1, 0, 1, 2} and set(np.unique(db)) <= {-1, 0, 1, 2}
    ta = np.array([(da == k).sum() for k in (-1, 0, 1, 2)])
    tb = np.array([(db == k).sum() for k in (-1, 0, 1, 2)])
    keep = (ta + tb) > 0
    assert stats.chi2_contingency(np.stack([ta[keep], tb[keep]])).pvalue > 1e-3
    for k in range(3):
        assert stats.ks_2samp(g["rel"][:, k], rel[:, k]).pvalue > 1e-3
    assert stats.ks_2samp(((g["rel"] - 0.5) ** 2).sum(1), ((rel - 0.5) ** 2).sum(1)).pvalue > 1e-3
    # unit Maxwellian at rest, Ir with mean 1/2
    n = int(g["n_v"])
    assert np.all(np.abs(v.mean(0) - g["v_mean"]) < 5 * np.sqrt(1.0 / len(v) + 1.0 / n))
    assert np.all(np.abs(v.var(0) - g["v_var"]) < 5 * np.sqrt(2.0 / len(v) + 2.0 / n))
    assert abs(ir.mean() - float(g["ir_mean"])) < 5 * np.sqrt(0.25 / len(v) + 0.25 / n)


def test_fill_barycentric_weights_follow_the_reference(oracle_lib):
    raw, dm, mess = I.capsule_small()
    g = golden("fill_pin.npz")
    o = _oracle(oracle_lib, dm, mess)
    o.fill(float(g["ppc"]), int(g["seed"]), at_rest=True)
    x, v, ir, cell = o.particles()
    ntet = int(g["tet_cells"])
    assert np.array_equal(np.bincount(cell, minlength=dm.ncell)[:ntet], g["tet_count"][:ntet])
    sel = cell < ntet
    from gen_golden import sorted_barycentric
    b = sorted_barycentric(dm, x[sel], cell[sel])
    a = g["bary"]
    assert b.min() > -1e-9 and b.max() < 1 + 1e-9
    for k in range(4):
        assert stats.ks_2samp(a[:, k], b[:, k]).pvalue > 1e-3
    # not uniform in the tetrahedron: the largest weight is far below the
    # Dirichlet(1,1,1,1) value (mean 25/48)
    assert a[:, 3].mean() < 0.45 and b[:, 3].mean() < 0.45


def test_placement_tetrahedra_fill_the_cells(block, oracle_lib):
    for raw, dm, mess in (block, I.capsule_small()):
        o = _oracle(oracle_lib, dm, mess)
        off, V, vol = o.placement()
        assert np.all(np.diff(off) > 0)
        assert np.abs(np.add.reduceat(vol, off[:-1]) / dm.cells["area"] - 1.0).max() < 1e-9


@pytest.fixture(scope="module")
def gsis_tet_case(oracle_lib):
    raw, dm, mess = I.capsule_small()
    g = golden("gsis_tet_pin.npz")
    parts, ns, acc, nan_cell, empty, neg = I.gsis_edge_inputs(dm, mess, int(g["ppc"]), int(g["seed"]), tets=True)
    o = _oracle(oracle_lib, dm, mess, seed=21)
    o.set_particles(*parts)
    rep = o.molecular_velocity_change(ns, acc)
    from gen_golden import gsis_summary
    mine = gsis_summary(dm, parts, o.particles(), tets=True)
    return dm, mess, parts, ns, acc, nan_cell, empty, neg, g, mine, rep


def test_update_on_tets_follows_the_reference(gsis_tet_case):
    """The update on the capsule tets: counts, kept particles and copies as
    on hexahedra, the moments equal to the NS values in both, and the moved
    particles' sorted barycentric weights (four uniforms over their sum, the
    reference's placement in a tetrahedron) with the same distribution."""
    from gen_golden import gsis_moment_errors
    dm, mess, parts, ns, acc, nan_cell, empty, neg, g, mine, rep = gsis_tet_case
    nc = dm.ncell
    n0 = np.bincount(parts[3], minlength=nc)
    upd = acc.astype(bool)
    upd[nan_cell:] = False
    x = ns[:, 0] * dm.cells["area"] * float(mess["n_ref"]) / float(mess["Neff"])
    fl = np.floor(x)
    regular = upd & ~np.isin(np.arange(nc), empty[:5]) & ~np.isin(np.arange(nc), neg)
    frac = (x - fl)[regular]
    for res in (g, mine):
        n = res["counts"]
        assert np.array_equal(n[~upd], n0[~upd])
        assert np.all(n[empty[:5]] == 0)
        assert np.array_equal(n[neg], n0[neg])
        assert np.all((n[regular] == fl[regular]) | (n[regular] == fl[regular] + 1))
        k = (n[regular] == fl[regular] + 1).sum()
        assert abs(k - frac.sum()) < 5 * np.sqrt((frac * (1 - frac)).sum())
        assert np.array_equal(res["kept"], np.minimum(n0, n))
        assert res["dup_ok"].all()
    assert rep["nan_cell"] == nan_cell and rep["cells_updated"] == int(upd.sum())
    err = gsis_moment_errors(dm, mess, parts[3], ns, acc, nan_cell, mine)
    for e in (g, err):
        assert float(e["ok_share"]) > 0.8
        assert float(e["u_err"]) < 1e-12 and float(e["T_err"]) < 1e-11 and float(e["Tr_err"]) < 1e-11
    a, b = g["rel"].astype(float), mine["rel"]
    assert len(b) > 5000 and abs(len(b) / int(g["n_rel"]) - 1) < 0.1
    assert b.min() > -1e-9 and b.max() < 1 + 1e-9
    for k in range(4):
        assert stats.ks_2samp(a[:, k], b[:, k]).pvalue > 1e-3
    # not uniform in the tetrahedron (Dirichlet(1,1,1,1): mean largest weight 25/48)
    assert a[:, 3].mean() < 0.45 and b[:, 3].mean() < 0.45
