"""The reference's initial fill and the GSIS particle update on the B200,
against the oracle's restatement on the same inputs.

- dsmc_fill_initial / dsmc_fill_freestream (Np_tri_inititial, meshfillpar,
  velocityLocationGenerate): counts per cell and per placement tetrahedron
  and every position bit for bit in FP64 (pure arithmetic on the same
  Philox draws); velocities and Ir, which go through log / sin / cos, within
  1e-13 relative (CUDA's and the host C library's last bits differ).
- dsmc_molecular_velocity_change (molecular_velocity_change, replication,
  deletion, MaxwellianSample, randomlocation): the report, the counts, which
  particles are kept, copied or deleted and every position bit for bit;
  velocities and Ir bit for bit where no Maxwellian sample entered the cell
  (copies and the linear map are IEEE arithmetic in the same order), within
  1e-12 of the velocity scale in the cells that were empty. After the
  update every updated cell's mean velocity, T and Tr equal the NS values
  (to rounding); gated-out cells and cells from the first NaN cell on are
  untouched.
- Edge cases the reference has: empty cells (Maxwellian sampling, refused
  for T < 0), negative densities (deletion refused), the acceptance gate,
  NaN stop, repeated updates, growth of the particle store, a fixed store
  that is too small and a density out of range (particles untouched).
- Mixed precision: same counts and choices, moments within FP32 rounding.
"""
import numpy as np
import pytest

import inputs as I
from gpu_util import make_case, make_oracle, rel_close
from pydsmc import gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tets():
    return I.capsule_small()


def _moments(v, ir, cell, ncell, dr):
    n = np.bincount(cell, minlength=ncell).astype(float)
    m = np.maximum(n, 1.0)
    u = np.stack([np.bincount(cell, v[:, k], ncell) for k in range(3)], 1) / m[:, None]
    s2 = np.bincount(cell, (v * v).sum(1), ncell)
    T = 2.0 / (3.0 * m) * (s2 - n * (u * u).sum(1))
    Tr = 4.0 / dr / m * np.bincount(cell, ir, ncell)
    return n, u, T, Tr


def _run_both(dm, mess, parts, ns, acc, precision=gpu.PRECISION_FP64, seed=9, updates=1):
    x, v, ir, cell = parts
    with make_case(dm, mess, seed=seed, precision=precision) as case:
        case.upload_particles(x, v, ir, cell)
        reps = [case.molecular_velocity_change(ns, acc) for _ in range(updates)]
        g = case.download_particles()
    o = make_oracle(dm, mess, seed=seed)
    o.set_particles(x, v, ir, cell)
    oreps = [o.molecular_velocity_change(ns, acc) for _ in range(updates)]
    return reps, g, oreps, o.particles()


def _compare_update(dm, mess, parts, ns, acc, nan_cell, updates=1):
    reps, (xg, vg, irg, cg), oreps, (xo, vo, iro, co) = _run_both(dm, mess, parts, ns, acc, updates=updates)
    for r, ro in zip(reps, oreps):
        assert r == ro
    assert np.array_equal(cg, co)
    assert np.array_equal(xg, xo)
    # cells that were empty before the update took Maxwellian samples
    n_in = np.bincount(parts[3], minlength=dm.ncell)
    sampled = np.isin(cg, np.flatnonzero(n_in == 0))
    assert np.array_equal(vg[~sampled], vo[~sampled])
    assert np.array_equal(irg[~sampled], iro[~sampled])
    # log / sin differ in the last bit; components near zero after the
    # linear map are compared on the scale of the cell's velocities
    assert rel_close(vg[sampled], vo[sampled], 1e-12, 1e-12 * np.abs(vo).max()).all()
    assert rel_close(irg[sampled], iro[sampled], 1e-12, 1e-12 * np.abs(iro).max()).all()
    # the NS state is reached in every updated cell; the others are untouched
    nc = dm.ncell
    upd = np.ones(nc, bool) if acc is None else acc.astype(bool)
    if nan_cell is not None:
        upd[nan_cell:] = False
    n, u, T, Tr = _moments(vg, irg, cg, nc, float(mess["dr"]))
    live = upd & (n > 1) & (T > 0)
    assert live.sum() > 0.5 * upd.sum()
    assert np.abs(u[live] - ns[live, 1:4]).max() < 1e-12 * np.abs(ns[live, 1:4]).max()
    assert np.abs(T[live] / ns[live, 4] - 1.0).max() < 1e-11
    assert np.abs(Tr[live] / ns[live, 5] - 1.0).max() < 1e-11
    x, v, ir, cell = parts
    keep = np.isin(cg, np.flatnonzero(~upd))
    keep_in = np.isin(cell, np.flatnonzero(~upd))
    assert np.array_equal(np.sort(vg[keep][:, 0]), np.sort(v[keep_in][:, 0]))
    return reps[-1]


def test_update_on_hexes_matches_oracle(block):
    raw, dm, mess = block
    parts = I.fill_inputs(dm, mess, 20, seed=11)
    ns, acc, nan_cell = I.gsis_inputs(dm, mess, 20, seed=5)
    rep = _compare_update(dm, mess, parts, ns, acc, nan_cell)
    assert rep["nan_cell"] == nan_cell and rep["cells_skipped"] > 0
    assert rep["added"] > 0 and rep["removed"] > 0


def test_update_on_tets_matches_oracle(tets):
    raw, dm, mess = tets
    x, v, ir, cell = I.fill_inputs_any(dm, mess, 8, seed=12)
    ns, acc, _ = I.gsis_inputs(dm, mess, 8, seed=6, nan=False)
    _compare_update(dm, mess, (x, v, ir, cell), ns, acc, None)


def test_update_edge_cases_match_oracle(block):
    """Empty cells (sampled; refused for T < 0), negative densities
    (deletion refused), the gate and NaN stop, two updates in a row; then
    the gate off."""
    raw, dm, mess = block
    parts, ns, acc, nan_cell, empty, neg = I.gsis_edge_inputs(dm, mess, 12, seed=13)
    rep = _compare_update(dm, mess, parts, ns, acc, nan_cell, updates=2)
    assert rep["nan_cell"] == nan_cell
    ns_all = ns.copy()
    ns_all[nan_cell, 2] = 1.0
    _compare_update(dm, mess, parts, ns_all, None, None)
    with make_case(dm, mess, seed=9) as case:
        case.upload_particles(*parts)
        case.molecular_velocity_change(ns, acc)
        _, _, _, cg = case.download_particles()
    n = np.bincount(cg, minlength=dm.ncell)
    assert np.all(n[empty[:5]] == 0) and np.all(n[empty[5:]] > 0)
    assert np.array_equal(n[neg], np.bincount(parts[3], minlength=dm.ncell)[neg])


def test_update_grows_the_store_and_refuses_bad_input(block):
    raw, dm, mess = block
    x, v, ir, cell = I.fill_inputs(dm, mess, 20, seed=15)
    ns, _, _ = I.gsis_inputs(dm, mess, 20, seed=8, gate=False, nan=False)
    big = ns.copy()
    big[:, 0] *= 90.0                            # about 1.4M particles: beyond the automatic store
    with make_case(dm, mess, seed=3) as case:
        case.upload_particles(x, v, ir, cell)
        rep = case.molecular_velocity_change(big)
        assert rep["particles"] > 1_200_000 and case.particle_count() == rep["particles"]
        xg, vg, irg, cg = case.download_particles()
        n, u, T, Tr = _moments(vg, irg, cg, dm.ncell, float(mess["dr"]))
        assert np.abs(T / big[:, 4] - 1.0).max() < 1e-11
        for s in range(1, 3):
            case.step(s)
        assert case.counters()["lost"] == 0
    for bad, code in ((1e12, "(-1)"), (None, "(-4)")):
        cap = 0 if bad is not None else len(cell) + 1000
        with make_case(dm, mess, seed=3, capacity=cap) as case:
            case.upload_particles(x, v, ir, cell)
            b = ns.copy()
            b[:, 0] *= 3.0 if bad is None else bad
            with pytest.raises(gpu.DsmcError) as e:
                case.molecular_velocity_change(b)
            assert code in str(e.value)
            xg, vg, irg, cg = case.download_particles()
            assert np.array_equal(cg, np.sort(cell, kind="stable")) and case.particle_count() == len(cell)
            case.step(1)                             # still usable


def test_update_mixed_precision(block):
    raw, dm, mess = block
    parts = I.fill_inputs(dm, mess, 20, seed=16)
    ns, acc, nan_cell = I.gsis_inputs(dm, mess, 20, seed=9)
    reps, (xg, vg, irg, cg), oreps, (xo, vo, iro, co) = _run_both(dm, mess, parts, ns, acc,
                                                                  precision=gpu.PRECISION_MIXED)
    assert reps[0] == oreps[0]
    assert np.array_equal(cg, co)
    assert np.abs(xg - xo).max() < 1e-5 * np.abs(xo).max()
    upd = acc.astype(bool)
    upd[nan_cell:] = False
    n, u, T, Tr = _moments(vg, irg, cg, dm.ncell, float(mess["dr"]))
    live = upd & (n > 1)
    assert np.abs(u[live] - ns[live, 1:4]).max() < 1e-5 * np.abs(ns[live, 1:4]).max()
    assert np.abs(T[live] / ns[live, 4] - 1.0).max() < 1e-4
    assert np.abs(Tr[live] / ns[live, 5] - 1.0).max() < 1e-5


@pytest.mark.parametrize("at_rest", [True, False])
def test_fill_matches_oracle(block, tets, at_rest):
    for raw, dm, mess in (block, tets):
        ppc, seed = 13, 4242
        with make_case(dm, mess) as case:
            (case.fill_initial if at_rest else case.fill_freestream)(ppc, seed)
            xg, vg, irg, cg = case.download_particles()
        o = make_oracle(dm, mess)
        o.fill(ppc, seed, at_rest=at_rest)
        xo, vo, iro, co = o.particles()
        assert np.array_equal(cg, co)
        assert np.array_equal(xg, xo)
        assert rel_close(vg, vo, 1e-13, 1e-14).all()
        assert rel_close(irg, iro, 1e-13, 1e-300).all()
        with make_case(dm, mess, precision=gpu.PRECISION_MIXED) as case:
            (case.fill_initial if at_rest else case.fill_freestream)(ppc, seed)
            xm, vm, irm, cm = case.download_particles()
        assert np.array_equal(cm, co)
        assert np.abs(xm - xo).max() < 1e-5 * np.abs(xo).max()
        assert np.abs(vm - vo).max() < 1e-6 * np.abs(vo).max()
