"""The device-side initial fill (dsmc_fill_freestream, dsmc_fill_initial);
the particle-by-particle comparison with the oracle is in test_gpu_gsis.py.

- Counts per cell follow setParticleMessage (src/meshImport.cpp:1399-1421):
  Np = floor(Ns) + [u < frac(Ns)], Ns = V_c * ppc * ncell / V_total, with u
  the 53-bit uniform of Philox block (c, 0, 4, 0) under the fill's seed,
  recomputed here with the oracle's Philox: exactly Np on tetrahedra (one
  placement tetrahedron per cell); on hexahedra the per-tetrahedron rounding
  and its clamp at zero (adjust_particles) can only add particles.
- Every particle lies in its cell: barycentric coordinates in [0, 1] for
  tetrahedra, inside the box for the block's hexahedra; positions are
  symmetric in the cell (mean barycentric coordinate 1/4, mean box-relative
  coordinate 1/2) and velocities follow the freestream Maxwellian (mean
  drift, variance T/2 per component) with Ir of mean T/2.
- The fill is deterministic in its seed, the same in FP64 and mixed
  precision up to FP32 rounding, and a case steps normally after it.
"""
import numpy as np
import pytest

import inputs as I
from gpu_util import make_case
from pydsmc import gpu
from pydsmc import workload as W

pytestmark = pytest.mark.gpu


def _expected_counts(dm, ppc, seed):
    from oracle import oracle as O
    vol = dm.cells["area"].astype(float)
    nps = ppc * dm.ncell
    key = [seed & 0xFFFFFFFF, seed >> 32]
    out = np.empty(dm.ncell, dtype=np.int64)
    vt = vol.sum()
    for c in range(dm.ncell):
        ns = vol[c] * nps / vt
        fl = np.floor(ns)
        b = O.philox([c, 0, 4, 0], key)
        k = (int(b[0]) << 21) ^ (int(b[1]) >> 11)
        u = (k + 0.5) * 2.0 ** -53
        out[c] = int(fl) + (1 if u < ns - fl else 0)
    return out


def _tet_vertices(dm):
    P = dm.points.reshape(-1, 3)
    f = dm.cells["cell2face"][:, :2]
    fm = dm.edges["faceMap"]
    a = fm[f[:, 0], :3]
    b = fm[f[:, 1], :3]
    in_a = (b[:, :, None] == a[:, None, :]).any(-1)
    extra = np.where(~in_a, b, -1).max(axis=1)
    return P[np.concatenate([a, extra[:, None]], axis=1)]          # [ncell, 4, 3]


def _fill(dm, mess, ppc, seed, precision):
    with make_case(dm, mess, precision=precision) as case:
        case.fill_freestream(ppc, seed)
        x, v, ir, cell = case.download_particles()
    return x, v, ir, cell


@pytest.fixture(scope="module")
def tets():
    return I.capsule_small()


def test_fill_on_tets(tets):
    raw, dm, mess = tets
    ppc, seed = 20, 12345
    x, v, ir, cell = _fill(dm, mess, ppc, seed, gpu.PRECISION_FP64)
    assert np.array_equal(np.bincount(cell, minlength=dm.ncell), _expected_counts(dm, ppc, seed))
    assert np.all(np.diff(cell) >= 0)                              # cell-major order
    V = _tet_vertices(dm)[cell]
    T = np.stack([V[:, 1] - V[:, 0], V[:, 2] - V[:, 0], V[:, 3] - V[:, 0]], axis=2)
    lam = np.linalg.solve(T, (x - V[:, 0])[:, :, None])[:, :, 0]
    bary = np.concatenate([1.0 - lam.sum(1, keepdims=True), lam], axis=1)
    assert bary.min() > -1e-9 and bary.max() < 1.0 + 1e-9
    assert np.all(np.abs(bary.mean(0) - 0.25) < 5e-3), bary.mean(0)
    u, sig, tN = W.freestream(mess, I.inflow_dir())
    n = len(cell)
    assert np.all(np.abs(v.mean(0) - u) < 5 * sig / np.sqrt(n))
    assert np.all(np.abs(v.var(0) / sig ** 2 - 1.0) < 0.02)
    assert abs(ir.mean() / (0.5 * tN) - 1.0) < 0.02
    # same seed, same fill; other seed, other fill
    x2, v2, ir2, cell2 = _fill(dm, mess, ppc, seed, gpu.PRECISION_FP64)
    assert np.array_equal(x, x2) and np.array_equal(v, v2) and np.array_equal(cell, cell2)
    x3, _, _, cell3 = _fill(dm, mess, ppc, seed + 1, gpu.PRECISION_FP64)
    assert not np.array_equal(cell3, cell) or not np.array_equal(x3, x)
    # mixed precision: the same particles up to FP32 rounding (cell-relative)
    xm, vm, irm, cellm = _fill(dm, mess, ppc, seed, gpu.PRECISION_MIXED)
    assert np.array_equal(cellm, cell)
    assert np.max(np.abs(xm - x)) < 1e-5 * np.abs(x).max()
    assert np.max(np.abs(vm - v)) < 1e-6 * np.abs(v).max()


def test_fill_on_hexes_then_steps(block):
    raw, dm, mess = block
    ppc, seed = 50, 7
    x, v, ir, cell = _fill(dm, mess, ppc, seed, gpu.PRECISION_FP64)
    excess = np.bincount(cell, minlength=dm.ncell) - _expected_counts(dm, ppc, seed)
    assert excess.min() >= 0 and excess.mean() < 0.5
    lo, hi = W.cell_boxes(dm)
    rel = (x - lo[cell]) / (hi[cell] - lo[cell])
    assert rel.min() >= -1e-9 and rel.max() <= 1.0 + 1e-9
    assert np.all(np.abs(rel.mean(0) - 0.5) < 5e-3)
    # stepping: fill at the density the case's Neff stands for (20 per cell
    # on average), so inflow and outflow balance
    with make_case(dm, mess, precision=gpu.PRECISION_MIXED, zones=I.REF_ZONES + [(7, gpu.ROLE_SPECULAR, 0)]) as case:
        case.fill_freestream(20, seed)
        n0 = case.particle_count()
        case.statistic_macroPre()
        for s in range(1, 6):
            case.step(s)
        c = case.counters()
        assert c["lost"] == 0 and c["overflow"] == 0 and c["collisions"] > 0 and c["injected"] > 0
        assert abs(case.particle_count() - n0) < 0.10 * n0
