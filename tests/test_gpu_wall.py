"""Wall statistics on the B200 (recordBoundaryStressHeat,
src/ProcessDSMC.cpp:1659-1689, read with dsmc_download_wall and converted as
outBoundaryStressHeat does, :3494-3552).

- Against the oracle (the same Philox streams): after one step of the
  block case and of the capsule tets, every wall face's hit count equals
  the oracle's and its five momentum / energy tallies agree to 1e-10 of
  their scale (the device adds them with FP64 atomics in another order, and
  CUDA's log / sincospi round the re-emitted velocities differently in the
  last bit); after three steps with collisions the totals agree to 1e-6.
- Kinetic theory, on a box of diffuse walls at the gas temperature, in both
  precisions: the hits per area are the one-sided flux n s / sqrt(2 pi), the
  normal stress is p = rho T, the shear and the heat flux vanish (within 4
  standard errors over the faces, and p within 3%).
"""
import math

import numpy as np
import pytest

import inputs as I
from gpu_util import make_case, make_oracle
from pydsmc import case as C
from pydsmc import gpu
from pydsmc import mesh as M

pytestmark = pytest.mark.gpu

DIFFUSE = [(3, 1, 0), (4, 4, 0), (5, 4, 0), (7, 4, 0)]


def _tallies_close(t, to, rtol):
    scale = np.abs(to).max(axis=0) + 1e-300
    return np.all(np.abs(t - to) <= rtol * scale)


def _compare_with_oracle(dm, mess, x, v, ir, cell, steps, exact_hits, rtol):
    with make_case(dm, mess, seed=5, nss=0, wall_stats=1) as case:
        case.upload_particles(x, v, ir, cell)
        for s in range(1, steps + 1):
            case.step(s)
        t = case.wall()
        c = case.counters()
    o = make_oracle(dm, mess, seed=5, nss=0, wall_stats=1)
    o.set_particles(x, v, ir, cell)
    for s in range(1, steps + 1):
        o.step(s)
    to = o.wall()
    walls = np.nonzero(to[:, 0] > 0)[0]
    print(f"wall faces hit: {len(walls)}, hits: {c['wall_hits']}")
    assert len(walls) > 5 and c["wall_hits"] > 100
    if exact_hits:
        assert np.array_equal(t[:, 0], to[:, 0])
        assert _tallies_close(t[:, 1:], to[:, 1:], rtol)
    else:
        tot, toto = t.sum(0), to.sum(0)
        assert abs(tot[0] - toto[0]) <= 1e-4 * toto[0]
        assert np.all(np.abs(tot[1:] - toto[1:]) <= rtol * np.abs(to[:, 1:]).sum(0))


def test_wall_tallies_match_the_oracle_block(block):
    raw, dm, mess = block
    x, v, ir, cell = I.fill_inputs(dm, mess, 60, seed=31)
    _compare_with_oracle(dm, mess, x, v, ir, cell, 1, True, 1e-10)
    _compare_with_oracle(dm, mess, x, v, ir, cell, 3, False, 1e-6)


def test_wall_tallies_match_the_oracle_capsule():
    raw, dm, mess = I.capsule_small()
    x, v, ir, cell = I.fill_inputs_any(dm, mess, 12, seed=32)
    _compare_with_oracle(dm, mess, x, v, ir, cell, 1, True, 1e-10)


@pytest.mark.parametrize("precision", [gpu.PRECISION_FP64, gpu.PRECISION_MIXED])
def test_wall_statistics_of_an_isothermal_box(precision):
    raw = M.hex_box(4, 4, 4, 0.4, 0.4, 0.4)
    dm = M.build_dsmc_mesh(raw)
    mess = C.mesh_message(dm, 5.0, 0.1, ppc=200, L0=0.4)
    tw = float(mess["Twall_ref"])
    rs = np.random.RandomState(1)
    cells = np.repeat(np.arange(dm.ncell, dtype=np.int32), 100)
    lo, hi = I.cell_boxes(dm)
    n = len(cells)
    x = lo[cells] + (hi[cells] - lo[cells]) * rs.random_sample((n, 3))
    v = math.sqrt(tw / 2) * rs.standard_normal((n, 3))           # in equilibrium with the walls
    ir = -np.log1p(-rs.random_sample(n)) * tw / 2
    steps = 100
    with make_case(dm, mess, zones=DIFFUSE, precision=precision, seed=3, nss=0, wall_stats=1) as case:
        case.upload_particles(x, v, ir, cells)
        for s in range(1, steps + 1):
            case.step(s)
        assert case.particle_count() == n and case.counters()["lost"] == 0
        t = case.wall()
    neff, nref, dt = float(mess["Neff"]), float(mess["n_ref"]), float(mess["dtime"])
    vol = dm.cells["area"].sum()
    rho = n * neff / (vol * nref)
    flux = n / vol * math.sqrt(tw / 2) / math.sqrt(2 * math.pi) * dt * steps
    hits, p, shear, q = [], [], [], []
    for f in np.nonzero(t[:, 0] > 0)[0]:
        e = dm.edges[f]
        nrm = np.array(e["edgeNormal"], dtype=float)
        nrm /= np.linalg.norm(nrm)
        pn = -(t[f, 1:4] * nrm).sum()
        scale = 2.0 * neff / (dt * steps) / float(e["length"]) / nref
        hits.append(t[f, 0] / float(e["length"]))
        p.append(pn * scale)
        shear.append((t[f, 1:4] + pn * nrm) * scale)
        q.append(-(t[f, 4] + t[f, 5]) * scale)
    nf = len(p)
    assert nf == 6 * 16                                        # every boundary face was hit
    se = lambda a: np.std(a, axis=0) / math.sqrt(nf)
    assert abs(np.mean(hits) - flux) < 4 * se(hits)
    assert abs(np.mean(p) - rho * tw) < 4 * se(p)
    assert abs(np.mean(p) / (rho * tw) - 1.0) < 0.03
    assert np.all(np.abs(np.mean(shear, axis=0)) < 4 * se(shear))
    assert abs(np.mean(q)) < 4 * se(q)
