"""Analytic checks of the oracle's step in a closed box, on the CPU. The
FP64 device step equals the oracle particle by particle with the
reference's zone roles (test_gpu_step.py), so the collision, relaxation and
conservation properties here hold for the library's FP64 path too; its
specular walls are checked on the device by conservation alone.

The box is 4x4x4 hexahedra with every boundary zone specular
(DSMC_ROLE_SPECULAR), filled at rest with the reference's initial fill
(velocity variance 1 per component, Ir of mean 1/2).

- Closed box: no particle is injected, removed, dropped or lost, every
  particle stays in the box, and the total energy sum(|v|^2 / 2 + Ir) is
  conserved by the whole step (specular walls and collisions).
- A collision (collisionVelocity, src/ProcessDSMC.cpp:2679-2744) conserves
  momentum and energy to rounding.
- NTC with the VHS cross-section (collision_diameter,
  src/ProcessDSMC.cpp:2603-2608) gives the equilibrium collision rate: the
  accepted collisions per cell and step equal
  n(n-1)/2 * Neff * dt / V * <sigma_T c_r>, where for a Maxwellian of
  per-component variance s^2/2 the mean of sigma_T c_r = K c_r^(2 - 2 omega)
  is K * E[(s chi_3)^(2 - 2 omega)] (Bird, Molecular Gas Dynamics, 4.63).
- Larsen-Borgnakke exchange relaxes a gas with no rotational energy to
  equipartition over 3 translational and 2 rotational degrees of freedom:
  translational variance = mean Ir = E / 2.5, a Maxwellian and an
  exponential Ir distribution.
- Specular reflection through axis-aligned faces flips the normal velocity
  component and keeps every speed component's magnitude bit for bit.
- Wall statistics (recordBoundaryStressHeat, src/ProcessDSMC.cpp:1659-1689,
  converted as outBoundaryStressHeat does, :3494-3552) in a box of diffuse
  walls at the gas temperature: the hits per area are the one-sided flux
  n s / sqrt(2 pi), the normal stress is p = rho T, and the shear and the
  heat flux vanish.
"""
import math

import numpy as np
import pytest
from scipy import stats
from scipy.special import gamma

import inputs as I
from conftest import OracleParams
from pydsmc import case as C
from pydsmc import mesh as M

SPECULAR = [(3, 1, 0), (4, 5, 0), (5, 5, 0), (7, 5, 0)]
DIFFUSE = [(3, 1, 0), (4, 4, 0), (5, 4, 0), (7, 4, 0)]
STAGE_MOVE, STAGE_SORT, STAGE_COLLIDE, STAGE_ALL = 0x2, 0x4, 0x8, 0x1F
PPC = 200


@pytest.fixture(scope="module")
def box():
    raw = M.hex_box(4, 4, 4, 0.4, 0.4, 0.4)
    dm = M.build_dsmc_mesh(raw)
    mess = C.mesh_message(dm, 5.0, 0.1, ppc=PPC, L0=0.4)
    return raw, dm, mess


def _filled(oracle_lib, box, seed=3):
    raw, dm, mess = box
    o = oracle_lib.Oracle(dm, mess, OracleParams(SPECULAR, I.inflow_dir(), seed=seed))
    o.fill(float(PPC), 5, at_rest=True)
    return o


def _energy(v, ir):
    return 0.5 * (v * v).sum() + ir.sum()


def _inside(dm, x):
    P = dm.points.reshape(-1, 3)
    return bool((x >= P.min(0)).all() and (x <= P.max(0)).all())


def test_closed_box_keeps_particles_and_energy(box, oracle_lib):
    raw, dm, mess = box
    o = _filled(oracle_lib, box)
    x, v, ir, cell = o.particles()
    n0, e0 = len(v), _energy(v, ir)
    for s in range(1, 31):
        o.step(s, STAGE_ALL)
    x, v, ir, cell = o.particles()
    ctr = o.counters()
    assert ctr["injected"] == ctr["removed"] == ctr["dropped"] == ctr["lost"] == 0
    assert ctr["wall_hits"] > 0 and ctr["collisions"] > 0
    assert len(v) == n0 and _inside(dm, x)
    assert abs(_energy(v, ir) / e0 - 1.0) < 1e-12


def test_collisions_conserve_momentum_and_energy(box, oracle_lib):
    o = _filled(oracle_lib, box)
    x, v, ir, cell = o.particles()
    p0, e0 = v.sum(0), _energy(v, ir)
    for s in range(1, 6):
        o.step(s, STAGE_COLLIDE)
    x1, v1, ir1, cell1 = o.particles()
    assert o.counters()["collisions"] > 1000
    assert np.array_equal(cell1, cell) and np.array_equal(x1, x)
    assert not np.array_equal(v1, v)
    scale = np.sqrt((v * v).sum())
    assert np.abs(v1.sum(0) - p0).max() < 1e-12 * scale
    assert abs(_energy(v1, ir1) / e0 - 1.0) < 1e-13


def test_collision_rate_is_the_vhs_equilibrium_rate(box, oracle_lib):
    raw, dm, mess = box
    o = _filled(oracle_lib, box)
    # crmax above every relative speed drawn (c_r / s > 6 has probability
    # ~1e-7), so no pair is accepted with a probability capped at one
    crmax = np.full(dm.ncell, 6.0)
    o.lib.oracle_set_cell_state(o.h, crmax.ctypes.data, None, None)
    om, eta = float(mess["omega"]), float(mess["eta"])
    K = math.pi * float(mess["d_ref"]) ** 2 * (2.0 * float(mess["kB"]) * float(mess["T_ref"]) /
                                                float(mess["p_mass_r"])) ** eta / gamma(2.5 - om)
    p = 2.0 - 2.0 * om
    vr = float(mess["v_rms"])
    per_pair = float(mess["Neff"]) * float(mess["dtime"]) * float(mess["dt_ref"]) / dm.cells["area"]
    expected = 0.0
    before = o.counters()["collisions"]
    for s in range(1, 31):
        o.step(s, STAGE_MOVE | STAGE_SORT)
        x, v, ir, cell = o.particles()
        n = np.bincount(cell, minlength=dm.ncell).astype(float)
        s_rel = math.sqrt(2.0 * v.var(0).mean())            # relative velocity: variance 2 s^2/2 per component
        mean_cr_p = (vr * s_rel) ** p * 2.0 ** (p / 2) * gamma((3.0 + p) / 2) / gamma(1.5)
        expected += (0.5 * n * (n - 1) * per_pair).sum() * K * mean_cr_p
        o.step(s, STAGE_COLLIDE)
    got = o.counters()["collisions"] - before
    assert got > 30000
    # accepted collisions are binomial draws: 4 sigma
    assert abs(got - expected) < 4.0 * math.sqrt(expected), (got, expected)


def test_larsen_borgnakke_relaxes_to_equipartition(box, oracle_lib):
    o = _filled(oracle_lib, box)
    x, v, ir, cell = o.particles()
    o.set_particles(x, v, np.zeros_like(ir), cell)
    e_mean = _energy(v, np.zeros_like(ir)) / len(v)
    t_eq = e_mean / 2.5
    assert abs(v.var(0).mean() / t_eq - 1.0) > 0.5      # far from equipartition at the start
    tt, tr = [], []
    for s in range(1, 181):
        o.step(s, STAGE_ALL)
        if s > 150:
            x, v, ir, cell = o.particles()
            tt.append(v.var(0).mean())
            tr.append(ir.mean())
    assert abs(np.mean(tt) / t_eq - 1.0) < 0.02
    assert abs(np.mean(tr) / t_eq - 1.0) < 0.02
    x, v, ir, cell = o.particles()
    assert abs(_energy(v, ir) / len(v) / e_mean - 1.0) < 1e-12
    for k in range(3):
        assert stats.kstest(v[:, k] / math.sqrt(tt[-1]), "norm").pvalue > 1e-3
    assert stats.kstest(ir / tr[-1], "expon").pvalue > 1e-3


def test_specular_reflection_keeps_speed_components(box, oracle_lib):
    raw, dm, mess = box
    o = _filled(oracle_lib, box)
    rs = np.random.RandomState(2)
    n = 5000
    cells = rs.randint(0, dm.ncell, n).astype(np.int32)
    lo, hi = I.cell_boxes(dm)
    x = lo[cells] + (hi[cells] - lo[cells]) * rs.random_sample((n, 3))
    v = 3.0 * rs.standard_normal((n, 3))
    dt = 20.0 * float(mess["dtime"]) * rs.random_sample(n)
    r = o.trace(x, v, dt, cells, stop_at_wall=False)
    assert set(np.unique(r["ifout"]).tolist()) <= {0, 1}
    assert r["ncross"].max() > 20
    assert np.array_equal(np.abs(r["v"]), np.abs(v))
    assert _inside(dm, r["x"])
    # an odd number of reflections off the x faces flips vx: some did
    assert (np.sign(r["v"][:, 0]) != np.sign(v[:, 0])).sum() > n // 10


def test_wall_statistics_of_an_isothermal_box(box, oracle_lib):
    raw, dm, mess = box
    tw = float(mess["Twall_ref"])
    o = oracle_lib.Oracle(dm, mess, OracleParams(DIFFUSE, I.inflow_dir(), seed=3, nss=0, wall_stats=1))
    rs = np.random.RandomState(1)
    cells = np.repeat(np.arange(dm.ncell, dtype=np.int32), 100)
    lo, hi = I.cell_boxes(dm)
    n = len(cells)
    x = lo[cells] + (hi[cells] - lo[cells]) * rs.random_sample((n, 3))
    v = math.sqrt(tw / 2) * rs.standard_normal((n, 3))           # in equilibrium with the walls
    ir = -np.log1p(-rs.random_sample(n)) * tw / 2
    o.set_particles(x, v, ir, cells)
    steps = 100
    for s in range(1, steps + 1):
        o.step(s, STAGE_ALL)
    assert len(o.particles()[3]) == n and o.counters()["lost"] == 0
    t = o.wall()
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
