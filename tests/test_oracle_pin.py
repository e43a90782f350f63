"""The oracle is pinned before it is trusted: the mesh builder, the case
constants and the C restatement of the step are checked against outputs of
the reference's own code (tests/golden/, made by gen_golden.py from
oracle/_ref/ref_harness) and against published Philox known answers."""
import numpy as np
import pytest
from scipy import stats

import inputs as I
from conftest import OracleParams, golden
from pydsmc import case as C
from pydsmc import mesh as M


def test_mesh_arrays_match_reference():
    g = golden("mesh_pin.npz")
    raw, dm = I.block_mesh(scale=8)
    for f in M.DSMC_CELL_DTYPE.names:
        if f == "no":
            continue
        assert np.array_equal(dm.cells[f], g["cells"][f]), f
    for f in M.DSMC_EDGE_DTYPE.names:
        assert np.array_equal(dm.edges[f], g["edges"][f]), f
    assert np.array_equal(dm.points, g["points"])
    assert np.array_equal(dm.split, g["split"])


def test_mesh_message_matches_reference():
    g = golden("mesh_pin.npz")
    raw, dm = I.block_mesh(scale=8)
    mine = C.mesh_message(dm, I.BLOCK_MA, I.BLOCK_KN)      # reference defaults: L0, T_in, T_w, 100 ppc
    ref = g["mess"].reshape(())
    for f in C.MESH_MESSAGE_DTYPE.names:
        if f == "Nk":          # never set by the reference (uninitialised)
            continue
        assert mine[f] == ref[f], f


def test_philox_known_answers(oracle_lib):
    # Random123 known-answer vectors for philox4x32-10
    kat = [
        ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
        ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
        ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
         [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
    ]
    for ctr, key, want in kat:
        assert list(oracle_lib.philox(ctr, key)) == want


def test_oracle_trace_bit_exact_vs_reference(block, oracle_lib):
    raw, dm, mess = block
    g = golden("trace_pin.npz")
    x, v, dt, cell = I.trace_inputs(dm, mess, len(g["cell_1"]), seed=1)
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir()))
    r = o.trace(x, v, dt, cell, stop_at_wall=True)
    for k in ("cell", "ifout", "face", "tri", "ncross"):
        assert np.array_equal(r[k], g[f"{k}_1"]), k
    assert np.array_equal(r["x"], g["x_1"])
    assert np.array_equal(r["dt"], g["dt_1"])
    # full trace (diffuse re-emission at walls): identical until a wall hit
    r0 = o.trace(x, v, dt, cell, stop_at_wall=False)
    nowall = g["face_0"] < 0
    for k in ("cell", "ifout", "ncross"):
        assert np.array_equal(r0[k][nowall], g[f"{k}_0"][nowall]), k
    assert np.array_equal(r0["face"], g["face_0"])
    # the check covers every outcome
    assert {-1, 0, 1} <= set(np.unique(g["ifout_1"]).tolist())
    assert (g["face_1"] >= 0).sum() > 100 and g["ncross_1"].max() >= 4


def test_oracle_advection_matches_reference(block, oracle_lib):
    raw, dm, mess = block
    g = golden("advect_pin.npz")
    x, v, ir, cell = I.fill_inputs(dm, mess, 10, seed=2)
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.NOWALL_ZONES, I.inflow_dir()))
    o.set_particles(x, v, ir, cell)
    o.step(1, 2 | 4)                    # advection + cache2chain
    xo, vo, iro, co = o.particles()
    assert np.array_equal(np.bincount(co, minlength=dm.ncell), g["ppc"])
    order = np.lexsort((vo[:, 2], vo[:, 1], vo[:, 0]))
    assert np.array_equal(vo[order], g["v"])
    assert np.array_equal(co[order], g["cell"])
    assert np.array_equal(xo[order], g["x"])


def test_oracle_inflow_remainders_match_reference(block, oracle_lib):
    raw, dm, mess = block
    g = golden("inflow_pin.npz")
    x, v, ir, cell = I.fill_inputs(dm, mess, 20, seed=3)
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir(), seed=5))
    o.set_particles(x, v, ir, cell)
    for s in range(1, int(g["steps"]) + 1):
        o.step(s)
    _, _, rem = o.cell_state()
    assert np.array_equal(rem, g["reminj"])
    assert (rem != 0).sum() > 10


def _band_check(fields, band, min_frac=0.95):
    """Per cell and field, |x - mean_ref| <= 3 sigma with sigma the reference
    seed-to-seed spread (inflated for K samples); most (cell, field) pairs
    must pass and the mean z must show no bias."""
    mean = band.mean(0)
    K = band.shape[0]
    sd = band.std(0, ddof=1) * np.sqrt(1.0 + 1.0 / K)
    ok = np.isfinite(mean) & np.isfinite(fields) & (sd > 0)
    z = (fields[ok] - mean[ok]) / sd[ok]
    frac = float(np.mean(np.abs(z) <= 3.0))
    return frac, float(np.mean(z)), z


@pytest.fixture(scope="module")
def oracle_stats_run(block, oracle_lib):
    """The oracle on the reference band's inputs: summed step moments over
    the averaging window, the particle count after every step and the
    candidate pairs and collisions of every step."""
    raw, dm, mess = block
    g = golden("stats_band.npz")
    x, v, ir, cell = I.fill_inputs(dm, mess, int(g["ppc"]), seed=3)
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir(), seed=11))
    o.set_particles(x, v, ir, cell)
    acc = np.zeros((dm.ncell, 18))
    steps, a0 = int(g["steps"]), int(g["avg_from"])
    counts, pairs, coll = [], [], []
    for s in range(1, steps + 1):
        o.step(s)
        if s >= a0:
            acc += o.step_moments()
        counts.append(len(o.particles()[3]))
        c = o.counters()
        pairs.append(c["candidate_pairs"])
        coll.append(c["collisions"])
    per_step = {"pairs": np.diff(np.concatenate([[0], pairs])), "collisions": np.diff(np.concatenate([[0], coll]))}
    return acc, steps - a0 + 1, counts, per_step


def test_oracle_statistics_within_reference_band(block, oracle_stats_run):
    raw, dm, mess = block
    g = golden("stats_band.npz")
    acc, nsteps, counts, _ = oracle_stats_run
    f = I.fields_from_moments(acc, nsteps, dm, mess)
    frac, zbar, _ = _band_check(f, g["fields"])
    assert frac >= 0.95, frac
    assert abs(zbar) < 0.3, zbar
    # particle inventory follows the reference's within its spread
    ref_n = g["nparticles"].astype(float)
    lo, hi = ref_n.min(0) * 0.97, ref_n.max(0) * 1.03
    assert np.all((np.array(counts) >= lo) & (np.array(counts) <= hi))


def test_oracle_statistics_on_tets_within_reference_band(oracle_lib):
    """The same band in the collision-dominated regime: the capsule tets at
    Kn 0.01 (about a dozen collisions per particle and step), time-averaged
    rho, u, T, Tr over steps 61-120 against 8 seeded reference runs, every
    third cell; and the particle count of each step within the runs'
    spread."""
    g = golden("stats_band_capsule.npz")
    raw, dm, mess = I.capsule_small()
    x, v, ir, cell = I.fill_inputs_any(dm, mess, int(g["ppc"]), 3)
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir(), seed=11))
    o.set_particles(x, v, ir, cell)
    acc = np.zeros((dm.ncell, 18))
    steps, a0 = int(g["steps"]), int(g["avg_from"])
    counts = []
    for s in range(1, steps + 1):
        o.step(s)
        if s >= a0:
            acc += o.step_moments()
        counts.append(int(o.lib.oracle_count(o.h)))
    f = I.fields_from_moments(acc, steps - a0 + 1, dm, mess)[g["cells"]]
    K = int(g["k"])
    mean = g["mean"].astype(float)
    sd = g["sd"].astype(float) * np.sqrt(1.0 + 1.0 / K)
    ok = np.isfinite(mean) & np.isfinite(f) & (sd > 0)
    assert ok.mean() > 0.95
    z = (f[ok] - mean[ok]) / sd[ok]
    assert np.mean(np.abs(z) <= 3.0) >= 0.95
    assert abs(np.mean(z)) < 0.3
    for j in range(6):
        zj = (f[ok[:, j], j] - mean[ok[:, j], j]) / sd[ok[:, j], j]
        assert abs(np.mean(zj)) < 0.3, j
    ref_n = g["nparticles"].astype(float)
    lo, hi = ref_n.min(0) * 0.97, ref_n.max(0) * 1.03
    assert np.all((np.array(counts) >= lo) & (np.array(counts) <= hi))


def test_oracle_stress_and_heat_flux_within_reference_band(block, oracle_stats_run):
    """Deviatoric stress, heat flux and rotational heat flux as
    writeAveragedMacro defines them, against the same 8 reference runs."""
    raw, dm, mess = block
    g = golden("macro_band.npz")
    acc, nsteps, counts, _ = oracle_stats_run
    assert nsteps == int(g["steps"]) - int(g["avg_from"]) + 1
    f = I.macro_from_moments(acc, nsteps, dm, mess)[:, g["columns"]]
    K = int(g["k"])
    sd = g["sd"] * np.sqrt(1.0 + 1.0 / K)
    ok = np.isfinite(f) & np.isfinite(g["mean"]) & (sd > 0)
    assert ok.mean() > 0.9
    z = (f[ok] - g["mean"][ok]) / sd[ok]
    assert np.mean(np.abs(z) <= 3.0) >= 0.95
    assert abs(np.mean(z)) < 0.3
    # each field on its own: no bias
    for j in range(f.shape[1]):
        zj = (f[ok[:, j], j] - g["mean"][ok[:, j], j]) / sd[ok[:, j], j]
        assert abs(np.mean(zj)) < 0.3, (int(g["columns"][j]), float(np.mean(zj)))


def test_oracle_collision_counts_within_reference_band(oracle_stats_run):
    """Particles, NTC candidate pairs (tol_collision_pairs) and accepted
    collisions (tol_collision_times, src/ProcessDSMC.cpp:2621-2666) summed
    over the 200 steps, and the acceptance fraction, against the 8 reference
    runs: within 4 seed-to-seed standard deviations."""
    g = golden("macro_band.npz")
    ref = g["per_step"].astype(float)                     # [seed, step, (particles, injected, pairs, collisions)]
    acc, nsteps, counts, per_step = oracle_stats_run
    K = ref.shape[0]
    mine = {
        "particles": float(np.sum(counts)),
        "pairs": float(per_step["pairs"].sum()),
        "collisions": float(per_step["collisions"].sum()),
    }
    mine["acceptance"] = mine["collisions"] / mine["pairs"]
    band = {
        "particles": ref[:, :, 0].sum(1),
        "pairs": ref[:, :, 2].sum(1),
        "collisions": ref[:, :, 3].sum(1),
    }
    band["acceptance"] = band["collisions"] / band["pairs"]
    for k, b in band.items():
        z = (mine[k] - b.mean()) / (b.std(ddof=1) * np.sqrt(1.0 + 1.0 / K))
        assert abs(z) < 4.0, (k, mine[k], b.mean(), z)
    assert mine["collisions"] > 50000


def test_oracle_trace_config_full_block(oracle_lib):
    """The TRACE configuration (10^6 particles on the full 48,640-cell block
    mesh, one dt, stop at the first non-interface face): the oracle's
    outputs are bit-exact with the reference's (SHA-256 digests of every
    array in trace_full_pin.npz), on the FP64 inputs and on the FP32-rounded
    state the mixed path stores."""
    g = golden("trace_full_pin.npz")
    raw, dm = I.block_mesh(scale=1)
    mess = I.block_mess(dm, 20)
    assert dm.ncell == int(g["ncell"])
    x, v, dt, cell = I.trace_inputs(dm, mess, int(g["n"]), seed=int(g["seed"]))
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir()))
    r = o.trace(x, v, dt, cell, stop_at_wall=True)
    for k in ("cell", "ifout", "face", "tri", "ncross", "dt", "x"):
        assert I.digest(r[k]) == str(g[f"fp64_{k}_sha"]), k
    x32, v32 = I.fp32_state(dm, x, v, cell)
    r = o.trace(x32, v32, dt, cell, stop_at_wall=True)
    for k in ("cell", "ifout", "face", "tri", "ncross", "dt"):
        assert I.digest(r[k]) == str(g[f"mixed_{k}_sha"]), k
    kept = r["cell"] >= 0
    assert I.digest(I.fp32_positions(dm, r["x"][kept], r["cell"][kept])) == str(g["mixed_x_sha"])
    assert np.array_equal(np.bincount(r["cell"][kept], minlength=dm.ncell), g["mixed_ppc"])
    # every outcome and many boundary hits
    assert np.all(g["fp64_ifout_counts"] > 10000) and int(g["fp64_hits"]) > 10000


def test_oracle_degenerate_trace_vs_reference(block, oracle_lib):
    """Exact paths through face centres (on the quads' split diagonals),
    edges and vertices, starts on faces, edges and corners, particles at
    rest, dt = 0, a denormal speed and a path along a face: bit-exact with
    the reference wherever its loop returns. Where it does not (it was given
    a few seconds per particle; the rest take milliseconds together) the
    path meets a split quad's diagonal on a face whose zone has no role in
    the reference's table (the block's sides, zone 7): CrossboundarySwitch
    leaves the particle where it is and the next search finds the other
    triangle of the same quad, without end. The oracle, like the CUDA path,
    stops such a particle at max_crossings and reports it lost; with zone 7
    given a role no particle reaches the bound."""
    raw, dm, mess = block
    g = golden("degenerate_trace_pin.npz")
    x, v, dt, cell = I.degenerate_trace_inputs(dm, mess, int(g["ncells"]), int(g["seed"]))
    assert len(g["ok"]) + len(g["spins"]) == len(cell)
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir()))
    r = o.trace(x, v, dt, cell, stop_at_wall=True)
    ok, spins = g["ok"], g["spins"]
    for k in ("cell", "ifout", "face", "tri", "ncross", "x", "dt"):
        assert np.array_equal(r[k][ok], g[k]), k
    # every outcome, drops (no exit found from a corner or face) among them
    assert {-1, 0, 1} <= set(np.unique(g["ifout"]).tolist())
    assert (g["face"] >= 0).sum() > 100
    assert len(spins) > 0
    lost = o.counters()["lost"]
    assert lost == len(spins) and np.all(r["ncross"][spins] == 4096)
    assert np.all(dm.edges["faceTag"][r["face"][spins]] == 7)
    o7 = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES + [(7, 3, 0)], I.inflow_dir()))
    o7.trace(x, v, dt, cell, stop_at_wall=True)
    assert o7.counters()["lost"] == 0


def test_oracle_degenerate_tet_trace_vs_reference(oracle_lib):
    """Paths along tetrahedron edges and faces and through vertices, from
    vertices, edge midpoints, face centroids and centroids: bit-exact with
    the reference on every particle (every zone of the capsule has a role,
    so the reference's loop always returns)."""
    g = golden("degenerate_trace_pin.npz")
    raw, dm, mess = I.capsule_small()
    x, v, dt, cell = I.degenerate_tet_trace_inputs(dm, mess, int(g["tet_ncells"]), int(g["seed"]))
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir()))
    r = o.trace(x, v, dt, cell, stop_at_wall=True)
    for k in ("cell", "ifout", "face", "tri", "ncross", "x", "dt"):
        assert np.array_equal(r[k], g["tet_" + k]), k
    c = o.counters()
    assert c["lost"] == 0 and c["dropped"] > len(cell) // 4 and c["crossings"] > 500
    assert {-1, 0, 1} <= set(np.unique(g["tet_ifout"]).tolist())


def test_oracle_sampling_bit_exact_vs_reference(oracle_lib):
    """statistic_macro (src/ProcessDSMC.cpp:2757-2861) over 5,200 steps of
    a particle sequence with no random draws (inputs.sampled_at: thinned
    and rescaled particles, cells that hold one particle on two steps of
    each 100-step window): the step-window average with its exponential
    weight after NSCHEME, the steady average after NSS, the GSIS window
    samples, validity and record, and the sparse-cell state machine, all
    bit-exact with the reference's; and the same when the host's GSIS
    exchange writes accumulating and released states back after each
    exchange step (ProcessGSIS::DSMC2NS, src/ProcessGSIS.cpp:1660-1674)."""
    from pydsmc import gpu
    g = golden("sample_pin.npz")
    raw, dm = I.block_mesh(scale=8)
    ppc = int(g["ppc"])
    mess = I.block_mess(dm, ppc)
    x, v, ir, cell = I.fill_inputs(dm, mess, ppc, int(g["seed"]))
    for pre in ("", "rule_"):
        o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir(), nss=5000, nscheme=2000, nevery=1,
                                                     nrepeat=100))
        o.macro_pre()
        for k in range(1, int(g["steps"]) + 1):
            keep, s = I.sampled_at(k, cell, ppc)
            o.set_particles(x[keep], v[keep] * s, ir[keep] * (s * s), cell[keep])
            o.step(k, 0x10)
            if pre and k % 100 == 0:      # the GSIS exchange's write-back (dsmc_upload_sparse_state)
                o.set_sparse_state(I.host_sparse_rule(o.counts()["sparse_state"], k))
        for name, which in (("local", gpu.MACRO_LOCAL), ("record", gpu.MACRO_RECORD),
                            ("final_record", gpu.MACRO_FINAL_RECORD)):
            assert np.array_equal(o.macro(which), g[pre + name]), pre + name
        cn = o.counts()
        for k in ("window_samples", "window_valid", "sparse_state"):
            assert np.array_equal(cn[k], g[pre + k]), pre + k
        # the sequence reaches the sparse states and fills every output
        assert (g[pre + "sparse_state"] == 1).sum() > 10 and (g[pre + "sparse_state"] == 0).sum() > 10
        for name in ("local", "record", "final_record"):
            assert (g[pre + name][:, 0] > 0).all()
    assert (g["rule_sparse_state"] == 2).sum() > 5


def test_oracle_ntc_pairs_bit_exact_vs_reference(oracle_lib):
    """One collisionDSMC (src/ProcessDSMC.cpp:2621-2666) on ragged cells
    (0 to ppc particles) of the block and the capsule tets, from the initial
    crmax and remainders: the NTC candidate pairs of every cell and the
    remainder each cell carries are bit-exact with the reference's (they
    depend on no draw); the accepted collisions, which do, agree within 4
    binomial sigma, and both conserve every cell's momentum and energy to
    rounding."""
    from gen_golden import collide_cases, collision_conservation
    g = golden("collide_pin.npz")
    for k, (raw, dm, mess, parts) in zip(("block", "tets"), collide_cases()):
        o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir(), seed=3))
        o.set_particles(*parts)
        o.step(1, 0x8)
        crmax, rem, _ = o.cell_state()
        c = o.counters()
        assert np.array_equal(rem, g[f"{k}_remcoll"]), k
        assert c["candidate_pairs"] == int(g[f"{k}_pairs"]), k
        pairs, ref = int(g[f"{k}_pairs"]), int(g[f"{k}_collisions"])
        p = ref / pairs
        assert abs(c["collisions"] - ref) < 4 * np.sqrt(pairs * p * (1 - p)) + 4, (k, c["collisions"], ref)
        dmom, den = collision_conservation(dm.ncell, parts, o.particles())
        assert dmom < 1e-13 and den < 1e-13
        assert float(g[f"{k}_dmom"]) < 1e-13 and float(g[f"{k}_den"]) < 1e-13
        assert (np.bincount(parts[3], minlength=dm.ncell) <= 1).sum() > 10      # empty and single cells too
    assert int(g["tets_pairs"]) > 500000


@pytest.mark.parametrize("pre", ["", "tet_"])
def test_oracle_injection_follows_the_reference(block, oracle_lib, pre):
    """preprocesseffquad (src/ProcessDSMC.cpp:2416-2570) on an empty domain
    for 40 steps, through the block's quad inlet and the capsule's triangle
    inlet at 30 degrees: the inflow remainders are bit-exact; the particles
    that stay in the domain after their r dt trace are as many (within 4
    binomial sigma of the share lost), spread over the inlet cells alike
    (chi-squared), and their positions, velocities and Ir have the same
    distributions (KS)."""
    raw, dm, mess = block if not pre else I.capsule_small()
    g = {k[len(pre):]: a for k, a in golden("inject_pin.npz").items() if k.startswith(pre)}
    gg = golden("inject_pin.npz")
    g["seed"], g["steps"] = gg["seed"], gg["steps"]
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir(), seed=int(g["seed"])))
    empty = np.zeros((0, 3))
    xs, vs, irs, cs = [], [], [], []
    for k in range(1, int(g["steps"]) + 1):
        o.set_particles(empty, empty, np.zeros(0), np.zeros(0, np.int32))
        o.step(k, 0x1 | 0x4)                        # inject, then merge into the cells
        x, v, ir, c = o.particles()
        xs.append(x); vs.append(v); irs.append(ir); cs.append(c)
    x, v, ir, c = (np.concatenate(a) for a in (xs, vs, irs, cs))
    _, _, rem = o.cell_state()
    assert np.array_equal(rem, g["reminj"])
    emitted = o.counters()["injected"]
    kept_ref = int(g["per_step"].sum())
    q = 1.0 - kept_ref / emitted
    assert abs(len(c) - kept_ref) < 4 * np.sqrt(emitted * q * (1 - q)) + 4
    cnt = np.bincount(c, minlength=dm.ncell)
    inlet = (cnt + g["cell_count"]) > 0
    assert stats.chi2_contingency(np.stack([cnt[inlet], g["cell_count"][inlet]])).pvalue > 1e-3
    for k in range(3):
        assert stats.ks_2samp(x[:, k], g["x"][:, k]).pvalue > 1e-3, ("x", k)
        assert stats.ks_2samp(v[:, k], g["v"][:, k]).pvalue > 1e-3, ("v", k)
    assert stats.ks_2samp(ir, g["ir"]).pvalue > 1e-3


@pytest.mark.parametrize("pre", ["", "tet_"])
def test_oracle_diffuse_wall_follows_the_reference(block, oracle_lib, pre):
    """Diffuse re-emission at the wall (CrossboundarySwitch's wall branch,
    src/ProcessDSMC.cpp:1702-1829), at the block's quad walls and the
    capsule's triangle walls: the paths up to the first wall hit are
    bit-exact (the first non-interface face of every particle is the
    reference's); the velocities after the hit follow the reference's
    (KS on the normal component, the speed and each component), with the
    flux-weighted Maxwellian's mean normal speed sqrt(Tw / 2) sqrt(pi / 2)."""
    raw, dm, mess = block if not pre else I.capsule_small()
    gg = golden("wall_pin.npz")
    g = {k: gg[pre + k] for k in ("first_face", "hit", "v")}
    g["n"], g["seed"] = gg["n"], gg["seed"]
    x, v, dt, c = I.wall_trace_inputs(dm, mess, int(g["n"]), int(g["seed"]), tets=bool(pre))
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir(), seed=3))
    first = o.trace(x, v, dt, c, stop_at_wall=True)
    assert np.array_equal(first["face"], g["first_face"])
    hit = g["hit"]
    assert len(hit) > 3000
    full = o.trace(x, v, dt, c, stop_at_wall=False)
    nrm = dm.edges["edgeNormal"][g["first_face"][hit]]
    nrm = nrm / np.linalg.norm(nrm, axis=1)[:, None]
    mine, ref = full["v"][hit], g["v"].astype(float)
    vn_m, vn_r = -(mine * nrm).sum(1), -(ref * nrm).sum(1)
    assert stats.ks_2samp(vn_m, vn_r).pvalue > 1e-3
    assert stats.ks_2samp(np.linalg.norm(mine, axis=1), np.linalg.norm(ref, axis=1)).pvalue > 1e-3
    for k in range(3):
        assert stats.ks_2samp(mine[:, k], ref[:, k]).pvalue > 1e-3
    want = np.sqrt(float(mess["Twall_ref"]) / 2) * np.sqrt(np.pi / 2)
    for vn in (vn_m, vn_r):
        assert abs(vn.mean() / want - 1) < 0.03


def test_oracle_tet_trace_bit_exact_vs_reference(oracle_lib):
    g = golden("tet_trace_pin.npz")
    raw, dm, mess = I.capsule_small()
    assert dm.ncell == int(g["ncell"])
    x, v, dt, cell = I.tet_trace_inputs(dm, mess, len(g["cell"]), seed=4)
    o = oracle_lib.Oracle(dm, mess, OracleParams(I.REF_ZONES, I.inflow_dir()))
    r = o.trace(x, v, dt, cell, stop_at_wall=True)
    for k in ("cell", "ifout", "face", "tri", "ncross"):
        assert np.array_equal(r[k], g[k]), k
    assert np.array_equal(r["x"], g["x"])
    assert np.array_equal(r["dt"], g["dt"])
    assert (g["face"] >= 0).sum() > 50      # wall and farfield hits are covered
