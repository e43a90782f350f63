"""Generate the golden fixtures of tests/golden/ from the reference's own code.

Runs oracle/_ref/ref_harness (built by ``make -C oracle ref`` from the
reference sources) on the inputs of tests/golden/inputs.py and stores its
outputs:

  mesh_pin.npz   DsmcCell/DsmcEdge/localPointXY/faceSplitTag/meshMessage the
                 reference builds from the CAS file of the 1/8 block mesh
  trace_pin.npz  tracing-check outputs on the 1/4 block mesh (16,000
                 particles, stop at the first wall hit, and full trace)
  advect_pin.npz advection + cache2chain on the 1/4 block mesh with the wall
                 zone as an outlet (no random draws): per-cell counts and the
                 particles sorted by velocity
  inflow_pin.npz per-cell inflow remainders after 60 full steps
  stats_band.npz time-averaged rho, u, T, Tr per cell over steps 101-200 of
                 8 independently seeded reference runs (20 per cell)
  tet_trace_pin.npz tracing-check outputs on the coarse capsule tet mesh
                 (16,000 particles, stop at the first wall hit)
  gsis_pin.npz   the reference's molecular_velocity_change on the 1/4 block
                 mesh (gsis_edge_inputs: gate, NaN cell, emptied cells,
                 negative densities): per-cell counts and moments after the
                 update, how many particles kept their input position, whether
                 every moved particle carries a kept particle's velocity, and
                 the box-relative positions of the moved particles
  gsis_tet_pin.npz the same on the capsule tets: counts, kept counts and
                 copies per cell, the largest deviations of the moments from
                 the NS values, and 8,000 of the moved particles' sorted
                 barycentric weights
  fill_pin.npz   the reference's initial fill (Np_tri_inititial + meshfillpar)
                 with the counts of the fill rule: per-tetrahedron counts and
                 box-relative positions on the 1/4 block mesh (centre-face
                 tetrahedra), sorted barycentric weights on the capsule tets,
                 velocity and Ir moments
  fluent_pin.npz out2Fluent_dsmc's file for given fields on the 1/8 block
                 mesh, with its zone list and mesh message
  pyramid_pin.npz the reference's arrays for a box of cubes split into six
                 pyramids each (mixed triangle / quad faces) and its initial
                 fill there (counts per placement tetrahedron, cube-relative
                 positions, velocity and Ir moments)
  pyramid_trace_pin.npz tracing-check outputs on that mesh (16,000
                 particles, dt uniform in [0, dtime])
  prism_pin.npz  the same for that box with each cube split into two wedges
                 (two triangles and three quads per cell): arrays, fill, and
                 tracing-check outputs (8,000 particles)
  degenerate_trace_pin.npz tracing-check outputs for exact, degenerate
                 paths on the 1/4 block mesh (degenerate_trace_inputs), the
                 particles on which the reference's loop does not return, and
                 the same on the capsule tets (degenerate_tet_trace_inputs)
  sample_pin.npz the reference's statistic_macro over 5,200 steps of a
                 deterministic particle sequence on the 1/8 block mesh
                 (inputs.sampled_at): local, record, final_record, window
                 samples and validity, sparse states; the same with the
                 sparse states changed after each exchange step by the
                 harness's host rule (inputs.host_sparse_rule), "rule_" keys
  collide_pin.npz one collisionDSMC of the reference on ragged particle
                 sets (block hexahedra and capsule tets): the NTC remainders,
                 candidate pairs, collisions, how many cells raised crmax,
                 and the largest per-cell momentum and energy changes
  inject_pin.npz the reference's injection on an empty 1/4 block mesh for
                 40 steps: particles kept per step and per cell, the inflow
                 remainders, and 6,000 of the kept particles (float32); the
                 same on the capsule tets ("tet_" keys)
  wall_pin.npz   particles traced near the block's wall (wall_trace_inputs):
                 the reference's first non-interface face of each, and the
                 final velocity (float32) of those whose first hit is the
                 wall, after its diffuse re-emission; the same near the
                 capsule's wall ("tet_" keys)
  trace_full_pin.npz the TRACE configuration: the reference's tracing
                 check (stop at the first non-interface face) of 10^6
                 particles on the full 48,640-cell block mesh
                 (inputs.trace_inputs, seed 1), on the FP64 inputs ("fp64_"
                 keys) and on the FP32-rounded state the mixed path stores
                 ("mixed_" keys): SHA-256 digests of every output array
                 (positions of the mixed run as the FP32 offsets from the
                 final cell's centre widen back), final per-cell counts,
                 outcome and hit counts, and 4,096 particles in full
  stats_band_capsule.npz the same band on the capsule tets (Kn 0.01), steps
                 61-120 of 8 seeded reference runs from 8 particles per
                 cell: float32 mean and spread of every third cell, and
                 the particle count of each step of each run
  macro_band.npz per-cell mean and seed-to-seed spread of the time-averaged
                 stress and heat-flux fields (writeAveragedMacro's
                 definitions) over the same 8 reference runs as stats_band,
                 and each run's per-step particles, injected particles,
                 candidate pairs and collisions

Usage: python tests/golden/gen_golden.py [fixture ...]   (default: all)
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import inputs as I  # noqa: E402
from oracle import harness as H  # noqa: E402
from pydsmc import case as C  # noqa: E402
from pydsmc import mesh as M  # noqa: E402

STATS_SEEDS = [101, 102, 103, 104, 105, 106, 107, 108]
STATS_STEPS = 200
STATS_AVG_FROM = 101
STATS_PPC = 20
TRACE_N = 16000


def roles_arg(zones):
    names = {1: "interface", 2: "inlet", 3: "outlet", 4: "wall", 0: "none"}
    return ",".join(f"{t}:{names[r]}" for t, r, _ in zones)


GSIS_PPC = 12
GSIS_SEED = 13
FILL_PPC = 7
FILL_SEED = 2024
FILL_TET_CELLS = 3000
FILL_TET_SAMPLE = 6000


def fill_counts(dm, ppc, seed):
    """Per-cell counts of the fill rule (setParticleMessage, with the
    Philox draw (c, 0, 4, 0) of the CUDA library and the oracle)."""
    from oracle import oracle as O
    O.load()
    vol = dm.cells["area"].astype(float)
    nps = ppc * dm.ncell
    vt = vol.sum()
    key = [seed & 0xFFFFFFFF, seed >> 32]
    out = np.empty(dm.ncell, dtype=np.int32)
    for c in range(dm.ncell):
        ns = vol[c] * nps / vt
        fl = np.floor(ns)
        b = O.philox([c, 0, 4, 0], key)
        u = (((int(b[0]) << 21) ^ (int(b[1]) >> 11)) + 0.5) * 2.0 ** -53
        out[c] = int(fl) + (1 if u < ns - fl else 0)
    return out


def gsis_summary(dm, before, after, tets=False):
    """Per-cell counts, moments and structure of a GSIS update's output; the
    moved particles' positions relative to their cell's box (hexahedra) or
    as sorted barycentric weights (tetrahedra)."""
    x0, v0, ir0, c0 = before
    x1, v1, ir1, c1 = after
    nc = dm.ncell
    lo, hi = (None, None) if tets else I.cell_boxes(dm)
    kept = np.zeros(nc, np.int32)
    dup_ok = np.ones(nc, bool)
    rel = []
    s0 = np.concatenate([[0], np.cumsum(np.bincount(c0, minlength=nc))])
    s1 = np.concatenate([[0], np.cumsum(np.bincount(c1, minlength=nc))])
    for c in range(nc):
        X0 = x0[s0[c]:s0[c + 1]]
        X1, V1 = x1[s1[c]:s1[c + 1]], v1[s1[c]:s1[c + 1]]
        known = {tuple(p) for p in X0}
        is_kept = np.array([tuple(p) in known for p in X1], dtype=bool)
        kept[c] = int(is_kept.sum())
        if len(X0) and (~is_kept).any():
            vk = {tuple(p) for p in V1[is_kept]}
            dup_ok[c] = all(tuple(p) in vk for p in V1[~is_kept])
        if (~is_kept).any():
            moved = X1[~is_kept]
            rel.append(sorted_barycentric(dm, moved, np.full(len(moved), c)) if tets else
                       (moved - lo[c]) / (hi[c] - lo[c]))
    n = np.bincount(c1, minlength=nc).astype(float)
    m = np.maximum(n, 1.0)
    u = np.stack([np.bincount(c1, v1[:, k], nc) for k in range(3)], 1) / m[:, None]
    return {"counts": n.astype(np.int32), "u": u, "kept": kept, "dup_ok": dup_ok,
            "sums": np.stack([np.bincount(c1, (v1 * v1).sum(1), nc), np.bincount(c1, ir1, nc)], 1),
            "rel": np.concatenate(rel) if rel else np.zeros((0, 3))}


GSIS_TET_REL = 8000


def gsis_moment_errors(dm, mess, cell0, ns, acc, nan_cell, summ):
    """How far a GSIS update's per-cell moments are from the NS values, over
    the updated cells holding more than one particle with T > 0: the largest
    velocity error relative to the largest |u|, the largest relative T and
    Tr errors, and the share of such cells among the updated ones."""
    upd = acc.astype(bool)
    upd[nan_cell:] = False
    n = summ["counts"].astype(float)
    live = upd & (n > 1)
    m = np.maximum(n, 1)
    T = 2.0 / (3.0 * m) * (summ["sums"][:, 0] - n * (summ["u"] ** 2).sum(1))
    Tr = 4.0 / float(mess["dr"]) / m * summ["sums"][:, 1]
    ok = live & (T > 0)
    return {"u_err": np.abs(summ["u"][ok] - ns[ok, 1:4]).max() / np.abs(ns[ok, 1:4]).max(),
            "T_err": np.abs(T[ok] / ns[ok, 4] - 1).max(), "Tr_err": np.abs(Tr[ok] / ns[ok, 5] - 1).max(),
            "ok_share": ok.sum() / max(live.sum(), 1)}


def sorted_barycentric(dm, x, cell):
    P = dm.points.reshape(-1, 3)
    V = P[I.tet_vertices(dm, cell)]
    T = np.stack([V[:, 1] - V[:, 0], V[:, 2] - V[:, 0], V[:, 3] - V[:, 0]], axis=2)
    lam = np.linalg.solve(T, (x - V[:, 0])[:, :, None])[:, :, 0]
    return np.sort(np.concatenate([1.0 - lam.sum(1, keepdims=True), lam], axis=1), axis=1)


def gen_gsis_fill(d):
    raw, dm = I.block_mesh()
    cas = os.path.join(d, "b4g.cas")
    M.write_cas(cas, raw)
    mess = I.block_mess(dm, STATS_PPC)
    parts, ns, acc, nan_cell, empty, neg = I.gsis_edge_inputs(dm, mess, GSIS_PPC, GSIS_SEED)
    r = H.gsis(cas, mess, *parts, ns, acc, seed=7)
    summ = gsis_summary(dm, parts, (r["x"], r["v"], r["ir"], r["cell"]))
    np.savez_compressed(os.path.join(HERE, "gsis_pin.npz"), ppc=GSIS_PPC, seed=GSIS_SEED, **summ)
    # the same on the capsule tets
    rawt, dmt, messt = I.capsule_small()
    cast = os.path.join(d, "capgs.cas")
    M.write_cas(cast, rawt)
    parts, ns, acc, nan_cell, empty, neg = I.gsis_edge_inputs(dmt, messt, GSIS_PPC, GSIS_SEED, tets=True)
    r = H.gsis(cast, messt, *parts, ns, acc, seed=7)
    summ = gsis_summary(dmt, parts, (r["x"], r["v"], r["ir"], r["cell"]), tets=True)
    err = gsis_moment_errors(dmt, messt, parts[3], ns, acc, nan_cell, summ)
    sub = np.random.RandomState(1).permutation(len(summ["rel"]))[:GSIS_TET_REL]
    np.savez_compressed(os.path.join(HERE, "gsis_tet_pin.npz"), ppc=GSIS_PPC, seed=GSIS_SEED,
                        counts=summ["counts"], kept=summ["kept"], dup_ok=summ["dup_ok"],
                        rel=summ["rel"][np.sort(sub)].astype(np.float32), n_rel=len(summ["rel"]), **err)

    counts = fill_counts(dm, FILL_PPC, FILL_SEED)
    f = H.fill(cas, mess, counts, seed=8)
    lo, hi = I.cell_boxes(dm)
    rel = (f["x"] - lo[f["cell"]]) / (hi[f["cell"]] - lo[f["cell"]])
    rawc, dmc, messc = I.capsule_small()
    casc = os.path.join(d, "capg.cas")
    M.write_cas(casc, rawc)
    countsc = fill_counts(dmc, FILL_PPC, FILL_SEED)
    countsc[FILL_TET_CELLS:] = 0
    fc = H.fill(casc, messc, countsc, seed=9)
    bary = sorted_barycentric(dmc, fc["x"], fc["cell"])[:FILL_TET_SAMPLE]
    vv = np.concatenate([f["v"], fc["v"]])
    irr = np.concatenate([f["ir"], fc["ir"]])
    np.savez_compressed(os.path.join(HERE, "fill_pin.npz"), ppc=FILL_PPC, seed=FILL_SEED, counts=counts,
                        cell_count=np.bincount(f["cell"], minlength=dm.ncell).astype(np.int32),
                        np_tri=f["np_tri"].astype(np.int16), rel=rel, tet_cells=FILL_TET_CELLS,
                        tet_count=np.bincount(fc["cell"], minlength=dmc.ncell).astype(np.int32), bary=bary,
                        v_mean=vv.mean(0), v_var=vv.var(0), ir_mean=irr.mean(), n_v=len(vv))


def fluent_fields(ncell, seed=17):
    rs = np.random.RandomState(seed)
    w = rs.standard_normal((ncell, 18)) * 10.0 ** rs.randint(-8, 8, (ncell, 18))
    w[0, 3] = np.nan
    w[1, 5] = 0.0
    w[2, 7] = -1e-300
    w[3, 0] = 1e300
    return w


def gen_fluent(d):
    raw8, dm8 = I.block_mesh(scale=8)
    cas8 = os.path.join(d, "b8f.cas")
    M.write_cas(cas8, raw8)
    mess = C.mesh_message(dm8, I.BLOCK_MA, I.BLOCK_KN, ppc=20, L0=I.BLOCK_L0)
    r = H.fluent(cas8, mess, fluent_fields(dm8.ncell))
    np.savez_compressed(os.path.join(HERE, "fluent_pin.npz"), text=np.frombuffer(r["text"], dtype=np.uint8),
                        zones=r["zones"], mess=np.asarray(mess))


PYR_N = (3, 2, 2)
PYR_L = (0.6, 0.4, 0.4)
PYR_PPC = 40
PYR_SEED = 77
PRISM_SEED = 78


def pyramid_case():
    raw = M.pyramid_box(*PYR_N, *PYR_L)
    dm = M.build_dsmc_mesh(raw)
    mess = C.mesh_message(dm, I.BLOCK_MA, I.BLOCK_KN, ppc=PYR_PPC, L0=0.1)
    return raw, dm, mess


def prism_case():
    """The same box as pyramid_case, each cube split into two wedges."""
    raw = M.prism_box(*PYR_N, *PYR_L)
    dm = M.build_dsmc_mesh(raw)
    mess = C.mesh_message(dm, I.BLOCK_MA, I.BLOCK_KN, ppc=PYR_PPC, L0=0.1)
    return raw, dm, mess


def cube_relative(x, cell, per_cube=6):
    """Positions relative to each cell's cube (per_cube cells per cube: 6
    pyramids or 2 wedges), in [0, 1]^3."""
    nx, ny, nz = PYR_N
    q = cell // per_cube
    i, j, k = q // (ny * nz), (q // nz) % ny, q % nz
    h = np.array([PYR_L[0] / nx, PYR_L[1] / ny, PYR_L[2] / nz])
    return (x - np.stack([i, j, k], 1) * h) / h


def _split_box_pins(d, name, case, per_cube, fill_seed, ref_seed, trace_seed, trace_n):
    raw, dm, mess = case()
    cas = os.path.join(d, name + ".cas")
    M.write_cas(cas, raw)
    ref = H.dump_mesh(cas, I.BLOCK_MA, I.BLOCK_KN, M.DSMC_CELL_DTYPE, M.DSMC_EDGE_DTYPE, C.MESH_MESSAGE_DTYPE)
    counts = fill_counts(dm, PYR_PPC, fill_seed)
    f = H.fill(cas, mess, counts, seed=ref_seed)
    fill = dict(cells=ref["cells"], edges=ref["edges"], points=ref["points"], split=ref["split"], counts=counts,
                cell_count=np.bincount(f["cell"], minlength=dm.ncell).astype(np.int32),
                np_tri=f["np_tri"].astype(np.int16), rel=cube_relative(f["x"], f["cell"], per_cube),
                v_mean=f["v"].mean(0), v_var=f["v"].var(0), ir_mean=f["ir"].mean(), n_v=len(f["v"]))
    x, v, dt, cell = I.split_box_trace_inputs(raw, mess, trace_n, seed=trace_seed)
    r = H.trace(cas, mess, x, v, dt, cell, True)
    trace = dict(ncell=dm.ncell, **{k: r[k] for k in ("cell", "ifout", "face", "tri", "ncross", "x", "dt")})
    return fill, trace


def gen_pyramid(d):
    fill, trace = _split_box_pins(d, "pyr", pyramid_case, 6, PYR_SEED, 11, 6, TRACE_N)
    np.savez_compressed(os.path.join(HERE, "pyramid_pin.npz"), **fill)
    np.savez_compressed(os.path.join(HERE, "pyramid_trace_pin.npz"), **trace)


def gen_prism(d):
    fill, trace = _split_box_pins(d, "prism", prism_case, 2, PRISM_SEED, 12, 7, TRACE_N // 2)
    np.savez_compressed(os.path.join(HERE, "prism_pin.npz"), **fill, **{"trace_" + k: v for k, v in trace.items()})


SAMPLE_PPC = 6
SAMPLE_SEED = 31
SAMPLE_STEPS = 5200          # past NSCHEME (2000) and NSS (5000), src/meshImport.h:48-59


def gen_sample(d):
    raw, dm = I.block_mesh(scale=8)
    cas = os.path.join(d, "b8s.cas")
    M.write_cas(cas, raw)
    mess = I.block_mess(dm, SAMPLE_PPC)
    x, v, ir, cell = I.fill_inputs(dm, mess, SAMPLE_PPC, SAMPLE_SEED)
    r = H.sample(cas, mess, x, v, ir, cell, SAMPLE_STEPS, SAMPLE_PPC)
    rr = H.sample(cas, mess, x, v, ir, cell, SAMPLE_STEPS, SAMPLE_PPC, host_rule=True)
    np.savez_compressed(os.path.join(HERE, "sample_pin.npz"), ppc=SAMPLE_PPC, seed=SAMPLE_SEED, steps=SAMPLE_STEPS,
                        **r, **{"rule_" + k: a for k, a in rr.items()})


COLLIDE_PPC = (20, 12)        # block hexahedra, capsule tets
COLLIDE_SEED = 41


def collide_cases():
    """Ragged particle sets for one collisionDSMC: the 1/4 block mesh and the
    capsule tets."""
    raw, dm = I.block_mesh()
    mess = I.block_mess(dm, STATS_PPC)
    rawc, dmc, messc = I.capsule_small()
    out = []
    for (r, m, ms, fill, ppc, k) in ((raw, dm, mess, I.fill_inputs, COLLIDE_PPC[0], 0),
                                     (rawc, dmc, messc, I.fill_inputs_any, COLLIDE_PPC[1], 1)):
        parts = I.ragged(fill(m, ms, ppc, COLLIDE_SEED + k), m.ncell, ppc, COLLIDE_SEED + 10 + k)
        out.append((r, m, ms, parts))
    return out


def collision_conservation(ncell, before, after):
    """The largest per-cell change of momentum (relative to the cell's
    momentum scale sqrt(sum |v|^2)) and of energy sum(|v|^2 / 2 + Ir)
    (relative) between two particle sets."""
    def sums(p):
        x, v, ir, c = p
        mom = np.stack([np.bincount(c, v[:, j], ncell) for j in range(3)], 1)
        return mom, np.bincount(c, 0.5 * (v * v).sum(1) + ir, ncell), np.sqrt(np.bincount(c, (v * v).sum(1), ncell))
    m0, e0, s0 = sums(before)
    m1, e1, _ = sums(after)
    live = s0 > 0
    return (float((np.abs(m1 - m0).max(1)[live] / s0[live]).max()),
            float((np.abs(e1 - e0)[live] / e0[live]).max()))


def gen_collide(d):
    res = {}
    for k, (raw, dm, mess, parts) in zip(("block", "tets"), collide_cases()):
        cas = os.path.join(d, f"col_{k}.cas")
        M.write_cas(cas, raw)
        r = H.collide(cas, mess, *parts, seed=3)
        after = (r["particles"]["x"], r["particles"]["v"], r["particles"]["ir"], r["particles"]["cell"])
        dmom, den = collision_conservation(dm.ncell, parts, after)
        res.update({f"{k}_remcoll": r["remcoll"], f"{k}_pairs": r["pairs"], f"{k}_collisions": r["collisions"],
                    f"{k}_crmax_raised": int((r["crmax"] > 3.0).sum()), f"{k}_dmom": dmom, f"{k}_den": den})
    np.savez_compressed(os.path.join(HERE, "collide_pin.npz"), **res)


INJECT_STEPS = 40
INJECT_SEED = 5
INJECT_SAMPLE = 6000


def gen_inject(d):
    raw, dm = I.block_mesh()
    cas = os.path.join(d, "b4i.cas")
    M.write_cas(cas, raw)
    mess = I.block_mess(dm, STATS_PPC)
    out = {}
    rawc, dmc, messc = I.capsule_small()
    casc = os.path.join(d, "capi.cas")
    M.write_cas(casc, rawc)
    for pre, path, m, ms in (("", cas, dm, mess), ("tet_", casc, dmc, messc)):
        r = H.inject(path, ms, INJECT_STEPS, INJECT_SEED)
        sub = np.sort(np.random.RandomState(2).permutation(len(r["cell"]))[:INJECT_SAMPLE])
        out.update({pre + "per_step": r["per_step"].astype(np.int32), pre + "reminj": r["reminj"],
                    pre + "cell_count": np.bincount(r["cell"], minlength=m.ncell).astype(np.int32),
                    pre + "x": r["x"][sub].astype(np.float32), pre + "v": r["v"][sub].astype(np.float32),
                    pre + "ir": r["ir"][sub].astype(np.float32)})
    np.savez_compressed(os.path.join(HERE, "inject_pin.npz"), steps=INJECT_STEPS, seed=INJECT_SEED, **out)


WALL_N = 20000
WALL_SEED = 12


def gen_wall(d):
    raw, dm = I.block_mesh()
    cas = os.path.join(d, "b4w.cas")
    M.write_cas(cas, raw)
    mess = I.block_mess(dm, STATS_PPC)
    rawc, dmc, messc = I.capsule_small()
    casc = os.path.join(d, "capw.cas")
    M.write_cas(casc, rawc)
    out = {}
    for pre, path, m, ms, tets in (("", cas, dm, mess, False), ("tet_", casc, dmc, messc, True)):
        x, v, dt, c = I.wall_trace_inputs(m, ms, WALL_N, WALL_SEED, tets=tets)
        first = H.trace(path, ms, x, v, dt, c, True)
        full = H.trace(path, ms, x, v, dt, c, False)
        hit = np.nonzero((first["face"] >= 0) & (m.edges["faceTag"][np.maximum(first["face"], 0)] == 6))[0]
        out.update({pre + "first_face": first["face"].astype(np.int32), pre + "hit": hit.astype(np.int32),
                    pre + "v": full["v"][hit].astype(np.float32)})
    np.savez_compressed(os.path.join(HERE, "wall_pin.npz"), n=WALL_N, seed=WALL_SEED, **out)


CAPBAND_SEEDS = [201, 202, 203, 204, 205, 206, 207, 208]
CAPBAND_PPC = 8
CAPBAND_STEPS = 120
CAPBAND_AVG_FROM = 61
CAPBAND_EVERY = 3             # cells kept in the fixture: every third


def gen_capband(d):
    """The statistics band on the capsule tets (Kn 0.01: collision-dominated),
    8 seeded reference runs side by side."""
    from concurrent.futures import ThreadPoolExecutor
    raw, dm, mess = I.capsule_small()
    cas = os.path.join(d, "capb.cas")
    M.write_cas(cas, raw)
    x, v, ir, cell = I.fill_inputs_any(dm, mess, CAPBAND_PPC, 3)

    def one(seed):
        return H.run(cas, mess, x, v, ir, cell, CAPBAND_STEPS, seed, "-", CAPBAND_AVG_FROM)

    with ThreadPoolExecutor(len(CAPBAND_SEEDS)) as ex:
        runs = list(ex.map(one, CAPBAND_SEEDS))
    band = np.stack([I.fields_from_moments(r["moments"], CAPBAND_STEPS - CAPBAND_AVG_FROM + 1, dm, mess)
                     for r in runs])
    keep = np.arange(0, dm.ncell, CAPBAND_EVERY)
    np.savez_compressed(os.path.join(HERE, "stats_band_capsule.npz"), cells=keep.astype(np.int32),
                        mean=band.mean(0)[keep].astype(np.float32),
                        sd=band.std(0, ddof=1)[keep].astype(np.float32), k=len(CAPBAND_SEEDS),
                        steps=CAPBAND_STEPS, avg_from=CAPBAND_AVG_FROM, ppc=CAPBAND_PPC,
                        nparticles=np.stack([r["steps"][:, 0] for r in runs]).astype(np.int32))


DEGEN_CELLS = 20
DEGEN_TET_CELLS = 12
DEGEN_SEED = 9
DEGEN_SPIN_SECONDS = 3


def gen_degenerate(d):
    """Degenerate tracing inputs on the 1/4 block mesh. The reference's loop
    has no iteration bound; the particles the oracle stops at its crossing
    bound are each given to the reference alone for DEGEN_SPIN_SECONDS (the
    rest finish together in well under a second) and recorded as spinning
    when it has not returned; the reference's outputs are stored for the
    rest."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle as O
    raw, dm = I.block_mesh()
    cas = os.path.join(d, "b4d.cas")
    M.write_cas(cas, raw)
    mess = I.block_mess(dm, STATS_PPC)
    x, v, dt, cell = I.degenerate_trace_inputs(dm, mess, DEGEN_CELLS, DEGEN_SEED)

    class P:                                 # DsmcCaseParams fields for the oracle
        nzones = len(I.REF_ZONES)
        zone_tag = [z[0] for z in I.REF_ZONES]
        zone_role = [z[1] for z in I.REF_ZONES]
        zone_inject = [z[2] for z in I.REF_ZONES]
        inflow_dir = tuple(I.inflow_dir())
        seed, nss, nscheme, nevery, nrepeat, wall_stats, max_crossings = 0, 5000, 2000, 1, 100, 0, 4096

    q = O.Oracle(dm, mess, P()).trace(x, v, dt, cell, stop_at_wall=True)
    cand = np.nonzero(q["ncross"] >= P.max_crossings)[0]

    def finishes(i):
        return H.trace_finishes(cas, mess, x[[i]], v[[i]], dt[[i]], cell[[i]], DEGEN_SPIN_SECONDS)

    with ThreadPoolExecutor(8) as ex:
        fin = list(ex.map(finishes, cand))
    if any(fin):
        raise SystemExit(f"the reference finished on {int(np.sum(fin))} particles the oracle bounds")
    ok = np.setdiff1d(np.arange(len(cell)), cand)
    r = H.trace(cas, mess, x[ok], v[ok], dt[ok], cell[ok], True, timeout=120)
    # the same on the capsule tetrahedra (every zone has a role there)
    rawc, dmc, messc = I.capsule_small()
    casc = os.path.join(d, "capd.cas")
    M.write_cas(casc, rawc)
    xt, vt, dtt, ct = I.degenerate_tet_trace_inputs(dmc, messc, DEGEN_TET_CELLS, DEGEN_SEED)
    rt = H.trace(casc, messc, xt, vt, dtt, ct, True, timeout=120)
    np.savez_compressed(os.path.join(HERE, "degenerate_trace_pin.npz"), ncells=DEGEN_CELLS, seed=DEGEN_SEED,
                        spin_seconds=DEGEN_SPIN_SECONDS, ok=ok.astype(np.int32), spins=cand.astype(np.int32),
                        tet_ncells=DEGEN_TET_CELLS,
                        **{k: r[k] for k in ("cell", "ifout", "face", "tri", "ncross", "x", "dt")},
                        **{"tet_" + k: rt[k] for k in ("cell", "ifout", "face", "tri", "ncross", "x", "dt")})


# the stress and heat-flux fields of macro_from_moments, banded like stats_band
MACRO_BAND_FIELDS = [5, 6, 7, 8, 9, 10, 11, 12, 13, 15, 16, 17]


def gen_band(d):
    raw, dm = I.block_mesh()
    cas = os.path.join(d, "b4.cas")
    M.write_cas(cas, raw)
    mess = I.block_mess(dm, STATS_PPC)
    xs, vs, irs, cs = I.fill_inputs(dm, mess, STATS_PPC, seed=3)
    fields, per_step = [], []
    for s in STATS_SEEDS:
        rr = H.run(cas, mess, xs, vs, irs, cs, STATS_STEPS, s, "-", STATS_AVG_FROM)
        f = I.macro_from_moments(rr["moments"], STATS_STEPS - STATS_AVG_FROM + 1, dm, mess)
        fields.append(f[:, MACRO_BAND_FIELDS])
        per_step.append(rr["steps"])
    fields = np.stack(fields)
    np.savez_compressed(os.path.join(HERE, "macro_band.npz"), mean=fields.mean(0), sd=fields.std(0, ddof=1),
                        k=len(STATS_SEEDS), columns=np.array(MACRO_BAND_FIELDS), steps=STATS_STEPS,
                        avg_from=STATS_AVG_FROM, ppc=STATS_PPC,
                        per_step=np.stack(per_step).astype(np.int32))


def main():
    if not H.available():
        raise SystemExit("oracle/_ref/ref_harness missing: make -C oracle ref")
    want = set(sys.argv[1:])
    if want - {"gsis", "fill", "fluent", "pyramid", "prism", "band", "degenerate", "sample", "collide", "inject",
               "wall", "capband", "core", "tracefull"}:
        raise SystemExit("fixtures: core (mesh, trace, advect, inflow, stats, tet trace), gsis, fill, fluent, pyramid, "
                         "prism, band, degenerate, sample, collide, inject, wall, capband, tracefull")
    with tempfile.TemporaryDirectory() as d:
        if not want or want & {"gsis", "fill"}:
            gen_gsis_fill(d)
        if not want or "fluent" in want:
            gen_fluent(d)
        if not want or "pyramid" in want:
            gen_pyramid(d)
        if not want or "prism" in want:
            gen_prism(d)
        if not want or "band" in want:
            gen_band(d)
        if not want or "degenerate" in want:
            gen_degenerate(d)
        if not want or "sample" in want:
            gen_sample(d)
        if not want or "collide" in want:
            gen_collide(d)
        if not want or "inject" in want:
            gen_inject(d)
        if not want or "wall" in want:
            gen_wall(d)
        if not want or "capband" in want:
            gen_capband(d)
        if not want or "core" in want:
            gen_core(d)
        if not want or "tracefull" in want:
            gen_trace_full(d)
    print("fixtures written to", HERE)


def gen_core(d):
    # -- mesh pin (1/8 block mesh)
    raw8, dm8 = I.block_mesh(scale=8)
    cas8 = os.path.join(d, "b8.cas")
    M.write_cas(cas8, raw8)
    ref = H.dump_mesh(cas8, I.BLOCK_MA, I.BLOCK_KN, M.DSMC_CELL_DTYPE, M.DSMC_EDGE_DTYPE, C.MESH_MESSAGE_DTYPE)
    np.savez_compressed(os.path.join(HERE, "mesh_pin.npz"), cells=ref["cells"], edges=ref["edges"],
                        points=ref["points"], split=ref["split"], mess=np.asarray(ref["mess"]))

    # -- trace pin (1/4 block mesh)
    raw, dm = I.block_mesh()
    cas = os.path.join(d, "b4.cas")
    M.write_cas(cas, raw)
    mess = I.block_mess(dm, STATS_PPC)
    x, v, dt, cell = I.trace_inputs(dm, mess, TRACE_N, seed=1)
    res = {}
    for stop in (1, 0):
        r = H.trace(cas, mess, x, v, dt, cell, bool(stop))
        for k in ("cell", "ifout", "face", "tri", "ncross"):
            res[f"{k}_{stop}"] = r[k]
        if stop:
            res["x_1"] = r["x"]
            res["dt_1"] = r["dt"]
    np.savez_compressed(os.path.join(HERE, "trace_pin.npz"), mess=np.asarray(mess), **res)

    # -- advection pin (wall zone as outlet, deterministic)
    xf, vf, irf, cf = I.fill_inputs(dm, mess, 10, seed=2)
    r = H.advect(cas, mess, xf, vf, irf, cf, 1, roles_arg(I.NOWALL_ZONES))
    order = np.lexsort((r["v"][:, 2], r["v"][:, 1], r["v"][:, 0]))
    ppc = np.bincount(r["cell"], minlength=dm.ncell)
    np.savez_compressed(os.path.join(HERE, "advect_pin.npz"), ppc=ppc, x=r["x"][order], v=r["v"][order],
                        cell=r["cell"][order])

    # -- inflow remainders and the statistics band (reference roles)
    xs, vs, irs, cs = I.fill_inputs(dm, mess, STATS_PPC, seed=3)
    fields = []
    reminj = None
    nper = []
    for s in STATS_SEEDS:
        rr = H.run(cas, mess, xs, vs, irs, cs, STATS_STEPS, s, "-", STATS_AVG_FROM)
        if reminj is None:
            reminj = rr["reminj"]
        elif not np.array_equal(reminj, rr["reminj"]):
            raise SystemExit("reference inflow remainders differ between seeds")
        fields.append(I.fields_from_moments(rr["moments"], STATS_STEPS - STATS_AVG_FROM + 1, dm, mess))
        nper.append(rr["steps"][:, 0])
    fields = np.stack(fields)
    np.savez_compressed(os.path.join(HERE, "stats_band.npz"), fields=fields, nparticles=np.stack(nper),
                        steps=STATS_STEPS, avg_from=STATS_AVG_FROM, ppc=STATS_PPC, seeds=np.array(STATS_SEEDS))
    # remainders after 60 steps
    r60 = H.run(cas, mess, xs, vs, irs, cs, 60, 5, "-", 61)
    np.savez_compressed(os.path.join(HERE, "inflow_pin.npz"), reminj=r60["reminj"], steps=60)

    # -- tetrahedral trace pin (coarse capsule)
    rawc, dmc, messc = I.capsule_small()
    casc = os.path.join(d, "cap.cas")
    M.write_cas(casc, rawc)
    refc = H.dump_mesh(casc, 5.0, 0.01, M.DSMC_CELL_DTYPE, M.DSMC_EDGE_DTYPE, C.MESH_MESSAGE_DTYPE)
    for f in M.DSMC_EDGE_DTYPE.names:
        if not np.array_equal(refc["edges"][f], dmc.edges[f]):
            raise SystemExit(f"capsule mesh differs from the reference's parse in edges.{f}")
    xt, vt, dtt, ct = I.tet_trace_inputs(dmc, messc, TRACE_N, seed=4)
    r = H.trace(casc, messc, xt, vt, dtt, ct, True)
    np.savez_compressed(os.path.join(HERE, "tet_trace_pin.npz"), ncell=dmc.ncell,
                        **{k: r[k] for k in ("cell", "ifout", "face", "tri", "ncross", "x", "dt")})


TRACE_FULL_SAMPLE = 4096


def gen_trace_full(d):
    """The TRACE configuration on the full block mesh, run through the
    reference's tracing on the FP64 inputs and on their FP32-rounded state."""
    raw, dm = I.block_mesh(scale=1)
    cas = os.path.join(d, "b1.cas")
    M.write_cas(cas, raw)
    mess = I.block_mess(dm, STATS_PPC)
    x, v, dt, cell = I.trace_inputs(dm, mess, I.TRACE_FULL_N, seed=I.TRACE_FULL_SEED)
    x32, v32 = I.fp32_state(dm, x, v, cell)
    rs = np.random.RandomState(77)
    pick = np.sort(rs.choice(len(cell), TRACE_FULL_SAMPLE, replace=False)).astype(np.int32)
    out = dict(ncell=dm.ncell, n=len(cell), seed=I.TRACE_FULL_SEED, pick=pick)
    for tag, (xi, vi) in (("fp64", (x, v)), ("mixed", (x32, v32))):
        r = H.trace(cas, mess, xi, vi, dt, cell, True, timeout=3600)
        for k in ("cell", "ifout", "face", "tri", "ncross", "dt"):
            out[f"{tag}_{k}_sha"] = np.array(I.digest(r[k]))
        kept = r["cell"] >= 0
        if tag == "fp64":
            out["fp64_x_sha"] = np.array(I.digest(r["x"]))
        else:
            out["mixed_x_sha"] = np.array(I.digest(I.fp32_positions(dm, r["x"][kept], r["cell"][kept])))
        out[f"{tag}_ppc"] = np.bincount(r["cell"][kept], minlength=dm.ncell).astype(np.int32)
        out[f"{tag}_ifout_counts"] = np.array([np.sum(r["ifout"] == k) for k in (-1, 0, 1)], dtype=np.int64)
        out[f"{tag}_hits"] = np.int64(np.sum(r["face"] >= 0))
        for k in ("cell", "ifout", "face", "tri", "ncross", "x", "dt"):
            out[f"{tag}_sample_{k}"] = r[k][pick]
    np.savez_compressed(os.path.join(HERE, "trace_full_pin.npz"), **out)


if __name__ == "__main__":
    main()
