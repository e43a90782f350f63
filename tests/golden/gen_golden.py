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

Usage: python tests/golden/gen_golden.py
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


def main():
    if not H.available():
        raise SystemExit("oracle/_ref/ref_harness missing: make -C oracle ref")
    out = {}
    with tempfile.TemporaryDirectory() as d:
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
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
