"""Runner for oracle/_ref/ref_harness, the reference's own DSMC code built
from its sources (ORACLE TEST INFRASTRUCTURE: used by tests/, the golden
fixture generator and bench.py's reference arm only).

Build recipe: ``make -C oracle ref`` (needs the reference sources; the built
binary is self-contained and travels with the repository snapshot).
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "ref_harness")


def available() -> bool:
    return os.path.exists(BIN) and os.access(BIN, os.X_OK)


def _run(args, timeout=3600):
    r = subprocess.run([BIN, *map(str, args)], capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"ref_harness {args[0]} failed ({r.returncode}): {r.stderr[-2000:]}")
    return r.stdout


def dump_mesh(cas: str, Ma: float, Kn: float, cell_dtype, edge_dtype, mess_dtype) -> dict:
    with tempfile.TemporaryDirectory() as d:
        _run(["mesh", cas, d, Ma, Kn])
        return {
            "cells": np.fromfile(os.path.join(d, "cells.bin"), dtype=cell_dtype),
            "edges": np.fromfile(os.path.join(d, "edges.bin"), dtype=edge_dtype),
            "points": np.fromfile(os.path.join(d, "points.bin"), dtype=np.float64),
            "split": np.fromfile(os.path.join(d, "split.bin"), dtype=np.uint8),
            "mess": np.fromfile(os.path.join(d, "mess.bin"), dtype=mess_dtype)[0],
        }


def _write_particles(path, x, v, ir, dt, cell):
    n = int(np.asarray(cell).shape[0])
    with open(path, "wb") as f:
        f.write(np.int64(n).tobytes())
        for k in range(3):
            f.write(np.ascontiguousarray(x[:, k], dtype=np.float64).tobytes())
        for k in range(3):
            f.write(np.ascontiguousarray(v[:, k], dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(ir, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(dt, dtype=np.float64).tobytes())
        f.write(np.ascontiguousarray(cell, dtype=np.int32).tobytes())


def _read_particles(path) -> dict:
    b = np.fromfile(path, dtype=np.uint8)
    n = int(b[:8].view(np.int64)[0])
    d = b[8:8 + n * 64].view(np.float64).reshape(8, n)
    cell = b[8 + n * 64:8 + n * 68].view(np.int32)
    return {"x": d[0:3].T.copy(), "v": d[3:6].T.copy(), "ir": d[6].copy(), "dt": d[7].copy(), "cell": cell.copy()}


def _write_mess(path, mess):
    np.asarray(mess).reshape(()).tofile(path)


def trace(cas: str, mess, x, v, dt, cell, stop_at_wall: bool = True, timeout: int = 3600) -> dict:
    """The reference's tracing loop on the given particles."""
    n = int(np.asarray(cell).shape[0])
    with tempfile.TemporaryDirectory() as d:
        pm, pp, po = (os.path.join(d, k) for k in ("mess.bin", "parts.bin", "out.bin"))
        _write_mess(pm, mess)
        _write_particles(pp, x, v, np.zeros(n), dt, cell)
        _run(["trace", cas, pm, pp, po, int(stop_at_wall)], timeout=timeout)
        b = np.fromfile(po, dtype=np.uint8)
        m = int(b[:8].view(np.int64)[0])
        ints = b[8:8 + 20 * m].view(np.int32).reshape(5, m)
        dbl = b[8 + 20 * m:].view(np.float64).reshape(7, m)
        return {"cell": ints[0].copy(), "ifout": ints[1].copy(), "face": ints[2].copy(), "tri": ints[3].copy(),
                "ncross": ints[4].copy(), "x": dbl[0:3].T.copy(), "v": dbl[3:6].T.copy(), "dt": dbl[6].copy()}


def trace_finishes(cas: str, mess, x, v, dt, cell, seconds: float) -> bool:
    """Whether the reference's tracing loop ends within the given time on
    these particles (its loop has no iteration bound)."""
    try:
        trace(cas, mess, x, v, dt, cell, True, timeout=seconds)
        return True
    except subprocess.TimeoutExpired:
        return False


def sample(cas: str, mess, x, v, ir, cell, nsteps: int, ppc: int, host_rule: bool = False) -> dict:
    """statistic_macroPre, then statistic_macro(k) for k = 1..nsteps on the
    particles of each step (the harness's sampledAt rule over the given
    ones, ppc per cell in input order), with host_rule the harness's
    hostRule changes of the sparse states after every exchange step; the
    macro arrays and window state after the last step."""
    n = int(np.asarray(cell).shape[0])
    with tempfile.TemporaryDirectory() as d:
        pm, pp = os.path.join(d, "mess.bin"), os.path.join(d, "parts.bin")
        _write_mess(pm, mess)
        _write_particles(pp, x, v, ir, np.zeros(n), cell)
        out = os.path.join(d, "out")
        os.makedirs(out)
        _run(["sample", cas, pm, pp, out, nsteps, ppc, int(host_rule)])
        res = {k: np.fromfile(os.path.join(out, k + ".bin"), dtype=np.float64).reshape(-1, 18)
               for k in ("local", "record", "final_record")}
        res["window_samples"] = np.fromfile(os.path.join(out, "window_samples.bin"), dtype=np.float64)
        res["window_valid"] = np.fromfile(os.path.join(out, "window_valid.bin"), dtype=np.float64).astype(np.int8)
        res["sparse_state"] = np.fromfile(os.path.join(out, "sparse_state.bin"), dtype=np.uint8)
        return res


def collide(cas: str, mess, x, v, ir, cell, seed: int = 1) -> dict:
    """One collisionDSMC() on the given particles from the initial crmax and
    remainders: remainders, crmax, candidate pairs, collisions and the
    buckets after it."""
    n = int(np.asarray(cell).shape[0])
    with tempfile.TemporaryDirectory() as d:
        pm, pp = os.path.join(d, "mess.bin"), os.path.join(d, "parts.bin")
        _write_mess(pm, mess)
        _write_particles(pp, x, v, ir, np.zeros(n), cell)
        out = os.path.join(d, "out")
        os.makedirs(out)
        _run(["collide", cas, pm, pp, out, seed])
        cnt = np.fromfile(os.path.join(out, "counts.bin"), dtype=np.float64)
        return {"remcoll": np.fromfile(os.path.join(out, "remcoll.bin"), dtype=np.float64),
                "crmax": np.fromfile(os.path.join(out, "crmax.bin"), dtype=np.float64),
                "pairs": int(cnt[0]), "collisions": int(cnt[1]),
                "particles": _read_particles(os.path.join(out, "particles.bin"))}


def inject(cas: str, mess, nsteps: int, seed: int = 1) -> dict:
    """preprocesseffquad on an empty domain for nsteps: the injected
    particles that stayed in the domain, their count per step and the
    inflow remainders."""
    with tempfile.TemporaryDirectory() as d:
        pm = os.path.join(d, "mess.bin")
        _write_mess(pm, mess)
        out = os.path.join(d, "out")
        os.makedirs(out)
        _run(["inject", cas, pm, out, nsteps, seed])
        res = _read_particles(os.path.join(out, "particles.bin"))
        res["per_step"] = np.fromfile(os.path.join(out, "steps.bin"), dtype=np.int64)
        res["reminj"] = np.fromfile(os.path.join(out, "reminj.bin"), dtype=np.float64)
        return res


def advect(cas: str, mess, x, v, ir, cell, istep: int = 1, roles: str = "-") -> dict:
    """The reference's advection(istep) + cache2chain(); buckets in order."""
    n = int(np.asarray(cell).shape[0])
    with tempfile.TemporaryDirectory() as d:
        pm, pp, po = (os.path.join(d, k) for k in ("mess.bin", "parts.bin", "out.bin"))
        _write_mess(pm, mess)
        _write_particles(pp, x, v, ir, np.zeros(n), cell)
        _run(["advect", cas, pm, pp, po, istep, roles])
        return _read_particles(po)


def run(cas: str, mess, x, v, ir, cell, nsteps: int, seed: int, roles: str = "-", avg_from: int = 1,
        timeout: int = 3600) -> dict:
    """The reference's five-call step loop for nsteps; returns its dumps and
    the timing line."""
    n = int(np.asarray(cell).shape[0])
    ncell = None
    with tempfile.TemporaryDirectory() as d:
        pm, pp = os.path.join(d, "mess.bin"), os.path.join(d, "parts.bin")
        _write_mess(pm, mess)
        _write_particles(pp, x, v, ir, np.zeros(n), cell)
        out = os.path.join(d, "out")
        os.makedirs(out)
        txt = _run(["run", cas, pm, pp, out, nsteps, seed, roles, avg_from], timeout=timeout)
        res = {"timing": json.loads(txt.strip().splitlines()[-1])}
        res["steps"] = np.fromfile(os.path.join(out, "steps.bin"), dtype=np.int64).reshape(nsteps, 4)
        for k in ("moments", "local", "record", "final_record"):
            a = np.fromfile(os.path.join(out, k + ".bin"), dtype=np.float64)
            res[k] = a.reshape(-1, 18)
        for k in ("crmax", "remcoll", "reminj", "window_samples"):
            res[k] = np.fromfile(os.path.join(out, k + ".bin"), dtype=np.float64)
        res["sparse_state"] = np.fromfile(os.path.join(out, "sparse_state.bin"), dtype=np.uint8)
        res["particles"] = _read_particles(os.path.join(out, "particles.bin"))
        return res


def gsis(cas: str, mess, x, v, ir, cell, nsresult, accepted=None, seed: int = 1, roles: str = "-") -> dict:
    """The reference's molecular_velocity_change on the given particles and
    NS solution; buckets in order."""
    n = int(np.asarray(cell).shape[0])
    with tempfile.TemporaryDirectory() as d:
        pm, pp, pn, pa, po = (os.path.join(d, k) for k in ("mess.bin", "parts.bin", "ns.bin", "acc.bin", "out.bin"))
        _write_mess(pm, mess)
        _write_particles(pp, x, v, ir, np.zeros(n), cell)
        np.ascontiguousarray(nsresult, dtype=np.float64).tofile(pn)
        if accepted is None:
            pa = "-"
        else:
            np.ascontiguousarray(accepted, dtype=np.int8).tofile(pa)
        _run(["gsis", cas, pm, pp, pn, pa, po, seed, roles])
        return _read_particles(po)


def fill(cas: str, mess, counts, seed: int = 1) -> dict:
    """The reference's initial fill of every cell with counts[c] particles
    (Np_tri_inititial + meshfillpar); buckets in order plus the
    per-tetrahedron counts."""
    with tempfile.TemporaryDirectory() as d:
        pm, pc = os.path.join(d, "mess.bin"), os.path.join(d, "counts.bin")
        _write_mess(pm, mess)
        np.ascontiguousarray(counts, dtype=np.int32).tofile(pc)
        out = os.path.join(d, "out")
        os.makedirs(out)
        _run(["fill", cas, pm, pc, out, seed])
        res = _read_particles(os.path.join(out, "particles.bin"))
        res["np_tri"] = np.fromfile(os.path.join(out, "np_tri.bin"), dtype=np.int32)
        return res


def fluent(cas: str, mess, fields) -> dict:
    """The reference's out2Fluent_dsmc of fields [ncell][18] on the mesh of
    cas; returns the file's bytes and the zone declarations (id, first, last)."""
    with tempfile.TemporaryDirectory() as d:
        pm, pf = os.path.join(d, "mess.bin"), os.path.join(d, "fields.bin")
        _write_mess(pm, mess)
        np.ascontiguousarray(fields, dtype=np.float64).tofile(pf)
        out = os.path.join(d, "out")
        os.makedirs(out)
        _run(["fluent", cas, pm, pf, out])
        with open(os.path.join(out, "fields.dat"), "rb") as fh:
            text = fh.read()
        zones = np.fromfile(os.path.join(out, "zones.bin"), dtype=np.int32).reshape(-1, 3)
        return {"text": text, "zones": zones}


def bench(cas: str, mess, counts, nsteps: int, seed: int, roles: str, drift, tN: float,
          timeout: int = 3600) -> dict:
    """The reference's own initial fill of counts[c] particles per cell,
    moved to the freestream (drift, temperature tN), then nsteps of its step
    loop, each timed (the harness's "bench" command); its JSON report."""
    with tempfile.TemporaryDirectory() as d:
        pm, pc = os.path.join(d, "mess.bin"), os.path.join(d, "counts.bin")
        _write_mess(pm, mess)
        np.ascontiguousarray(counts, dtype=np.int32).tofile(pc)
        out = _run(["bench", cas, pm, pc, nsteps, seed, roles, float(drift[0]), float(drift[1]), float(drift[2]),
                    float(tN)], timeout=timeout)
        return json.loads(out.strip().splitlines()[-1])
