"""DSMC particle-step benchmark (B200).

One "step" is one full DSMC step (inflow injection, move with face-crossing
tracing, cell sort, NTC collisions, 18-moment sampling) over every particle
of the case. The metric is particle-steps/s: particles at the start of each
step summed over the timed steps, divided by the device time (CUDA events on
the library's stream, max over ranks). Mixed precision is the production
path; the all-FP64 path is timed on the same case for the mixed/FP64 ratio.

Default workload: the capsule case (Ma 5, Kn 0.01, AoA 30 deg) on the
generated 371,214-tet mesh at 100 particles per cell (37.1M particles);
--workload block runs the 48,640-hex block case (200 particles per cell by
default).

Multi-GPU runs are independent replicas (one case per GPU, no collective on
the data path): value = the sum of all ranks' particle-steps / the slowest
rank's time.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload capsule|block|batch|serve]
                  [--ppc P] [--impl ours|reference] [--no-cpu-baseline]
                  [--cases N] [--batch-seed S] [--no-autotune]

--workload batch runs the batched form instead: --cases seeded hex-box
cases advanced together, one CUDA graph per step, against the same cases
stepped one after another. --workload serve runs the served form: --requests
capsule cases arriving at --rate per second, served with continuous batching
(p50/p99 time-to-result, cases/hour, particle-steps/s).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "dig-appolo_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

from pydsmc import case as C  # noqa: E402
from pydsmc import mesh as M  # noqa: E402
from pydsmc import workload as W  # noqa: E402

METRIC = "DSMC particle-steps/s (mixed vs FP64 plain, 1 B200)"


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def block_workload(ppc: int):
    """The block case: 48x32x32 hexes, central 8^3 block removed (48,640
    cells), Ma 5, Kn 0.1 on the block edge, T_in 142.2 K, T_w 300 K, inflow
    on x-min, outflow x-max, specular sides, AoA 0."""
    raw = M.block_case_mesh(scale=1)
    dm = M.build_dsmc_mesh(raw)
    mess = C.mesh_message(dm, 5.0, 0.1, ppc=ppc, L0=0.5 / 32 * 8)
    zones = [(3, 1, 0), (4, 2, 1), (5, 3, 0), (6, 4, 0), (7, 5, 0)]
    return {"name": "block", "dm": dm, "mess": mess, "zones": zones, "inflow_dir": C.inflow_direction(0.0),
            "desc": {"workload": "block-48640", "cells": dm.ncell, "ppc": ppc,
                     "mesh": "hex box 1.0x0.5x0.5 m, 48x32x32 minus central 8^3 diffuse block",
                     "Ma": 5.0, "Kn": 0.1, "aoa_deg": 0.0, "sides": "specular"}}


def make_workload(name: str, ppc: int):
    if name == "block":
        return block_workload(ppc)
    if name == "capsule":
        from pydsmc import capsule
        return capsule.capsule_workload(ppc)
    raise SystemExit(f"unknown workload {name}")


def algorithmic_bytes(n_particles: float, ncell: int, ntri_per_cell: float, mixed: bool) -> dict:
    """Algorithmic bytes of one step and of one launch of each stage's main
    kernel.

    - step: each particle's state read and written once, 32 B (mixed: x, v,
      Ir as FP32 + cell id) or 60 B (FP64: x, v, Ir as FP64 + cell id); each
      cell's triangles read once (9 words + 8 B of face id/tag per
      triangle); the per-cell collision and sampling state (3 x 18 FP64
      accumulators + crmax + 2 remainders) read and written.
    - move: the particle state read and written, the triangles read.
    - collide: velocities and internal energy read and written (16 B mixed,
      32 B FP64 per particle); crmax and the collision remainder read and
      written, the cell volume and the cell's start read.
    - sample: velocities and internal energy read; the accumulators read and
      written and the record fields written (18 FP64) per cell.
    - sort (gather): the state read from the source and written to the
      sorted slot, plus the source index."""
    sp = 32 if mixed else 60
    word = 4 if mixed else 8
    vi = 4 * word
    geom = ntri_per_cell * (9 * word + 8)
    acc = 3 * 18 * 8 + 3 * 8
    move = n_particles * 2 * sp + ncell * geom
    step = move + ncell * 2 * acc
    collide = n_particles * 2 * vi + ncell * (2 * 8 + 2 * 8 + 8 + 4)
    sample = n_particles * vi + ncell * (2 * 54 * 8 + 18 * 8 + 4)
    sort = n_particles * (2 * sp + 4)
    return {"step": step, "move": move, "collide": collide, "sample": sample, "sort": sort, "inject": None,
            "per_particle_state": sp, "geom_per_cell": geom}


def measured_traffic(kernel: str, workload: str, particles: float):
    """DRAM bytes per launch of a kernel on this workload from the committed
    ncu summaries (profiles/<kernel>_<mesh>_ppc<N>.md, lines
    'dram_bytes_per_launch: B' and 'particles: P'): the summary of this very
    workload if there is one, else one of the same mesh at another particle
    count, scaled to this launch by the particle ratio (full captures are
    taken on a smaller case). Returns (bytes or None, source note)."""
    mesh, _, _ = workload.rpartition("_ppc")
    pdir = os.path.join(ROOT, "profiles")

    def read(path):
        vals = {}
        with open(path) as f:
            for line in f:
                k, sep, v = line.strip().partition(":")
                if sep and k in ("dram_bytes_per_launch", "particles"):
                    vals[k] = float(v.strip().split()[0])
        return vals

    exact = os.path.join(pdir, f"{kernel}_{workload}.md")
    cands = [exact] if os.path.exists(exact) else sorted(
        os.path.join(pdir, f) for f in (os.listdir(pdir) if os.path.isdir(pdir) else [])
        if f.startswith(f"{kernel}_{mesh}_ppc") and f.endswith(".md"))
    for path in cands:
        vals = read(path)
        if "dram_bytes_per_launch" not in vals:
            continue
        rel = os.path.relpath(path, ROOT)
        if path == exact or "particles" not in vals:
            return vals["dram_bytes_per_launch"], rel
        scale = particles / vals["particles"]
        return vals["dram_bytes_per_launch"] * scale, f"{rel}, scaled by particles x{scale:.3f}"
    return None, None


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        q = ("--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                r = subprocess.run(["nvidia-smi", "-i", str(self.index), q, "--format=csv,noheader,nounits"],
                                   capture_output=True, text=True, timeout=5)
                if r.returncode == 0 and r.stdout.strip():
                    self.samples.append([s.strip() for s in r.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, n in enumerate(names):
                if len(s) > 3 + k and s[3 + k].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# our implementation
# ---------------------------------------------------------------------------
def run_case(wl, fill, precision, steps, warmup, seed, timing=False):
    import torch
    from pydsmc import gpu
    p = gpu.default_params(precision=precision, seed=seed, zones=wl["zones"], inflow_dir=wl["inflow_dir"],
                           nss=10 ** 9, nscheme=max(1, (steps + warmup) // 5), nrepeat=100)
    case = gpu.Case(wl["dm"], wl["mess"], p, device=torch.cuda.current_device())
    if "device" in fill:
        case.fill_freestream(*fill["device"])
    else:
        case.upload_particles(fill["x"], fill["v"], fill["ir"], fill["cell"])
    case.statistic_macroPre()
    # launch shapes picked on this case (ordinary steps; results do not
    # depend on them), then the warm-up steps
    istep, _ = case.autotune(1, trial_steps=1)
    istep -= 1
    for _ in range(warmup):
        istep += 1
        case.step(istep)
    case.sync()
    stream = torch.cuda.ExternalStream(case.lib.dsmc_stream(case.h))
    n_before = []
    case.set_timing(timing)
    case.stage_ms(reset=True)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    counts = []
    # particle counts are device-resident; read them at the end from the counters
    c0 = case.counters()
    n0 = case.particle_count()
    ev0.record(stream)
    for _ in range(steps):
        istep += 1
        case.step(istep)
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    c1 = case.counters()
    n1 = case.particle_count()
    stage = case.stage_ms(reset=True) if timing else None
    case.sync()
    res = {"ms": ms, "n0": n0, "n1": n1, "counters0": c0, "counters1": c1, "stage": stage, "istep": istep,
           "case": case}
    return res


def over_ranks(x: float, op: str, device: str) -> float:
    """x reduced over the ranks of the process group (max or sum); x itself
    without a group or with one rank. Replica runs report the slowest
    rank's time and the sum of all ranks' particle-steps."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return x
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def particle_steps(res, steps):
    # particles at the start of each timed step: n0 + injected - removed... use the
    # inventory at both ends (the inventory drifts slowly) times the step count
    return 0.5 * (res["n0"] + res["n1"]) * steps


def run_ours(args):
    import torch
    import torch.distributed as dist
    from pydsmc import gpu
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if not torch.cuda.is_available():
        raise SystemExit("no CUDA device")
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    gpu.load()
    wl = make_workload(args.workload, args.ppc)
    dm, mess = wl["dm"], wl["mess"]
    # the reference's initial state: a mean of ppc particles per cell in
    # proportion to the cell volumes, drawn on the device
    fill = {"device": (float(args.ppc), 1000 + rank)}

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return over_ranks(x, "max", "cuda")

    def sum_over_ranks(x):
        return over_ranks(x, "sum", "cuda")

    peak, peak_kind = load_peaks()
    # --- headline: mixed precision, graph replay
    barrier()
    with ClockSampler(local) as clk:
        mixed = run_case(wl, fill, gpu.PRECISION_MIXED, args.steps, args.warmup, seed=1000 + rank)
    barrier()
    ms_mixed = max_over_ranks(mixed["ms"])
    ps_mixed = sum_over_ranks(particle_steps(mixed, args.steps))
    value = ps_mixed / (ms_mixed / 1e3)
    case_m = mixed.pop("case")
    nparts = int(mixed["n0"])
    # --- the GSIS particle update on the same case (between steps): an NS
    # state of +-10% density around the current counts, drift and
    # temperatures perturbed around the freestream; host wall time of the
    # call (NS upload, count pass and scan, one read-back, rebuild)
    gsis = gsis_timing(case_m, wl, seed=3000 + rank)
    # --- stage timing pass (events between stages, no graph) for the roofline
    barrier()
    tim = run_case(wl, fill, gpu.PRECISION_MIXED, max(3, args.steps // 2), 1, seed=2000 + rank, timing=True)
    tim.pop("case").close()
    stage_ms, tsteps = tim["stage"]
    stage_avg = stage_ms / max(tsteps, 1)
    # --- FP64 path on the same case
    barrier()
    fp64 = run_case(wl, fill, gpu.PRECISION_FP64, args.steps, args.warmup, seed=1000 + rank)
    fp64.pop("case").close()
    barrier()
    ms_fp64 = max_over_ranks(fp64["ms"])
    ps_fp64 = sum_over_ranks(particle_steps(fp64, args.steps))
    value_fp64 = ps_fp64 / (ms_fp64 / 1e3)
    # --- e2e through the C ABI with host buffers
    barrier()
    e2e = run_e2e(wl, fill, args, rank)
    e2e_ms = max_over_ranks(e2e["ms"])
    e2e_ps = sum_over_ranks(e2e["particle_steps"])
    case_m.close()

    tri_per_cell = 12.0 if wl["name"] == "block" else 4.0
    n_mean = 0.5 * (mixed["n0"] + mixed["n1"])
    ab = algorithmic_bytes(n_mean, dm.ncell, tri_per_cell, mixed=True)
    names = ["inject", "move", "sort", "collide", "sample"]
    kernels = {"inject": "inject_gen_kernel", "move": "move_kernel", "sort": "gather_kernel",
               "collide": "collide_kernel", "sample": "sample_kernel"}
    dom = names[int(np.argmax(stage_avg))]
    dom_ms = float(stage_avg[names.index(dom)])
    dom_bytes = ab.get(dom)
    achieved = (dom_bytes / (dom_ms / 1e3)) / 1e9 if (dom_bytes and dom_ms > 0) else None
    traffic, traffic_src = measured_traffic(kernels[dom], wl["desc"]["workload"] + f"_ppc{args.ppc}", n_mean)
    step_achieved = (ab["step"] / (ms_mixed / args.steps / 1e3)) / 1e9
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "particle-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_mixed / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64acc",
        "data": "synthetic (generated mesh; device initial fill: the reference's per-cell counts and placement, freestream velocities)",
        "config": dict(wl["desc"], particles_per_gpu=nparts, parallelism=f"replicas x{world}",
                       l2="particle state > L2 (126 MB)", precision="mixed"),
        "fp64": {"value": value_fp64, "ms_per_step": ms_fp64 / args.steps, "dtype": "f64"},
        "mixed_over_fp64": value / value_fp64 if value_fp64 > 0 else None,
        "stage_ms_per_step": dict(zip(names, [float(x) for x in stage_avg])),
        "roofline": {"bound": "hbm", "kernel": kernels[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "traffic_source": traffic_src, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": dom_bytes, "launch_ms": dom_ms,
                     "step": {"algorithmic_bytes": ab["step"], "achieved": step_achieved,
                              "frac": step_achieved / peak}},
        "e2e": {"value": e2e_ps / (e2e_ms / 1e3), "unit": "particle-steps/s",
                "h2d_bytes_per_step": e2e["h2d"] / args.steps, "d2h_bytes_per_step": e2e["d2h"] / args.steps},
        "gpu_launches": None,
        "gsis_update": gsis,
        "clocks": clk.summary(),
        "counters": {k: mixed["counters1"][k] - mixed["counters0"][k] for k in mixed["counters1"]},
    }
    line["gpu_launches"] = launches_per_step(wl) * args.steps
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl, fill, args)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def gsis_timing(case, wl, seed: int, repeats: int = 3) -> dict:
    dm, mess = wl["dm"], wl["mess"]
    rs = np.random.default_rng(seed)
    n = case.counts()["ppc"].astype(float)
    vol = dm.cells["area"].astype(float)
    u, sig, tN = W.freestream(mess, wl["inflow_dir"])
    ns = np.empty((dm.ncell, 6))
    ns[:, 0] = np.maximum(n, 1.0) * rs.uniform(0.9, 1.1, dm.ncell) * float(mess["Neff"]) / (vol * float(mess["n_ref"]))
    ns[:, 1:4] = u + 0.05 * rs.standard_normal((dm.ncell, 3))
    ns[:, 4] = tN * rs.uniform(0.95, 1.05, dm.ncell)
    ns[:, 5] = tN * rs.uniform(0.95, 1.05, dm.ncell)
    case.sync()
    ms = []
    rep = None
    for _ in range(repeats):
        t0 = time.perf_counter()
        rep = case.molecular_velocity_change(ns)
        ms.append((time.perf_counter() - t0) * 1e3)
    return {"ms": float(np.median(ms)), "particles": int(rep["particles"]), "cells_updated": int(rep["cells_updated"]),
            "added": int(rep["added"]), "removed": int(rep["removed"]),
            "note": "host wall time of dsmc_molecular_velocity_change (NS upload included), median of 3"}


def launches_per_step(wl) -> int:
    # inject: count, scan, generate; move; sort: rank, scan x2, scatter,
    # far-slot order, gather; collide: classify, collide; sample
    return 3 + 1 + 6 + 2 + 1


def run_e2e(wl, fill, args, rank):
    """The same step count through the C ABI with host buffers: upload the
    particles from host memory, run the steps, read each step's counters
    and the sampled fields (the GSIS hand-off, [cell][18] FP64) back."""
    import torch
    from pydsmc import gpu
    p = gpu.default_params(precision=gpu.PRECISION_MIXED, seed=3000 + rank, zones=wl["zones"],
                           inflow_dir=wl["inflow_dir"], nss=10 ** 9, nscheme=100, nrepeat=100)
    case = gpu.Case(wl["dm"], wl["mess"], p, device=torch.cuda.current_device())
    # the same initial particles as host arrays (made on the device, read
    # back before the timed region); the graph is warmed on them
    case.fill_freestream(*fill["device"])
    hx, hv, hir, hcell = case.download_particles()
    # the C ABI's layout: one contiguous column per coordinate
    cols = [np.ascontiguousarray(hx[:, k]) for k in range(3)] + [np.ascontiguousarray(hv[:, k]) for k in range(3)]
    for s in range(1, args.warmup + 1):
        case.step(s)
    case.sync()
    t0 = time.perf_counter()
    case.upload_columns(*cols, hir, hcell)
    n0 = case.particle_count()
    h2d = int(n0) * (7 * 8 + 4)
    d2h = 0
    total = 0
    for s in range(args.warmup + 1, args.warmup + args.steps + 1):
        case.step(s)
        c = case.counters()
        d2h += 12 * 8
        total += n0
    local = case.macro(gpu.MACRO_LOCAL)
    d2h += local.nbytes
    case.sync()
    ms = (time.perf_counter() - t0) * 1e3
    case.close()
    return {"ms": ms, "particle_steps": total, "h2d": h2d, "d2h": d2h}


def cpu_baseline(wl, fill, args):
    """The reference's own DSMC step (oracle/_ref, one compute rank = one
    core) on a bounded sample: the same mesh and constants with a reduced
    particle count, a few steps."""
    sys.path.insert(0, ROOT)
    from oracle import harness as H
    if not H.available():
        return {"value": None, "unit": "particle-steps/s", "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref/ref_harness not built"}
    dm, mess = wl["dm"], wl["mess"]
    ppc_s = max(2, min(args.ppc, 10))
    sub = W.initial_fill(dm, mess, ppc_s, seed=7, inflow_dir=wl["inflow_dir"], proportional=True)
    nsteps = 5
    roles = {1: "interface", 2: "inlet", 3: "outlet", 4: "wall", 5: "none", 0: "none"}
    r_arg = ",".join(f"{t}:{roles[r]}" for t, r, _ in wl["zones"])
    with tempfile.TemporaryDirectory() as d:
        cas = os.path.join(d, "case.cas")
        M.write_cas(cas, wl["dm"].raw)
        r = H.run(cas, mess, sub["x"], sub["v"], sub["ir"], sub["cell"], nsteps, 1, r_arg, nsteps + 1, timeout=600)
    t = r["timing"]
    return {"value": t["particle_steps_per_s"], "unit": "particle-steps/s", "cores": 1, "kind": "reference",
            "sample": f"{wl['desc']['workload']} mesh, {ppc_s} particles/cell on average in proportion to the cell "
                      f"volumes ({len(sub['cell'])} particles), "
                      f"{nsteps} steps, {t['seconds']:.2f} s of one core"}


# ---------------------------------------------------------------------------
# batched form: many independent cases in one CUDA graph per step
# ---------------------------------------------------------------------------
BLOCK_ZONES = [(3, 1, 0), (4, 2, 1), (5, 3, 0), (6, 4, 0), (7, 5, 0)]


def batch_specs(n: int, seed: int):
    """Seeded hex-box obstacle cases: cells log-uniform in 5k-80k (a box of
    3k x 2k x 2k hexes, 1.0 x 0.5 x 0.5 m, with the central (k/2)^3 block
    removed as a diffuse wall, k even), particles per cell uniform in
    20-200, Ma uniform in 3-10, angle of attack uniform in 0-40 deg, Kn on
    the block edge log-uniform in 0.01-1."""
    rs = np.random.default_rng(seed)
    out = []
    for j in range(n):
        cells = math.exp(rs.uniform(math.log(5e3), math.log(8e4)))
        k = max(4, 2 * int(round((cells / 11.875) ** (1.0 / 3.0) / 2.0)))
        out.append({"k": k, "ppc": float(rs.uniform(20, 200)), "Ma": float(rs.uniform(3, 10)),
                    "aoa": float(rs.uniform(0, 40)), "Kn": float(math.exp(rs.uniform(math.log(0.01), 0.0))),
                    "seed": j})
    return out


def batch_mesh(k: int):
    h = k // 2
    nx, ny, nz = 3 * k, 2 * k, 2 * k
    i0, j0, k0 = (nx - h) // 2, (ny - h) // 2, (nz - h) // 2
    raw = M.hex_box(nx, ny, nz, 1.0, 0.5, 0.5, (i0, i0 + h, j0, j0 + h, k0, k0 + h))
    return M.build_dsmc_mesh(raw), h * 0.5 / ny


def make_batch_cases(specs, precision, autotune=True):
    import torch
    from pydsmc import gpu
    meshes = {}
    cases, steps = [], []
    for sp in specs:
        if sp["k"] not in meshes:
            meshes[sp["k"]] = batch_mesh(sp["k"])
        dm, L0 = meshes[sp["k"]]
        mess = C.mesh_message(dm, sp["Ma"], sp["Kn"], ppc=int(round(sp["ppc"])), L0=L0)
        p = gpu.default_params(precision=precision, seed=7000 + sp["seed"], zones=BLOCK_ZONES,
                               inflow_dir=C.inflow_direction(sp["aoa"]), nss=10 ** 9, nscheme=50, nrepeat=100)
        case = gpu.Case(dm, mess, p, device=torch.cuda.current_device())
        case.fill_freestream(sp["ppc"], 9000 + sp["seed"])
        case.statistic_macroPre()
        nxt = 1
        if autotune:
            nxt, _ = case.autotune(1, trial_steps=1)
        cases.append(case)
        steps.append(nxt - 1)
    return cases, steps


def run_batch(args):
    """The batched form: args.cases cases (batch_specs), autotuned, advanced
    (a) one after another, each by its own per-step graph, and (b) together,
    one CUDA graph per step whose branches are the cases. value = total
    particle-steps / device time of (b)."""
    import torch
    from pydsmc import gpu
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    gpu.load()
    specs = batch_specs(args.cases, args.batch_seed)
    t0 = time.perf_counter()
    cases, steps = make_batch_cases(specs, gpu.PRECISION_MIXED, autotune=not args.no_autotune)
    setup_s = time.perf_counter() - t0
    K, W0 = args.steps, args.warmup
    # (a) one after another: device time summed over the cases
    seq_ms, seq_ps = 0.0, 0.0
    for j, case in enumerate(cases):
        for _ in range(W0):
            steps[j] += 1
            case.step(steps[j])
        case.sync()
        st = torch.cuda.ExternalStream(case.lib.dsmc_stream(case.h))
        n0 = case.particle_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(K):
            steps[j] += 1
            case.step(steps[j])
        e1.record(st)
        e1.synchronize()
        seq_ms += e0.elapsed_time(e1)
        seq_ps += 0.5 * (n0 + case.particle_count()) * K
    # (b) together
    batch = gpu.Batch(cases)
    batch.step(W0)
    batch.sync()
    bs = torch.cuda.ExternalStream(batch.stream())
    n0 = sum(c.particle_count() for c in cases)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(bs)
        batch.step(K)
        e1.record(bs)
        e1.synchronize()
    b_ms = e0.elapsed_time(e1)
    batch.sync()
    n1 = sum(c.particle_count() for c in cases)
    b_ps = 0.5 * (n0 + n1) * K
    shapes = [c.launch_shape() for c in cases]
    batch.close()
    for c in cases:
        c.close()
    cells = [batch_mesh_cells(sp["k"]) for sp in specs]
    line = {
        "metric": f"DSMC particle-steps/s, {len(specs)}-case batch (one CUDA graph per step, 1 B200)",
        "value": b_ps / (b_ms / 1e3), "unit": "particle-steps/s", "n_gpus": 1, "steps": K, "warmup": W0,
        "ms_per_step": b_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64acc", "data": "synthetic (seeded cases, device freestream fill)",
        "sequential": {"value": seq_ps / (seq_ms / 1e3), "ms_per_step": seq_ms / K,
                       "how": "each case on its own, one after another, its own per-step graph"},
        "batch_over_sequential": (b_ps / (b_ms / 1e3)) / (seq_ps / (seq_ms / 1e3)),
        "config": {"workload": f"batch-{len(specs)}", "cases": len(specs), "cells_total": int(sum(cells)),
                   "particles_total": int(n0), "cells_range": [int(min(cells)), int(max(cells))],
                   "autotuned": not args.no_autotune, "batch_seed": args.batch_seed, "setup_s": setup_s,
                   "move_threads_chosen": sorted({s["move_threads"] for s in shapes})},
        "gpu_launches": None,
        "gsis_update": gsis,
        "clocks": clk.summary(),
    }
    line["gpu_launches"] = launches_per_step(None) * K * len(specs) + K * len(specs)
    print(json.dumps(line), flush=True)


def batch_mesh_cells(k: int) -> int:
    h = k // 2
    return 12 * k ** 3 - h ** 3


# ---------------------------------------------------------------------------
# served form: continuous batching of arriving capsule cases
# ---------------------------------------------------------------------------
SERVE_SCALES = (2.65, 1.8, 1.4, 1.15, 1.0)   # mesh spacing factors: about 20k to 371k tets


def serve_pool():
    """Capsule meshes at several resolutions (the request stream resamples
    among them)."""
    from pydsmc import capsule
    pool = []
    for f in SERVE_SCALES:
        raw = capsule.capsule_mesh(h_fine=0.215 * f, h_coarse=0.60 * f, seed=0)
        pool.append(M.build_dsmc_mesh(raw))
    return pool


def run_serve(args):
    """The served form: args.requests capsule cases arriving as a Poisson
    stream (args.rate per second), each on a mesh drawn from the pool, with
    10-100 particles per cell and 200-2000 steps (mixed precision, Ma 5,
    Kn 0.01, AoA 30 deg); admission by a 160 GB device-memory budget; fields
    handed to the host every 100 steps; sampling window 20%, steady sampling
    from 50% of each case's steps."""
    import torch
    from pydsmc import capsule, gpu, serve
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    gpu.load()
    t0 = time.perf_counter()
    pool = serve_pool()
    setup_s = time.perf_counter() - t0
    rs = np.random.default_rng(args.batch_seed)
    zones = [(3, 1, 0), (4, 2, 1), (5, 3, 0), (6, 4, 0)]
    reqs, t = [], 0.0
    for j in range(args.requests):
        t += rs.exponential(1.0 / args.rate)
        dm = pool[int(rs.integers(0, len(pool)))]
        ppc = float(rs.uniform(10, 100))
        steps = int(rs.integers(200, 2001))
        mess = C.mesh_message(dm, 5.0, 0.01, ppc=int(round(ppc)), L0=capsule.L0)
        reqs.append((t, serve.CaseRequest(dm=dm, mess=mess, zones=zones, inflow_dir=C.inflow_direction(30.0),
                                          steps=steps, ppc=ppc, seed=j, precision=gpu.PRECISION_MIXED,
                                          name=f"req{j}")))
    be = serve.GpuBackend(device=torch.cuda.current_device())
    srv = serve.Server(be, hbm_budget=160e9, max_active=64, handoff_every=100)
    with ClockSampler(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        start = time.perf_counter()
        for ta, r in reqs:
            srv.submit(r, start + ta)
        srv.run()
    be.close()
    s = srv.summary()
    line = {
        "metric": "DSMC served capsule cases (continuous batching, 1 B200): particle-steps/s; p50/p99 time-to-result",
        "value": s["particle_steps_per_s"], "unit": "particle-steps/s", "n_gpus": 1,
        "p50_s": s["p50_s"], "p99_s": s["p99_s"], "cases_per_hour": s["cases_per_hour"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64acc",
        "data": "synthetic (seeded Poisson request stream, generated meshes, device freestream fill)",
        "config": {"workload": "serve-capsule", "requests": args.requests, "rate_per_s": args.rate,
                   "mesh_cells": sorted(int(d.ncell) for d in pool), "ppc": [10, 100], "steps": [200, 2000],
                   "hbm_budget_gb": 160, "handoff_every": 100, "max_concurrent": s["max_concurrent"],
                   "rounds": s["rounds"], "span_s": s["span_s"], "mesh_setup_s": setup_s,
                   "timing": "wall clock from each request's arrival to its result on the host"},
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, ROOT)
    from oracle import harness as H
    if not H.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness (the reference's DSMC "
                          "code built against a one-rank MPI shim) is not built"}))
        return
    wl = make_workload(args.workload, args.ppc)
    dm, mess = wl["dm"], wl["mess"]
    cores = os.cpu_count() or 1
    ppc_s = max(2, min(args.ppc, 10))
    roles = {1: "interface", 2: "inlet", 3: "outlet", 4: "wall", 5: "none", 0: "none"}
    r_arg = ",".join(f"{t}:{roles[r]}" for t, r, _ in wl["zones"])
    nsteps = args.warmup + args.steps
    with tempfile.TemporaryDirectory() as d:
        cas = os.path.join(d, "case.cas")
        M.write_cas(cas, dm.raw)
        from concurrent.futures import ThreadPoolExecutor
        fills = [W.initial_fill(dm, mess, ppc_s, seed=100 + k, inflow_dir=wl["inflow_dir"], proportional=True)
                 for k in range(cores)]
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=cores) as ex:
            futs = [ex.submit(H.run, cas, mess, f["x"], f["v"], f["ir"], f["cell"], nsteps, 1 + k, r_arg, nsteps + 1, 3600)
                    for k, f in enumerate(fills)]
            res = [f.result() for f in futs]
        wall = time.perf_counter() - t0
    per = [r["timing"]["particle_steps_per_s"] for r in res]
    agg = float(sum(per))
    # n_gpus: the N this arm was launched for (the reference itself runs on
    # the host cores; "device" says so)
    line = {"impl": "reference", "metric": METRIC, "value": agg, "unit": "particle-steps/s",
            "n_gpus": int(os.environ.get("WORLD_SIZE", args.gpus)), "device": f"host ({cores} cores)",
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": wl["desc"],
            "cpu_baseline": {"value": agg, "unit": "particle-steps/s", "cores": cores, "kind": "reference",
                             "sample": f"{cores} independent single-rank processes, {ppc_s} particles/cell on "
                                       f"average each, "
                                       f"{nsteps} steps each, {wall:.1f} s wall"},
            "e2e": {"value": agg, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="capsule")
    ap.add_argument("--ppc", type=int, default=None)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cases", type=int, default=64, help="batch workload: number of cases")
    ap.add_argument("--batch-seed", type=int, default=0)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--requests", type=int, default=16, help="serve workload: number of requests")
    ap.add_argument("--rate", type=float, default=4.0, help="serve workload: arrivals per second")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.ppc is None:
        args.ppc = 100 if args.workload == "capsule" else 200
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
