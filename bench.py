"""DSMC particle-step benchmark (B200).

One "step" is one full DSMC step (inflow injection, move with face-crossing
tracing, cell sort, NTC collisions, 18-moment sampling) over every particle
of the case. The metric is particle-steps/s: particles at the start of each
step summed over the timed steps, divided by the device time (CUDA events on
the library's stream, max over ranks). Mixed precision is the production
path; the all-FP64 path is timed on the same case for the mixed/FP64 ratio.

Default workload: the capsule case (Ma 5, Kn 0.01, AoA 30 deg) on the
generated 372,500-tet mesh at a mean of 100 particles per cell (37.25M
particles), run for its 2,000 steps with the served sampling rule (NSCHEME
at 20% of the steps, NSS at 50%) and the wall statistics on; the K timed
steps follow a spin-up to NSS and the W warm-up steps. Both precisions run
the whole case from the same host particles; the mixed run's fields are
compared with the FP64 run's per field. --workload block runs the
48,640-hex block case (200 particles per cell by default, 500 steps).

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


def stage_rooflines(ab: dict, stage_ms, names, kernels: dict, peak: float) -> dict:
    """Algorithmic bytes over the event-timed stage time, for every stage
    with a byte model (the dominant one is the line's `roofline`)."""
    out = {}
    for k, name in enumerate(names):
        b = ab.get(name)
        ms = float(stage_ms[k])
        if not b or ms <= 0:
            continue
        gbs = (b / (ms / 1e3)) / 1e9
        out[name] = {"kernel": kernels[name], "ms": ms, "algorithmic_bytes": b, "achieved": gbs, "frac": gbs / peak}
    return out


def measured_traffic(kernel: str, workload: str, particles: float):
    """DRAM bytes per launch of a kernel on this workload from the committed
    ncu summaries (profiles/<kernel>_<mesh>_ppc<N>.md, lines
    'dram_bytes_per_launch: B' and 'particles: P'): the summary of this very
    workload if there is one, else one of the same mesh at another particle
    count (full captures are taken on a smaller case), scaled to this launch
    by the particle ratio (the captured steps hold a slightly different
    count than the timed ones). Returns (bytes or None, source note)."""
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
        if "particles" not in vals:
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
def run_plan(wl, args) -> dict:
    """The case's run: the configuration's step count (2,000 on the capsule,
    500 on the block), with the served sampling rule (the exponential window
    NSCHEME from 20% of the steps, steady sampling NSS from 50%). The timed
    steps follow a spin-up to NSS and the warm-up steps, so they see the
    developed flow (shock layer, wake) and every sampler running."""
    total = args.run_steps if args.run_steps else (2000 if wl["name"] == "capsule" else 500)
    total = max(total, args.warmup + args.steps)
    nss, nscheme = total // 2, max(1, total // 5)
    spin = min(nss, total - args.warmup - args.steps)
    return {"total": total, "nss": nss, "nscheme": nscheme, "spinup": spin, "exchange_every": 100}


def bench_config(wl, plan) -> dict:
    """The workload as both arms report it."""
    dm = wl["dm"]
    return dict(wl["desc"], steps_run=plan["total"], nss=plan["nss"], nscheme=plan["nscheme"], wall_stats=True,
                particles_nominal=int(round(wl["desc"]["ppc"] * dm.ncell)),
                l2="inputs larger than L2 (particle state >= 1.2 GB per step)")


def case_params(wl, plan, precision, seed):
    from pydsmc import gpu
    return gpu.default_params(precision=precision, seed=seed, zones=wl["zones"], inflow_dir=wl["inflow_dir"],
                              nss=plan["nss"], nscheme=plan["nscheme"], nrepeat=plan["exchange_every"],
                              wall_stats=1)


def pinned_copy(a):
    """A numpy array in page-locked host memory (the host buffers a caller
    hands to the C ABI)."""
    import torch
    dt = {np.dtype(np.float64): torch.float64, np.dtype(np.int32): torch.int32}[np.asarray(a).dtype]
    t = torch.empty(np.asarray(a).shape, dtype=dt, pin_memory=True)
    out = t.numpy()
    out[...] = a
    return out


def initial_state(wl, plan, args, rank):
    """The initial particles as host arrays (the reference's fill rule: a mean
    of ppc per cell in proportion to the cell volumes, freestream
    velocities; drawn on the device and read back), in pinned memory."""
    import torch
    from pydsmc import gpu
    case = gpu.Case(wl["dm"], wl["mess"], case_params(wl, plan, gpu.PRECISION_MIXED, 1000 + rank),
                    device=torch.cuda.current_device())
    case.fill_freestream(float(args.ppc), 1000 + rank)
    hx, hv, hir, hcell = case.download_particles()
    cols = [pinned_copy(np.ascontiguousarray(hx[:, k])) for k in range(3)] + \
           [pinned_copy(np.ascontiguousarray(hv[:, k])) for k in range(3)] + [pinned_copy(hir), pinned_copy(hcell)]
    case.close()
    return cols


def full_run(wl, plan, args, precision, init, shape, rank, barrier, clock_index=None, stage_steps=0, tune=False):
    """One run of the case through the C ABI: the host arrays uploaded,
    steps 1..total, the GSIS hand-off at every exchange step after NSS (the
    window-averaged `record` fields and the particle count read back), the
    sampled fields at the end. Wall time of all of it is the run's
    end-to-end figure; steps spinup+warmup+1 .. +steps are timed on the
    device with CUDA events (barrier and synchronise on both sides). With
    `tune`, the autotuner picks the launch shapes on 29 ordinary steps of
    the run ending some 30 steps before the warm-up, on the developed flow
    the timed steps see."""
    import torch
    from pydsmc import gpu
    case = gpu.Case(wl["dm"], wl["mess"], case_params(wl, plan, precision, 1000 + rank),
                    device=torch.cuda.current_device())
    if shape:
        case.set_launch_shape(**shape)
    stream = torch.cuda.ExternalStream(case.lib.dsmc_stream(case.h))
    first = plan["spinup"] + args.warmup + 1
    last = first + args.steps - 1
    windows, nsamp = [], []
    h2d = sum(int(c.nbytes) for c in init)
    d2h = 0
    res = {}
    barrier()
    t0 = time.perf_counter()
    case.upload_columns(*init)
    case.statistic_macroPre()
    n = case.particle_count()
    nsamp.append((0, n))
    # the autotuner runs 29 steps (14 shapes, two steps each, and one to
    # warm up): tune where that ends well before the warm-up, or not at all
    # on runs too short for it
    tune_at = -1
    if tune:
        tune_at = plan["spinup"] - 60 if plan["spinup"] > 60 else (1 if first > 45 else -1)
    istep = 0
    while istep < plan["total"]:
        istep += 1
        if istep == tune_at:
            nxt, res["launch_shape"] = case.autotune(istep, trial_steps=2)
            istep = nxt - 1
            continue
        if istep == first:
            case.sync()
            barrier()
            res["n0"] = case.particle_count()
            res["c0"] = case.counters()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            clk = ClockSampler(clock_index) if clock_index is not None else None
            if clk:
                clk.__enter__()
            # a named range around the timed steps, for profilers
            torch.cuda.nvtx.range_push(f"timed-{'mixed' if precision == gpu.PRECISION_MIXED else 'fp64'}")
            ev0.record(stream)
        case.step(istep)
        if istep == last:
            ev1.record(stream)
            ev1.synchronize()
            torch.cuda.nvtx.range_pop()
            if clk:
                clk.__exit__()
                res["clocks"] = clk.summary()
            barrier()
            res["ms"] = ev0.elapsed_time(ev1)
            res["n1"] = case.particle_count()
            res["c1"] = case.counters()
        if istep % plan["exchange_every"] == 0:
            n = case.particle_count()
            nsamp.append((istep, n))
            d2h += 8
            if istep > plan["nss"]:
                windows.append(case.macro(gpu.MACRO_RECORD))
                d2h += windows[-1].nbytes
    final = case.macro(gpu.MACRO_FINAL_RECORD)
    d2h += final.nbytes
    case.sync()
    wall = time.perf_counter() - t0
    # particle-steps of the run: the inventory read at each exchange, between
    # two reads the mean of the two
    ps = 0.0
    for (sa, na), (sb, nb) in zip(nsamp, nsamp[1:]):
        ps += 0.5 * (na + nb) * (sb - sa)
    if nsamp[-1][0] < plan["total"]:
        ps += nsamp[-1][1] * (plan["total"] - nsamp[-1][0])
    res.update(case=case, windows=np.stack(windows) if windows else None, final=final, wall_s=wall,
               particle_steps=ps, h2d=h2d, d2h=d2h, counters_end=case.counters())
    if stage_steps:
        case.set_timing(True)
        case.stage_ms(reset=True)
        for k in range(stage_steps):
            case.step(plan["total"] + 1 + k)
        ms, nst = case.stage_ms(reset=True)
        case.set_timing(False)
        res["stage"] = ms / max(nst, 1)
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


def run_ours(args):
    import torch
    import torch.distributed as dist
    from pydsmc import fields, gpu
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
    dm = wl["dm"]
    plan = run_plan(wl, args)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return over_ranks(x, "max", "cuda")

    def sum_over_ranks(x):
        return over_ranks(x, "sum", "cuda")

    peak, peak_kind = load_peaks()
    init = initial_state(wl, plan, args, rank)
    # --- mixed precision: the full run, the headline steps timed inside it
    mixed = full_run(wl, plan, args, gpu.PRECISION_MIXED, init, None, rank, barrier, clock_index=local,
                     stage_steps=max(3, args.steps // 2), tune=not args.no_autotune)
    shape = mixed.get("launch_shape")
    ms_mixed = max_over_ranks(mixed["ms"])
    ps_mixed = sum_over_ranks(0.5 * (mixed["n0"] + mixed["n1"]) * args.steps)
    value = ps_mixed / (ms_mixed / 1e3)
    case_m = mixed.pop("case")
    # --- the GSIS particle update on the developed case (between steps)
    gsis = gsis_timing(case_m, wl, seed=3000 + rank)
    case_m.close()
    # --- the all-FP64 path: the same run from the same host particles
    barrier()
    fp64 = full_run(wl, plan, args, gpu.PRECISION_FP64, init, None, rank, barrier, tune=not args.no_autotune)
    fp64.pop("case").close()
    ms_fp64 = max_over_ranks(fp64["ms"])
    ps_fp64 = sum_over_ranks(0.5 * (fp64["n0"] + fp64["n1"]) * args.steps)
    value_fp64 = ps_fp64 / (ms_fp64 / 1e3)
    field_err = fields.compare_windows(mixed["windows"], fp64["windows"], dm.cells["area"]) \
        if mixed["windows"] is not None and fp64["windows"] is not None else None
    # --- end to end over K steps only: upload, K steps, counters every step,
    # the sampled fields at the end
    barrier()
    e2e_k = run_e2e_k(wl, plan, args, init, shape, rank)
    e2e_full_s = max_over_ranks(mixed["wall_s"])
    e2e_full_ps = sum_over_ranks(mixed["particle_steps"])
    e2e_k_s = max_over_ranks(e2e_k["s"])
    e2e_k_ps = sum_over_ranks(e2e_k["particle_steps"])

    tri_per_cell = 12.0 if wl["name"] == "block" else 4.0
    n_mean = 0.5 * (mixed["n0"] + mixed["n1"])
    ab = algorithmic_bytes(n_mean, dm.ncell, tri_per_cell, mixed=True)
    names = ["inject", "move", "sort", "collide", "sample"]
    kernels = {"inject": "inject_gen_kernel", "move": "move_kernel", "sort": "gather_kernel",
               "collide": "collide_kernel", "sample": "sample_warp_kernel"}
    stage_avg = mixed["stage"]
    dom = names[int(np.argmax(stage_avg))]
    dom_ms = float(stage_avg[names.index(dom)])
    dom_bytes = ab.get(dom)
    achieved = (dom_bytes / (dom_ms / 1e3)) / 1e9 if (dom_bytes and dom_ms > 0) else None
    traffic, traffic_src = measured_traffic(kernels[dom], wl["desc"]["workload"] + f"_ppc{args.ppc}", n_mean)
    step_achieved = (ab["step"] / (ms_mixed / args.steps / 1e3)) / 1e9
    cnt = {k: mixed["c1"][k] - mixed["c0"][k] for k in mixed["c1"]}
    searches = n_mean * args.steps + cnt["crossings"]
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
        "data": "synthetic (generated mesh; initial state: the reference's per-cell counts and placement with "
                "freestream velocities, drawn on the device and handed to the run as host arrays)",
        "config": bench_config(wl, plan),
        "timed_steps": [plan["spinup"] + args.warmup + 1, plan["spinup"] + args.warmup + args.steps],
        "launch_shape": shape,
        "particles": {"at_timed_start": int(mixed["n0"]), "initial": int(init[-1].shape[0]),
                      "parallelism": f"replicas x{world}"},
        "fp64": {"value": value_fp64, "ms_per_step": ms_fp64 / args.steps, "dtype": "f64",
                 "launch_shape": fp64.get("launch_shape")},
        "mixed_over_fp64": value / value_fp64 if value_fp64 > 0 else None,
        "field_error_vs_fp64": field_err,
        "stage_ms_per_step": dict(zip(names, [float(x) for x in stage_avg])),
        "roofline": {"bound": "hbm", "kernel": kernels[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                     "traffic_source": traffic_src, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": dom_bytes, "launch_ms": dom_ms,
                     "step": {"algorithmic_bytes": ab["step"], "achieved": step_achieved,
                              "frac": step_achieved / peak},
                     "stages": stage_rooflines(ab, stage_avg, names, kernels, peak)},
        "e2e": {"value": e2e_full_ps / e2e_full_s, "unit": "particle-steps/s",
                "h2d_bytes_per_step": mixed["h2d"] / plan["total"], "d2h_bytes_per_step": mixed["d2h"] / plan["total"],
                "how": f"the whole {plan['total']}-step run through the C ABI: host arrays (pinned) uploaded, every "
                       f"step, the record fields and the particle count read at every exchange step, the final "
                       f"fields read; wall time",
                "k_steps": {"value": e2e_k_ps / e2e_k_s, "steps": args.steps,
                            "h2d_bytes_per_step": e2e_k["h2d"] / args.steps,
                            "d2h_bytes_per_step": e2e_k["d2h"] / args.steps,
                            "how": "upload of the host arrays, K steps with the counters read after each, the "
                                   "local fields read; wall time"}},
        "gpu_launches": launches_per_step(wl) * args.steps,
        "gsis_update": gsis,
        "clocks": mixed.get("clocks"),
        "counters": cnt,
        "fp64_fallback_rate": cnt["fp64_fallbacks"] / searches if searches else None,
    }
    if not args.no_forms:
        barrier()
        line["forms"] = short_forms(args, rank)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl, plan, args)
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
    # inject: count, scan, generate; move: stay pass, tracing pass; sort:
    # rank, scan x2, scatter, far-slot order, gather; collide: classify,
    # collide; sample
    return 3 + 2 + 6 + 2 + 1


def run_e2e_k(wl, plan, args, init, shape, rank):
    """K steps end to end through the C ABI: upload the host arrays
    (pinned), run the steps, read each step's counters and the sampled
    fields ([cell][18] FP64) back; wall time. The graphs are warmed by W
    steps on the same case before the timed region."""
    import torch
    from pydsmc import gpu
    case = gpu.Case(wl["dm"], wl["mess"], case_params(wl, plan, gpu.PRECISION_MIXED, 3000 + rank),
                    device=torch.cuda.current_device())
    if shape:
        case.set_launch_shape(**shape)
    case.upload_columns(*init)
    case.statistic_macroPre()
    for s in range(1, args.warmup + 1):
        case.step(s)
    case.sync()
    t0 = time.perf_counter()
    case.upload_columns(*init)
    n0 = case.particle_count()
    h2d = sum(int(c.nbytes) for c in init)
    d2h = 0
    total = 0
    for s in range(args.warmup + 1, args.warmup + args.steps + 1):
        case.step(s)
        case.counters()
        d2h += 12 * 8
        total += n0
    local = case.macro(gpu.MACRO_LOCAL)
    d2h += local.nbytes
    case.sync()
    sec = time.perf_counter() - t0
    case.close()
    return {"s": sec, "particle_steps": total, "h2d": h2d, "d2h": d2h}


def reference_roles(wl) -> str:
    roles = {1: "interface", 2: "inlet", 3: "outlet", 4: "wall", 5: "none", 0: "none"}
    return ",".join(f"{t}:{roles[r]}" for t, r, _ in wl["zones"])


def reference_bench(wl, args, nproc: int, nsteps: int, seed0: int) -> dict:
    """The reference's own step (oracle/_ref) on the full case: nproc
    independent single-rank processes at once, each filling the case with
    the reference's own initial fill (a mean of ppc particles per cell in
    proportion to the volumes, moved to the freestream) and running nsteps
    steps; the first step of each is its warm-up, the rest are timed."""
    sys.path.insert(0, ROOT)
    from concurrent.futures import ThreadPoolExecutor
    from oracle import harness as H
    dm, mess = wl["dm"], wl["mess"]
    u, _, tN = W.freestream(mess, wl["inflow_dir"])
    r_arg = reference_roles(wl)
    with tempfile.TemporaryDirectory() as d:
        cas = os.path.join(d, "case.cas")
        M.write_cas(cas, dm.raw)
        counts = [W.proportional_counts(dm, float(args.ppc), np.random.default_rng(seed0 + k)) for k in range(nproc)]
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=nproc) as ex:
            futs = [ex.submit(H.bench, cas, mess, counts[k], nsteps, seed0 + k, r_arg, u, tN, 3600)
                    for k in range(nproc)]
            res = [f.result() for f in futs]
        wall = time.perf_counter() - t0
    rates = []
    for r in res:
        sec = r["step_seconds"][1:] if nsteps > 1 else r["step_seconds"]
        parts = r["step_particles"][1:] if nsteps > 1 else r["step_particles"]
        rates.append(sum(parts) / sum(sec))
    return {"value": float(sum(rates)), "per_process": rates, "particles": [r["particles"] for r in res],
            "fill_s": [r["fill_seconds"] for r in res], "wall_s": wall,
            "step_s": [r["step_seconds"] for r in res]}


def cpu_baseline(wl, plan, args):
    """The reference's own DSMC step (oracle/_ref, one compute rank = one
    core) on the full case: its own fill, one warm-up step, one timed step."""
    sys.path.insert(0, ROOT)
    from oracle import harness as H
    if not H.available():
        return {"value": None, "unit": "particle-steps/s", "cores": 1, "kind": "reference",
                "sample": "unavailable: oracle/_ref/ref_harness not built"}
    r = reference_bench(wl, args, 1, 2, 7)
    return {"value": r["value"], "unit": "particle-steps/s", "cores": 1, "kind": "reference",
            "sample": f"the full {wl['desc']['workload']} case ({r['particles'][0]} particles from the reference's "
                      f"own fill, moved to the freestream), one warm-up step and one timed step "
                      f"({r['step_s'][0][-1]:.1f} s) on one core"}


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


def batch_leg(specs, K, W0, autotune=True, clock_index=None) -> dict:
    """The batched form on the given cases (batch_specs), autotuned,
    advanced (a) one after another, each by its own per-step graph, and (b)
    together, one CUDA graph per step whose branches are the cases; device
    time of each (CUDA events)."""
    import torch
    from pydsmc import gpu
    t0 = time.perf_counter()
    cases, steps = make_batch_cases(specs, gpu.PRECISION_MIXED, autotune=autotune)
    setup_s = time.perf_counter() - t0
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
    clk = ClockSampler(clock_index) if clock_index is not None else None
    if clk:
        clk.__enter__()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(bs)
    batch.step(K)
    e1.record(bs)
    e1.synchronize()
    if clk:
        clk.__exit__()
    b_ms = e0.elapsed_time(e1)
    batch.sync()
    n1 = sum(c.particle_count() for c in cases)
    b_ps = 0.5 * (n0 + n1) * K
    shapes = [c.launch_shape() for c in cases]
    batch.close()
    for c in cases:
        c.close()
    cells = [batch_mesh_cells(sp["k"]) for sp in specs]
    return {"value": b_ps / (b_ms / 1e3), "ms_per_step": b_ms / K, "particles": int(n0),
            "sequential": {"value": seq_ps / (seq_ms / 1e3), "ms_per_step": seq_ms / K,
                           "how": "each case on its own, one after another, its own per-step graph"},
            "batch_over_sequential": (b_ps / (b_ms / 1e3)) / (seq_ps / (seq_ms / 1e3)),
            "cases": len(specs), "cells_total": int(sum(cells)), "cells_range": [int(min(cells)), int(max(cells))],
            "setup_s": setup_s, "move_threads_chosen": sorted({s["move_threads"] for s in shapes}),
            "clocks": clk.summary() if clk else None}


def run_batch(args):
    """The batched form: args.cases cases (batch_specs). value = total
    particle-steps / device time of the batched steps."""
    import torch
    from pydsmc import gpu
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    gpu.load()
    specs = batch_specs(args.cases, args.batch_seed)
    K, W0 = args.steps, args.warmup
    r = batch_leg(specs, K, W0, autotune=not args.no_autotune, clock_index=int(os.environ.get("LOCAL_RANK", "0")))
    line = {
        "metric": f"DSMC particle-steps/s, {len(specs)}-case batch (one CUDA graph per step, 1 B200)",
        "value": r["value"], "unit": "particle-steps/s", "n_gpus": 1, "steps": K, "warmup": W0,
        "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64acc", "data": "synthetic (seeded cases, device freestream fill)",
        "sequential": r["sequential"], "batch_over_sequential": r["batch_over_sequential"],
        "config": {"workload": f"batch-{len(specs)}", "cases": len(specs), "cells_total": r["cells_total"],
                   "particles_total": r["particles"], "cells_range": r["cells_range"],
                   "autotuned": not args.no_autotune, "batch_seed": args.batch_seed, "setup_s": r["setup_s"],
                   "move_threads_chosen": r["move_threads_chosen"]},
        "gpu_launches": launches_per_step(None) * K * len(specs) + K * len(specs),
        "clocks": r["clocks"],
    }
    print(json.dumps(line), flush=True)


def batch_mesh_cells(k: int) -> int:
    h = k // 2
    return 12 * k ** 3 - h ** 3


# ---------------------------------------------------------------------------
# served form: continuous batching of arriving capsule cases
# ---------------------------------------------------------------------------
SERVE_SCALES = (2.65, 1.8, 1.4, 1.15, 1.0)   # mesh spacing factors: about 20k to 371k tets


def serve_pool(scales=None):
    """Capsule meshes at several resolutions (the request stream resamples
    among them)."""
    from pydsmc import capsule
    pool = []
    for f in (SERVE_SCALES if scales is None else scales):
        raw = capsule.capsule_mesh(h_fine=0.215 * f, h_coarse=0.60 * f, seed=0)
        pool.append(M.build_dsmc_mesh(raw))
    return pool


def serve_leg(pool, requests: int, rate: float, seed: int, steps_range=(200, 2001), ppc_range=(10, 100),
              round_steps: int = 20, clock_index=None) -> dict:
    """The served form: `requests` capsule cases arriving as a Poisson stream
    (`rate` per second), each on a mesh drawn from the pool, with particles
    per cell and steps uniform in the given ranges (mixed precision, Ma 5,
    Kn 0.01, AoA 30 deg); admission by a 160 GB device-memory budget; rounds
    of at most `round_steps` steps, arrivals admitted while a round runs;
    fields handed to the host every 100 steps; sampling window 20%, steady
    sampling from 50% of each case's steps."""
    import torch
    from pydsmc import capsule, gpu, serve
    rs = np.random.default_rng(seed)
    zones = [(3, 1, 0), (4, 2, 1), (5, 3, 0), (6, 4, 0)]
    reqs, t = [], 0.0
    for j in range(requests):
        t += rs.exponential(1.0 / rate)
        dm = pool[int(rs.integers(0, len(pool)))]
        ppc = float(rs.uniform(*ppc_range))
        steps = int(rs.integers(*steps_range))
        mess = C.mesh_message(dm, 5.0, 0.01, ppc=int(round(ppc)), L0=capsule.L0)
        reqs.append((t, serve.CaseRequest(dm=dm, mess=mess, zones=zones, inflow_dir=C.inflow_direction(30.0),
                                          steps=steps, ppc=ppc, seed=j, precision=gpu.PRECISION_MIXED,
                                          name=f"req{j}")))
    be = serve.GpuBackend(device=torch.cuda.current_device())
    srv = serve.Server(be, hbm_budget=160e9, max_active=64, handoff_every=100, max_round_steps=round_steps)
    clk = ClockSampler(clock_index) if clock_index is not None else None
    if clk:
        clk.__enter__()
    start = time.perf_counter()
    for ta, r in reqs:
        srv.submit(r, start + ta)
    srv.run()
    if clk:
        clk.__exit__()
    be.close()
    s = srv.summary()
    return {"value": s["particle_steps_per_s"], "p50_s": s["p50_s"], "p99_s": s["p99_s"],
            "cases_per_hour": s["cases_per_hour"], "requests": requests, "rate_per_s": rate,
            "mesh_cells": sorted(int(d.ncell) for d in pool), "ppc": list(ppc_range),
            "steps": [steps_range[0], steps_range[1] - 1], "hbm_budget_gb": 160, "handoff_every": 100,
            "round_steps": round_steps, "max_concurrent": s["max_concurrent"],
            "joined_while_running": s["joined_while_running"], "rounds": s["rounds"], "span_s": s["span_s"],
            "clocks": clk.summary() if clk else None}


def run_serve(args):
    """The served form (serve_leg) as its own line: args.requests requests
    at args.rate per second on the full pool of capsule meshes."""
    import torch
    from pydsmc import gpu
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    gpu.load()
    t0 = time.perf_counter()
    pool = serve_pool()
    setup_s = time.perf_counter() - t0
    r = serve_leg(pool, args.requests, args.rate, args.batch_seed, clock_index=int(os.environ.get("LOCAL_RANK", "0")))
    line = {
        "metric": "DSMC served capsule cases (continuous batching, 1 B200): particle-steps/s; p50/p99 time-to-result",
        "value": r["value"], "unit": "particle-steps/s", "n_gpus": 1,
        "p50_s": r["p50_s"], "p99_s": r["p99_s"], "cases_per_hour": r["cases_per_hour"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64acc",
        "data": "synthetic (seeded Poisson request stream, generated meshes, device freestream fill)",
        "config": dict({k: r[k] for k in ("requests", "rate_per_s", "mesh_cells", "ppc", "steps", "hbm_budget_gb",
                                          "handoff_every", "round_steps", "max_concurrent", "joined_while_running",
                                          "rounds", "span_s")},
                       workload="serve-capsule", mesh_setup_s=setup_s,
                       timing="wall clock from each request's arrival to its result on the host"),
        "clocks": r["clocks"],
    }
    print(json.dumps(line), flush=True)


def short_forms(args, rank) -> dict:
    """The batched and served forms, short, for the headline line: 8 seeded
    batch cases for W + K steps, and 8 served capsule requests (about 20k
    and 50k tets, 10-60 particles per cell, 200-400 steps) arriving at 4 per
    second."""
    out = {}
    specs = batch_specs(8, 1000 + rank)
    out["batch"] = batch_leg(specs, args.steps, args.warmup, autotune=not args.no_autotune)
    pool = serve_pool((2.65, 1.8))
    out["serve"] = serve_leg(pool, 8, 4.0, 2000 + rank, steps_range=(200, 401), ppc_range=(10, 60))
    return out


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def mem_available_gb() -> float:
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) / 1e6
    except OSError:
        pass
    return 8.0


def run_reference(args):
    """The reference arm: the reference's own CPU implementation of the step
    (oracle/_ref: its sources built against a one-rank MPI stand-in) on the
    same case as our arm, on the host cores: as many concurrent single-rank
    processes as the cores and the host memory allow (about 6 GB each at the
    capsule's 37 million particles), each with the reference's own initial
    fill, one warm-up step and up to three timed steps (one step takes about
    14 s of one core). Rank 0 runs it; other ranks exit."""
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
    plan = run_plan(wl, args)
    cores = os.cpu_count() or 1
    per_gb = 8.0 if wl["name"] == "capsule" else 2.0
    nproc = max(1, min(cores, 16, int(mem_available_gb() // per_gb)))
    nsteps = min(4, max(2, -(-(args.steps + args.warmup) // nproc)))
    r = reference_bench(wl, args, nproc, nsteps, 100)
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": "particle-steps/s",
            "n_gpus": int(os.environ.get("WORLD_SIZE", args.gpus)), "device": f"host ({nproc} of {cores} cores)",
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": bench_config(wl, plan),
            "cpu_baseline": {"value": r["value"], "unit": "particle-steps/s", "cores": nproc, "kind": "reference",
                             "sample": f"{nproc} concurrent single-rank processes of the reference, each the full "
                                       f"case ({int(np.mean(r['particles']))} particles on average from its own "
                                       f"fill, moved to the freestream), 1 warm-up and {nsteps - 1} timed steps "
                                       f"each, {r['wall_s']:.1f} s wall"},
            "e2e": {"value": r["value"], "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
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
    ap.add_argument("--no-forms", action="store_true", help="leave out the short batched and served legs")
    ap.add_argument("--run-steps", type=int, default=0,
                    help="steps of the case's run (default: 2000 capsule, 500 block); the timed steps follow a "
                         "spin-up to half of it")
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
