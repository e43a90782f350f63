"""Serving DSMC cases with continuous batching.

Requests (a mesh, its case constants and a step count) arrive over time. The
server admits them in arrival order while their device-memory footprint fits
the budget and a batch slot is free, keeps every admitted case resident on
the GPU between steps, and advances all admitted cases together: each round
is one batched step call (dsmc_batch_step: one CUDA graph per step whose
branches are the cases). A round stops at the next point where some case
must hand its sampled fields to the host (every `handoff_every` of its own
steps, the GSIS exchange of the reference's coupled loop), finishes, or has
run `max_round_steps`; a finished case releases its memory and slot before
the next admission, so new requests join the batch while others are
running. A backend that can launch a round without waiting for it
(`launch` / `wait`) lets the server admit the requests that arrive during
the round while the GPU works: their set-up (mesh upload, device fill) runs
on their own streams beside the batch, and they join the next round.

Every case keeps its own step count, constants and random streams, and a
batched step equals the same step taken alone, so a case's result does not
depend on which other cases shared the GPU with it.

The scheduling logic talks to a backend (create, batched step, hand-off,
finish, footprint); `GpuBackend` drives the CUDA library, and tests may
substitute their own.
"""
from __future__ import annotations

import heapq
import itertools
import time
from dataclasses import dataclass, field

import numpy as np


@dataclass
class CaseRequest:
    """One case: the mesh and constants of a pydsmc.gpu.Case, the initial
    fill (mean particles per cell, seed) and the number of steps. Sampling
    follows the served configuration: the exponential window is 20% of the
    steps (NSCHEME) and steady sampling starts at 50% (NSS)."""
    dm: object
    mess: np.ndarray
    zones: list
    inflow_dir: tuple
    steps: int
    ppc: float
    seed: int = 0
    precision: int = 1
    name: str = ""


@dataclass
class CaseResult:
    request: CaseRequest
    t_arrival: float
    t_admit: float
    t_done: float
    handoffs: int
    final_record: np.ndarray
    local: np.ndarray
    particle_steps: float
    counters: dict

    @property
    def time_to_result(self) -> float:
        return self.t_done - self.t_arrival


@dataclass
class _Active:
    rid: int
    req: CaseRequest
    handle: object
    t_arrival: float
    t_admit: float
    footprint: int
    step: int = 0
    handoffs: int = 0
    particle_steps: float = 0.0


class GpuBackend:
    """Backend on the CUDA library (one device)."""

    def __init__(self, device: int = 0):
        from . import gpu
        self.gpu = gpu
        self.device = device
        self._batch = None
        self._members = ()
        gpu.load()

    def footprint(self, req: CaseRequest) -> int:
        """Upper bound of the device bytes of one case: two particle buffers
        and the sort scratch at the automatic capacity (1.5 x the expected
        particles + 65536), plus per-cell state and geometry."""
        n = req.ppc * req.dm.ncell
        cap = max(int(n * 1.5) + (1 << 16), 1 << 20)
        per_particle = (2 * 32 + 8) if req.precision == self.gpu.PRECISION_MIXED else (2 * 60 + 8)
        per_cell = 4096 + 12 * 160
        return int(cap * per_particle + req.dm.ncell * per_cell + (8 << 20))

    def create(self, req: CaseRequest):
        g = self.gpu
        nss = max(1, int(0.5 * req.steps))
        p = g.default_params(precision=req.precision, seed=req.seed, zones=req.zones, inflow_dir=req.inflow_dir,
                             nss=nss, nscheme=max(1, int(0.2 * req.steps)), nevery=1, nrepeat=100)
        case = g.Case(req.dm, req.mess, p, device=self.device)
        case.fill_freestream(req.ppc, 1_000_003 * req.seed + 17)
        case.statistic_macroPre()
        return case

    def launch(self, handles, n: int):
        """Enqueue n batched steps of these cases and return."""
        if n <= 0 or not handles:
            return
        members = tuple(id(h) for h in handles)
        if members != self._members:
            # membership changed: a new batch (its graphs are captured on
            # first use and then replayed while the membership holds)
            if self._batch is not None:
                self._batch.close()
            self._batch = self.gpu.Batch(handles)
            self._members = members
        self._batch.step(n)

    def wait(self):
        """Wait for the last launched round."""
        if self._batch is not None:
            self._batch.sync()

    def step(self, handles, n: int):
        self.launch(handles, n)
        self.wait()

    def particles(self, handle) -> int:
        return handle.particle_count()

    def handoff(self, handle):
        # the sampled fields the host GSIS step receives
        return handle.macro(self.gpu.MACRO_LOCAL)

    def finish(self, handle):
        g = self.gpu
        out = (handle.macro(g.MACRO_FINAL_RECORD), handle.macro(g.MACRO_LOCAL), handle.counters())
        if self._batch is not None and id(handle) in self._members:
            # the batch refers to the case: release it first
            self._batch.close()
            self._batch = None
            self._members = ()
        handle.close()
        return out

    def close(self):
        if self._batch is not None:
            self._batch.close()
            self._batch = None
            self._members = ()


class Server:
    """Continuous-batching request loop (see the module docstring)."""

    def __init__(self, backend, hbm_budget: float = 160e9, max_active: int = 64, handoff_every: int = 100,
                 clock=time.perf_counter, max_round_steps: int | None = None):
        self.backend = backend
        self.budget = int(hbm_budget)
        self.max_active = max_active
        self.handoff_every = handoff_every
        self.max_round_steps = max_round_steps
        self.clock = clock
        self.joined_running = 0     # admissions while other cases were on the GPU
        self._queue = []            # (t_arrival, rid, request)
        self._ids = itertools.count()
        self.active: list[_Active] = []
        self.results: dict[int, CaseResult] = {}
        self.used = 0
        self.rounds = 0
        self.max_concurrent = 0
        self.admit_order: list[int] = []
        self._joining: list[_Active] = []

    def submit(self, req: CaseRequest, t_arrival: float | None = None) -> int:
        rid = next(self._ids)
        t = self.clock() if t_arrival is None else t_arrival
        fp = self.backend.footprint(req)
        if fp > self.budget:
            raise ValueError(f"case needs {fp} bytes, more than the whole budget {self.budget}")
        heapq.heappush(self._queue, (t, rid, req))
        return rid

    def _admit(self, now: float, into: list | None = None):
        # arrival order; a case that does not fit blocks the ones behind it
        into = self.active if into is None else into
        while self._queue and self._queue[0][0] <= now and len(self.active) + len(self._joining) < self.max_active:
            t, rid, req = self._queue[0]
            fp = self.backend.footprint(req)
            if self.used + fp > self.budget:
                break
            heapq.heappop(self._queue)
            if self.active:
                self.joined_running += 1
            handle = self.backend.create(req)
            self.used += fp
            into.append(_Active(rid, req, handle, t, self.clock(), fp))
            self.admit_order.append(rid)
        self.max_concurrent = max(self.max_concurrent, len(self.active) + len(self._joining))

    def _round_steps(self) -> int:
        n = None
        for a in self.active:
            to_end = a.req.steps - a.step
            to_handoff = self.handoff_every - (a.step % self.handoff_every)
            m = min(to_end, to_handoff)
            n = m if n is None else min(n, m)
        if n and self.max_round_steps:
            n = min(n, self.max_round_steps)
        return n or 0

    def run(self, sleep=time.sleep):
        """Serve until every submitted request has finished."""
        overlap = hasattr(self.backend, "launch") and hasattr(self.backend, "wait")
        self._joining = []
        while self._queue or self.active:
            now = self.clock()
            self._admit(now)
            if not self.active:
                sleep(max(0.0, self._queue[0][0] - now))
                continue
            n = self._round_steps()
            counts = [self.backend.particles(a.handle) for a in self.active]
            if overlap:
                self.backend.launch([a.handle for a in self.active], n)
                # requests that arrived meanwhile are set up while the round runs
                self._admit(self.clock(), into=self._joining)
                self.backend.wait()
            else:
                self.backend.step([a.handle for a in self.active], n)
            self.rounds += 1
            still = []
            for a, c in zip(self.active, counts):
                a.step += n
                a.particle_steps += float(c) * n
                if a.step % self.handoff_every == 0 and a.step < a.req.steps:
                    self.backend.handoff(a.handle)
                    a.handoffs += 1
                if a.step >= a.req.steps:
                    final, local, counters = self.backend.finish(a.handle)
                    self.used -= a.footprint
                    self.results[a.rid] = CaseResult(a.req, a.t_arrival, a.t_admit, self.clock(), a.handoffs + 1,
                                                     final, local, a.particle_steps, counters)
                else:
                    still.append(a)
            self.active = still + self._joining
            self._joining = []
        return self.results

    def summary(self) -> dict:
        r = list(self.results.values())
        ttr = np.array([x.time_to_result for x in r]) if r else np.zeros(0)
        span = (max(x.t_done for x in r) - min(x.t_arrival for x in r)) if r else 0.0
        ps = float(sum(x.particle_steps for x in r))
        return {"cases": len(r), "p50_s": float(np.percentile(ttr, 50)) if r else None,
                "p99_s": float(np.percentile(ttr, 99)) if r else None,
                "cases_per_hour": len(r) / span * 3600.0 if span > 0 else None,
                "particle_steps_per_s": ps / span if span > 0 else None, "span_s": span,
                "rounds": self.rounds, "max_concurrent": self.max_concurrent,
                "joined_while_running": self.joined_running}
