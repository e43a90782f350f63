"""The continuous-batching request loop (dig-appolo_b200/pydsmc/serve.py).

CPU, with a backend that only counts: requests are admitted in arrival
order while their footprint fits the budget and a slot is free; a request
that arrives while others run joins them as soon as memory frees up; every
round stops at the next hand-off (every 100 of a case's own steps) or end
of some case; every case runs exactly its steps with its hand-offs.

GPU: cases served together give the same fields and particle inventory as
the same cases run alone with plain steps (a batched step equals the same
step taken alone).
"""
import numpy as np
import pytest

import inputs as I
from pydsmc import serve


class CountingBackend:
    def __init__(self, sizes):
        self.sizes = sizes
        self.log = []          # (round, sorted active names, n)
        self.rounds = 0

    def footprint(self, req):
        return self.sizes[req.name]

    def create(self, req):
        return {"name": req.name, "step": 0, "handoffs": []}

    def step(self, handles, n):
        self.rounds += 1
        self.log.append((sorted(h["name"] for h in handles), n))
        for h in handles:
            h["step"] += n

    def particles(self, h):
        return 1000

    def handoff(self, h):
        h["handoffs"].append(h["step"])

    def finish(self, h):
        return np.full((1, 18), float(h["step"])), np.zeros((1, 18)), {"steps": h["step"], "handoffs": list(h["handoffs"])}


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


def _req(name, steps):
    return serve.CaseRequest(dm=None, mess=None, zones=[], inflow_dir=(1.0, 0.0), steps=steps, ppc=10, name=name)


def test_admission_by_footprint_and_rounds_at_handoffs():
    sizes = {"a": 60, "b": 50, "c": 30, "d": 80}
    be = CountingBackend(sizes)
    clk = FakeClock()
    srv = serve.Server(be, hbm_budget=100, max_active=8, handoff_every=100, clock=clk)
    srv.submit(_req("a", 250), 0.0)
    srv.submit(_req("b", 120), 0.0)       # does not fit beside a (60 + 50 > 100): waits
    srv.submit(_req("c", 310), 0.0)       # behind b in arrival order: waits too
    srv.submit(_req("d", 90), 5.0)        # arrives later
    res = srv.run(sleep=clk.sleep)
    assert sorted(res) == [0, 1, 2, 3]
    assert srv.admit_order == [0, 1, 2, 3]
    for rid, name, steps in ((0, "a", 250), (1, "b", 120), (2, "c", 310), (3, "d", 90)):
        r = res[rid]
        assert r.counters["steps"] == steps
        assert r.counters["handoffs"] == [s for s in range(100, steps, 100)]
    # memory: never more than the budget at once
    for names, n in be.log:
        assert sum(sizes[x] for x in names) <= 100
        assert n >= 1
    # b joined while a was still running (continuous batching)
    first_b = next(i for i, (names, _) in enumerate(be.log) if "b" in names)
    assert "a" in be.log[first_b][0] or first_b > 0
    assert srv.used == 0 and not srv.active


def test_rejects_a_case_larger_than_the_budget():
    be = CountingBackend({"x": 500})
    srv = serve.Server(be, hbm_budget=100, clock=FakeClock())
    with pytest.raises(ValueError):
        srv.submit(_req("x", 10), 0.0)


def test_slots_limit_concurrency():
    sizes = {f"c{k}": 1 for k in range(6)}
    be = CountingBackend(sizes)
    clk = FakeClock()
    srv = serve.Server(be, hbm_budget=100, max_active=2, clock=clk)
    for k in range(6):
        srv.submit(_req(f"c{k}", 50 + 10 * k), 0.0)
    srv.run(sleep=clk.sleep)
    assert max(len(names) for names, _ in be.log) == 2
    assert srv.max_concurrent == 2


@pytest.mark.gpu
def test_served_cases_equal_cases_run_alone():
    from pydsmc import case as CS
    from pydsmc import gpu
    raw4, dm4 = I.block_mesh(scale=4)
    raw8, dm8 = I.block_mesh(scale=8)
    zones = I.REF_ZONES + [(7, gpu.ROLE_SPECULAR, 0)]
    reqs = []
    for k, (dm, ma, kn, ppc, steps) in enumerate([(dm4, 5.0, 0.1, 20, 230), (dm8, 7.0, 0.05, 30, 140),
                                                   (dm4, 4.0, 0.3, 15, 100), (dm8, 9.0, 0.02, 25, 260)]):
        mess = CS.mesh_message(dm, ma, kn, ppc=ppc, L0=I.BLOCK_L0)
        reqs.append(serve.CaseRequest(dm=dm, mess=mess, zones=zones, inflow_dir=I.inflow_dir(), steps=steps,
                                      ppc=float(ppc), seed=100 + k, precision=gpu.PRECISION_MIXED, name=f"r{k}"))
    be = serve.GpuBackend()
    # alone: each case by itself, plain per-case steps
    alone = []
    for r in reqs:
        h = be.create(r)
        for s in range(1, r.steps + 1):
            h.step(s)
        alone.append(be.finish(h))
    # served: staggered arrivals, two slots, so cases join and leave the batch
    t0 = 0.0
    srv = serve.Server(be, max_active=2)
    ids = [srv.submit(r, t0) for r in reqs]
    res = srv.run()
    be.close()
    for rid, (final, local, counters) in zip(ids, alone):
        got = res[rid]
        assert np.array_equal(got.final_record, final, equal_nan=True)
        assert np.array_equal(got.local, local, equal_nan=True)
        for k in ("injected", "removed", "collisions", "crossings"):
            assert got.counters[k] == counters[k], k
    s = srv.summary()
    assert s["cases"] == 4 and s["max_concurrent"] == 2 and s["p99_s"] >= s["p50_s"] > 0


@pytest.mark.gpu
def test_cases_arriving_while_others_run_equal_cases_run_alone():
    """Requests that arrive while another case is on the GPU: the server
    admits them during the running round (their device fill overlaps it)
    and they join the next round; every result equals the same case run
    alone. Time is counted in rounds, so the arrivals fall in mid-run."""
    from pydsmc import case as CS
    from pydsmc import gpu
    raw4, dm4 = I.block_mesh(scale=4)
    raw8, dm8 = I.block_mesh(scale=8)
    zones = I.REF_ZONES + [(7, gpu.ROLE_SPECULAR, 0)]
    specs = [(dm4, 5.0, 0.1, 20, 160, 0.0), (dm8, 7.0, 0.05, 30, 90, 2.5), (dm4, 4.0, 0.3, 15, 70, 5.5)]
    reqs = []
    for k, (dm, ma, kn, ppc, steps, _) in enumerate(specs):
        mess = CS.mesh_message(dm, ma, kn, ppc=ppc, L0=I.BLOCK_L0)
        reqs.append(serve.CaseRequest(dm=dm, mess=mess, zones=zones, inflow_dir=I.inflow_dir(), steps=steps,
                                      ppc=float(ppc), seed=200 + k, precision=gpu.PRECISION_MIXED, name=f"a{k}"))
    class Backend(serve.GpuBackend):
        in_round = False

        def launch(self, handles, n):
            super().launch(handles, n)
            self.in_round = True

        def wait(self):
            super().wait()
            self.in_round = False

    be = Backend()
    alone = []
    for r in reqs:
        h = be.create(r)
        for s in range(1, r.steps + 1):
            h.step(s)
        alone.append(be.finish(h))

    class RoundClock:
        """Rounds done, plus one half while a round is on the GPU."""
        srv = None
        slept = 0.0

        def __call__(self):
            return (self.srv.rounds if self.srv else 0) + (0.5 if be.in_round else 0.0) + self.slept

        def sleep(self, dt):
            self.slept += dt

    clk = RoundClock()
    srv = serve.Server(be, max_active=4, max_round_steps=10, clock=clk)
    clk.srv = srv
    ids = [srv.submit(r, t) for r, (*_, t) in zip(reqs, specs)]
    res = srv.run(sleep=clk.sleep)
    be.close()
    for rid, (final, local, counters) in zip(ids, alone):
        got = res[rid]
        assert np.array_equal(got.final_record, final, equal_nan=True)
        assert np.array_equal(got.local, local, equal_nan=True)
        for k in ("injected", "removed", "collisions", "crossings"):
            assert got.counters[k] == counters[k], k
    # the later requests were admitted while a round of the first one ran
    assert srv.joined_running == 2
    for k in (1, 2):
        assert res[ids[k]].t_admit % 1.0 == 0.5 and res[ids[k]].t_admit < res[ids[0]].t_done
    assert srv.max_concurrent == 3
