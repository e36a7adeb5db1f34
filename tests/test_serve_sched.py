"""Serving scheduler on CPU: a fake engine with a virtual clock stands in for the GPU.

Checks the continuous-batching rules of gschism_b200/serve.py: FIFO admission of the longest
prefix that fits the memory budget, requests that arrive while others run join as memory frees
up, the budget is never exceeded, every request gets its own results and a time-to-forecast."""
import types

import numpy as np
import pytest

from gschism_b200.serve import Request, Server, summary


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-4)


def _case(n):
    return types.SimpleNamespace(n_nodes=n, vgrid=types.SimpleNamespace(nvrt=20), ntracers=1,
                                 params=types.SimpleNamespace(dt=150.0))


class FakeEngine:
    """Footprint 100 bytes per node; a step costs 1 us per 1000 nodes of the cohort."""

    def __init__(self, clock):
        self.clock = clock
        self.live = {}
        self.max_live_bytes = 0
        self.next = 0
        self.steps = {}

    def footprint(self, cases):
        return 100 * sum(c.n_nodes for c in cases)

    def free_bytes(self):
        return 10**9

    def build(self, reqs):
        h = self.next
        self.next += 1
        self.live[h] = (list(reqs), self.footprint([r.case for r in reqs]))
        self.steps[h] = 0
        self.max_live_bytes = max(self.max_live_bytes, sum(b for _, b in self.live.values()))
        return h

    def advance(self, h, k):
        reqs, _ = self.live[h]
        self.clock.t += 1e-6 * k * sum(r.case.n_nodes for r in reqs) / 1000.0
        self.steps[h] += k

    def wait(self):
        pass

    def results(self, h, n):
        reqs, _ = self.live[h]
        assert self.steps[h] == reqs[0].nsteps
        return [{"ETA2": np.full(3, float(r.rid))} for r in reqs]

    def close(self, h):
        del self.live[h]


def _run(reqs, budget, steps_per_turn=4):
    clk = Clock()
    eng = FakeEngine(clk)
    srv = Server(eng, budget_bytes=budget, steps_per_turn=steps_per_turn, background_build=False,
                 clock=clk, sleep=clk.sleep)
    srv.run(reqs)
    return srv, eng, clk


def test_every_request_served_with_its_own_result_and_budget_kept():
    sizes = [50_000, 200_000, 10_000, 400_000, 30_000, 120_000]
    reqs = [Request(rid=i, case=_case(n), nsteps=40, arrival=0.01 * i) for i, n in enumerate(sizes)]
    budget = 100 * 500_000                      # at most 500k nodes resident
    srv, eng, clk = _run(reqs, budget)
    assert eng.max_live_bytes <= budget
    assert srv.peak_used <= budget
    for r in reqs:
        assert r.result["ETA2"][0] == r.rid
        assert r.finished >= r.started >= r.admitted >= r.arrival
    s = summary(reqs, clk.t)
    assert s["requests"] == len(reqs) and s["ttf_p99_s"] >= s["ttf_p50_s"] > 0


def test_late_arrivals_join_while_earlier_cohorts_run():
    # a long request first, then short ones arriving while it runs: they are admitted as new
    # cohorts and finish before it
    reqs = [Request(rid=0, case=_case(100_000), nsteps=400, arrival=0.0)]
    reqs += [Request(rid=i, case=_case(10_000), nsteps=8, arrival=0.001 * i) for i in range(1, 4)]
    srv, eng, clk = _run(reqs, budget=10**9, steps_per_turn=4)
    assert len({r.cohort for r in reqs}) >= 2
    assert all(reqs[i].finished < reqs[0].finished for i in range(1, 4))
    admits = [e for e in srv.log if e[0] == "admit"]
    assert admits[0][3] == [0]


def test_fifo_prefix_and_memory_wait():
    # the budget holds one big request at a time: the second waits for the first to finish
    reqs = [Request(rid=i, case=_case(300_000), nsteps=16, arrival=0.0) for i in range(3)]
    srv, eng, clk = _run(reqs, budget=100 * 350_000)
    assert reqs[0].finished <= reqs[1].admitted <= reqs[1].finished <= reqs[2].admitted
    assert eng.max_live_bytes <= 100 * 350_000


def test_request_larger_than_budget_is_an_error():
    reqs = [Request(rid=0, case=_case(1_000_000), nsteps=4, arrival=0.0)]
    with pytest.raises(RuntimeError):
        _run(reqs, budget=1000)


def test_turn_share_by_node_steps():
    clk = Clock()
    srv = Server(FakeEngine(clk), budget_bytes=10**9, turn_node_steps=2_000_000, background_build=False,
                 clock=clk, sleep=clk.sleep)
    from gschism_b200.serve import _Cohort
    big = _Cohort(cid=0, reqs=[Request(rid=0, case=_case(2_000_000), nsteps=10)], nbytes=0, target=10)
    small = _Cohort(cid=1, reqs=[Request(rid=1, case=_case(25_000), nsteps=10)], nbytes=0, target=10)
    assert srv._turn_steps(big) == 1
    assert srv._turn_steps(small) == 80


def test_large_request_gets_its_own_cohort():
    reqs = [Request(rid=0, case=_case(2_000_000), nsteps=8, arrival=0.0)]
    reqs += [Request(rid=i, case=_case(20_000), nsteps=8, arrival=0.0) for i in range(1, 4)]
    srv, eng, clk = _run(reqs, budget=10**12)
    assert reqs[0].cohort != reqs[1].cohort
    assert reqs[1].cohort == reqs[2].cohort == reqs[3].cohort
    assert all(r.finished < reqs[0].finished for r in reqs[1:])
