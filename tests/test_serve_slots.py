"""Slot serving on CPU: a fake engine with a virtual clock stands in for the GPU.

Checks the slot-level rules of gschism_b200/serve.py:SlotServer: a request is admitted at a step
boundary into a free slot of its own region, in arrival order, while other forecasts keep
running; every forecast runs exactly its horizon from its own step 1 and hands back its own
results; a finished slot is parked and taken by the next request of its region."""
import types

import numpy as np
import pytest

from gschism_b200.serve import Request, SlotServer, summary


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-4)


def _region(n):
    return types.SimpleNamespace(n_nodes=n, vgrid=types.SimpleNamespace(nvrt=20), ntracers=1,
                                 params=types.SimpleNamespace(dt=150.0))


class FakeSlotEngine:
    """One fake context per region: a context step costs 1 us per 1000 nodes of its slots (parked
    ones included); each slot counts its own steps since admission, the way the member clock
    does."""

    def __init__(self, clock):
        self.clock = clock
        self.ctx = {}
        self.closed = set()

    def build(self, slot_cases):
        h = len(self.ctx)
        self.ctx[h] = {"sizes": [c.n_nodes for c in slot_cases], "own": [None] * len(slot_cases),
                       "owner": [None] * len(slot_cases), "steps": 0}
        return h

    def admit(self, h, slot, r):
        c = self.ctx[h]
        assert c["own"][slot] is None, "admitted into a busy slot"
        c["own"][slot], c["owner"][slot] = 0, r.rid

    def advance(self, h, k):
        c = self.ctx[h]
        self.clock.t += 1e-6 * k * sum(c["sizes"]) / 1000.0
        c["steps"] += k
        for sl in range(len(c["own"])):
            if c["own"][sl] is not None:
                c["own"][sl] += k

    def wait(self):
        pass

    def result(self, h, slot):
        c = self.ctx[h]
        return {"rid": c["owner"][slot], "steps": c["own"][slot]}

    def park(self, h, slot):
        c = self.ctx[h]
        c["own"][slot], c["owner"][slot] = None, None

    def close(self, h):
        self.closed.add(h)


def _reqs(spec, regions=None):
    """spec: (arrival, region, nsteps) per request."""
    return [Request(rid=i, case=regions[g] if regions and g < len(regions) else None, nsteps=n, arrival=t, region=g)
            for i, (t, g, n) in enumerate(spec)]


def test_slots_run_every_forecast_its_horizon():
    clk = Clock()
    eng = FakeSlotEngine(clk)
    regions = [_region(50_000), _region(400_000)]
    srv = SlotServer(eng, regions, [2, 1], steps_per_turn=8, clock=clk, sleep=clk.sleep)
    reqs = _reqs([(0.0, 0, 30), (0.0, 1, 20), (0.001, 0, 13), (0.002, 0, 40), (0.003, 1, 5), (0.5, 0, 9)], regions)
    srv.run(reqs)
    for r in reqs:
        assert r.result == {"rid": r.rid, "steps": r.nsteps}      # its own slot, exactly its horizon
        assert r.arrival <= r.admitted <= r.finished
        assert r.cohort == r.region                              # a slot of its own region's context
    assert eng.closed == set(eng.ctx)
    # region 0 has two slots: the third region-0 request waits for one to free up
    first_free = min(r.finished for r in reqs[:3] if r.region == 0)
    assert reqs[3].admitted >= first_free - 1e-12
    # region 1's second request waits for its single slot
    assert reqs[4].admitted >= reqs[1].finished - 1e-12
    # a request of another region is not held up by a full region
    assert reqs[4].admitted <= reqs[3].admitted
    s = summary(reqs, max(r.finished for r in reqs))
    assert s["requests"] == 6 and s["ttf_p50_s"] > 0


def test_admission_happens_while_others_run():
    """A request arriving mid-run is admitted at the next step boundary, not after the running
    forecast ends."""
    clk = Clock()
    eng = FakeSlotEngine(clk)
    srv = SlotServer(eng, [_region(1_000_000)], 2, steps_per_turn=4, clock=clk, sleep=clk.sleep)
    reqs = _reqs([(0.0, 0, 400), (0.01, 0, 8)])
    srv.run(reqs)
    assert reqs[1].admitted < reqs[0].finished
    assert reqs[1].finished < reqs[0].finished
    # turns never step past a forecast's horizon, nor beyond steps_per_turn
    turns = [e for e in srv.log if e[0] == "turn"]
    ks = [k for *_, gk in turns for g, k in gk]
    assert all(1 <= k <= 4 for k in ks)
    assert sum(ks) == 400


def test_regions_step_separately_and_idle_regions_not_at_all():
    """A small region's context takes more steps per turn than a large one's (about the same
    node-steps), and a region with nothing running is not stepped."""
    clk = Clock()
    eng = FakeSlotEngine(clk)
    regions = [_region(20_000), _region(800_000), _region(50_000)]
    srv = SlotServer(eng, regions, 2, steps_per_turn=64, turn_node_steps=4_000_000, clock=clk, sleep=clk.sleep)
    reqs = _reqs([(0.0, 0, 200), (0.0, 1, 30)], regions)
    srv.run(reqs)
    turns = [e for e in srv.log if e[0] == "turn"]
    first = dict(turns[0][3])
    assert first[0] > first[1]                    # 64 steps of the small context, 2 of the large
    assert eng.ctx[2]["steps"] == 0               # region 2 had no request
    assert eng.ctx[0]["steps"] == 200 and eng.ctx[1]["steps"] == 30


def test_unknown_region_is_refused():
    clk = Clock()
    srv = SlotServer(FakeSlotEngine(clk), [_region(1000)], 1, clock=clk, sleep=clk.sleep)
    with pytest.raises(ValueError):
        srv.run(_reqs([(0.0, 3, 5)]))
