"""Forecast serving on one GPU: continuous batching of storm-surge requests.

    python -m gschism_b200.serve --requests 16 --rate 2 --hours 48 [--seed 1] [--budget-gb 150]

Requests (a mesh with its forcing and a horizon in steps) arrive over time.  The server keeps a
FIFO queue and, at every scheduling turn, admits the longest prefix of the queue whose device
memory (`footprint_bytes`, an upper bound of what the context allocates) fits in the memory left
by the running work: the admitted requests become one cohort, a batch context holding them all
as members.  A new cohort's host preparation (connectivity, ordering, matrix layout: the bulk of
the set-up, no CUDA call) runs on worker threads while the running cohorts keep stepping; its
device half (allocation, upload, cold start: well under a second) runs on the stepping thread
between two turns, so building never competes with stepping on the device.  Every turn
advances each running cohort by a few steps; a cohort whose requests reach their horizon hands
back its results, releases its memory and leaves.  So requests that arrive while others run are
admitted as memory frees up and their steps interleave with the running ones, turn by turn.

Every turn a cohort advances about the same number of node-steps (a 2M-node forecast one step,
a 30k-node one dozens), so the GPU is shared among the running forecasts and short ones finish
early.  All cohorts step on one CUDA stream: the step's persistent kernels (elevation solve,
transport) wait on each other's blocks and are never run concurrently with another such kernel.
A member's results do not depend on the batch it runs in (per-member reductions in a fixed
order), so each forecast is the same alone and in the mix.

Reported: time-to-forecast per request (arrival to results on the host), its p50/p99, and the
node-level-steps/s of the whole run.

Slot serving (`SlotServer`, `--regions R`): for a service over a fixed set of region meshes, each
region has one context of member slots on its mesh, and a request joins its region's running
launch sequence at the next step boundary, with its own clock on the device
(gs_set_member_start); see the class.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import dataclasses
import json
import math
import sys
import time
from typing import Any, Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np


@dataclasses.dataclass
class Request:
    rid: int
    case: Any                      # cases.Case
    nsteps: int
    vortex: Optional[dict] = None
    arrival: float = 0.0           # seconds after the start of the run
    # filled in by the server
    admitted: float = math.nan
    started: float = math.nan      # its cohort began stepping
    finished: float = math.nan     # results on the host
    cohort: int = -1
    result: Optional[np.ndarray] = None
    region: int = -1               # slot serving: the index of the request's mesh among the regions
    slot: int = -1                 # slot serving: the member slot it ran in

    @property
    def time_to_forecast(self) -> float:
        return self.finished - self.arrival

    def node_level_steps(self) -> int:
        return int(self.case.n_nodes) * int(self.case.vgrid.nvrt) * int(self.nsteps)


class ModelEngine:
    """GPU engine: one batch context (`Model`) per cohort, all stepping on one shared stream."""

    def __init__(self, precision: str = "fp32_ir", device: int = 0, fields: Sequence[str] = ("ETA2",)):
        import torch
        from .model import footprint_bytes
        self.torch = torch
        self.precision, self.device, self.fields = precision, device, tuple(fields)
        torch.cuda.set_device(device)
        self.stream = torch.cuda.Stream(device)
        self._footprint = footprint_bytes

    def footprint(self, cases) -> int:
        return self._footprint(cases)

    def free_bytes(self) -> int:
        return int(self.torch.cuda.mem_get_info(self.device)[0])

    def build(self, reqs: Sequence[Request]):
        """Host preparation only (worker thread): no CUDA call, so it never competes with the
        running steps for the device."""
        from .model import Model
        return Model([r.case for r in reqs], precision=self.precision, device=self.device, defer_device=True)

    def activate(self, h, reqs: Sequence[Request]) -> None:
        """Device half on the stepping thread, between turns: allocation, upload, cold start,
        storm forcing, and the shared stream."""
        self.torch.cuda.set_device(self.device)
        h.finalize()
        for i, r in enumerate(reqs):
            if r.vortex is not None:
                h.set_vortex(i, r.vortex)
        h.sync()
        h.set_stream(self.stream.cuda_stream)

    def advance(self, h, k: int) -> None:
        h.step(k)

    def wait(self) -> None:
        self.stream.synchronize()

    def results(self, h, n: int) -> List[Dict[str, np.ndarray]]:
        h.sync()
        return [{f: h.get(i, f).copy() for f in self.fields} for i in range(n)]

    def close(self, h) -> None:
        h.close()


@dataclasses.dataclass
class _Cohort:
    cid: int
    reqs: List[Request]
    nbytes: int
    target: int
    future: Any = None
    handle: Any = None
    done: int = 0


class Server:
    """Continuous-batching scheduler over an engine (see the module docstring)."""

    def __init__(self, engine, budget_bytes: Optional[int] = None, max_members: int = 64,
                 steps_per_turn: int = 8, turn_node_steps: Optional[int] = 2_000_000, build_workers: int = 2,
                 max_cohort_nodes: int = 1_000_000,
                 background_build: bool = True,
                 clock: Callable[[], float] = time.perf_counter, sleep: Callable[[float], None] = time.sleep,
                 on_finish: Optional[Callable[[Request], None]] = None):
        self.engine = engine
        self.budget = int(budget_bytes if budget_bytes is not None else 0.9 * engine.free_bytes())
        self.max_members = max_members
        self.steps_per_turn = max(1, steps_per_turn)
        self.turn_node_steps = turn_node_steps
        self.max_cohort_nodes = max_cohort_nodes
        self.clock, self.sleep = clock, sleep
        self.pool = cf.ThreadPoolExecutor(max_workers=max(1, build_workers)) if background_build else None
        self._t0 = 0.0
        self.used = 0
        self.peak_used = 0
        self.log: List[tuple] = []
        self.on_finish = on_finish

    def _admit(self, queue: List[Request], now: float, cid: int) -> Optional[_Cohort]:
        """Longest FIFO prefix of same-horizon requests that fits in the free budget and in
        max_cohort_nodes (a request above it gets a cohort of its own, so small forecasts neither
        wait for its set-up nor step at its pace)."""
        if not queue:
            return None
        group: List[Request] = []
        nbytes = 0
        nodes = 0
        for r in queue:
            if group and nodes + int(r.case.n_nodes) > self.max_cohort_nodes:
                break
            if group and (r.nsteps != group[0].nsteps or r.case.vgrid.nvrt != group[0].case.vgrid.nvrt
                          or r.case.ntracers != group[0].case.ntracers or r.case.params.dt != group[0].case.params.dt):
                break
            if len(group) >= self.max_members:
                break
            nb = self.engine.footprint([q.case for q in group + [r]])
            if self.used + nb > self.budget:
                break
            group.append(r)
            nbytes = nb
            nodes += int(r.case.n_nodes)
        if not group:
            if self.used == 0:
                raise RuntimeError(f"request {queue[0].rid} needs more device memory than the budget")
            return None
        del queue[:len(group)]
        for r in group:
            r.admitted = now
            r.cohort = cid
        self.used += nbytes
        self.peak_used = max(self.peak_used, self.used)
        c = _Cohort(cid=cid, reqs=group, nbytes=nbytes, target=group[0].nsteps)
        if self.pool is not None:
            c.future = self.pool.submit(self._build, cid, group)
        else:
            c.handle = self._build(cid, group)
        self.log.append(("admit", now, cid, [r.rid for r in group], nbytes))
        return c

    def _turn_steps(self, c: _Cohort) -> int:
        """Steps a cohort advances in one turn: about turn_node_steps node-steps (a large cohort
        one step, a small one many), so every running forecast gets a similar share of the GPU per
        turn and short ones finish early; steps_per_turn when no share is set."""
        if not self.turn_node_steps:
            return self.steps_per_turn
        nodes = sum(int(r.case.n_nodes) for r in c.reqs)
        return max(1, int(self.turn_node_steps // max(1, nodes)))

    def _build(self, cid: int, group: Sequence[Request]):
        t = self.clock()
        h = self.engine.build(group)
        self.log.append(("build", cid, t - self._t0, self.clock() - t))
        return h

    def run(self, requests: Sequence[Request]) -> List[Request]:
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        queue: List[Request] = []
        building: List[_Cohort] = []
        active: List[_Cohort] = []
        t0 = self._t0 = self.clock()
        cid = 0
        try:
            while pending or queue or building or active:
                now = self.clock() - t0
                while pending and pending[0].arrival <= now:
                    queue.append(pending.pop(0))
                while True:
                    c = self._admit(queue, now, cid)
                    if c is None:
                        break
                    cid += 1
                    building.append(c)
                # cohorts whose build finished join the stepping
                for c in list(building):
                    if c.future is not None:
                        if not c.future.done():
                            continue
                        c.handle = c.future.result()
                    ta = self.clock()
                    if hasattr(self.engine, "activate"):
                        self.engine.activate(c.handle, c.reqs)
                    self.log.append(("activate", c.cid, ta - t0, self.clock() - ta))
                    building.remove(c)
                    active.append(c)
                    t = self.clock() - t0
                    for r in c.reqs:
                        r.started = t
                if not active:
                    # nothing to step: wait for a build or the next arrival
                    waits = []
                    if pending and not building:
                        waits.append(pending[0].arrival - now)
                    self.sleep(max(0.0, min(waits)) if waits else 0.002)
                    continue
                tt = self.clock()
                for c in active:
                    k = min(self._turn_steps(c), c.target - c.done)
                    self.engine.advance(c.handle, k)
                    c.done += k
                self.engine.wait()
                self.log.append(("turn", tt - t0, self.clock() - tt, len(active)))
                for c in list(active):
                    if c.done < c.target:
                        continue
                    res = self.engine.results(c.handle, len(c.reqs))
                    t = self.clock() - t0
                    for r, x in zip(c.reqs, res):
                        r.result = x
                        r.finished = t
                        if self.on_finish is not None:
                            self.on_finish(r)
                    self.engine.close(c.handle)
                    active.remove(c)
                    self.used -= c.nbytes
                    self.log.append(("finish", t, c.cid))
        finally:
            if self.pool is not None:
                self.pool.shutdown(wait=True)
        return list(requests)


class SlotEngine:
    """GPU engine for slot serving: one batch context per region, its members the region's slots
    on the region's mesh; each slot keeps its cold-start state in page-locked memory, so an
    admission puts it back with one direct copy per field.  All contexts step on one stream."""

    def __init__(self, precision: str = "fp32_ir", device: int = 0, fields: Sequence[str] = ("ETA2",),
                 jcg_tiles: Optional[Tuple[int, int]] = None):
        import torch
        self.torch = torch
        self.precision, self.device, self.fields = precision, device, tuple(fields)
        self.jcg_tiles = jcg_tiles            # (tiles of a large member, smallest tile), or the default
        torch.cuda.set_device(device)
        self.stream = torch.cuda.Stream(device)
        self.cold: Dict[int, List[Dict[str, np.ndarray]]] = {}

    def build(self, slot_cases):
        from .model import Model
        h = Model(list(slot_cases), precision=self.precision, device=self.device)
        if self.jcg_tiles is not None:
            h.set_launch("JCG_TILES", *self.jcg_tiles)
        cold = [h.member_state(i, pinned=True) for i in range(len(slot_cases))]
        for i in range(len(slot_cases)):
            h.park(i, cold[i])
        h.sync()
        h.set_stream(self.stream.cuda_stream)
        self.cold[id(h)] = cold
        return h

    def admit(self, h, slot: int, r: Request) -> None:
        h.admit(slot, self.cold[id(h)][slot], vortex=r.vortex)

    def advance(self, h, k: int) -> None:
        h.step(k)

    def wait(self) -> None:
        self.stream.synchronize()

    def check(self, h) -> None:
        """Raise if a bounded device wait ran out during the turn (gs_sync)."""
        h.sync()

    def result(self, h, slot: int) -> Dict[str, np.ndarray]:
        return {f: h.get(slot, f).copy() for f in self.fields}

    def park(self, h, slot: int) -> None:
        h.park(slot, self.cold[id(h)][slot])

    def close(self, h) -> None:
        self.cold.pop(id(h), None)
        h.close()


@dataclasses.dataclass
class _Region:
    g: int                          # region index
    nodes: int                      # nodes of one slot
    handle: Any = None              # its context
    free: List[int] = dataclasses.field(default_factory=list)
    running: Dict[int, list] = dataclasses.field(default_factory=dict)   # slot -> [request, steps left]


class SlotServer:
    """Slot-level continuous batching.  Every region a forecast service covers (one mesh each)
    gets one context of `slots_per_region` member slots on its mesh, built once; a request names
    its region, its forcing and its horizon.  At every step boundary the server admits queued
    requests, in arrival order, into free slots of their region (a request whose region is full
    waits; requests behind it for other regions go ahead): the slot's cold-start state is put back
    and its clock starts, so the forecast joins the running launch sequence of its region and
    steps alongside the forecasts already there, exactly as it would alone.  Each turn advances
    every region that has forecasts running by about `turn_node_steps` node-steps (a small
    region's context many steps, a large one's few; at most `steps_per_turn`, and never past the
    next horizon); regions with nothing running are not stepped.  A finished forecast hands back
    its results and its slot is parked (at rest, no forcing) until the next admission."""

    def __init__(self, engine, regions: Sequence[Any], slots_per_region: Sequence[int] | int = 2,
                 steps_per_turn: int = 32, turn_node_steps: Optional[int] = 4_000_000,
                 clock: Callable[[], float] = time.perf_counter,
                 sleep: Callable[[float], None] = time.sleep, on_finish: Optional[Callable[[Request], None]] = None):
        self.engine, self.regions = engine, list(regions)
        if isinstance(slots_per_region, int):
            slots_per_region = [slots_per_region] * len(self.regions)
        self.nslots = [int(n) for n in slots_per_region]
        if not any(self.nslots):
            raise ValueError("no slots")
        self.steps_per_turn, self.turn_node_steps = int(steps_per_turn), turn_node_steps
        self.clock, self.sleep, self.on_finish = clock, sleep, on_finish
        self.log: List[tuple] = []
        self.setup_s = math.nan

    def _turn_steps(self, reg: _Region) -> int:
        k = self.steps_per_turn
        if self.turn_node_steps:
            ctx_nodes = reg.nodes * len(reg.free) + reg.nodes * len(reg.running)
            k = max(1, min(k, int(self.turn_node_steps // max(1, ctx_nodes))))
        return min(k, min(left for _, left in reg.running.values()))

    def run(self, requests: Sequence[Request]) -> List[Request]:
        for r in requests:
            if not (0 <= r.region < len(self.regions)) or self.nslots[r.region] < 1:
                raise ValueError(f"request {r.rid}: no slot for region {r.region}")
        pending = sorted(requests, key=lambda r: (r.arrival, r.rid))
        queue: List[Request] = []
        ts = self.clock()
        regs: List[_Region] = []
        for g, n in enumerate(self.nslots):
            if n < 1:
                continue
            reg = _Region(g=g, nodes=int(self.regions[g].n_nodes), free=list(range(n)))
            reg.handle = self.engine.build([self.regions[g]] * n)
            regs.append(reg)
        by_g = {reg.g: reg for reg in regs}
        self.setup_s = self.clock() - ts
        t0 = self.clock()
        try:
            while pending or queue or any(reg.running for reg in regs):
                now = self.clock() - t0
                while pending and pending[0].arrival <= now:
                    queue.append(pending.pop(0))
                for r in list(queue):
                    reg = by_g[r.region]
                    if reg.free:
                        slot = reg.free.pop(0)
                        self.engine.admit(reg.handle, slot, r)
                        r.slot, r.cohort = slot, r.region
                        r.admitted = r.started = self.clock() - t0
                        reg.running[slot] = [r, int(r.nsteps)]
                        queue.remove(r)
                        self.log.append(("admit", r.admitted, r.rid, r.region, slot))
                active = [reg for reg in regs if reg.running]
                if not active:
                    self.sleep(max(0.0, pending[0].arrival - now) if pending else 0.002)
                    continue
                tt = self.clock()
                ks = []
                for reg in active:
                    k = self._turn_steps(reg)
                    self.engine.advance(reg.handle, k)
                    ks.append((reg, k))
                self.engine.wait()
                for reg, _ in ks:
                    if hasattr(self.engine, "check"):
                        self.engine.check(reg.handle)
                self.log.append(("turn", tt - t0, self.clock() - tt, [(reg.g, k) for reg, k in ks]))
                for reg, k in ks:
                    for slot in sorted(reg.running):
                        reg.running[slot][1] -= k
                    for slot in [sl for sl in sorted(reg.running) if reg.running[sl][1] == 0]:
                        r = reg.running.pop(slot)[0]
                        r.result = self.engine.result(reg.handle, slot)
                        r.finished = self.clock() - t0
                        self.engine.park(reg.handle, slot)
                        reg.free.append(slot)
                        self.log.append(("finish", r.finished, r.rid, r.region, slot))
                        if self.on_finish is not None:
                            self.on_finish(r)
        finally:
            for reg in regs:
                self.engine.close(reg.handle)
        return list(requests)


def slot_requests(n: int, rate: float, seed: int, regions: Sequence[Any], hours: float = 48.0,
                  dt: float = 150.0, horizons: Optional[Sequence[float]] = None) -> List[Request]:
    """n storm-surge requests over the regions' meshes: Poisson arrivals (mean gap 1/rate), a
    uniformly drawn region, a seeded storm on its mesh (cases.storm_on) and a horizon of `hours`,
    or one drawn uniformly from `horizons` (hours) when given."""
    from . import cases
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        if i > 0:
            t += rng.exponential(1.0 / rate)
        g = int(rng.integers(0, len(regions)))
        v = cases.storm_on(regions[g], int(rng.integers(1, 2**31 - 1)))
        h = hours if not horizons else float(horizons[int(rng.integers(0, len(horizons)))])
        out.append(Request(rid=i, case=regions[g], nsteps=int(round(h * 3600.0 / dt)), vortex=v, arrival=t,
                           region=g))
    return out


def region_meshes(nregions: int, nmin: int, nmax: int, seed: int, nvrt: int = 20, dt: float = 150.0) -> List[Any]:
    """The regions' storm meshes, node counts log-spaced over [nmin, nmax]."""
    from . import cases
    out = []
    for g in range(nregions):
        target = nmin * (nmax / nmin) ** (g / max(1, nregions - 1))
        c, _, _ = cases.storm(seed * 1000 + g, nmin=int(target), nmax=int(target) + 1, nvrt=nvrt, dt=dt)
        out.append(c)
    return out


def summary(reqs: Sequence[Request], makespan: float) -> dict:
    ttf = np.array([r.time_to_forecast for r in reqs])
    nls = sum(r.node_level_steps() for r in reqs)
    return {
        "requests": len(reqs),
        "ttf_p50_s": float(np.percentile(ttf, 50)),
        "ttf_p99_s": float(np.percentile(ttf, 99)),
        "ttf_max_s": float(ttf.max()),
        "makespan_s": makespan,
        "node_level_steps_per_s": nls / makespan if makespan > 0 else math.nan,
        "cohorts": len({r.cohort for r in reqs}),
    }


def poisson_requests(n: int, rate: float, seed: int, hours: float = 48.0, nmin: int = 10_000,
                     nmax: int = 2_000_000, nvrt: int = 20, dt: float = 150.0) -> List[Request]:
    """n storm-surge requests (cases.storm) with exponential inter-arrival times of mean 1/rate."""
    from . import cases
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        if i > 0:
            t += rng.exponential(1.0 / rate)
        c, v, nsteps = cases.storm(int(rng.integers(1, 2**31 - 1)), nmin=nmin, nmax=nmax, nvrt=nvrt, dt=dt,
                                   hours=hours)
        out.append(Request(rid=i, case=c, nsteps=nsteps, vortex=v, arrival=t))
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--requests", type=int, default=16)
    ap.add_argument("--rate", type=float, default=2.0, help="mean arrivals per second (Poisson)")
    ap.add_argument("--hours", type=float, default=48.0, help="forecast horizon")
    ap.add_argument("--nmin", type=int, default=10_000)
    ap.add_argument("--nmax", type=int, default=2_000_000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--budget-gb", type=float, default=None)
    ap.add_argument("--steps-per-turn", type=int, default=8)
    ap.add_argument("--precision", choices=["fp64", "fp32_ir"], default="fp32_ir")
    ap.add_argument("--regions", type=int, default=0,
                    help="slot serving over this many region meshes (node counts log-spaced over "
                         "[nmin, nmax]); 0 = one mesh per request, served in cohorts")
    ap.add_argument("--slots-per-region", type=int, default=2)
    ap.add_argument("--region-cohorts", action="store_true",
                    help="with --regions: serve the same requests in cohorts instead of slots (comparison)")
    ap.add_argument("--horizons", type=str, default="",
                    help="slot serving: comma-separated horizons in hours drawn per request (mixed horizons)")
    a = ap.parse_args(argv)
    if a.regions > 0:
        return _main_slots(a)
    reqs = poisson_requests(a.requests, a.rate, a.seed, hours=a.hours, nmin=a.nmin, nmax=a.nmax)
    eng = ModelEngine(precision=a.precision)

    def progress(r: Request) -> None:
        # one line per finished forecast, so a run cut short still reports what it did
        print(json.dumps({"rid": r.rid, "nodes": int(r.case.n_nodes), "arrival_s": round(r.arrival, 3),
                          "started_s": round(r.started, 3), "ttf_s": round(r.time_to_forecast, 3)}),
              file=sys.stderr, flush=True)

    srv = Server(eng, budget_bytes=None if a.budget_gb is None else int(a.budget_gb * 1e9),
                 steps_per_turn=a.steps_per_turn, on_finish=progress)
    t0 = time.perf_counter()
    srv.run(reqs)
    out = summary(reqs, time.perf_counter() - t0)
    out.update({"horizon_hours": a.hours, "rate_per_s": a.rate, "nodes": [int(r.case.n_nodes) for r in reqs],
                "ttf_s": [round(r.time_to_forecast, 3) for r in reqs], "peak_budget_gb": srv.peak_used / 1e9})
    print(json.dumps(out))
    return 0


def _main_slots(a) -> int:
    regions = region_meshes(a.regions, a.nmin, a.nmax, a.seed)
    horizons = [float(x) for x in a.horizons.split(",") if x.strip()]
    reqs = slot_requests(a.requests, a.rate, a.seed, regions, hours=a.hours, horizons=horizons or None)
    if a.region_cohorts:
        srv = Server(ModelEngine(precision=a.precision), steps_per_turn=a.steps_per_turn)
        t0 = time.perf_counter()
        srv.run(reqs)
        out = summary(reqs, time.perf_counter() - t0)
        out.update({"mode": "cohorts", "horizon_hours": horizons or a.hours, "rate_per_s": a.rate,
                    "nsteps": [r.nsteps for r in reqs], "region": [r.region for r in reqs],
                    "region_nodes": [int(c.n_nodes) for c in regions],
                    "ttf_s": [round(r.time_to_forecast, 3) for r in reqs]})
        print(json.dumps(out))
        return 0

    def progress(r: Request) -> None:
        print(json.dumps({"rid": r.rid, "region": r.region, "slot": r.slot, "nodes": int(r.case.n_nodes),
                          "arrival_s": round(r.arrival, 3), "admitted_s": round(r.admitted, 3),
                          "ttf_s": round(r.time_to_forecast, 3)}), file=sys.stderr, flush=True)

    srv = SlotServer(SlotEngine(precision=a.precision), regions, a.slots_per_region, on_finish=progress)
    t0 = time.perf_counter()
    srv.run(reqs)
    out = summary(reqs, time.perf_counter() - t0 - srv.setup_s)
    out.update({"mode": "slots", "horizon_hours": horizons or a.hours, "rate_per_s": a.rate,
                "nsteps": [r.nsteps for r in reqs], "region": [r.region for r in reqs],
                "region_nodes": [int(c.n_nodes) for c in regions], "slots_per_region": a.slots_per_region,
                "setup_s": round(srv.setup_s, 3), "ttf_s": [round(r.time_to_forecast, 3) for r in reqs],
                "wait_s": [round(r.admitted - r.arrival, 3) for r in reqs]})
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
