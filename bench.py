"""Benchmark: SCHISM semi-implicit step on one B200, node-level-steps/s.

Workload (single large mesh, the configuration the metric is quoted on that fits one GPU):
1M-node jittered-lattice basin, 500 km x 500 km, 30 SZ levels (10 z + 21 sigma), Gaussian-
random-field bathymetry 2..4000 m, M2+S2 1.2 m on the west side, 2 tracers (T, S); dt = 120 s;
JCG rtol 1e-12.  Inputs are seeded synthetic data (no dataset involved).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--n 1000]

value    = node-level-steps/s of the timed steps (sum of nodes x levels x steps / device time),
           FP32-inner JCG with FP64 refinement ("fp32_ir"), state resident in HBM.
e2e      = the same steps (a fresh context from the same cold start, the same step indices)
           through the C ABI with page-locked host buffers: every step uploads the surface stress
           field from host memory (gs_set_tau), steps (gs_step) and reads the elevation back
           (gs_state_get).
roofline = the JCG persistent kernel (dominant), algorithmic bytes per launch / launch time.
The plain FP64 single-instance form is measured on the same GPU and reported under "fp64".
ensemble = the batched form: 64 members on meshes of uneven size (20k-500k nodes, 20 levels,
           1 tracer, per-member tide and wind), all members in one launch per phase, FP32+IR and
           FP64, against the plain FP64 single-instance form run member by member.
error_vs_oracle = the FP64 and FP32+IR forms after 3 steps of the benchmarked mesh against the
           CPU oracle (oracle/, pinned to the reference's own kernels by tests/test_ref_pinned.py)
           after the same 3 steps: elevation max |difference| in m, tracers and velocities relative.
serving = storm-surge forecast requests served in cohorts (p50/p99 time-to-forecast);
serving_slots = the same kind of requests over four region meshes, admitted into free member
           slots of one running context at step boundaries.
cpu_baseline = the oracle on the benchmarked mesh itself (all host threads), 2 timed steps.
--impl reference = the same oracle on the benchmarked mesh, 1 warm-up + up to 6 timed steps (a
           bounded sample of the run), plus a single-thread figure on a 200 x 200 sample.
Multi-GPU (torchrun): every rank steps its own replica of the mesh (no data exchange exists in
the step); value = all ranks' node-level-steps / the max over ranks of the device time.  The
64-member ensemble is then sharded over the ranks by device footprint (`ensemble_sharded`).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "node-level-steps/s"


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=1000, help="lattice side (n x n nodes)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline sample")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the 64-member ensemble comparison")
    ap.add_argument("--no-serve", action="store_true", help="skip the forecast-serving run")
    return ap.parse_args()


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region (raw samples in a temporary file, or in the
    file GS_CLOCK_LOG names)."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = os.environ.get("GS_CLOCK_LOG") or os.path.join(
            tempfile.gettempdir(), f"gschism_clocks_gpu{gpu}_{os.getpid()}.csv")

    def __enter__(self):
        d = os.path.dirname(self.path)
        if d:
            os.makedirs(d, exist_ok=True)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return out
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        if sm:
            out["sm_mhz"] = statistics.median(sm)
        if mx:
            out["sm_max_mhz"] = max(mx)
        out["reasons"] = sorted(reasons)
        out["samples"] = len(sm)
        return out


# DRAM bytes (reads + writes, dram__bytes.sum) per inner iteration of k_jcg_ir on the 1M-node
# basin, from one ncu capture of that kernel (the second step's solve of the same 1,000,000-row
# system with 6 levels: launch bytes / inner iterations of that launch); scaled here by the timed
# launches' inner iterations.
JCG_DRAM_BYTES_PER_INNER_ITER = 23.9e6


def _jcg_bytes_per_iter(N, nnz, mode):
    """Algorithmic bytes of one JCG iteration: matrix values + column indices + row pointers,
    and seven vector passes (read p, invD, x, r; write x, r, p), s_v = 8 (FP64) or 4 (FP32)."""
    sv = 8 if mode == "fp64" else 4
    return nnz * (sv + 4) + 4 * (N + 1) + 7 * N * sv


def run_ours(a):
    import torch
    from gschism_b200 import cases
    from gschism_b200.model import Model
    from gschism_b200.shard import max_over_ranks
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    case = cases.basin(seed=2 + 0, n=a.n, nvrt=30, nz=10, ntr=2)
    nodes, nvrt = case.n_nodes, case.nvrt
    res = {}
    modes = ["fp32_ir"] + ([] if a.no_fp64 else ["fp64"])
    stream = torch.cuda.Stream()
    peak, peak_kind = _peaks()
    for mode in modes:
        m = Model([case], precision=mode, device=local)
        m.set_stream(stream.cuda_stream)
        it = 0
        for _ in range(a.warmup):
            it += 1
            m.step(1)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        jev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
        iters = []
        phases = ["BTRACK", "PREPARE", "ASSEMBLE", "SOLVE", "UPDATE_ELEV", "MOMENTUM", "VVEL", "TRANSPORT",
                  "LEVELS", "NODAL_VEL"]
        with Clocks(local) as clk:
            ev[0].record(stream)
            for k in range(a.steps):
                it += 1
                m.phase("BEGIN", it)
                for ph in phases:
                    if ph == "SOLVE":
                        jev[k][0].record(stream)
                        m.phase(ph, it)
                        jev[k][1].record(stream)
                    else:
                        m.phase(ph, it)
            ev[1].record(stream)
            torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1])
        jms = [s.elapsed_time(e) for s, e in jev]
        st = m.stats(0)
        m.sync()
        ms_max = max_over_ranks(ms, dist, device="cuda")
        total = nodes * nvrt * a.steps * ws
        res[mode] = dict(value=total / (ms_max / 1e3), ms_per_step=ms_max / a.steps, jcg_ms=jms, stats=st,
                         clocks=clk.summary(), nnz=m.sizes[0]["nnz"])
        # per-step JCG iteration counts (device-side)
        res[mode]["jcg_iters_last"] = st["jcg_iters"]
        res[mode]["jcg_outer_last"] = st["jcg_outer"]
        if mode == "fp32_ir":
            # end-to-end through the C ABI with page-locked host buffers: upload tau, step, read
            # eta back; a fresh context from the same cold start, warmed up and timed over the same
            # step indices as the device-timed loop above (the flow, and with it the work of a
            # step, grows while the tide ramps up)
            import ctypes
            m.close()
            m = Model([case], precision=mode, device=local)
            m.set_stream(stream.cuda_stream)
            tau_t = torch.from_numpy(np.ascontiguousarray(case.tau)).pin_memory()
            eta_t = torch.zeros(nodes, dtype=torch.float64).pin_memory()
            tau, eta = tau_t.numpy(), eta_t.numpy()

            def e2e_step():
                m.set_tau(0, tau)
                m.step(1)
                m.lib.gs_state_get(m.h, 0, 1, eta.ctypes.data_as(ctypes.c_void_p), eta.nbytes)

            # untimed warm-up of this path (its first gs_step captures the step graph)
            for _ in range(a.warmup):
                e2e_step()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t0 = time.perf_counter()
            for k in range(a.steps):
                e2e_step()
            e1.record(stream)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            ems = max(e0.elapsed_time(e1), wall * 1e3)
            res[mode]["e2e"] = dict(value=total / (max_over_ranks(ems, dist, device="cuda") / 1e3), unit=METRIC,
                                    h2d_bytes_per_step=int(tau.nbytes), d2h_bytes_per_step=int(eta.nbytes))
        m.close()
        del m
    # several GPUs: the 64-member ensemble sharded by device footprint (every rank steps its own
    # members; the device time is the max over ranks)
    ens_sharded = run_ensemble_sharded(a, stream, local, dist, ws, rank) if (ws > 1 and not a.no_ensemble) else None
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    # the batched-ensemble comparison is a one-GPU measurement (rank 0 of a one-rank run)
    ens = run_ensemble(a, stream, local) if (ws == 1 and not a.no_ensemble) else None
    srv = run_serving(local) if (ws == 1 and not a.no_serve) else None
    slots = run_slot_serving(local) if (ws == 1 and not a.no_serve) else None
    r = res["fp32_ir"]
    # roofline of the dominant kernel (JCG): algorithmic bytes / average launch time
    nnz = r["nnz"]
    it_in = max(r["jcg_iters_last"], 1)
    outer = max(r["jcg_outer_last"], 1)
    bytes_launch = it_in * _jcg_bytes_per_iter(nodes, nnz, "fp32") + outer * (nnz * 12 + 4 * nodes + 3 * 8 * nodes)
    jms_avg = statistics.mean(r["jcg_ms"])
    achieved = bytes_launch / (jms_avg / 1e3) / 1e9
    line = {
        "metric": METRIC, "value": r["value"], "unit": METRIC, "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (JCG inner f32, f64 refinement)",
        "data": "synthetic (seeded GRF bathymetry, lattice mesh)",
        "config": {"workload": f"basin {a.n}x{a.n} nodes ({nodes}), 30 SZ levels, 2 tracers, dt=120 s, JCG rtol 1e-12",
                   "nodes": nodes, "levels": nvrt, "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (state ~10 GB per replica)"},
        "e2e": r["e2e"],
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": (None if JCG_DRAM_BYTES_PER_INNER_ITER is None
                                 else JCG_DRAM_BYTES_PER_INNER_ITER * it_in), "kernel": "k_jcg_ir",
                     "peak_kind": peak_kind, "iters_per_launch": it_in, "bytes_per_launch": bytes_launch},
        "clocks": r["clocks"],
        # per step, issued phase by phase: clock, btrack, elevation BC, side preparation, ghat, assembly,
        # solve, elevation update, momentum, vertical velocity, transport, nodal tracers, 6 level kernels,
        # 2 density kernels (two tracers), nodal velocities (the launch list in profiles/)
        "gpu_launches": a.steps * 22,
        "jcg": {"inner_iters": r["jcg_iters_last"], "outer": r["jcg_outer_last"], "ms_avg": jms_avg},
    }
    if "fp64" in res:
        f = res["fp64"]
        line["fp64"] = {"value": f["value"], "ms_per_step": f["ms_per_step"], "jcg_iters": f["jcg_iters_last"],
                        "jcg_ms_avg": statistics.mean(f["jcg_ms"])}
    if ens is not None:
        line["ensemble"] = ens
    if ens_sharded is not None:
        line["ensemble_sharded"] = ens_sharded
    if srv is not None:
        line["serving"] = srv
    if slots is not None:
        line["serving_slots"] = slots
    if not a.no_cpu:
        cb, ofields, case_full = cpu_sample(a)
        line["cpu_baseline"] = cb
        line["error_vs_oracle"] = error_vs_oracle(case_full, ofields, 3, local)
    print(json.dumps(line))


def run_ensemble(a, stream, local):
    """64-member ensemble: batched FP32+IR and FP64 (one launch per phase for all members) and
    the plain FP64 single-instance form (one member at a time), same steps, device time."""
    import torch
    from gschism_b200 import cases
    from gschism_b200.model import Model
    ens = cases.ensemble(n_members=64)
    nodes = sum(c.n_nodes for c in ens)
    nvrt = ens[0].vgrid.nvrt
    steps, warm = min(a.steps, 5), max(3, min(a.warmup, 3))

    def timed(m):
        m.set_stream(stream.cuda_stream)
        for _ in range(warm):
            m.step(1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            m.step(1)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    out = {"workload": f"64 members, {nodes} nodes in total (20k-500k each, log-uniform), {nvrt} levels, "
                       f"1 tracer, per-member tide 0.3-2 m and wind stress 0-0.3 N/m2, dt=120 s",
           "nodes": nodes, "levels": nvrt, "steps": steps, "warmup": warm}
    phases = ["BEGIN", "BTRACK", "PREPARE", "ASSEMBLE", "SOLVE", "UPDATE_ELEV", "MOMENTUM", "VVEL", "TRANSPORT",
              "LEVELS", "NODAL_VEL"]
    peak, peak_kind = _peaks()

    def breakdown(m, it0, nstep=2):
        """Device time of every phase over `nstep` steps issued phase by phase (CUDA events on the
        launching stream), in ms per step, and the per-member solver counters of the last step."""
        acc = {p: 0.0 for p in phases}
        for k in range(nstep):
            evs = [torch.cuda.Event(enable_timing=True) for _ in range(len(phases) + 1)]
            evs[0].record(stream)
            for i, p in enumerate(phases):
                m.phase(p, it0 + k)
                evs[i + 1].record(stream)
            torch.cuda.synchronize()
            for i, p in enumerate(phases):
                acc[p] += evs[i].elapsed_time(evs[i + 1]) / nstep
        st = [m.stats(i) for i in range(len(ens))]
        return acc, st

    eta = {}
    small = sorted(range(len(ens)), key=lambda i: ens[i].n_nodes)[:2]
    for prec in ("fp32_ir", "fp64"):
        m = Model(ens, precision=prec, device=local)
        ms = timed(m)
        its = [m.stats(i)["jcg_iters"] for i in range(len(ens))]
        eta[prec] = [m.get(i, "ETA2").copy() for i in range(len(ens))]
        ph, st = breakdown(m, warm + steps + 1)
        # roofline of the batched solve: algorithmic bytes of every member's iterations / phase time
        byts = 0.0
        for i, sz in enumerate(m.sizes):
            if prec == "fp32_ir":
                byts += st[i]["jcg_iters"] * _jcg_bytes_per_iter(sz["np"], sz["nnz"], "fp32") + \
                    st[i]["jcg_outer"] * (sz["nnz"] * 12 + 4 * sz["np"] + 3 * 8 * sz["np"])
            else:
                byts += st[i]["jcg_iters"] * _jcg_bytes_per_iter(sz["np"], sz["nnz"], "fp64")
        ach = byts / (ph["SOLVE"] / 1e3) / 1e9
        out[f"{prec}_batched"] = {"value": nodes * nvrt / (ms / 1e3), "ms_per_step": ms,
                                  "jcg_iters_min": min(its), "jcg_iters_max": max(its),
                                  "phase_ms": {p: round(v, 3) for p, v in ph.items()},
                                  "solve_roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                                                     "frac": ach / peak, "peak_kind": peak_kind,
                                                     "bytes_per_launch": byts,
                                                     "kernel": "k_jcg_ir" if prec == "fp32_ir" else "k_jcg64"}}
        m.close()
        del m
        torch.cuda.empty_cache()
    out["max_eta_diff_fp32_ir_vs_fp64_m"] = max(float(np.max(np.abs(x - y))) for x, y in zip(eta["fp32_ir"], eta["fp64"]))
    # the two smallest members (their own tide and wind) against the CPU oracle, same steps
    from oracle.step_api import OracleModel
    errs = []
    for i in small:
        o = OracleModel(ens[i])
        o.run(warm + steps)
        oe = o.get("ETA2")
        errs.append({"member": i, "nodes": int(ens[i].n_nodes),
                     "fp32_ir_eta_max_abs_m": float(np.abs(eta["fp32_ir"][i] - oe).max()),
                     "fp64_eta_max_abs_m": float(np.abs(eta["fp64"][i] - oe).max())})
        del o
    out["error_vs_oracle"] = {"steps": warm + steps, "members": errs}
    tot = 0.0
    for c in ens:
        m = Model([c], precision="fp64", device=local)
        tot += timed(m)
        m.close()
        del m
    out["fp64_single_instance"] = {"value": nodes * nvrt / (tot / 1e3), "ms_per_step": tot,
                                   "note": "members stepped one at a time, sum of their device times"}
    out["speedup_fp32_ir_batched_vs_fp64_single"] = tot / out["fp32_ir_batched"]["ms_per_step"]
    return out


def run_ensemble_sharded(a, stream, local, dist, ws, rank):
    """The 64-member ensemble over `ws` ranks (gschism_b200/shard.py): members assigned by device
    footprint, each rank steps its share batched (FP32+IR), device time max over ranks.  Every rank
    takes the same collective steps (a barrier, one max)."""
    import torch
    from gschism_b200 import cases
    from gschism_b200.model import Model, footprint_bytes
    from gschism_b200.shard import max_over_ranks, shard_members
    ens = cases.ensemble(n_members=64)
    mine = shard_members([footprint_bytes([c]) for c in ens], ws)[rank]
    steps, warm = min(a.steps, 5), 3
    m = Model([ens[i] for i in mine], precision="fp32_ir", device=local) if mine else None
    if m is not None:
        m.set_stream(stream.cuda_stream)
        for _ in range(warm):
            m.step(1)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    if m is not None:
        for _ in range(steps):
            m.step(1)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, device="cuda")
    if m is not None:
        m.close()
    nodes = sum(c.n_nodes for c in ens)
    nvrt = ens[0].vgrid.nvrt
    return {"workload": f"the 64-member ensemble ({nodes} nodes, {nvrt} levels) sharded over {ws} GPUs by device footprint",
            "value": nodes * nvrt * steps / (ms / 1e3), "unit": METRIC, "ms_per_step": ms / steps, "steps": steps,
            "warmup": warm, "scaling": "strong", "members_on_rank0": len(mine) if rank == 0 else None}


def run_serving(local, n=8, rate=2.0, hours=6.0, seed=1):
    """Forecast serving (gschism_b200/serve.py): n storm-surge requests (10k-2M nodes, 20 levels,
    tide + vortex) arriving as a Poisson process of `rate` per second, continuous batching on this
    GPU; time-to-forecast = arrival to results on the host.  The horizon is `hours` instead of the
    scenario's 48 h, to keep this run to about a minute of GPU time."""
    from gschism_b200.serve import ModelEngine, Server, poisson_requests, summary
    reqs = poisson_requests(n, rate, seed, hours=hours)
    srv = Server(ModelEngine(precision="fp32_ir", device=local))
    t0 = time.perf_counter()
    srv.run(reqs)
    out = summary(reqs, time.perf_counter() - t0)
    builds = [e[3] for e in srv.log if e[0] == "build"]
    out.update({"workload": f"{n} storm-surge requests, Poisson arrivals {rate}/s, 10k-2M nodes, 20 levels, "
                            f"{hours:g} h horizon at dt=150 s (the full scenario's horizon is 48 h)",
                "nodes": [int(r.case.n_nodes) for r in reqs], "ttf_s": [round(r.time_to_forecast, 3) for r in reqs],
                "build_s_total": round(sum(builds), 2)})
    return out


def run_slot_serving(local, n=16, rate=2.0, hours=(3.0, 6.0), seed=1, regions=4, slots=2):
    """Slot-level serving (gschism_b200/serve.py:SlotServer): one context with `slots` member
    slots on each of `regions` storm meshes (30k-600k nodes, 20 levels); n requests (a region, a
    storm, a horizon drawn from `hours`) arriving as a Poisson process of `rate` per second, each
    admitted into a free slot of its region at a step boundary while the others run.  Horizons
    are a few hours instead of the scenario's 48 h, to keep this run to about half a minute."""
    from gschism_b200.serve import SlotEngine, SlotServer, region_meshes, slot_requests, summary
    regs = region_meshes(regions, 30_000, 600_000, seed)
    reqs = slot_requests(n, rate, seed, regs, horizons=list(hours))
    srv = SlotServer(SlotEngine(precision="fp32_ir", device=local), regs, slots)
    t0 = time.perf_counter()
    srv.run(reqs)
    out = summary(reqs, time.perf_counter() - t0 - srv.setup_s)
    out.update({"workload": f"{n} storm-surge requests over {regions} region meshes "
                            f"({', '.join(str(int(c.n_nodes)) for c in regs)} nodes, 20 levels), {slots} slots each, "
                            f"Poisson arrivals {rate}/s, horizons {'/'.join(f'{h:g}' for h in hours)} h at dt=150 s",
                "setup_s": round(srv.setup_s, 2), "ttf_s": [round(r.time_to_forecast, 3) for r in reqs],
                "wait_s": [round(r.admitted - r.arrival, 3) for r in reqs]})
    out.pop("cohorts", None)
    return out


def _cpu_info():
    """Host CPU model and logical core count (recorded beside every CPU number)."""
    model = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except Exception:
        pass
    return model, os.cpu_count() or 1


def _omp_threads(n):
    """Set the OpenMP thread count of the already loaded oracle library (libgomp)."""
    import ctypes
    try:
        ctypes.CDLL("libgomp.so.1").omp_set_num_threads(int(n))
        return True
    except OSError:
        return False


def _fields_of(get):
    return {f: np.array(get(f), copy=True) for f in ("ETA2", "ELEM_TR", "SIDE_U2")}


def _errors(g, o):
    def rel(x, y):
        s_ = float(np.abs(y).max())
        return float(np.abs(x - y).max()) / (s_ if s_ > 0 else 1.0)
    return {"eta_max_abs_m": float(np.abs(g["ETA2"] - o["ETA2"]).max()),
            "tracer_rel": rel(g["ELEM_TR"], o["ELEM_TR"]), "velocity_rel": rel(g["SIDE_U2"], o["SIDE_U2"])}


def cpu_sample(a, steps=3):
    """The CPU oracle on the benchmarked mesh itself (all host threads): step 1 untimed, steps
    2..`steps` timed.  Returns the cpu_baseline entry and the oracle's fields after `steps` steps
    (the error_vs_oracle comparison)."""
    from gschism_b200 import cases
    from oracle.step_api import OracleModel
    case = cases.basin(seed=2, n=a.n, nvrt=30, nz=10, ntr=2)
    o = OracleModel(case)
    o.run(1)
    t0 = time.perf_counter()
    o.run(steps - 1, start=2)
    dtm = time.perf_counter() - t0
    fields = _fields_of(o.get)
    cpu, ncores = _cpu_info()
    cores = int(os.environ.get("OMP_NUM_THREADS", ncores))
    out = {"value": case.n_nodes * case.nvrt * (steps - 1) / dtm, "unit": METRIC, "cores": cores, "kind": "port",
           "sample": f"the benchmarked basin {a.n}x{a.n} ({case.n_nodes} nodes, 30 levels, 2 tracers): steps 2-{steps} "
                     f"timed after one untimed step, {dtm:.1f} s", "cpu_model": cpu}
    del o
    return out, fields, case


def error_vs_oracle(case, oracle_fields, steps, device):
    """The FP64 and FP32+IR forms after `steps` steps of `case` against the oracle's fields after
    the same steps."""
    from gschism_b200.model import Model
    out = {"workload": f"the benchmarked mesh ({case.n_nodes} nodes), {steps} steps from the cold start",
           "oracle": "oracle/ (CPU FP64 restatement, pinned to the reference's own kernels)"}
    for prec in ("fp64", "fp32_ir"):
        m = Model([case], precision=prec, device=device)
        m.step(steps)
        m.sync()
        out[prec] = _errors(_fields_of(lambda f: m.get(0, f)), oracle_fields)
        m.close()
        del m
    out["fp32_ir_within_1e-6_m"] = out["fp32_ir"]["eta_max_abs_m"] <= 1e-6
    return out


def run_reference(a):
    """The reference arm: the CPU oracle (the reference has no CPU path of its own; the oracle is
    pinned to its kernels) on the benchmarked mesh, all host threads, 1 warm-up step and up to 6
    timed steps; plus one step single-threaded on a 200 x 200 sample."""
    ws, rank, local = _dist()
    if rank != 0:
        return
    from gschism_b200 import cases
    from oracle.step_api import OracleModel
    case = cases.basin(seed=2, n=a.n, nvrt=30, nz=10, ntr=2)
    o = OracleModel(case)
    warm = max(1, min(a.warmup, 1))
    o.run(warm)
    k = max(1, min(a.steps, 6))
    t0 = time.perf_counter()
    o.run(k, start=warm + 1)
    dtm = time.perf_counter() - t0
    del o
    v = case.n_nodes * case.nvrt * k / dtm
    cpu, ncores = _cpu_info()
    cores = int(os.environ.get("OMP_NUM_THREADS", ncores))
    single = None
    small = cases.basin(seed=2, n=200, nvrt=30, nz=10, ntr=2, length=500e3 * 200 / 1000)
    if _omp_threads(1):
        o1 = OracleModel(small)
        o1.run(1)
        t1 = time.perf_counter()
        o1.run(1, start=2)
        d1 = time.perf_counter() - t1
        single = {"value": small.n_nodes * small.nvrt / d1, "unit": METRIC, "cores": 1,
                  "sample": f"basin 200x200 ({small.n_nodes} nodes), 30 levels, 2 tracers, step 2 after one untimed step"}
        _omp_threads(cores)
        del o1
    sample = (f"CPU oracle (the reference has no CPU path; the oracle is pinned to the reference's own kernels): "
              f"the benchmarked basin {a.n}x{a.n} ({case.n_nodes} nodes), 30 levels, 2 tracers, {k} timed steps "
              f"after {warm} warm-up step")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": ws, "steps": k,
        "warmup": warm, "ms_per_step": dtm / k * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"basin {a.n}x{a.n} nodes ({case.n_nodes}), 30 SZ levels, 2 tracers, dt=120 s, "
                               f"JCG rtol 1e-12", "nodes": case.n_nodes, "levels": case.nvrt,
                   "parallelism": f"{cores} host threads"},
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": cores, "kind": "port", "sample": sample,
                         "cpu_model": cpu, "single_thread": single},
        "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def main():
    a = _args()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
