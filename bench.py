"""Benchmark: SCHISM semi-implicit step on one B200, node-level-steps/s.

Workload (single large mesh, the configuration the metric is quoted on that fits one GPU):
1M-node jittered-lattice basin, 500 km x 500 km, 30 SZ levels (10 z + 21 sigma), Gaussian-
random-field bathymetry 2..4000 m, M2+S2 1.2 m on the west side, 2 tracers (T, S); dt = 120 s;
JCG rtol 1e-12.  Inputs are seeded synthetic data (no dataset involved).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--n 1000]

value    = node-level-steps/s of the timed steps (sum of nodes x levels x steps / device time),
           FP32-inner JCG with FP64 refinement ("fp32_ir"), state resident in HBM.
e2e      = the same loop through the C ABI with host buffers: every step uploads the surface
           stress field from host memory (gs_set_tau) and reads the elevation back (gs_state_get).
roofline = the JCG persistent kernel (dominant), algorithmic bytes per launch / launch time.
The plain FP64 single-instance form is measured on the same GPU and reported under "fp64".
ensemble = the batched form: 64 members on meshes of uneven size (20k-500k nodes, 20 levels,
           1 tracer, per-member tide and wind), all members in one launch per phase, FP32+IR and
           FP64, against the plain FP64 single-instance form run member by member.
Multi-GPU (torchrun): every rank steps its own replica of the mesh (no data exchange exists in
the step); value = all ranks' node-level-steps / the max over ranks of the device time.
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


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per inner iteration of k_jcg_ir on
# the 1M-node basin, from the ncu capture summarised in profiles/k_jcg_ir_basin1M.md (launch
# bytes / inner iterations of that launch); scaled here by the timed launches' inner iterations.
JCG_DRAM_BYTES_PER_INNER_ITER = 31.6e6


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
            # end-to-end through the C ABI with host buffers: upload tau, step, read eta back
            tau = np.ascontiguousarray(case.tau.copy())
            eta = np.zeros(nodes)
            import ctypes
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            t0 = time.perf_counter()
            for k in range(a.steps):
                m.set_tau(0, tau)
                m.step(1)
                m.lib.gs_state_get(m.h, 0, 1, eta.ctypes.data_as(ctypes.c_void_p), eta.nbytes)
            e1.record(stream)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            ems = max(e0.elapsed_time(e1), wall * 1e3)
            res[mode]["e2e"] = dict(value=total / (max_over_ranks(ems, dist, device="cuda") / 1e3), unit=METRIC,
                                    h2d_bytes_per_step=int(tau.nbytes), d2h_bytes_per_step=int(eta.nbytes))
        m.close()
        del m
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    # the batched-ensemble comparison is a one-GPU measurement (rank 0 of a one-rank run)
    ens = run_ensemble(a, stream, local) if (ws == 1 and not a.no_ensemble) else None
    srv = run_serving(local) if (ws == 1 and not a.no_serve) else None
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
        "gpu_launches": a.steps * 18,
        "jcg": {"inner_iters": r["jcg_iters_last"], "outer": r["jcg_outer_last"], "ms_avg": jms_avg},
    }
    if "fp64" in res:
        f = res["fp64"]
        line["fp64"] = {"value": f["value"], "ms_per_step": f["ms_per_step"], "jcg_iters": f["jcg_iters_last"],
                        "jcg_ms_avg": statistics.mean(f["jcg_ms"])}
    if ens is not None:
        line["ensemble"] = ens
    if srv is not None:
        line["serving"] = srv
    if not a.no_cpu:
        line["cpu_baseline"] = cpu_sample(a)
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
    eta = {}
    for prec in ("fp32_ir", "fp64"):
        m = Model(ens, precision=prec, device=local)
        ms = timed(m)
        its = [m.stats(i)["jcg_iters"] for i in range(len(ens))]
        eta[prec] = [m.get(i, "ETA2").copy() for i in range(len(ens))]
        out[f"{prec}_batched"] = {"value": nodes * nvrt / (ms / 1e3), "ms_per_step": ms,
                                  "jcg_iters_min": min(its), "jcg_iters_max": max(its)}
        m.close()
        del m
        torch.cuda.empty_cache()
    out["max_eta_diff_fp32_ir_vs_fp64_m"] = max(float(np.max(np.abs(x - y))) for x, y in zip(eta["fp32_ir"], eta["fp64"]))
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


def cpu_sample(a, steps=6, n=500):
    """The CPU restatement (oracle) on a bounded sample of the same workload: a n x n basin with
    the same levels, tracers and physics, all host threads, `steps` steps."""
    from gschism_b200 import cases
    from oracle.step_api import OracleModel
    case = cases.basin(seed=2, n=n, nvrt=30, nz=10, ntr=2, length=500e3 * n / 1000)
    o = OracleModel(case)
    t0 = time.perf_counter()
    o.run(steps)
    dtm = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": case.n_nodes * case.nvrt * steps / dtm, "unit": METRIC, "cores": cores, "kind": "port",
            "sample": f"basin {n}x{n} ({case.n_nodes} nodes), 30 levels, 2 tracers, {steps} steps, {dtm:.1f} s"}


def run_reference(a):
    ws, rank, local = _dist()
    if rank != 0:
        return
    from gschism_b200 import cases
    from oracle.step_api import OracleModel
    n = 500
    case = cases.basin(seed=2, n=n, nvrt=30, nz=10, ntr=2, length=500e3 * n / 1000)
    o = OracleModel(case)
    for _ in range(min(a.warmup, 1)):
        o.run(1)
    t0 = time.perf_counter()
    o.run(a.steps)
    dtm = time.perf_counter() - t0
    v = case.n_nodes * case.nvrt * a.steps / dtm
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    sample = (f"CPU restatement of the reference kernels (the reference has no CPU path): basin {n}x{n} "
              f"({case.n_nodes} nodes), 30 levels, 2 tracers, {a.steps} steps")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": METRIC, "n_gpus": ws, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": dtm / a.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"basin {a.n}x{a.n} nodes, 30 SZ levels, 2 tracers, dt=120 s (sampled at {n}x{n})"},
        "cpu_baseline": {"value": v, "unit": METRIC, "cores": cores, "kind": "port", "sample": sample},
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
