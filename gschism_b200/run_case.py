"""Run a synthetic case for a few steps and print the per-step solver statistics.

    python -m gschism_b200.run_case --case basin --n 1000 --levels 6 --steps 2 --precision fp32_ir

Used to drive profiler captures of one phase on a chosen size: the elevation solve depends on
the horizontal mesh only, so `--levels` can shrink the device state without changing it.

    python -m gschism_b200.run_case --n 1000 --steps 12 --time-phase BTRACK --repeat 20
    python -m gschism_b200.run_case --case ensemble --members 12 --levels 3 --steps 2

times one phase alone on the state reached after the steps (CUDA events around `--repeat`
launches after 3 untimed ones).  Only phases that do not modify their own inputs give a
repeatable figure this way (BTRACK does: it reads velocities and writes only its own output).
"""
from __future__ import annotations

import argparse
import time

from . import cases
from .model import Model


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--case", choices=["basin", "channel", "ensemble"], default="basin")
    ap.add_argument("--members", type=int, default=64, help="ensemble: the first members of the 64-member set")
    ap.add_argument("--n", type=int, default=1000, help="basin lattice side (n x n nodes)")
    ap.add_argument("--levels", type=int, default=30, help="vertical levels (basin)")
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--precision", choices=["fp64", "fp32_ir"], default="fp32_ir")
    ap.add_argument("--inner-rtol", type=float, default=0.1)
    ap.add_argument("--time-phase", default=None, help="phase to time after the steps (e.g. BTRACK)")
    ap.add_argument("--repeat", type=int, default=20)
    a = ap.parse_args(argv)
    t0 = time.time()
    if a.case == "basin":
        cs = [cases.basin(n=a.n, nvrt=a.levels, nz=max(2, min(10, a.levels // 3)))]
    elif a.case == "ensemble":
        cs = cases.ensemble(n_members=64, nvrt=a.levels)[:a.members]
    else:
        cs = [cases.channel()]
    m = Model(cs, precision=a.precision, ir_inner_rtol=a.inner_rtol)
    print(f"case {a.case}: {sum(z['np'] for z in m.sizes)} nodes in {len(cs)} member(s), {cs[0].vgrid.nvrt} "
          f"levels, set-up {time.time() - t0:.1f} s", flush=True)
    for s in range(a.steps):
        m.step(1)
        m.sync()
        its = [m.stats(k)["jcg_iters"] for k in range(len(cs))]
        print("step", s, m.stats(), "iters per member", min(its), "..", max(its), flush=True)
    if a.time_phase:
        import torch
        st = torch.cuda.Stream()
        m.set_stream(st.cuda_stream)
        for _ in range(3):
            m.phase(a.time_phase)
        m.sync()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(st)
        for _ in range(a.repeat):
            m.phase(a.time_phase)
        ev[1].record(st)
        ev[1].synchronize()
        print(f"phase {a.time_phase}: {ev[0].elapsed_time(ev[1]) / a.repeat:.3f} ms per launch "
              f"({a.repeat} launches after {a.steps} steps)", flush=True)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
