"""Autotuner of the step's launch shapes (gs_set_launch).

Every stream kernel of the step strides over its entities, so its launch shape (threads per
block, grid cap in blocks per SM) changes only its speed; the JCG tiling (tiles of a large member,
smallest tile) changes the speed and the order of the solver's partial sums.  The tuner steps a
context phase by phase with CUDA events between the phases and, one kernel at a time, tries
every candidate shape for a few interleaved rounds (the flow develops while it runs, so
candidates are compared round by round, never one block of steps against another), keeps the
shape with the smallest median time of the kernel's phase (for the solver: time per inner
iteration), and moves to the next kernel.

    shapes = autotune.tuned_shapes(cases, precision="fp32_ir")   # cache, or tune a scratch copy
    model = Model(cases, precision="fp32_ir")
    autotune.apply(model, shapes)

Results are cached in a JSON file (``GSCHISM_TUNE_CACHE`` or ``_build/tune_cache.json`` next to
the library) keyed by the GPU, the precision, the vertical grid, the tracer count and the size
class (log2 of the node count), so a serving loop tunes a size class once.
"""
from __future__ import annotations

import json
import math
import os
import statistics
from typing import Callable, Dict, List, Optional, Sequence, Tuple

Shape = Tuple[int, int]

# phases of one step in order, as gs_step runs them
STEP_PHASES = ["BTRACK", "PREPARE", "ASSEMBLE", "SOLVE", "UPDATE_ELEV", "MOMENTUM", "VVEL", "TRANSPORT",
               "LEVELS", "NODAL_VEL"]
# the phase whose time a kernel's shape moves
KERNEL_PHASE = {"BTRACK": "BTRACK", "SIDE_PREP": "PREPARE", "GHAT": "PREPARE", "ASSEMBLE": "ASSEMBLE",
                "MOMENTUM": "MOMENTUM", "VVEL": "VVEL", "NODAL_VEL": "NODAL_VEL", "NODAL_TRACER": "TRANSPORT",
                "LEVELS": "LEVELS", "JCG_TILES": "SOLVE"}
TUNE_ORDER = ["BTRACK", "JCG_TILES", "MOMENTUM", "SIDE_PREP", "GHAT", "VVEL", "NODAL_VEL", "NODAL_TRACER",
              "ASSEMBLE", "LEVELS"]


def candidates(kernel: str) -> List[Shape]:
    """Shapes tried for a kernel (the library rejects those its compiled kernel cannot run)."""
    if kernel == "JCG_TILES":
        return [(592, 1024), (296, 1024), (444, 1024), (888, 1024), (1184, 512), (888, 512)]
    return [(b, g) for b in (64, 128, 256, 512) for g in (16, 32)]


class PhaseTimer:
    """Runs one step phase by phase on a torch stream with an event between phases."""

    def __init__(self, model, first_step: int):
        import torch
        self.torch = torch
        self.model = model
        self.it = first_step
        self.stream = torch.cuda.Stream()
        model.set_stream(self.stream.cuda_stream)
        self.ev = [torch.cuda.Event(enable_timing=True) for _ in range(len(STEP_PHASES) + 1)]

    def step(self) -> Dict[str, float]:
        m, it = self.model, self.it
        m.phase("BEGIN", it)
        self.ev[0].record(self.stream)
        for i, ph in enumerate(STEP_PHASES):
            m.phase(ph, it if ph == "LEVELS" else 0)
            self.ev[i + 1].record(self.stream)
        self.ev[-1].synchronize()
        self.it += 1
        out = {ph: self.ev[i].elapsed_time(self.ev[i + 1]) for i, ph in enumerate(STEP_PHASES)}
        # the solve lasts as long as its slowest member
        out["jcg_iters"] = max(1, max(int(m.stats(j)["jcg_iters"]) for j in range(len(m.cases))))
        return out


def _cost(kernel: str, times: Dict[str, float]) -> float:
    t = times[KERNEL_PHASE[kernel]]
    return t / times["jcg_iters"] if kernel == "JCG_TILES" else t


def tune_model(model, kernels: Sequence[str] = TUNE_ORDER, rounds: int = 3,
               measure: Optional[Callable[[], Dict[str, float]]] = None, first_step: int = 1,
               log: Optional[Callable[[str], None]] = None) -> Dict[str, Shape]:
    """Tune the launch shapes of `model` in place (it is stepped while tuning, from step
    `first_step` on) and return the chosen shape of every kernel.  `measure()` runs one step and
    returns per-phase times in ms (and "jcg_iters"); by default a PhaseTimer on the model."""
    from ._lib import GsError
    if measure is None:
        measure = PhaseTimer(model, first_step=first_step).step
    chosen: Dict[str, Shape] = {}
    for k in kernels:
        start = model.get_launch(k)
        valid = []
        for c in candidates(k):
            try:
                model.set_launch(k, *c)
                valid.append(c)
            except GsError:
                continue
        if not valid:
            model.set_launch(k, *start)
            chosen[k] = start
            continue
        samples: Dict[Shape, List[float]] = {c: [] for c in valid}
        for _ in range(rounds):
            for c in valid:
                model.set_launch(k, *c)
                samples[c].append(_cost(k, measure()))
        best = min(valid, key=lambda c: statistics.median(samples[c]))
        model.set_launch(k, *best)
        chosen[k] = best
        if log:
            base = statistics.median(samples[start]) if start in samples else float("nan")
            log(f"{k}: {best} {statistics.median(samples[best]):.4g} (default {start} {base:.4g})")
    return chosen


def apply(model, shapes: Dict[str, Shape]) -> None:
    for k, (a, b) in shapes.items():
        model.set_launch(k, a, b)


# --------------------------------------------------------------------------------- cache
def cache_path() -> str:
    env = os.environ.get("GSCHISM_TUNE_CACHE")
    if env:
        return env
    from . import build
    return os.path.join(build.BUILD, "tune_cache.json")


def cache_key(cases, precision: str, gpu: str) -> str:
    c0 = cases[0]
    nodes = sum(int(c.n_nodes) for c in cases)
    cls = int(round(math.log2(max(nodes, 1))))
    p = c0.params
    return (f"{gpu}|{precision}|nvrt={c0.vgrid.nvrt}|ntr={c0.ntracers}|itr_met={p.itr_met}|"
            f"nodes~2^{cls}")


def load_cache(path: Optional[str] = None) -> Dict[str, Dict[str, List[int]]]:
    path = path or cache_path()
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def store_cache(key: str, shapes: Dict[str, Shape], path: Optional[str] = None) -> None:
    path = path or cache_path()
    data = load_cache(path)
    data[key] = {k: list(v) for k, v in shapes.items()}
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    tmp = f"{path}.tmp{os.getpid()}"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def tuned_shapes(cases, precision: str = "fp32_ir", warmup: int = 4, rounds: int = 2,
                 path: Optional[str] = None, retune: bool = False,
                 log: Optional[Callable[[str], None]] = None) -> Dict[str, Shape]:
    """Shapes for a batch of these cases: from the cache, or tuned on a scratch context built
    from the same cases (stepped `warmup` steps first) and stored."""
    import torch
    from .model import Model
    key = cache_key(cases, precision, torch.cuda.get_device_name())
    if not retune:
        hit = load_cache(path).get(key)
        if hit:
            return {k: (int(v[0]), int(v[1])) for k, v in hit.items()}
    scratch = Model(list(cases), precision=precision)
    try:
        scratch.step(warmup)
        scratch.sync()
        timer = PhaseTimer(scratch, first_step=warmup + 1)
        shapes = tune_model(scratch, rounds=rounds, measure=timer.step, log=log)
    finally:
        scratch.close()
    store_cache(key, shapes, path)
    return shapes
