"""Checks against the fixtures made by the reference's own kernels (tests/golden/make_step_golden.py).

Shared by the CPU test of the oracle (tests/test_ref_pinned.py) and the GPU test of the CUDA path
(tests/test_gpu_ref_pinned.py).  Two kinds of check:

* trajectory: from the same cold start, every snapshot field after k steps must agree with the
  reference within `TRAJ_FACTOR` times the reference's own reproducibility envelope at that step
  (the spread between reference runs that differ only in summation orders a GPU may take), and
  never worse than the fixed bounds in `TRAJ_CAP`; the JCG iteration counts must be the
  reference's;
* per phase: from the reference's state before one step, every phase's output must agree with
  the reference's output of the same phase within `PHASE_TOL` (relative to the field's largest
  magnitude); integer fields bit for bit.
"""
from __future__ import annotations

import os

import numpy as np

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

TRAJ_FACTOR = 10.0
# floors (relative to the field's largest magnitude) for fields whose envelope is at rounding level
TRAJ_FLOOR = {"ETA2": 1e-12, "NODE_TR": 1e-12, "ELEM_TR": 1e-12, "SIDE_U2": 1e-11, "NODE_U2": 1e-11,
              "NODE_W2": 1e-10, "ELEM_W": 1e-10, "NODE_RHO": 1e-14, "ELEM_RHO": 1e-14}
# the targets: elevation and tracers 1e-10, velocities (horizontal and vertical) 1e-8 over 100 steps
TRAJ_CAP = {"ETA2": 1e-10, "NODE_TR": 1e-10, "ELEM_TR": 1e-10, "SIDE_U2": 1e-8, "NODE_U2": 1e-8,
            "NODE_W2": 1e-7, "ELEM_W": 1e-7, "NODE_RHO": 1e-12, "ELEM_RHO": 1e-12}
PHASE_TOL = 1e-12
PHASE_TOL_FIELD = {"NODE_W2": 1e-11, "ELEM_W": 1e-11, "ELEM_QV": 1e-11}

PHASES = ("BTRACK", "PREPARE", "ASSEMBLE", "SOLVE", "UPDATE_ELEV", "MOMENTUM", "VVEL", "TRANSPORT", "LEVELS",
          "NODAL_VEL")
INT_FIELDS = {"NODE_KB", "NODE_DRY", "SIDE_KB", "SIDE_DRY", "ELEM_KB", "ELEM_DRY"}


def load(name: str) -> dict:
    return dict(np.load(os.path.join(GOLD, f"step_{name}.npz")))


def rel(a, b) -> float:
    s = float(np.abs(b).max())
    return float(np.abs(np.asarray(a, float) - np.asarray(b, float)).max()) / (s if s > 0 else 1.0)


def cut(g: dict, name: str, a: np.ndarray) -> np.ndarray:
    """The fixture's entity subset of a full field (fixtures of meshes above 300 nodes)."""
    if f"subset_{name[0]}" not in g or name == "ETA2":
        return a
    idx = g[f"subset_{name[0]}"]
    return a[:, :, idx] if name in ("NODE_TR", "ELEM_TR") else a[:, idx]


def traj_tolerance(g: dict, step_index: int, field: str) -> float:
    fields = [str(f) for f in g["envelope_fields"]]
    env = float(g["envelope"][step_index, fields.index(field)])
    return min(max(TRAJ_FACTOR * env, TRAJ_FLOOR[field]), TRAJ_CAP[field])


def check_trajectory(g: dict, step, get, nsteps: int, iters=None):
    """step(it) advances one step; get(field) returns a full field.  Returns the report rows
    (step, field, error, tolerance) and raises AssertionError on the first failure."""
    snaps = [int(s) for s in g["snap_steps"]]
    rows = []
    for it in range(1, nsteps + 1):
        its = step(it)
        if iters is not None:
            its = iters()
        if its is not None:
            assert int(its) == int(g["iters"][it - 1]), (it, its, int(g["iters"][it - 1]))
        if it in snaps:
            i = snaps.index(it)
            for f in [str(x) for x in g["envelope_fields"]]:
                e = rel(cut(g, f, get(f)), g[f"snap{it}_{f}"])
                tol = traj_tolerance(g, i, f)
                rows.append((it, f, e, tol))
                assert e <= tol, f"step {it} {f}: rel err {e:.3e} > tolerance {tol:.3e}"
    return rows


def state_fields(g: dict):
    return [k[len("state_"):] for k in g if k.startswith("state_")]


def check_phases(g: dict, put, run_phase, get):
    """Start from the reference's state before the fixture's phase step, run every phase and
    compare its outputs.  Returns the rows (phase, field, error)."""
    for f in state_fields(g):
        put(f, g[f"state_{f}"])
    rows = []
    for ph in PHASES:
        run_phase(ph)
        for key in [k for k in g if k.startswith(f"phase_{ph}_")]:
            f = key[len(f"phase_{ph}_"):]
            a, b = get(f), g[key]
            if f in INT_FIELDS:
                assert np.array_equal(np.asarray(a), np.asarray(b)), f"{ph} {f} differs"
                rows.append((ph, f, 0.0))
                continue
            e = rel(a, b)
            rows.append((ph, f, e))
            assert e <= PHASE_TOL_FIELD.get(f, PHASE_TOL), f"{ph} {f}: rel err {e:.3e}"
    return rows
