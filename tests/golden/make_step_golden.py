"""Generate the step fixtures from the reference's own kernels.

The reference's step kernels (src/kernels/meshdata.cu) are compiled for the host CPU from the
reference tree (oracle/refemu/build.py) and driven in the order of src/python/schism_step.py
(oracle/refemu/refstep.py).  For each case below this script stores, in tests/golden/step_<name>.npz:

* trajectory snapshots (from the cold start) of elevation, tracers and velocities at the listed
  steps (fields of meshes above 300 nodes on a fixed seeded subset of entities, all levels), with the JCG
  iteration count and transport sub-step count of every step;
* the reference's reproducibility envelope: for every snapshot field, the largest relative
  difference between this run and three runs that differ only in choices a GPU run of the
  reference makes (its atomic nodal-velocity sums in reversed thread order; its solver dot
  products in 32-entry blocks added pairwise; its kernels compiled with contracted
  multiply-adds, as nvcc/NVRTC do by default);
* for the cases with `phase_step`, the complete state before that step and every phase's output
  within it, for per-phase checks from an identical state.

Needs the reference tree ($GS_REFERENCE_ROOT, default /root/reference); the fixtures are
committed so the tests run without it.

    python tests/golden/make_step_golden.py            # all cases
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)

from gschism_b200 import cases  # noqa: E402

SNAP_FIELDS = ("ETA2", "NODE_TR", "ELEM_TR", "SIDE_U2", "NODE_U2", "NODE_W2", "ELEM_W")
RHO_FIELDS = ("NODE_RHO", "ELEM_RHO")   # cases with T and S (two tracers or more)
STATE_FIELDS = ("ETA1", "ETA2", "NODE_Z", "NODE_U2", "NODE_W2", "NODE_TR", "NODE_KB", "NODE_DRY", "SIDE_U2",
                "SIDE_ZC", "SIDE_KB", "SIDE_DRY", "ELEM_Z", "ELEM_TR", "ELEM_KB", "ELEM_DRY", "JCG_X", "JCG_X1",
                "JCG_X2")
PHASE_OUT = {
    "BTRACK": ("SIDE_BTU",),
    "PREPARE": ("ELBC", "SIDE_U", "SIDE_HHAT", "SIDE_CHI", "ELEM_GHAT"),
    "ASSEMBLE": ("CSR_DATA", "QEL"),
    "SOLVE": (),
    "UPDATE_ELEV": ("ETA2", "NODE_KB", "JCG_X"),
    "MOMENTUM": ("SIDE_U2",),
    "VVEL": ("ELEM_W", "ELEM_QV"),
    "TRANSPORT": ("SIDE_QH", "ELEM_TR", "NODE_TR"),
    "LEVELS": ("NODE_Z", "SIDE_ZC", "ELEM_Z", "NODE_KB", "NODE_DRY", "SIDE_KB", "SIDE_DRY", "ELEM_KB", "ELEM_DRY"),
    "NODAL_VEL": ("NODE_U2", "NODE_W2"),
}
SUBSET = 400   # entities kept per field for meshes above 300 nodes


def _uniform_tracers(c):
    """The reference's cold start sets tracers per node, uniform in the vertical
    (temp.ic/salt.ic, main.py:344-372); use the surface value on every level."""
    c.tr_init[:] = c.tr_init[:, -1:, :]
    return c


def step_cases():
    """name -> (case, steps, snapshot steps, phase step or None)."""
    return {
        # the plain FP64 configuration: 10 km x 5 km channel, 10 sigma levels, M2 0.5 m, 100 steps
        "channel": (cases.channel(seed=1), 100, (1, 2, 5, 10, 20, 30, 50, 75, 100), None),
        # SZ levels (3 z + 6 sigma) over Gaussian-random-field depths, M2+S2, T and S
        "basin16": (_uniform_tracers(cases.basin(seed=5, n=16, nvrt=8, nz=3, ntr=2, length=15e3, nsteps=20)),
                    20, (1, 2, 5, 10, 20), 6),
        # an ensemble-like member: its own tide amplitude and a uniform wind stress
        "member": (_uniform_tracers(cases.basin(seed=6, n=16, nvrt=10, nz=3, ntr=1, length=15e3, amp=0.7,
                                                tau=(1.5e-4, -0.8e-4), nsteps=20)),
                   20, (1, 5, 10, 20), 6),
    }


def subset_indices(case, seed=11):
    """Fixed entity subsets (nodes, sides, elements) for meshes above 300 nodes."""
    rng = np.random.default_rng(seed)
    npn, ne = case.n_nodes, case.n_elems
    ns = npn + ne - 1
    if npn <= 300:
        return None
    pick = lambda n: np.sort(rng.choice(n, size=min(SUBSET, n), replace=False)).astype(np.int64)
    return {"N": pick(npn), "S": pick(ns), "E": pick(ne)}


def _cut(name, a, sub):
    if sub is None or name == "ETA2":
        return a
    idx = sub[name[0]]
    if name in ("NODE_TR", "ELEM_TR"):
        return a[:, :, idx]
    return a[:, idx]


def snap_fields(case):
    return SNAP_FIELDS + (RHO_FIELDS if case.ntracers >= 2 else ())


def _run_variant(name, atomic_order, dot_order, fma, out):
    """Child process: one reference run (the mesh is a process-wide global there)."""
    from oracle.refemu.refstep import RefStep
    c, nsteps, snaps, phase_step = step_cases()[name]
    fields = snap_fields(c)
    sub = subset_indices(c)
    r = RefStep(c, atomic_order=atomic_order, dot_order=dot_order, fma=bool(fma))
    res = {"iters": [], "substeps": []}
    for it in range(1, nsteps + 1):
        if phase_step is not None and it == phase_step and atomic_order == 0 and dot_order == 0 and not fma:
            for f in STATE_FIELDS:
                res[f"state_{f}"] = r.get(f)
            time = r.begin_step(it)
            seq = [("BTRACK", r.btrack), ("PREPARE", lambda: r.prepare_elevation(time)),
                   ("ASSEMBLE", lambda: (r.assemble(time), r.essential_bc())), ("SOLVE", r.solve),
                   ("UPDATE_ELEV", r.update_elevation), ("MOMENTUM", lambda: r.momentum(time)),
                   ("VVEL", r.vertical_velocity), ("TRANSPORT", r.transport), ("LEVELS", lambda: r.levels(it)),
                   ("NODAL_VEL", r.nodal_velocities)]
            for ph, fn in seq:
                fn()
                for f in PHASE_OUT[ph] + (RHO_FIELDS if ph == "LEVELS" and c.ntracers >= 2 else ()):
                    res[f"phase_{ph}_{f}"] = r.get(f)
            cnt = r.counts()
        else:
            r.step(it)
            cnt = r.counts()
        res["iters"].append(cnt["jcg_iters"])
        res["substeps"].append(cnt["substeps"])
        if it in snaps:
            for f in fields:
                res[f"snap{it}_{f}"] = _cut(f, r.get(f), sub)
    res["iters"] = np.asarray(res["iters"], np.int32)
    res["substeps"] = np.asarray(res["substeps"], np.int32)
    if sub is not None:
        for k, v in sub.items():
            res[f"subset_{k}"] = v
    np.savez(out, **res)


def _rel(a, b):
    s = float(np.abs(b).max())
    return float(np.abs(a - b).max()) / (s if s > 0 else 1.0)


def make(name):
    with tempfile.TemporaryDirectory() as d:
        outs = {}
        for tag, ao, do, fm in (("base", 0, 0, 0), ("atomic", 1, 0, 0), ("dots", 0, 1, 0), ("fma", 0, 0, 1)):
            outs[tag] = os.path.join(d, f"{tag}.npz")
            subprocess.run([sys.executable, os.path.abspath(__file__), "--variant", name, str(ao), str(do), str(fm),
                            outs[tag]], check=True, stdout=subprocess.DEVNULL)
        base = dict(np.load(outs["base"]))
        var = [dict(np.load(outs[t])) for t in ("atomic", "dots", "fma")]
    c, nsteps, snaps, phase_step = step_cases()[name]
    if phase_step is not None:
        base["phase_step"] = np.int32(phase_step)
    fields = snap_fields(c)
    env = np.zeros((len(snaps), len(fields)))
    for i, s in enumerate(snaps):
        for j, f in enumerate(fields):
            key = f"snap{s}_{f}"
            env[i, j] = max(_rel(v[key], base[key]) for v in var)
    base["envelope"] = env
    base["envelope_fields"] = np.array(fields)
    base["snap_steps"] = np.asarray(snaps, np.int32)
    base["variant_iters"] = np.stack([v["iters"] for v in var])
    np.savez_compressed(os.path.join(HERE, f"step_{name}.npz"), **base)
    print(name, "steps", nsteps, "iters", base["iters"][:5], "...", "envelope at last snapshot:",
          {f: f"{env[-1, j]:.1e}" for j, f in enumerate(fields)})


def main(argv):
    if len(argv) >= 2 and argv[1] == "--variant":
        _run_variant(argv[2], int(argv[3]), int(argv[4]), int(argv[5]), argv[6])
        return
    names = argv[1:] or list(step_cases())
    for n in names:
        make(n)


if __name__ == "__main__":
    main(sys.argv)
