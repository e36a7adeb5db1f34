"""The CUDA path against the reference's own kernels (gpu; fixtures: tests/golden/make_step_golden.py).

Same checks as tests/test_ref_pinned.py, through the C ABI: per phase from the reference's state
(every phase's output within 1e-12 of the reference's, 1e-10 after the solve, whose reductions
run in another order; integer fields bit for bit), and whole trajectories from the cold start
(the 100-step channel, an SZ basin, a wind-driven member) within the reference's own
reproducibility envelope, with the reference's JCG iteration counts."""
import numpy as np
import pytest

from tests import _refpin as R
from tests.golden.make_step_golden import step_cases

pytestmark = pytest.mark.gpu

SOLVE_TOL = 1e-10


@pytest.mark.parametrize("name", ["channel", "basin16", "member"])
def test_cuda_trajectory_matches_reference(name, native):
    from gschism_b200.model import Model
    g = R.load(name)
    c, nsteps, _, _ = step_cases()[name]
    m = Model([c], precision="fp64")
    try:
        def step(it):
            m.step(1)
            return m.stats(0)["jcg_iters"]
        rows = R.check_trajectory(g, step, lambda f: m.get(0, f), nsteps)
    finally:
        m.close()
    worst = {}
    for it, f, e, tol in rows:
        worst[f] = max(worst.get(f, 0.0), e / tol)
    print(name, {f: round(v, 3) for f, v in worst.items()})


@pytest.mark.parametrize("name", ["basin16", "member"])
def test_cuda_phases_match_reference(name, native):
    from gschism_b200.model import Model
    g = R.load(name)
    c, _, _, _ = step_cases()[name]
    m = Model([c], precision="fp64")
    it = int(g["phase_step"])
    try:
        for f in R.state_fields(g):
            m.put(0, f, g[f"state_{f}"])
        m.phase("BEGIN", it)
        rows = _phases(g, m, it)
    finally:
        m.close()
    print(name, [(ph, f, f"{e:.1e}") for ph, f, e in rows])


def _phases(g, m, it):
    """Every phase after BEGIN; the fields after the solve are compared at SOLVE_TOL."""
    rows = []
    after_solve = False
    for ph in R.PHASES:
        m.phase(ph, it)
        if ph == "SOLVE":
            after_solve = True
        for key in [k for k in g if k.startswith(f"phase_{ph}_")]:
            f = key[len(f"phase_{ph}_"):]
            a, b = m.get(0, f), g[key]
            if f in R.INT_FIELDS:
                assert np.array_equal(a, b), f"{ph} {f} differs"
                continue
            e = R.rel(a, b)
            rows.append((ph, f, e))
            tol = SOLVE_TOL if after_solve else R.PHASE_TOL_FIELD.get(f, R.PHASE_TOL)
            assert e <= tol, f"{ph} {f}: rel err {e:.3e} > {tol:.1e}"
    return rows
