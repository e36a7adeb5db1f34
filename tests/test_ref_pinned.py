"""The CPU oracle against the reference's own kernels (fixtures: tests/golden/make_step_golden.py).

The fixtures come from the reference's src/kernels/meshdata.cu compiled for the host and driven in
the order of src/python/schism_step.py; these tests pin oracle/step.c, btrack.c and transport.c to
them: per phase from the reference's state (every phase's output within 1e-12, integer fields bit
for bit), and along whole trajectories from the cold start (within the reference's own
reproducibility envelope; equal JCG iteration counts)."""
import numpy as np
import pytest

from tests import _refpin as R
from tests.golden.make_step_golden import step_cases

CASES = ["channel", "basin16", "member"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_trajectory_matches_reference(name):
    from oracle.step_api import OracleModel
    g = R.load(name)
    c, nsteps, _, _ = step_cases()[name]
    o = OracleModel(c)
    rows = R.check_trajectory(g, o.step, o.get, nsteps)
    assert rows


@pytest.mark.parametrize("name", ["basin16", "member"])
def test_oracle_phases_match_reference(name):
    from oracle.step_api import OracleModel
    g = R.load(name)
    c, _, _, _ = step_cases()[name]
    p = c.params
    o = OracleModel(c)
    it = int(g["phase_step"])
    time = it * p.dt
    o.begin_step(it)
    run = {
        "BTRACK": o.btrack, "PREPARE": lambda: o.prepare_elevation(time),
        "ASSEMBLE": lambda: (o.assemble(time), o.essential_bc()),
        "SOLVE": lambda: o.jcg_solve(p.rtol, p.maxiter, p.check_every), "UPDATE_ELEV": o.update_elevation,
        "MOMENTUM": lambda: o.momentum(time), "VVEL": o.vertical_velocity, "TRANSPORT": lambda: o.transport(p.dt),
        "LEVELS": lambda: o.levels(it), "NODAL_VEL": o.nodal_velocities,
    }
    # put the state after begin_step: begin_step only sets forcing and ramps, no state field
    rows = R.check_phases(g, o.put, lambda ph: run[ph](), o.get)
    worst = max(e for _, _, e in rows)
    assert worst <= 1e-12


def test_reference_iteration_counts_are_order_independent():
    """The reference's JCG iteration counts do not move with the summation orders a GPU may use."""
    for name in CASES:
        g = R.load(name)
        assert (g["variant_iters"] == g["iters"][None, :]).all(), name
