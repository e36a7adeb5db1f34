"""CUDA path vs the CPU oracle (gpu).

Per phase: both sides start from the bit-identical state of the oracle after a few steps of the
10 km channel case (the state is copied into the GPU member in reference numbering), then run
the same phases of one step.  Integer outputs (backtracked element ids, bottom levels, wet/dry
flags) must match exactly; FP64 fields within the stated relative tolerances (the CUDA kernels
contract multiply-adds, the oracle does not; the JCG reductions use a different order).
"""
import numpy as np
import pytest

from gschism_b200 import cases
from tests._parity import copy_state, level_mask, relerr

pytestmark = pytest.mark.gpu

TOL_PHASE = 1e-12     # single phase from identical inputs (FMA contraction only)
TOL_SOLVE = 1e-10     # after the JCG solve (reduction order; rtol = 1e-12)


@pytest.fixture(scope="module")
def channel_pair(native, oracle_lib):
    from gschism_b200.model import Model
    from oracle.step_api import OracleModel
    c = cases.channel()
    o = OracleModel(c)
    o.run(4)
    g = Model([c])
    copy_state(o, g)
    return c, o, g


def test_phases_match_oracle_from_identical_state(channel_pair):
    c, o, g = channel_pair
    it = 5
    dt = c.params.dt
    nv = c.nvrt
    # backtracking first: inputs bit-identical, element ids must match exactly
    o.begin_step(it); g.phase("BEGIN", it)
    o.btrack(); g.phase("BTRACK", it)
    assert np.array_equal(g.get(0, "SIDE_BTELEM"), o.get("SIDE_BTELEM"))
    assert relerr(g.get(0, "SIDE_BTU"), o.get("SIDE_BTU")) <= TOL_PHASE
    n_walks = int((o.get("SIDE_BTELEM") >= 0).sum())
    assert n_walks > 1000
    o.prepare_elevation(it * dt); g.phase("PREPARE", it)
    assert relerr(g.get(0, "ELBC"), o.get("ELBC")) <= 1e-14
    assert relerr(g.get(0, "SIDE_U"), o.get("SIDE_U")) <= TOL_PHASE
    assert relerr(g.get(0, "SIDE_HHAT"), o.get("SIDE_HHAT")) <= TOL_PHASE
    assert relerr(g.get(0, "ELEM_GHAT"), o.get("ELEM_GHAT")) <= TOL_PHASE
    o.assemble(it * dt); o.essential_bc(); g.phase("ASSEMBLE", it)
    assert np.array_equal(g.get(0, "CSR_INDPTR"), o.get("CSR_INDPTR"))
    assert np.array_equal(g.get(0, "CSR_INDICES"), o.get("CSR_INDICES"))
    assert relerr(g.get(0, "CSR_DATA"), o.get("CSR_DATA")) <= TOL_PHASE
    assert relerr(g.get(0, "QEL"), o.get("QEL")) <= TOL_PHASE
    its_o, _ = o.jcg_solve(c.params.rtol, c.params.maxiter, c.params.check_every)
    g.phase("SOLVE", it)
    assert g.stats(0)["jcg_iters"] == its_o
    o.update_elevation(); g.phase("UPDATE_ELEV", it)
    assert relerr(g.get(0, "ETA2"), o.get("ETA2")) <= TOL_SOLVE
    assert np.array_equal(g.get(0, "NODE_KB"), o.get("NODE_KB"))
    # continue from the oracle's solution so the later phases again see identical inputs
    copy_state(o, g)
    o.momentum(it * dt); g.phase("MOMENTUM", it)
    assert relerr(g.get(0, "SIDE_U2"), o.get("SIDE_U2")) <= TOL_PHASE
    assert relerr(g.get(0, "SIDE_GRADETA2"), o.get("SIDE_GRADETA2")) <= TOL_PHASE
    o.vertical_velocity(); g.phase("VVEL", it)
    kbe = o.get("ELEM_KB")
    assert relerr(g.get(0, "ELEM_W"), o.get("ELEM_W")) <= 1e-11
    assert relerr(g.get(0, "ELEM_QV"), o.get("ELEM_QV"), level_mask(kbe, nv)) <= 1e-11
    o.transport(dt); g.phase("TRANSPORT", it)
    assert g.stats(0)["transport_substeps"] == o.counters()[1]
    assert relerr(g.get(0, "SIDE_QH"), o.get("SIDE_QH")) <= TOL_PHASE
    assert relerr(g.get(0, "ELEM_TR"), o.get("ELEM_TR")) <= TOL_PHASE
    assert relerr(g.get(0, "NODE_TR"), o.get("NODE_TR")) <= TOL_PHASE
    o.levels(it); g.phase("LEVELS", it)
    for f in ("NODE_KB", "NODE_DRY", "ELEM_KB", "ELEM_DRY", "SIDE_KB", "SIDE_DRY"):
        assert np.array_equal(g.get(0, f), o.get(f)), f
    kb = o.get("NODE_KB")
    assert relerr(g.get(0, "NODE_Z"), o.get("NODE_Z"), level_mask(kb, nv)) <= TOL_PHASE
    assert relerr(g.get(0, "ELEM_Z"), o.get("ELEM_Z"), level_mask(o.get("ELEM_KB"), nv)) <= TOL_PHASE
    assert relerr(g.get(0, "SIDE_ZC"), o.get("SIDE_ZC"), level_mask(o.get("SIDE_KB"), nv)) <= TOL_PHASE
    o.nodal_velocities(); g.phase("NODAL_VEL", it)
    assert relerr(g.get(0, "NODE_U2"), o.get("NODE_U2")) <= TOL_PHASE
    assert relerr(g.get(0, "NODE_W2"), o.get("NODE_W2")) <= 1e-11


def test_btrack_ids_bit_exact_on_basin(native, oracle_lib):
    """SZ levels, irregular bathymetry: every backtracked element id equals the oracle's."""
    from gschism_b200.model import Model
    from oracle.step_api import OracleModel
    c = cases.basin(seed=9, n=48, nvrt=12, nz=4, ntr=1, length=48e3, amp=1.5)
    o = OracleModel(c)
    o.run(3)
    g = Model([c])
    copy_state(o, g)
    o.begin_step(4); g.phase("BEGIN", 4)
    o.btrack(); g.phase("BTRACK", 4)
    ids = o.get("SIDE_BTELEM")
    assert (ids >= 0).sum() > 10000
    assert np.array_equal(g.get(0, "SIDE_BTELEM"), ids)
    assert relerr(g.get(0, "SIDE_BTU"), o.get("SIDE_BTU")) <= TOL_PHASE


def test_multistep_channel_fp64(native, oracle_lib):
    """Whole steps through gs_step against og_step: the channel configuration's full 100 steps.
    Elevation and tracers stay within 1e-10 relative at steps 30 and 100; velocities within 1e-8.  The 1e-10 velocity target is not reachable
    over a trajectory by any implementation whose sums run in another order than one particular
    run of the reference: the reference's own kernels, run twice with only their atomic sums or
    their solver dot products in another order, drift apart to 1e-9 (horizontal) and 2e-8
    (vertical) over 100 steps of this channel (tests/golden/step_channel.npz, envelope).  From an
    identical state every phase meets 1e-12 (test_phases_match_oracle_from_identical_state and
    tests/test_gpu_ref_pinned.py)."""
    from gschism_b200.model import Model
    from oracle.step_api import OracleModel
    c = cases.channel(seed=3)
    o = OracleModel(c)
    g = Model([c])
    done = 0
    for n in (30, 100):
        its_o = o.run(n - done, start=done + 1)
        g.step(n - done)
        done = n
        assert relerr(g.get(0, "ETA2"), o.get("ETA2")) <= 1e-10, n
        assert relerr(g.get(0, "SIDE_U2"), o.get("SIDE_U2")) <= 1e-8, n
        assert relerr(g.get(0, "ELEM_TR"), o.get("ELEM_TR")) <= 1e-10, n
        assert relerr(g.get(0, "NODE_TR"), o.get("NODE_TR")) <= 1e-10, n
        assert abs(g.stats(0)["jcg_iters"] - its_o[-1]) <= c.params.check_every, n


def test_batch_members_independent_of_the_mix(native):
    """Each member's state after several steps is bit-identical alone and inside a batch."""
    from gschism_b200.model import Model
    a = cases.channel(seed=11, nx=40, ny=21, nvrt=10)
    b = cases.channel(seed=12, nx=63, ny=32, nvrt=10)
    d = cases.channel(seed=13, nx=25, ny=17, nvrt=10)
    mix = Model([a, b, d])
    mix.step(6)
    for k, c in enumerate([a, b, d]):
        alone = Model([c])
        alone.step(6)
        for f in ("ETA2", "SIDE_U2", "ELEM_TR", "NODE_U2"):
            assert np.array_equal(mix.get(k, f), alone.get(0, f)), (k, f)
        assert mix.stats(k)["jcg_iters"] == alone.stats(0)["jcg_iters"]
        alone.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_basin_62k_nodes_against_oracle(native, oracle_lib, precision):
    """A 250 x 250 basin (62,500 nodes, 8 levels): a member of many solver tiles, renumbered along
    a Hilbert curve whose first and last quadrants share an edge (rows there gather columns
    31,000-62,000 rows away).  Both precisions against the FP64 oracle over 3 steps."""
    from gschism_b200.model import Model
    from oracle.step_api import OracleModel
    c = cases.basin(seed=5, n=250, nvrt=8, nz=3, ntr=1, length=125e3)
    o = OracleModel(c)
    g = Model([c], precision=precision)
    its_o = o.run(3)
    g.step(3)
    if precision == "fp64":
        assert relerr(g.get(0, "ETA2"), o.get("ETA2")) <= 1e-10
        assert abs(g.stats(0)["jcg_iters"] - its_o[-1]) <= c.params.check_every
    else:
        assert np.abs(g.get(0, "ETA2") - o.get("ETA2")).max() <= 1e-6
    assert relerr(g.get(0, "ELEM_TR"), o.get("ELEM_TR")) <= 1e-8
    g.close()


def test_mixed_precision_elevation_within_1e6_m(native, oracle_lib):
    """FP32 inner JCG with FP64 refinement: elevation within 1e-6 m of the FP64 oracle."""
    from gschism_b200.model import Model
    from oracle.step_api import OracleModel
    c = cases.channel(seed=4)
    o = OracleModel(c)
    g = Model([c], precision="fp32_ir")
    n = 20
    o.run(n)
    g.step(n)
    err = np.abs(g.get(0, "ETA2") - o.get("ETA2")).max()
    assert err <= 1e-6, err
    st = g.stats(0)
    assert st["jcg_outer"] >= 1


def test_graph_step_equals_phase_by_phase(native):
    """gs_step (one captured step replayed as a CUDA graph) gives the same bits as the same
    steps issued phase by phase, also across a recapture when storm forcing switches on."""
    from gschism_b200.model import Model
    c, v, _ = cases.storm(41, nmin=2500, nmax=2500, hours=1.0)
    a, b = Model([c]), Model([c])
    phases = ["BTRACK", "PREPARE", "ASSEMBLE", "SOLVE", "UPDATE_ELEV", "MOMENTUM", "VVEL", "TRANSPORT",
              "LEVELS", "NODAL_VEL"]

    def by_phase(m, it):
        m.phase("BEGIN", it)
        for ph in phases:
            m.phase(ph, it)

    a.step(3)
    for it in range(1, 4):
        by_phase(b, it)
    a.set_vortex(0, v)
    b.set_vortex(0, v)
    a.step(3)
    for it in range(4, 7):
        by_phase(b, it)
    for f in ("ETA2", "SIDE_U2", "ELEM_TR", "NODE_TAU"):
        assert np.array_equal(a.get(0, f), b.get(0, f)), f


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_member_at_rest_beside_a_forced_one(native, precision):
    """A member without forcing (zero right-hand side: retired before the first iteration) in the
    same batch as a forced member: the solve ends, the resting member stays at rest and the forced
    one gets the same bits as alone."""
    from gschism_b200.model import Model
    rest = cases.channel(seed=51, nx=30, ny=16)
    rest.emo = [np.zeros_like(a) for a in rest.emo]
    rest.tau = np.zeros_like(rest.tau)
    forced = cases.channel(seed=52, nx=40, ny=21)
    mix = Model([rest, forced], precision=precision)
    mix.step(3)
    mix.sync()
    assert mix.stats(0)["jcg_iters"] == 0
    assert mix.stats(0)["error_flags"] == 0
    assert np.all(mix.get(0, "ETA2") == 0.0)
    alone = Model([forced], precision=precision)
    alone.step(3)
    assert np.array_equal(mix.get(1, "ETA2"), alone.get(0, "ETA2"))
    assert mix.stats(1)["jcg_iters"] == alone.stats(0)["jcg_iters"]


def test_transport_members_with_different_substep_counts(native):
    """Members of one batch that need different numbers of transport sub-steps (one many, one a
    single sub-step): the sub-cycling ends, and each member's tracers equal those of the same
    member alone (a member that finished early must stay finished)."""
    from gschism_b200.model import Model
    a = cases.channel(seed=61, nx=30, ny=16)
    b = cases.channel(seed=62, nx=40, ny=21)
    for c in (a, b):
        c.params.dramp = 0.0              # full tide from the first step: real flow by step 3
    before = ["BTRACK", "PREPARE", "ASSEMBLE", "SOLVE", "UPDATE_ELEV", "MOMENTUM", "VVEL"]

    def third_step(m, scaled):
        m.step(2)
        m.phase("BEGIN", 3)
        for ph in before:
            m.phase(ph, 3)
        for k in scaled:                      # 50x the fluxes: many more transport sub-steps
            qh = m.get(k, "SIDE_QH")
            m.put(k, "SIDE_QH", np.where(qh > -1e30, 50.0 * qh, qh))
        m.phase("TRANSPORT", 3)
        m.sync()

    mix = Model([a, b])
    third_step(mix, [0])
    alone_a, alone_b = Model([a]), Model([b])
    third_step(alone_a, [0])
    third_step(alone_b, [])
    assert mix.stats(0)["transport_substeps"] >= 3
    assert mix.stats(1)["transport_substeps"] == 1
    assert np.array_equal(mix.get(0, "ELEM_TR"), alone_a.get(0, "ELEM_TR"))
    assert np.array_equal(mix.get(1, "ELEM_TR"), alone_b.get(0, "ELEM_TR"))
