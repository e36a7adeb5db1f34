"""Slot-level admission on the GPU (gpu): a forecast admitted into a member slot of a running
context, at a step boundary, runs from its own step 1 and equals the same forecast run alone, bit
for bit; the forecast already running is not disturbed by the admission or by the slot's
retirement; a parked slot stays at rest without errors."""
import numpy as np
import pytest

from gschism_b200 import _lib as L
from gschism_b200 import cases

pytestmark = pytest.mark.gpu

CHECK = ("ETA2", "NODE_TR", "SIDE_U2", "ELEM_W", "NODE_U2", "SIDE_BTELEM", "NODE_KB", "ELEM_DRY")


def _same(m, k, solo):
    for f in CHECK:
        a, b = m.get(k, f), solo.get(0, f)
        assert np.array_equal(a, b), f"{f}: max diff {np.abs(a.astype(float) - b.astype(float)).max():.3e}"


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_member_admitted_mid_run_equals_its_solo_run(native, precision):
    from gschism_b200.model import Model
    a, va, _ = cases.storm(4, nmin=4000, nmax=4500, nvrt=10, dt=100.0, hours=1.0)   # already running
    b, _, _ = cases.storm(5, nmin=6000, nmax=6500, nvrt=10, dt=100.0, hours=1.0)
    vb = cases.storm_on(b, 11)
    solo_a = Model([a], precision=precision)
    solo_a.set_vortex(0, va)
    solo_b = Model([b], precision=precision)
    solo_b.set_tau(0, np.zeros(solo_b.shape(0, "NODE_TAU")))
    solo_b.set_vortex(0, vb)

    m = Model([a, b], precision=precision)
    m.set_vortex(0, va)
    cold = m.member_state(1, pinned=True)
    ref_cold = solo_b.member_state(0)
    for f in cold:                                               # a slot's cold start is the member's own
        assert np.array_equal(cold[f], ref_cold[f]), f
    m.park(1, cold)
    m.step(5)
    assert m.current_step() == 5
    assert np.abs(m.get(1, "ETA2")).max() == 0.0                 # parked: at rest
    assert np.abs(m.get(1, "SIDE_U2")).max() == 0.0
    assert m.stats(1)["error_flags"] == 0

    assert m.admit(1, cold, vortex=vb) == 5
    m.step(8)
    solo_b.step(8)
    solo_a.step(13)
    _same(m, 1, solo_b)
    _same(m, 0, solo_a)

    m.park(1, cold)                                              # retire the storm forecast
    m.step(3)
    solo_a.step(3)
    _same(m, 0, solo_a)
    assert np.abs(m.get(1, "ETA2")).max() == 0.0
    assert m.stats(1)["error_flags"] == 0 and m.stats(0)["error_flags"] == 0

    # the slot takes a second forecast: again its solo run
    solo_b2 = Model([b], precision=precision)
    solo_b2.set_tau(0, np.zeros(solo_b2.shape(0, "NODE_TAU")))
    v2 = cases.storm_on(b, 12)
    solo_b2.set_vortex(0, v2)
    assert m.admit(1, cold, vortex=v2) == 16
    m.step(4)
    solo_b2.step(4)
    _same(m, 1, solo_b2)
    for x in (m, solo_a, solo_b, solo_b2):
        x.close()


def _parked_beside_active(precision):
    """Eight storm members of ~10k nodes, the even ones parked (at rest: zero right-hand side,
    done before their first iteration), the odd ones forced; 32-row solver tiles, so ~2,600 tiles
    over the cooperative grid's blocks put several member boundaries inside a block."""
    from gschism_b200.model import Model
    cs = [cases.storm(20 + i, nmin=10000, nmax=10500, nvrt=10, dt=100.0, hours=1.0)[0] for i in range(8)]
    m = Model(cs, precision=precision)
    m.set_launch("JCG_TILES", 592, 32)
    for k in range(8):
        m.set_tau(k, np.zeros(m.shape(k, "NODE_TAU")))
        if k % 2 == 0:
            m.park(k, m.member_state(k))
        else:
            m.set_vortex(k, cases.storm_on(cs[k], 100 + k))
    return cs, m


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_retired_member_sharing_solver_blocks_with_an_active_one(native, precision):
    """Parked members whose solver tiles share blocks with active members' tiles: every active
    member's solve runs to convergence without a bounded wait running out (a block holding a
    finished member's tiles must not wait for that member's next iteration), and gives the bits
    of its solo run with the same tiling."""
    from gschism_b200.model import Model
    cs, m = _parked_beside_active(precision)
    solo = Model([cs[1]], precision=precision)
    solo.set_launch("JCG_TILES", 592, 32)
    solo.set_tau(0, np.zeros(solo.shape(0, "NODE_TAU")))
    solo.set_vortex(0, cases.storm_on(cs[1], 101))
    for _ in range(3):
        m.step(1)
        solo.step(1)
        m.sync()                                                 # GS_ERR_TIMEOUT if a wait ran out
        for k in range(8):
            st = m.stats(k)
            assert st["error_flags"] == 0, k
            assert (st["jcg_iters"] == 0) if k % 2 == 0 else (st["jcg_iters"] > 0), k
        assert m.stats(1)["jcg_iters"] == solo.stats(0)["jcg_iters"]
    _same(m, 1, solo)
    m.close()
    solo.close()


def test_members_of_one_context_share_the_vertical_grid(native):
    from gschism_b200.model import Model
    s, _, _ = cases.storm(4, nmin=4000, nmax=4500, nvrt=10, dt=100.0, hours=1.0)
    with pytest.raises(ValueError):
        Model([cases.channel(), s])


def test_member_start_rejects_bad_arguments(native):
    from gschism_b200.model import Model
    m = Model([cases.channel()])
    with pytest.raises(L.GsError):
        m.set_member_start(1, 0)
    with pytest.raises(L.GsError):
        m.set_member_start(0, -1)
    m.set_member_start(0, L.GS_MEMBER_PARKED)
    m.step(2)
    assert np.abs(m.get(0, "ETA2")).max() == 0.0                 # parked from the cold start: no tide
    m.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_slot_server_on_gpu(native, precision):
    """The slot server end to end on two small regions, with 32-row solver tiles so that parked
    and running slots share solver blocks: every forecast equals its solo run (same tiling)."""
    from gschism_b200.model import Model
    from gschism_b200.serve import SlotEngine, SlotServer, slot_requests
    regions = [cases.storm(7, nmin=9000, nmax=9500, nvrt=10, dt=100.0, hours=1.0)[0],
               cases.storm(8, nmin=12000, nmax=12500, nvrt=10, dt=100.0, hours=1.0)[0]]
    reqs = slot_requests(6, rate=200.0, seed=4, regions=regions, hours=0.25, dt=100.0)
    eng = SlotEngine(precision=precision, fields=("ETA2", "NODE_TR"), jcg_tiles=(592, 32))
    srv = SlotServer(eng, regions, 2, steps_per_turn=3)
    srv.run(reqs)
    for r in reqs:
        solo = Model([r.case], precision=precision)
        solo.set_launch("JCG_TILES", 592, 32)
        solo.set_tau(0, np.zeros(solo.shape(0, "NODE_TAU")))
        solo.set_vortex(0, r.vortex)
        solo.step(r.nsteps)
        assert np.array_equal(r.result["ETA2"], solo.get(0, "ETA2")), r.rid
        assert np.array_equal(r.result["NODE_TR"], solo.get(0, "NODE_TR")), r.rid
        solo.close()
