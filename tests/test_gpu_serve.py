"""Storm forcing and the serving loop on the GPU.

* the device's vortex stress equals the oracle's (same formula, gs_set_vortex vs og_set_vortex)
* storm steps on the GPU (FP64) match the oracle within the step-parity tolerances
* served forecasts are bit-identical to the same requests run alone, whatever the cohorts
"""
import numpy as np
import pytest

from gschism_b200 import cases

from tests._parity import relerr

pytestmark = pytest.mark.gpu


def _storm(seed, n=2500, steps=6):
    c, v, _ = cases.storm(seed, nmin=n, nmax=n, hours=steps * 150.0 / 3600.0)
    # a storm centred on the domain, so the stress is strong everywhere in a few steps
    L = c.x.max()
    v.update(x0=0.5 * L, y0=0.5 * L, rmax=0.3 * L)
    return c, v, steps


def test_vortex_stress_matches_oracle(native, oracle_lib):
    from gschism_b200.model import Model
    from oracle.step_api import OracleModel
    c, v, _ = _storm(21)
    g = Model([c])
    g.set_vortex(0, v)
    g.phase("BEGIN", 40)
    g.phase("BTRACK", 40)
    g.phase("PREPARE", 40)
    o = OracleModel(c)
    o.set_vortex(v)
    o.L.og_begin_step(o.h, 40)
    tg, to = g.get(0, "NODE_TAU"), o.get("NODE_TAU")
    assert np.abs(to).max() > 1e-6
    assert relerr(tg, to) <= 1e-13


def test_storm_steps_match_oracle(native, oracle_lib):
    from gschism_b200.model import Model
    from oracle.step_api import OracleModel
    c, v, n = _storm(22)
    g = Model([c])
    g.set_vortex(0, v)
    o = OracleModel(c)
    o.set_vortex(v)
    o.run(n)
    g.step(n)
    assert relerr(g.get(0, "ETA2"), o.get("ETA2")) <= 1e-10
    assert relerr(g.get(0, "SIDE_U2"), o.get("SIDE_U2")) <= 1e-8
    # switching the storm off restores the member's own stress
    g.set_vortex(0, None)
    assert np.array_equal(g.get(0, "NODE_TAU"), c.tau)


def test_served_forecasts_equal_alone(native):
    from gschism_b200.model import Model, footprint_bytes
    from gschism_b200.serve import ModelEngine, Request, Server, summary
    reqs = []
    for i, (seed, n) in enumerate([(31, 1800), (32, 3000), (33, 2200), (34, 2600)]):
        c, v, steps = _storm(seed, n=n, steps=10)
        reqs.append(Request(rid=i, case=c, nsteps=steps, vortex=v, arrival=0.02 * i))
    # room for about two requests at a time: later ones wait for memory and form new cohorts
    budget = footprint_bytes([reqs[1].case, reqs[3].case]) + 1
    eng = ModelEngine(precision="fp32_ir")
    srv = Server(eng, budget_bytes=budget, steps_per_turn=3)
    srv.run(reqs)
    assert len({r.cohort for r in reqs}) >= 2
    assert srv.peak_used <= budget
    for r in reqs:
        m = Model([r.case], precision="fp32_ir")
        m.set_vortex(0, r.vortex)
        m.step(r.nsteps)
        assert np.array_equal(r.result["ETA2"], m.get(0, "ETA2")), r.rid
        m.close()
    s = summary(reqs, max(r.finished for r in reqs))
    assert s["ttf_p99_s"] >= s["ttf_p50_s"] > 0


def test_footprint_bounds_a_tvd_fct_context(native):
    """The bound includes the TVD and vertical-FCT scratch arrays (itr_met = 4)."""
    import dataclasses
    import torch
    from gschism_b200.model import Model, footprint_bytes
    c = cases.transport_stress(n=150, nsteps=10)
    c.params = dataclasses.replace(c.params, itr_met=4)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    m = Model([c])
    m.sync()
    used = free0 - torch.cuda.mem_get_info()[0]
    est = footprint_bytes([c])
    m.close()
    assert used <= est


def test_footprint_bounds_the_allocation(native):
    import torch
    from gschism_b200.model import Model, footprint_bytes
    ens = cases.ensemble(n_members=3, nmin=20_000, nmax=60_000)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    m = Model(ens)
    m.sync()
    used = free0 - torch.cuda.mem_get_info()[0]
    est = footprint_bytes(ens)
    m.close()
    assert used <= est <= 2.0 * used + 512 * 2**20
