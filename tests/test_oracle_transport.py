"""Transport options of the CPU oracle (no GPU): the TVD scheme with limiter 0 is the upwind
scheme, every limiter keeps tracers within their initial bounds, and the implicit vertical
diffusion conserves tracer mass when nothing moves."""
import dataclasses

import numpy as np
import pytest

from gschism_b200 import cases


def _run(case, nsteps):
    from oracle.step_api import OracleModel
    o = OracleModel(case)
    for it in range(1, nsteps + 1):
        o.step(it)
    return o


def _with(case, **kw):
    case.params = dataclasses.replace(case.params, **kw)
    return case


def test_tvd_without_limiter_is_upwind(oracle_lib):
    up = _run(cases.channel(), 6)
    tv = _run(_with(cases.channel(), itr_met=3, tvd_limiter=0), 6)
    assert np.array_equal(up.get("ELEM_TR"), tv.get("ELEM_TR"))
    assert np.array_equal(up.get("NODE_TR"), tv.get("NODE_TR"))


@pytest.mark.parametrize("limiter", [1, 2, 3, 4])
def test_tvd_keeps_tracers_within_bounds(oracle_lib, limiter):
    c = cases.transport_stress(n=40, nvrt=12, ntr=3, limiter=limiter, tau_mag=0.3)
    from oracle.step_api import OracleModel
    o = OracleModel(c)
    tr0 = o.get("ELEM_TR")
    lo, hi = tr0.min(), tr0.max()
    up = _run(_with(cases.transport_stress(n=40, nvrt=12, ntr=3, tau_mag=0.3), tvd_limiter=0), 8)
    for it in range(1, 9):
        o.step(it)
    tr = o.get("ELEM_TR")
    assert tr.min() >= lo - 1e-12 and tr.max() <= hi + 1e-12
    # a limiter adds anti-diffusive flux: the result differs from first order
    assert np.abs(tr - up.get("ELEM_TR")).max() > 1e-9


def test_vertical_diffusion_conserves_mass_at_rest(oracle_lib):
    c = cases.transport_stress(n=30, nvrt=12, ntr=2, tau_mag=0.0, dfh0=1e-2)
    from oracle.step_api import OracleModel
    o = OracleModel(c)
    m0 = o.tracer_mass()
    tr0 = o.get("ELEM_TR")
    for it in range(1, 6):
        o.step(it)
    m1 = o.tracer_mass()
    assert np.abs(o.get("ELEM_TR") - tr0).max() > 1e-6          # the columns mix
    assert np.all(np.abs(m1 - m0) <= 1e-13 * np.abs(m0))
