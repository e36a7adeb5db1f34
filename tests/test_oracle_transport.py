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


def _upwind_column(c, nu):
    """Implicit upwind of one column of equal prisms under a uniform upward flux with Courant
    number nu, in the reference's inflow-only form (closed bottom and top)."""
    out = np.empty_like(c)
    out[0] = c[0]
    for j in range(1, len(c)):
        out[j] = (c[j] + nu * out[j - 1]) / (1.0 + nu)
    return out


@pytest.mark.parametrize("nu,steps", [(0.2, 20), (0.5, 8), (3.0, 2)])
def test_fct_column_bounded_conservative_and_sharper(oracle_lib, nu, steps):
    """The flux-corrected vertical step (itr_met = 4) on a step profile carried upward: the
    correction keeps the field in [0, 1], leaves the column's mass that of the upwind solve, and
    lands closer to the exact translated profile than implicit upwind alone."""
    from oracle.step_api import fct_column
    n = 40
    c0 = (np.arange(n) < 8).astype(float)
    up, fc = c0.copy(), c0.copy()
    for _ in range(steps):
        up = _upwind_column(up, nu)
        cl = _upwind_column(fc, nu)
        fc = fct_column(nu, np.ones(n - 1), np.ones(n), fc, cl)
        assert abs(fc.sum() - cl.sum()) <= 1e-14 * cl.sum()
        assert fc.min() >= 0.0 and fc.max() <= 1.0
    x = np.arange(n)
    exact = np.clip(8 + nu * steps - x, 0.0, 1.0)
    keep = x < 30                               # away from the closed top
    e_up, e_fc = np.abs(up - exact)[keep].sum(), np.abs(fc - exact)[keep].sum()
    assert e_fc < (0.95 if nu > 1 else 0.8) * e_up, (e_fc, e_up)


def test_fct_column_leaves_uniform_and_monotone_fields(oracle_lib):
    from oracle.step_api import fct_column
    rng = np.random.default_rng(3)
    n = 12
    q = rng.normal(size=n - 1)
    v = rng.uniform(0.5, 2.0, n)
    flat = np.full(n, 0.7)
    assert np.array_equal(fct_column(50.0, q, v, flat, flat), flat)
    # any field: the result stays within the bounds of the prism, its neighbours, before and after
    co, cl = rng.uniform(size=n), rng.uniform(size=n)
    out = fct_column(50.0, q, v, co, cl)
    both = np.stack([co, cl])
    lo = np.array([both[:, max(i - 1, 0):i + 2].min() for i in range(n)])
    hi = np.array([both[:, max(i - 1, 0):i + 2].max() for i in range(n)])
    assert np.all(out >= lo - 1e-15) and np.all(out <= hi + 1e-15)
    assert abs((v * out).sum() - (v * cl).sum()) <= 1e-14 * (v * cl).sum()


def test_vertical_fct_in_the_step(oracle_lib):
    """itr_met = 4 against itr_met = 3 on the wind-driven closed basin: one step from the same
    state changes the tracers but not their mass (the correction is column-conservative), and the
    tracers stay within their initial bounds over 10 steps."""
    from oracle.step_api import OracleModel

    def mk(itr):
        return OracleModel(_with(cases.transport_stress(n=30, nvrt=12, ntr=2, tau_mag=0.3), itr_met=itr))

    tv, fc = mk(3), mk(4)
    tr0 = tv.get("ELEM_TR")
    lo, hi = tr0.min(), tr0.max()
    tv.step(1)
    fc.step(1)
    assert np.abs(fc.get("ELEM_TR") - tv.get("ELEM_TR")).max() > 1e-7
    assert np.all(np.abs(fc.tracer_mass() - tv.tracer_mass()) <= 1e-14 * np.abs(tv.tracer_mass()))
    for it in range(2, 11):
        fc.step(it)
    tr = fc.get("ELEM_TR")
    assert tr.min() >= lo - 1e-12 and tr.max() <= hi + 1e-12
