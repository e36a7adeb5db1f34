"""Known-answer tests of the CPU oracle (no reference golden vectors exist for the step).

* lake at rest: no forcing -> elevation and velocities stay exactly zero, tracers unchanged;
* uniform flow: with a spatially uniform horizontal velocity and w = 0, backtracking from a side
  centre lands at x0 - dt*u and returns u;
* closed basin with wind: no open boundary -> the elevation integral stays zero to rounding.
"""
import numpy as np
import pytest

from gschism_b200 import cases


@pytest.fixture(scope="module")
def lib(oracle_lib):
    return oracle_lib


def _still(c):
    c.emo = [np.zeros_like(e) for e in c.emo]
    c.tau = np.zeros_like(c.tau)
    return c


def test_lake_at_rest(lib):
    from oracle.step_api import OracleModel
    c = _still(cases.channel(nx=20, ny=12, nvrt=6))
    o = OracleModel(c)
    tr0 = o.get("ELEM_TR")
    o.run(5)
    assert np.all(o.get("ETA2") == 0.0)
    assert np.all(o.get("SIDE_U2") == 0.0)
    assert np.array_equal(o.get("ELEM_TR"), tr0)


def test_uniform_flow_backtracking(lib):
    from oracle.step_api import OracleModel
    c = _still(cases.channel(nx=30, ny=16, nvrt=5, shuffle=False))
    o = OracleModel(c)
    u = np.array([0.05, 0.02])
    nv = c.nvrt
    o.put("NODE_U2", np.broadcast_to(u, (nv, o.np, 2)).copy())
    o.put("NODE_W2", np.zeros((nv, o.np)))
    o.put("SIDE_U2", np.broadcast_to(u, (nv, o.ns, 2)).copy())
    o.begin_step(1)
    o.btrack()
    btu = o.get("SIDE_BTU")
    ids = o.get("SIDE_BTELEM")
    walked = ids >= 0
    assert walked.sum() > 0.8 * walked.size
    np.testing.assert_allclose(btu[walked], np.broadcast_to(u, btu.shape)[walked], rtol=0, atol=1e-14)
    # foot points of interior sides: x0 - dt*u lies inside the element reported by the walk
    sc = None
    x, y, el = c.x, c.y, c.elnode
    from oracle import oracle as O
    isb = O.grid_isbnd(c.n_nodes, c.open_bnd, c.land_bnd)
    g = O.grid_build(c.elnode, c.n_nodes, isb)
    mid = 0.5 * (x[g["isidenode"][:, 0]] + x[g["isidenode"][:, 1]]), 0.5 * (y[g["isidenode"][:, 0]] + y[g["isidenode"][:, 1]])
    foot = mid[0] - c.params.dt * u[0], mid[1] - c.params.dt * u[1]
    k = nv - 1
    inside_domain = (foot[0] > 1.0) & (foot[0] < 9999.0) & (foot[1] > 1.0) & (foot[1] < 4999.0)
    sel = np.where(walked[k] & inside_domain)[0][:500]
    for s in sel:
        e = ids[k, s]
        a, b, d = el[e]
        px, py = foot[0][s], foot[1][s]

        def cr(i, j):
            return (x[j] - x[i]) * (py - y[i]) - (y[j] - y[i]) * (px - x[i])
        assert min(cr(a, b), cr(b, d), cr(d, a)) >= -1e-6
    del sc


def test_closed_basin_volume(lib):
    from oracle.step_api import OracleModel
    c = cases.channel(nx=24, ny=14, nvrt=6, shuffle=False)
    # close the open boundary: one land loop, wind stress drives the flow
    land = np.concatenate([c.land_bnd[0], c.open_bnd[0][1:]])
    c.land_bnd = [land]
    c.open_bnd = []
    c.iettype = np.zeros(0, np.int64)
    c.emo, c.efa = [], []
    c.tau = np.broadcast_to(np.array([2e-4, 1e-4]), c.tau.shape).copy()
    o = OracleModel(c)
    o.run(10)
    eta = o.get("ETA2")
    assert np.abs(eta).max() > 1e-6          # the wind moved the surface
    from oracle import oracle as O
    isb = O.grid_isbnd(c.n_nodes, c.open_bnd, c.land_bnd)
    assert (isb >= 0).sum() == 0
    # mass matrix lumped: sum of nodal eta weighted by their patch areas ~ 0
    x, y, el = c.x, c.y, c.elnode
    area = 0.5 * np.abs((x[el[:, 1]] - x[el[:, 0]]) * (y[el[:, 2]] - y[el[:, 0]])
                        - (x[el[:, 2]] - x[el[:, 0]]) * (y[el[:, 1]] - y[el[:, 0]]))
    vol = sum((area * eta[el[:, j]]).sum() for j in range(3)) / 3.0
    assert abs(vol) <= 1e-6 * area.sum() * np.abs(eta).max()
