"""Connectivity against golden vectors produced by the reference's own grid reader
(src/grid/read_and_process_grid.cpp readHGrid/readVGrid; fixtures made by tests/golden/make_golden.py)."""
import ctypes
import os

import numpy as np
import pytest

from gschism_b200 import cases
from tests.golden.make_golden import golden_cases

GOLD = os.path.join(os.path.dirname(__file__), "golden")
NAMES = ["channel", "basin24", "tiny"]


def _gold(name):
    return dict(np.load(os.path.join(GOLD, f"grid_{name}.npz")))


@pytest.fixture(scope="module")
def gcases():
    return golden_cases()


@pytest.mark.parametrize("name", NAMES)
def test_oracle_connectivity_matches_reference(name, gcases, oracle_lib):
    from oracle import oracle as O
    g = _gold(name)
    c = gcases[name]
    isb = O.grid_isbnd(c.n_nodes, c.open_bnd, c.land_bnd)
    assert np.array_equal(isb, g["isbnd"])
    o = O.grid_build(c.elnode, c.n_nodes, isb)
    assert np.array_equal(o["nne"], g["nodeNeighElems_data"])
    assert np.array_equal(o["nne_start"], g["nodeNeighElems_start"])
    assert np.array_equal(o["nnp"], g["nodeNeighNodes_data"])
    assert np.array_equal(o["nnp_start"], g["nodeNeighNodes_start"])
    assert np.array_equal(o["elside"].T, g["elside"])
    assert np.array_equal(o["ic3"].T, g["ic3"])
    assert np.array_equal(o["isdel"].T, g["isdel"])
    assert np.array_equal(o["isidenode"].T, g["isidenode"])


@pytest.mark.parametrize("name", NAMES)
def test_product_connectivity_matches_reference(name, gcases, native):
    from gschism_b200 import _lib as L
    from oracle import oracle as O
    g = _gold(name)
    c = gcases[name]
    ne, np_ = c.n_elems, c.n_nodes
    el4 = np.full((ne, 4), -1, np.int32)
    el4[:, :3] = c.elnode
    i34 = np.full(ne, 3, np.int32)
    isb = np.ascontiguousarray(g["isbnd"], dtype=np.int32)
    out = [np.zeros(np_ + 1, np.int32), np.zeros(4 * ne, np.int32), np.zeros(np_ + 1, np.int32),
           np.zeros(4 * ne + np_, np.int32), np.zeros(4 * ne, np.int32), np.zeros(4 * ne, np.int32),
           np.zeros(8 * ne, np.int32), np.zeros(8 * ne, np.int32), np.zeros(1, np.int32)]
    P = lambda a: a.ctypes.data_as(L.PI)
    el = np.ascontiguousarray(el4.ravel())
    assert native.gs_grid_build(np_, ne, P(el), P(i34), P(isb), *[P(a) for a in out]) == 0
    ns = int(out[8][0])
    assert ns == g["isdel"].shape[1]
    assert np.array_equal(out[1][:out[0][-1]], g["nodeNeighElems_data"])
    assert np.array_equal(out[3][:out[2][-1]], g["nodeNeighNodes_data"])
    assert np.array_equal(out[5].reshape(ne, 4).T, g["elside"])
    assert np.array_equal(out[4].reshape(ne, 4).T, g["ic3"])
    assert np.array_equal(out[6][:2 * ns].reshape(ns, 2).T, g["isdel"])
    assert np.array_equal(out[7][:2 * ns].reshape(ns, 2).T, g["isidenode"])


@pytest.mark.parametrize("name", NAMES)
def test_vgrid_matches_reference(name, gcases):
    g = _gold(name)
    vg = gcases[name].vgrid
    assert list(g["vgrid_ints"]) == [2, vg.nvrt, vg.nz, vg.nsiglev]
    np.testing.assert_array_equal(g["vgrid_ztot"][:vg.nz], vg.ztot)
    np.testing.assert_array_equal(g["vgrid_params"], [vg.h_c, vg.h_s, vg.theta_b, vg.theta_f])
    np.testing.assert_array_equal(g["vgrid_sigma"][:vg.nsiglev], vg.sigma)
    np.testing.assert_allclose(g["vgrid_cs"][:vg.nsiglev], vg.cs(), rtol=0, atol=1e-15)


def test_product_rejects_broken_mesh(native):
    from gschism_b200 import _lib as L
    c = cases.channel(nx=6, ny=5, nvrt=4, shuffle=False)
    el = c.elnode.copy()
    el[0] = el[0][::-1]                      # flip one triangle: opposite orientation
    ne, np_ = el.shape[0], c.n_nodes
    el4 = np.full((ne, 4), -1, np.int32); el4[:, :3] = el
    i34 = np.full(ne, 3, np.int32)
    from oracle import oracle as O
    isb = O.grid_isbnd(np_, c.open_bnd, c.land_bnd)
    out = [np.zeros(np_ + 1, np.int32), np.zeros(4 * ne, np.int32), np.zeros(np_ + 1, np.int32),
           np.zeros(4 * ne + np_, np.int32), np.zeros(4 * ne, np.int32), np.zeros(4 * ne, np.int32),
           np.zeros(8 * ne, np.int32), np.zeros(8 * ne, np.int32), np.zeros(1, np.int32)]
    P = lambda a: a.ctypes.data_as(L.PI)
    assert native.gs_grid_build(np_, ne, P(np.ascontiguousarray(el4.ravel())), P(i34), P(isb),
                                *[P(a) for a in out]) == L.GS_ERR_BAD_MESH


@pytest.mark.parametrize("name", NAMES)
def test_readhgrid_shim_matches_reference_tuple(name, gcases, tmp_path, native):
    """gschism_b200.grid.readHGrid returns the reference's tuple on the same hgrid.gr3."""
    from gschism_b200 import grid
    g = _gold(name)
    c = gcases[name]
    cases.write_case(c, str(tmp_path))
    out = grid.readHGrid(str(tmp_path / "hgrid.gr3"), "", 1, 0)
    names = ["i34", "partElements", "partNodes", "partSides", "elnode", "elside", "nodeCoords", "nodeCoords_ll",
             "ic3", "isdel", "isidenode", "isbnd", "nond", "nlnd", "iond", "ilnd"]
    for k, nm in enumerate(names):
        if nm == "nodeCoords_ll":
            continue
        np.testing.assert_array_equal(np.asarray(out[k]), g[nm], err_msg=nm)
    for k, nm in ((16, "nodeNeighElems"), (17, "nodeNeighNodes")):
        np.testing.assert_array_equal(out[k][0], g[nm + "_data"])
        np.testing.assert_array_equal(out[k][1], g[nm + "_start"])
    v = grid.readVGrid(str(tmp_path / "vgrid.in"), c.n_nodes)
    np.testing.assert_array_equal(v[0], g["vgrid_ints"])
    np.testing.assert_array_equal(v[1], g["vgrid_ztot"])
    np.testing.assert_array_equal(v[3], g["vgrid_params"])
    np.testing.assert_array_equal(v[5], g["vgrid_sigma"])
    np.testing.assert_allclose(v[6], g["vgrid_cs"], rtol=0, atol=1e-15)
