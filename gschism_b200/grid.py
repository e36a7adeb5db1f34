"""Grid entry points with the reference's signatures (src/grid/read_and_process_grid.cpp).

readHGrid(filename, filename_ll, nPartitions, ncor) returns the same 23-tuple as the reference
(:829-855, tuple order :1223-1248); the connectivity comes from gs_grid_build, which reproduces
the reference numbering exactly.  readVGrid(filename, nNodes) returns the reference's 8-tuple
(:1322-1520) for SZ grids; readHGridData(filename, nNodes, nElements) the node column of a .gr3.
Only one partition is supported (nPartitions = 1): multi-GPU runs shard whole members.
"""
from __future__ import annotations

import math
from typing import Tuple

import numpy as np

from . import _lib as L


def _read_lines(filename):
    with open(filename) as f:
        return f.read().splitlines()


def _ints(line):
    out = []
    for tok in line.split():
        try:
            out.append(int(tok))
        except ValueError:
            break
    return out


def _isbnd(np_, open_segs, land_segs):
    isb = np.full(np_, -1, dtype=np.int32)
    for k, seg in enumerate(open_segs):
        isb[np.asarray(seg, dtype=np.int64)] = k
    for seg in land_segs:
        for v in seg:
            if isb[v] == -1:
                isb[v] = -2
    return isb


def read_hgrid_file(filename):
    """Parse hgrid.gr3: coordinates/depth, triangles (0-based), open and land segments."""
    lines = _read_lines(filename)
    ne, np_ = _ints(lines[1])[:2]
    xyz = np.array([[float(t) for t in lines[2 + i].split()[1:4]] for i in range(np_)], dtype=np.float64)
    el = np.full((ne, 4), -1, dtype=np.int32)
    i34 = np.zeros(ne, dtype=np.int32)
    for e in range(ne):
        toks = _ints(lines[2 + np_ + e])
        n = toks[1]
        i34[e] = n
        el[e, :n] = np.asarray(toks[2:2 + n]) - 1
    p = 2 + np_ + ne
    nope = _ints(lines[p])[0]
    p += 2
    open_segs = []
    for _ in range(nope):
        nn = _ints(lines[p])[0]
        open_segs.append([_ints(lines[p + 1 + j])[0] - 1 for j in range(nn)])
        p += 1 + nn
    land_segs = []
    if p < len(lines):
        nland = _ints(lines[p])[0]
        p += 2
        for _ in range(nland):
            toks = _ints(lines[p])
            nn, isl = toks[0], (toks[1] if len(toks) > 1 else 0)
            seg = [_ints(lines[p + 1 + j])[0] - 1 for j in range(nn)]
            if isl == 1:
                seg.append(seg[0])
            land_segs.append(seg)
            p += 1 + nn
    return xyz, el, i34, open_segs, land_segs


def build_connectivity(el4: np.ndarray, i34: np.ndarray, isbnd: np.ndarray, np_: int):
    lib = L.load()
    ne = el4.shape[0]
    out = [np.zeros(np_ + 1, np.int32), np.zeros(4 * ne, np.int32), np.zeros(np_ + 1, np.int32),
           np.zeros(4 * ne + np_, np.int32), np.zeros(4 * ne, np.int32), np.zeros(4 * ne, np.int32),
           np.zeros(8 * ne, np.int32), np.zeros(8 * ne, np.int32), np.zeros(1, np.int32)]
    P = lambda a: a.ctypes.data_as(L.PI)
    el = np.ascontiguousarray(el4.reshape(-1), dtype=np.int32)
    st = lib.gs_grid_build(np_, ne, P(el), P(np.ascontiguousarray(i34, np.int32)),
                           P(np.ascontiguousarray(isbnd, np.int32)), *[P(a) for a in out])
    L.check(st, None, "gs_grid_build")
    ns = int(out[8][0])
    return dict(nne_start=out[0], nne=out[1][:out[0][-1]], nnp_start=out[2], nnp=out[3][:out[2][-1]],
                ic3=out[4].reshape(ne, 4), elside=out[5].reshape(ne, 4),
                isdel=out[6][:2 * ns].reshape(ns, 2), isidenode=out[7][:2 * ns].reshape(ns, 2), ns=ns)


def readHGrid(filename: str, filename_ll: str = "", nPartitions: int = 1, ncor: int = 0) -> Tuple:
    """The reference's 23-tuple: i34, partElements, partNodes, partSides, elnode(4,ne), elside(4,ne),
    nodeCoords(3,np), nodeCoords_ll, ic3(4,ne), isdel(2,ns), isidenode(2,ns), isbnd, nond, nlnd,
    iond(nope,mnond), ilnd(nland,mnlnd), (nodeNeighElems, starts), (nodeNeighNodes, starts),
    numPartElements, numPartNodes, numPartSides, numPartBoundaryNodes, numPartBoundarySides."""
    if nPartitions != 1:
        raise NotImplementedError("one partition per device")
    xyz, el4, i34, open_segs, land_segs = read_hgrid_file(filename)
    np_, ne = xyz.shape[0], el4.shape[0]
    isb = _isbnd(np_, open_segs, land_segs)
    c = build_connectivity(el4, i34, isb, np_)
    ns = c["ns"]
    mnond = max([len(s) for s in open_segs], default=0)
    mnlnd = max([len(s) for s in land_segs], default=0)
    iond = np.full((len(open_segs), mnond), -1, np.int32)
    for k, s in enumerate(open_segs):
        iond[k, :len(s)] = s
    ilnd = np.full((len(land_segs), mnlnd), -1, np.int32)
    for k, s in enumerate(land_segs):
        ilnd[k, :len(s)] = s
    nb_nodes = int((isb >= 0).sum())
    nb_sides = 0
    pairs = set()
    for segs in (land_segs, open_segs):
        for s in segs:
            for a, b in zip(s[:-1], s[1:]):
                pairs.add((min(a, b), max(a, b)))
    for a, b in c["isidenode"]:
        if (min(a, b), max(a, b)) in pairs:
            nb_sides += 1
    ll = np.zeros((0, 0)) if not (filename_ll and ncor > 0) else \
        np.array([[float(t) for t in ln.split()[1:3]] for ln in _read_lines(filename_ll)[2:2 + np_]]).T
    return (i34, np.zeros(ne, np.int32), np.zeros(np_, np.int32), np.zeros(ns, np.int32),
            np.ascontiguousarray(el4.T), np.ascontiguousarray(c["elside"].T), np.ascontiguousarray(xyz.T), ll,
            np.ascontiguousarray(c["ic3"].T), np.ascontiguousarray(c["isdel"].T),
            np.ascontiguousarray(c["isidenode"].T), isb,
            np.array([len(s) for s in open_segs], np.int32), np.array([len(s) for s in land_segs], np.int32),
            iond, ilnd, (c["nne"], c["nne_start"]), (c["nnp"], c["nnp_start"]),
            np.array([ne], np.int32), np.array([np_], np.int32), np.array([ns], np.int32),
            np.array([nb_nodes], np.int32), np.array([nb_sides], np.int32))


def readVGrid(filename: str, nNodes: int) -> Tuple:
    """SZ vgrid.in (ivcor = 2) as the reference tuple: (ivcor, nvrt, nz, nsiglev), ztot[nvrt],
    kb (empty), (h_c, h_s, theta_b, theta_f), sigma_lcl (empty), sigma[nvrt], cs[nvrt], dcs[nvrt].
    Accepts the standard layout (with or without the level-nz line)."""
    lines = [ln for ln in _read_lines(filename) if ln.strip()]
    ivcor = _ints(lines[0])[0]
    if ivcor != 2:
        raise NotImplementedError("only SZ grids (ivcor = 2)")
    toks = lines[1].split()
    nvrt, nz, h_s = int(toks[0]), int(toks[1]), float(toks[2])
    ztot = np.zeros(nvrt)
    p = 2
    if lines[p].strip().lower().startswith("z"):
        p += 1
    for k in range(nz - 1):
        ztot[k] = float(lines[p].split()[1])
        p += 1
    ztot[nz - 1] = -h_s
    if not lines[p].strip().lower().startswith("s"):
        p += 1                                            # optional level-nz line
    p += 1                                                # "S levels"
    h_c, theta_b, theta_f = (float(t) for t in lines[p].split()[:3])
    p += 1
    nsig = nvrt - nz + 1
    sigma = np.zeros(nvrt)
    for k in range(nsig):
        sigma[k] = float(lines[p + k].split()[1])
    s = sigma[:nsig]
    cs = np.zeros(nvrt)
    dcs = np.zeros(nvrt)
    cs[:nsig] = ((1.0 - theta_b) * np.sinh(theta_f * s) / math.sinh(theta_f)
                 + theta_b * (np.tanh(theta_f * (s + 0.5)) - math.tanh(theta_f * 0.5)) / 2.0 / math.tanh(theta_f * 0.5))
    dcs[:nsig] = ((1.0 - theta_b) * theta_f * np.cosh(theta_f * s) / math.sinh(theta_f)
                  + theta_b * theta_f / 2.0 / math.tanh(theta_f * 0.5) / np.cosh((theta_f * (s + 0.5)) ** 2.0))
    return (np.array([ivcor, nvrt, nz, nsig], np.int32), ztot, np.zeros(0, np.int32),
            np.array([h_c, h_s, theta_b, theta_f]), np.zeros((0, 0)), sigma, cs, dcs)


def readHGridData(filename: str, nNodes: int, nElements: int) -> np.ndarray:
    """Fourth column of a .gr3 node block (drag.gr3, temp.ic, ...)."""
    lines = _read_lines(filename)
    ne, np_ = _ints(lines[1])[:2]
    if np_ != nNodes or ne != nElements:
        raise RuntimeError("node/element counts do not match")
    return np.array([float(lines[2 + i].split()[3]) for i in range(np_)], dtype=np.float64)
