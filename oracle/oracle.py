"""ctypes front end of the C oracle (test infrastructure only: tests, smoke check, CPU baseline).

The grid functions restate the reference's readHGrid connectivity
(src/grid/read_and_process_grid.cpp:27-574); the step functions restate the hydrodynamic
step kernels of src/kernels/meshdata.cu in FP64 (see oracle/step.c for per-function citations).
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, List

import numpy as np

from . import build as _build

_lib = None

I32P = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
F64P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


def lib():
    global _lib
    if _lib is None:
        path = _build.build_oracle() if not os.path.exists(_build.LIB) else _build.LIB
        _lib = ctypes.CDLL(path)
        _lib.og_grid_build.restype = ctypes.c_int
        _lib.og_grid_build.argtypes = [ctypes.c_int, ctypes.c_int, I32P, I32P, I32P,
                                       I32P, I32P, I32P, I32P, I32P, I32P, I32P, I32P, I32P]
        _lib.og_grid_isbnd.restype = None
        _lib.og_grid_isbnd.argtypes = [ctypes.c_int, ctypes.c_int, I32P, I32P,
                                       ctypes.c_int, I32P, I32P, I32P]
        _setup_step(_lib)
    return _lib


def _setup_step(L) -> None:
    """Signatures of the step functions (filled in by oracle/step.c when present)."""
    if not hasattr(L, "og_model_create"):
        return
    from . import step_api
    step_api.declare(L)


def _flat(segs):
    start = np.zeros(len(segs) + 1, dtype=np.int32)
    for k, s in enumerate(segs):
        start[k + 1] = start[k] + len(s)
    nodes = (np.concatenate([np.asarray(s, dtype=np.int32) for s in segs])
             if segs else np.zeros(0, dtype=np.int32))
    return start, np.ascontiguousarray(nodes, dtype=np.int32)


def grid_isbnd(np_: int, open_bnd: List[np.ndarray], land_bnd: List[np.ndarray]) -> np.ndarray:
    os_, on = _flat(open_bnd)
    ls_, ln = _flat(land_bnd)
    out = np.empty(np_, dtype=np.int32)
    lib().og_grid_isbnd(np_, len(open_bnd), os_, on if on.size else np.zeros(1, np.int32),
                        len(land_bnd), ls_, ln if ln.size else np.zeros(1, np.int32), out)
    return out


def grid_build(elnode: np.ndarray, np_: int, isbnd: np.ndarray) -> Dict[str, np.ndarray]:
    """Connectivity of a triangle/quad mesh; elnode is [ne, 3] or [ne, 4] (-1 padded)."""
    ne = elnode.shape[0]
    el4 = np.full((ne, 4), -1, dtype=np.int32)
    el4[:, :elnode.shape[1]] = elnode
    i34 = (el4 >= 0).sum(axis=1).astype(np.int32)
    cap_s = 4 * ne + 4
    out = dict(
        nne_start=np.zeros(np_ + 1, np.int32), nne=np.zeros(4 * ne + 1, np.int32),
        nnp_start=np.zeros(np_ + 1, np.int32), nnp=np.zeros(4 * ne + np_ + 1, np.int32),
        ic3=np.zeros(4 * ne, np.int32), elside=np.zeros(4 * ne, np.int32),
        isdel=np.zeros(2 * cap_s, np.int32), isidenode=np.zeros(2 * cap_s, np.int32),
        ns=np.zeros(1, np.int32))
    rc = lib().og_grid_build(np_, ne, np.ascontiguousarray(el4.ravel()), i34,
                             np.ascontiguousarray(isbnd, dtype=np.int32),
                             out["nne_start"], out["nne"], out["nnp_start"], out["nnp"],
                             out["ic3"], out["elside"], out["isdel"], out["isidenode"], out["ns"])
    if rc != 0:
        raise RuntimeError(f"og_grid_build failed with code {rc}")
    ns = int(out["ns"][0])
    return dict(
        i34=i34,
        nne_start=out["nne_start"], nne=out["nne"][:out["nne_start"][-1]].copy(),
        nnp_start=out["nnp_start"], nnp=out["nnp"][:out["nnp_start"][-1]].copy(),
        ic3=out["ic3"].reshape(ne, 4), elside=out["elside"].reshape(ne, 4),
        isdel=out["isdel"][:2 * ns].reshape(ns, 2), isidenode=out["isidenode"][:2 * ns].reshape(ns, 2),
        ns=ns)
