"""Generate the connectivity golden vectors from the reference's own grid reader.

Runs the reference readHGrid / readVGrid (src/grid/read_and_process_grid.cpp, compiled from the
reference sources by oracle/build.py into oracle/_ref) on seeded synthetic cases written in
SCHISM's file formats, and stores their outputs as .npz fixtures next to this script.  Needs the
reference tree; the fixtures are committed so the tests run without it.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))

from gschism_b200 import cases  # noqa: E402
from oracle import build as ob  # noqa: E402

NAMES = ("i34 partElements partNodes partSides elnode elside nodeCoords nodeCoords_ll ic3 isdel isidenode "
         "isbnd nond nlnd iond ilnd nodeNeighElems nodeNeighNodes").split()


def golden_cases():
    """Small seeded cases: the 63x32 channel, a 24x20 basin (SZ levels), an unshuffled 9x7 channel."""
    return {
        "channel": cases.channel(seed=1),
        "basin24": cases.basin(seed=5, n=24, nvrt=12, nz=4, ntr=2, length=20e3, nsteps=1),
        "tiny": cases.channel(seed=7, nx=9, ny=7, nvrt=5, shuffle=False),
    }


def main():
    ob.build_ref()
    ref = ob.load_ref()
    if ref is None:
        raise SystemExit("reference grid module not available")
    for name, case in golden_cases().items():
        with tempfile.TemporaryDirectory() as d:
            cases.write_case(case, d)
            out = ref.readHGrid(os.path.join(d, "hgrid.gr3"), "", 1, 0)
            v = ref.readVGrid(os.path.join(d, "vgrid.in"), case.n_nodes)
        arr = {}
        for k, val in zip(NAMES, out[:18]):
            if isinstance(val, tuple):
                arr[k + "_data"] = np.asarray(val[0])
                arr[k + "_start"] = np.asarray(val[1])
            else:
                arr[k] = np.asarray(val)
        arr["vgrid_ints"] = np.asarray(v[0])
        arr["vgrid_ztot"] = np.asarray(v[1])
        arr["vgrid_params"] = np.asarray(v[3])
        arr["vgrid_sigma"] = np.asarray(v[5])
        arr["vgrid_cs"] = np.asarray(v[6])
        np.savez_compressed(os.path.join(HERE, f"grid_{name}.npz"), **arr)
        print(name, {k: a.shape for k, a in arr.items() if k in ("elside", "isdel", "nodeNeighNodes_data")})


if __name__ == "__main__":
    main()
