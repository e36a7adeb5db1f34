"""The output writer's NetCDF files (no GPU): the reference's file and variable layout
(src/iop/writeOutput.py:288-711), records every nspool steps, ihfskip / nspool records per file,
values equal to the fields written (float32)."""
import numpy as np
import pytest

from gschism_b200 import cases
from gschism_b200.output import NetcdfSink, grid_of, record_to_variables

FIELDS = ("ETA2", "NODE_DRY", "ELEM_DRY", "SIDE_DRY", "NODE_U2", "NODE_W2", "NODE_Z", "ELEM_W", "NODE_TR")


def test_files_hold_the_records(tmp_path, native):
    from scipy.io import netcdf_file
    from oracle.step_api import OracleModel
    c = cases.channel()
    o = OracleModel(c)
    g = grid_of(c)
    g["kb"] = o.get("NODE_KB")
    sink = NetcdfSink(str(tmp_path), g, c.nvrt, c.ntracers, c.params.dt, nspool=2, ihfskip=4)
    recs = {}
    for it in range(1, 7):
        o.step(it)
        if it % 2 == 0:
            fields = {f: o.get(f) for f in FIELDS}
            recs[it] = fields
            sink.write(it, record_to_variables(fields, c.ntracers))
    sink.close()
    names = sorted(p.name for p in tmp_path.iterdir())
    assert names == sorted(f"{b}_{n}.nc" for b in ("out2d", "horizontalVelX", "horizontalVelY", "verticalVelocity",
                                                   "zCoordinates", "verticalVelAtElement", "temperature")
                           for n in (1, 2))
    # file 1 holds steps 2 and 4, file 2 holds step 6
    for fnum, steps in ((1, (2, 4)), (2, (6,))):
        with netcdf_file(str(tmp_path / f"out2d_{fnum}.nc"), "r", mmap=False) as f:
            assert f.dimensions["nSCHISM_hgrid_node"] == c.n_nodes
            assert f.dimensions["nSCHISM_vgrid_layers"] == c.nvrt
            assert list(f.variables["time"][:]) == [s * c.params.dt for s in steps]
            fn = f.variables["SCHISM_hgrid_face_nodes"][:]
            assert fn.shape == (c.n_elems, 4) and fn[:, :3].min() == 1 and (fn[:, 3] == -1).all()
            assert np.array_equal(fn[:, :3] - 1, c.elnode)
            for r, s in enumerate(steps):
                assert np.array_equal(f.variables["elevation"][r], recs[s]["ETA2"].astype(np.float32))
                assert np.array_equal(f.variables["dryFlagElement"][r], recs[s]["ELEM_DRY"].astype(np.float32))
        with netcdf_file(str(tmp_path / f"horizontalVelY_{fnum}.nc"), "r", mmap=False) as f:
            v = f.variables["horizontalVelY"]
            assert v.dimensions == ("time", "nSCHISM_hgrid_node", "nSCHISM_vgrid_layers")
            for r, s in enumerate(steps):
                assert np.array_equal(v[r], recs[s]["NODE_U2"][:, :, 1].T.astype(np.float32))
        with netcdf_file(str(tmp_path / f"temperature_{fnum}.nc"), "r", mmap=False) as f:
            for r, s in enumerate(steps):
                assert np.array_equal(f.variables["temperature"][r], recs[s]["NODE_TR"][0].T.astype(np.float32))
