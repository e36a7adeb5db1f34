"""Streamed output through the C ABI (gpu): gs_state_get_async into page-locked buffers, marks and a
writer thread; the files hold exactly the fields a synchronous read gives at the same steps."""
import numpy as np
import pytest

from gschism_b200 import cases

pytestmark = pytest.mark.gpu


def test_streamed_output_equals_synchronous_reads(tmp_path, native):
    from scipy.io import netcdf_file
    from gschism_b200.model import Model
    from gschism_b200.output import OutputWriter
    c = cases.channel()
    m = Model([c])
    ref = Model([c])
    w = OutputWriter(m, 0, str(tmp_path), nspool=2, ihfskip=4, ring=2)
    expect = {}
    try:
        for it in range(1, 7):
            m.step(1)
            w.step_done(it)
            ref.step(1)
            if it % 2 == 0:
                expect[it] = {f: ref.get(0, f) for f in ("ETA2", "NODE_U2", "ELEM_W", "NODE_TR", "SIDE_DRY")}
        w.close()
        assert w.written == 3
    finally:
        m.close()
        ref.close()
    for fnum, steps in ((1, (2, 4)), (2, (6,))):
        with netcdf_file(str(tmp_path / f"out2d_{fnum}.nc"), "r", mmap=False) as f:
            for r, s in enumerate(steps):
                assert np.array_equal(f.variables["elevation"][r], expect[s]["ETA2"].astype(np.float32))
                assert np.array_equal(f.variables["dryFlagSide"][r], expect[s]["SIDE_DRY"].astype(np.float32))
        with netcdf_file(str(tmp_path / f"horizontalVelX_{fnum}.nc"), "r", mmap=False) as f:
            for r, s in enumerate(steps):
                assert np.array_equal(f.variables["horizontalVelX"][r], expect[s]["NODE_U2"][:, :, 0].T.astype(np.float32))
        with netcdf_file(str(tmp_path / f"verticalVelAtElement_{fnum}.nc"), "r", mmap=False) as f:
            for r, s in enumerate(steps):
                assert np.array_equal(f.variables["verticalVelAtElement"][r], expect[s]["ELEM_W"].T.astype(np.float32))
