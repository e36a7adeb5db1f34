"""Recovery after a device wait runs out (gpu).

The solve of one member is made to wait for a block arrival that never comes
(gs_test_stall_solve), with the context's wait bound cut to ~16k polls (a few milliseconds).
Every wait of the persistent kernels is bounded, so the kernels return; the step reports
GS_ERR_TIMEOUT once, the flag and the barrier word are cleared, and after the saved state is put
back the same context steps on bit for bit like a context that never failed.  No device fault,
trap or endless wait is involved."""
import numpy as np
import pytest

from gschism_b200 import cases
from gschism_b200 import _lib as L

pytestmark = pytest.mark.gpu

STATE = ("ETA1", "ETA2", "NODE_Z", "NODE_U2", "NODE_W2", "NODE_TR", "NODE_KB", "NODE_DRY", "SIDE_U2", "SIDE_ZC",
         "SIDE_KB", "SIDE_DRY", "ELEM_Z", "ELEM_TR", "ELEM_KB", "ELEM_DRY", "JCG_X", "JCG_X1", "JCG_X2")
CHECK = ("ETA2", "NODE_TR", "SIDE_U2", "ELEM_W", "NODE_U2", "SIDE_BTELEM")


@pytest.mark.parametrize("precision", ["fp64", "fp32_ir"])
def test_timed_out_solve_is_reported_and_context_recovers(native, precision):
    from gschism_b200.model import Model
    members = [cases.channel(seed=1), cases.channel(seed=2, nx=31, ny=16)]
    ref = Model(members, precision=precision)
    m = Model(members, precision=precision)
    try:
        ref.step(4)
        m.step(3)
        saved = [{f: m.get(k, f) for f in STATE} for k in range(len(members))]
        m.set_wait_limit(1 << 14)
        m.test_stall_solve(0)
        m.step(1)
        with pytest.raises(L.GsError) as ei:
            m.sync()
        assert ei.value.status == L.GS_ERR_TIMEOUT
        # reported once: the flag is cleared and the context answers again
        m.sync()
        m.test_stall_solve(-1)
        m.set_wait_limit(0)
        for k in range(len(members)):
            for f in STATE:
                m.put(k, f, saved[k][f])
        m.phase("BEGIN", 3)      # the device clock back to step 3; gs_step advances it to 4
        m.step(1)
        m.sync()
        for k in range(len(members)):
            for f in CHECK:
                assert np.array_equal(m.get(k, f), ref.get(k, f)), (k, f)
            assert m.stats(k)["jcg_iters"] == ref.stats(k)["jcg_iters"]
            assert m.stats(k)["error_flags"] == 0
    finally:
        m.close()
        ref.close()


def test_not_converged_is_reported_per_solve(native):
    """ERR_JCG_NOT_CONVERGED describes the last solve only: set when maxiter stops it, cleared by
    the next solve that converges."""
    from gschism_b200.model import Model
    c = cases.channel()
    m = Model([c], precision="fp64", maxiter=5)
    try:
        m.step(1)
        st = m.stats(0)
        assert st["jcg_iters"] == 5 and st["error_flags"] & 2
    finally:
        m.close()
    m = Model([c], precision="fp64")
    try:
        m.step(1)
        assert m.stats(0)["error_flags"] == 0
    finally:
        m.close()
