"""The reference's call order through the `cufunc` shim on the device (gpu): three steps issued
kernel by kernel give the same bits as three gs_step calls."""
import numpy as np
import pytest

from gschism_b200 import cases
from gschism_b200.kernels import Kernels
from tests.test_kernels_shim import reference_step

pytestmark = pytest.mark.gpu


def test_shim_call_order_equals_gs_step(native):
    from gschism_b200.model import Model
    c = cases.channel()
    a, b = Model([c]), Model([c])
    try:
        k = Kernels(a)
        for it in (1, 2, 3):
            its, _ = reference_step(k, it, c.params.dt)
            assert its == a.stats(0)["jcg_iters"]
        b.step(3)
        for f in ("ETA2", "NODE_TR", "SIDE_U2", "ELEM_W", "NODE_U2", "SIDE_BTELEM"):
            assert np.array_equal(a.get(0, f), b.get(0, f)), f
    finally:
        a.close()
        b.close()
