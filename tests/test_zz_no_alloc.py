"""The allocation-free JCG entry point (gs_jcg_solve_csr_noalloc) against the solver that owns its
buffers (gs_jcg_solve_csr), on the same elevation system, twice in a row (gpu).

The allocation-free entry point serves callers that cannot allocate device memory while they
run (their device memory is handed out by their own pool, or allocation latency is not allowed
in their loop); its work space is a fixed array inside the library that every call reuses, so the
second call checks that nothing left over from the first one leaks into the result.
"""
import ctypes

import numpy as np
import pytest

from gschism_b200 import cases

pytestmark = pytest.mark.gpu

TOL = 1e-12     # same kernel, same tiles: the two entry points agree to rounding


@pytest.fixture(scope="module")
def system(oracle_lib):
    from oracle.step_api import OracleModel
    c = cases.channel(seed=31)
    o = OracleModel(c)
    o.run(2)
    o.begin_step(3)
    o.btrack()
    o.prepare_elevation(3 * c.params.dt)
    o.assemble(3 * c.params.dt)
    o.essential_bc()
    return o.get("CSR_INDPTR"), o.get("CSR_INDICES"), o.get("CSR_DATA"), o.get("QEL")


def test_noalloc_matches_allocating_solver_twice(native, system):
    import torch
    from gschism_b200.solver import PCGSolverMultiGPU
    ip, ix, da, b = system
    n = b.size
    dev = torch.device("cuda", 0)
    d_ip, d_ix = torch.as_tensor(ip, device=dev), torch.as_tensor(ix, device=dev)
    d_da, d_b = torch.as_tensor(da, device=dev), torch.as_tensor(b, device=dev)
    P = lambda t: ctypes.c_void_p(t.data_ptr())
    for rhs_scale in (1.0, -0.5):
        ref = PCGSolverMultiGPU(None, [n], [da.size])
        ref.csr_indptr(0).copy_(d_ip)
        ref.csr_indices(0).copy_(d_ix)
        ref.csr_data(0).copy_(d_da)
        ref.b_m[0].copy_(d_b * rhs_scale)
        its_ref = ref.solve(rtol=1e-12, maxiter=1500, checkEvery=10)
        x_ref = ref.x_m[0].cpu().numpy()
        ref.close()
        x = torch.zeros(n, dtype=torch.float64, device=dev)
        bb = (d_b * rhs_scale).contiguous()
        torch.cuda.synchronize()
        its = ctypes.c_int(0)
        st = native.gs_jcg_solve_csr_noalloc(n, P(d_ip), P(d_ix), P(d_da), P(bb), P(x), ctypes.c_double(1e-12),
                                             1500, 10, None, ctypes.byref(its))
        assert st == 0
        assert its.value == its_ref
        xs = x.cpu().numpy()
        assert np.abs(xs - x_ref).max() <= TOL * np.abs(x_ref).max()


def test_noalloc_rejects_oversize(native):
    its = ctypes.c_int(0)
    st = native.gs_jcg_solve_csr_noalloc(65537, ctypes.c_void_p(8), ctypes.c_void_p(8), ctypes.c_void_p(8),
                                         ctypes.c_void_p(8), ctypes.c_void_p(8), ctypes.c_double(1e-12), 10, 10,
                                         None, ctypes.byref(its))
    assert st == 1   # GS_ERR_ARG: beyond the fixed work space, nothing is launched
