"""The allocation-free JCG entry point (gs_jcg_solve_csr_noalloc) against the solver that owns its
buffers (gs_jcg_solve_csr) and against the CPU oracle's JCG, two calls in a row each (gpu).

The allocation-free entry point serves callers that cannot allocate device memory while they
run (their device memory is handed out by their own pool, or allocation latency is not allowed
in their loop); its work space is a fixed array inside the library that every call reuses, so the
second call checks that nothing left over from the first one leaks into the result.

The allocation-free solve cuts rows into 256-row tiles and the allocating one into tiles of at
least 1,024 rows, so their dot products add partial sums in different orders: solutions agree to
the solver tolerance (1e-10 relative at rtol 1e-12), and iteration counts by up to one test
interval (check_every).  Systems: the 10 km channel (2,016 rows) and a 250 x 250 basin (62,500
rows, close to the 65,536-row limit), from a zero and from a nonzero initial guess.
"""
import ctypes

import numpy as np
import pytest

from gschism_b200 import cases

pytestmark = pytest.mark.gpu

TOL = 1e-10     # relative to the largest |x|: tolerance-level agreement (different reduction orders)
CHECK = 10      # check_every: iteration counts may differ by one test interval


def _system(case, steps):
    """The elevation system of step steps+1 from the oracle, the parabolic initial guess the
    oracle's solve starts from, and the oracle's solutions from that guess and from zero."""
    from oracle.step_api import OracleModel
    o = OracleModel(case)
    o.run(steps)
    it = steps + 1
    o.begin_step(it)
    o.btrack()
    o.prepare_elevation(it * case.params.dt)
    o.assemble(it * case.params.dt)
    o.essential_bc()
    hist = [o.get(f) for f in ("JCG_X", "JCG_X1", "JCG_X2")]
    guess = 3.0 * hist[0] - 3.0 * hist[1] + hist[2]
    its_g, _ = o.jcg_solve(1e-12, 1500, CHECK)
    x_g = o.get("JCG_X")
    for f, v in zip(("JCG_X", "JCG_X1", "JCG_X2"), hist):
        o.put(f, np.zeros_like(v))
    its_0, _ = o.jcg_solve(1e-12, 1500, CHECK)
    x_0 = o.get("JCG_X")
    return dict(ip=o.get("CSR_INDPTR"), ix=o.get("CSR_INDICES"), da=o.get("CSR_DATA"), b=o.get("QEL"),
                guess=guess, x_guess=x_g, its_guess=its_g, x_zero=x_0, its_zero=its_0)


@pytest.fixture(scope="module")
def systems(oracle_lib):
    return {"channel": _system(cases.channel(seed=31), 2),
            "basin250": _system(cases.basin(seed=7, n=250, nvrt=4, nz=2, ntr=1, length=125e3), 1)}


def _noalloc(native, s, x0):
    import torch
    dev = torch.device("cuda", 0)
    t = {k: torch.as_tensor(np.ascontiguousarray(s[k]), device=dev) for k in ("ip", "ix", "da", "b")}
    x = torch.as_tensor(np.ascontiguousarray(x0, dtype=np.float64), device=dev).clone()
    P = lambda a: ctypes.c_void_p(a.data_ptr())
    torch.cuda.synchronize()
    its = ctypes.c_int(0)
    st = native.gs_jcg_solve_csr_noalloc(int(s["b"].size), P(t["ip"]), P(t["ix"]), P(t["da"]), P(t["b"]), P(x),
                                         ctypes.c_double(1e-12), 1500, CHECK, None, ctypes.byref(its))
    assert st == 0
    return x.cpu().numpy(), its.value


def _close(x, ref):
    return np.abs(x - ref).max() <= TOL * np.abs(ref).max()


@pytest.mark.parametrize("name", ["channel", "basin250"])
def test_noalloc_matches_allocating_solver_twice(native, systems, name):
    import torch
    from gschism_b200.solver import PCGSolverMultiGPU
    s = systems[name]
    n = s["b"].size
    dev = torch.device("cuda", 0)
    for rhs_scale in (1.0, -0.5):
        ref = PCGSolverMultiGPU(None, [n], [s["da"].size])
        ref.csr_indptr(0).copy_(torch.as_tensor(s["ip"], device=dev))
        ref.csr_indices(0).copy_(torch.as_tensor(s["ix"], device=dev))
        ref.csr_data(0).copy_(torch.as_tensor(s["da"], device=dev))
        ref.b_m[0].copy_(torch.as_tensor(s["b"] * rhs_scale, device=dev))
        its_ref = ref.solve(rtol=1e-12, maxiter=1500, checkEvery=CHECK)
        x_ref = ref.x_m[0].cpu().numpy()
        ref.close()
        sr = dict(s, b=s["b"] * rhs_scale)
        x, its = _noalloc(native, sr, np.zeros(n))
        assert abs(its - its_ref) <= CHECK, (its, its_ref)
        assert _close(x, x_ref)


@pytest.mark.parametrize("name", ["channel", "basin250"])
def test_noalloc_matches_oracle_from_zero_and_nonzero_guess(native, systems, name):
    s = systems[name]
    assert np.abs(s["guess"]).max() > 0.0
    x, its = _noalloc(native, s, s["guess"])
    assert abs(its - s["its_guess"]) <= CHECK and _close(x, s["x_guess"])
    x, its = _noalloc(native, s, np.zeros_like(s["guess"]))
    assert abs(its - s["its_zero"]) <= CHECK and _close(x, s["x_zero"])


def test_noalloc_rejects_oversize(native):
    its = ctypes.c_int(0)
    st = native.gs_jcg_solve_csr_noalloc(65537, ctypes.c_void_p(8), ctypes.c_void_p(8), ctypes.c_void_p(8),
                                         ctypes.c_void_p(8), ctypes.c_void_p(8), ctypes.c_double(1e-12), 10, 10,
                                         None, ctypes.byref(its))
    assert st == 1   # GS_ERR_ARG: beyond the fixed work space, nothing is launched
