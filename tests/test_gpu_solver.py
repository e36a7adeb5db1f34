"""Stand-alone JCG on a caller CSR (PCGSolverMultiGPU drop-in) against the oracle's JCG (gpu)."""
import numpy as np
import pytest

from gschism_b200 import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system(oracle_lib):
    """An elevation system assembled by the oracle after a few channel steps."""
    from oracle.step_api import OracleModel
    c = cases.channel(seed=21)
    o = OracleModel(c)
    o.run(3)
    o.begin_step(4)
    o.btrack()
    o.prepare_elevation(4 * c.params.dt)
    o.assemble(4 * c.params.dt)
    o.essential_bc()
    A = (o.get("CSR_INDPTR"), o.get("CSR_INDICES"), o.get("CSR_DATA"))
    b = o.get("QEL")
    hist = (o.get("JCG_X"), o.get("JCG_X1"), o.get("JCG_X2"))
    its, rel = o.jcg_solve(1e-12, 1500, 10)
    return A, b, hist, its, o.get("JCG_X"), rel


def _fill(s, A, b):
    import torch
    ip, ix, da = A
    s.csr_indptr(0).copy_(torch.as_tensor(ip))
    s.csr_indices(0).copy_(torch.as_tensor(ix))
    s.csr_data(0).copy_(torch.as_tensor(da))
    s.b_m[0].copy_(torch.as_tensor(b))


def test_jcg_csr_matches_oracle(native, system):
    from gschism_b200.solver import PCGSolverMultiGPU
    A, b, hist, its_o, x_o, rel_o = system
    s = PCGSolverMultiGPU(None, [b.size], [A[2].size])
    _fill(s, A, b)
    # a fresh solver starts from x = 0 (empty history), the oracle from its parabolic guess:
    # both solutions meet rtol = 1e-12 and agree to the conditioning of the system
    its = s.solve(rtol=1e-12, maxiter=1500, checkEvery=10)
    assert 0 < its < 1500
    x = s.x_m[0].cpu().numpy()
    assert s.checkSolution() <= 1e-11
    assert rel_o <= 1e-11
    assert np.abs(x - x_o).max() <= 1e-9 * np.abs(x_o).max()
    s.close()


def test_jcg_csr_zero_rhs_returns_zero(native, system):
    from gschism_b200.solver import PCGSolverMultiGPU
    A, b, *_ = system
    s = PCGSolverMultiGPU(None, [b.size], [A[2].size])
    _fill(s, A, np.zeros_like(b))
    assert s.solve(rtol=1e-12, maxiter=100) == 0
    assert np.all(s.x_m[0].cpu().numpy() == 0.0)
    s.close()


def test_jcg_csr_maxiter_cap(native, system):
    from gschism_b200.solver import PCGSolverMultiGPU
    A, b, *_ = system
    s = PCGSolverMultiGPU(None, [b.size], [A[2].size])
    _fill(s, A, b)
    assert s.solve(rtol=1e-14, maxiter=3, checkEvery=10) == 3     # not converged: returns maxiter
    s.close()


def test_jcg_csr_mixed_precision(native, system):
    from gschism_b200.solver import PCGSolverMultiGPU
    A, b, hist, its_o, x_o, rel_o = system
    s = PCGSolverMultiGPU(None, [b.size], [A[2].size], precision="fp32_ir")
    _fill(s, A, b)
    s.solve(rtol=1e-12, maxiter=1500, checkEvery=10)
    assert s.checkSolution() <= 1e-11
    s.close()
