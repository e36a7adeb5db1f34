"""Drop-in for the reference JCG solver class (src/solver/pcg_solver.py:538-1148).

    solver = PCGSolverMultiGPU(configCuda, N=[n], NNZ=[nnz])
    solver.csr_indptr(0)[:] = ...;  solver.csr_indices(0)[:] = ...;  solver.csr_data(0)[:] = ...
    solver.b_m[0][:] = rhs                       # the reference gathers b from the mesh (qel)
    iters = solver.solve(rtol=1e-12, maxiter=1500, checkEvery=10)
    rel = solver.checkSolution()

Same names, argument meaning and return values as the reference.  The matrix and vectors live in
device buffers owned by the native solver (gs_jcg); csr_data(m) & co. return torch tensors that
view them, as the reference returns CuPy arrays its populate kernels fill.  One partition per
device: the reference's row-block multi-GPU split is not needed for meshes that fit one B200
(a 180 GB part holds every benchmark configuration), so len(N) must be 1.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from . import _lib as L


class _DevArray:
    """__cuda_array_interface__ view of a raw device pointer (for torch.as_tensor)."""

    def __init__(self, ptr: int, n: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3, "strides": None}


class PCGSolverMultiGPU:
    TPB = 256
    useNative = True

    def __init__(self, configCuda=None, N: Sequence[int] = (), NNZ: Sequence[int] = (), precision: str = "fp64",
                 device: int | None = None):
        import torch
        N, NNZ = list(N), list(NNZ)
        if len(N) != 1 or len(NNZ) != 1:
            raise NotImplementedError("one partition per device (len(N) == 1)")
        self.lib = L.load()
        dev = device if device is not None else (getattr(configCuda, "devices", [0]) or [0])[0]
        self.N_m, self.NNZ_m, self.N_total = N, NNZ, int(N[0])
        h = ctypes.c_void_p()
        prec = {"fp64": L.GS_FP64, "fp32_ir": L.GS_FP32_IR}[precision]
        L.check(self.lib.gs_jcg_create(int(N[0]), int(NNZ[0]), prec, int(dev), ctypes.byref(h)), None, "gs_jcg_create")
        self.h = h
        ptrs = [ctypes.c_void_p() for _ in range(5)]
        L.check(self.lib.gs_jcg_buffers(self.h, *[ctypes.byref(p) for p in ptrs]), None, "gs_jcg_buffers")
        ip, ix, da, b, x = (p.value for p in ptrs)
        dv = torch.device("cuda", int(dev))
        n, nnz = int(N[0]), int(NNZ[0])
        self.indptr_m = [torch.as_tensor(_DevArray(ip, n + 1, "<i4"), device=dv)]
        self.indices_m = [torch.as_tensor(_DevArray(ix, nnz, "<i4"), device=dv)]
        self.data_m = [torch.as_tensor(_DevArray(da, nnz, "<f8"), device=dv)]
        self.b_m = [torch.as_tensor(_DevArray(b, n, "<f8"), device=dv)]
        self.x_m = [torch.as_tensor(_DevArray(x, n, "<f8"), device=dv)]
        self.last_iters = 0

    def csr_data(self, m):
        return self.data_m[m]

    def csr_indices(self, m):
        return self.indices_m[m]

    def csr_indptr(self, m):
        return self.indptr_m[m]

    def solve(self, rtol=1e-5, maxiter=None, ensureSymmetric=False, checkEvery=10) -> int:
        """Jacobi-PCG with the reference semantics (pcg_solver.py:1075-1124): atol = rtol*|b|,
        parabolic initial guess from the last three solutions, convergence tested every
        checkEvery iterations on the device; returns the iteration count."""
        import torch
        torch.cuda.synchronize()
        if maxiter is None:
            maxiter = self.N_total * 10
        it = ctypes.c_int(0)
        st = self.lib.gs_jcg_solve_csr(self.h, float(rtol), int(maxiter), int(checkEvery), ctypes.byref(it))
        if st != L.GS_OK:
            raise L.GsError(st, self.lib.gs_jcg_last_error(self.h).decode())
        self.last_iters = it.value
        return it.value

    def checkSolution(self, label="") -> float:
        """|b - A x| / |b| (pcg_solver.py:1127-1143)."""
        rel = ctypes.c_double(0.0)
        L.check(self.lib.gs_jcg_check(self.h, ctypes.byref(rel)), None, "gs_jcg_check")
        return rel.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.gs_jcg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
