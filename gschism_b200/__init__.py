"""gschism_b200: B200-native SCHISM semi-implicit hydrodynamic step.

Native library: gschism_b200/_build/libgschism_b200.so (C ABI, include/gschism_b200.h), built
by gschism_b200/build.py for sm_100a.  Python modules:

* cases   -- seeded synthetic SCHISM cases and SCHISM file writers
* model   -- Model: a batch of members resident on one GPU (gs_ctx)
* solver  -- PCGSolverMultiGPU: drop-in for src/solver/pcg_solver.py on a caller CSR (gs_jcg)
* grid    -- readHGrid / readVGrid with the reference's signatures (src/grid)
* kernels -- the reference's cufunc kernel names mapped onto phases of a Model
"""
from . import cases  # noqa: F401

__all__ = ["cases", "model", "solver", "grid", "kernels"]
