"""Recipe: the reference's step kernels compiled for the host CPU (test infrastructure only).

For one case this script
  1. fills the reference's own constants template (src/kernels/constants_template.h) with the
     case's compile-time constants, the way src/iop/processConstantsHeader.py:3-209 does from a
     namelist, into oracle/_ref/refemu/<tag>/constants.h;
  2. compiles oracle/refemu/ref_step.cpp, which includes src/kernels/meshdata.cu unchanged from
     the reference tree, with g++ (asserts on, FMA contraction off) into
     oracle/_ref/refemu/<tag>/libref_step.so; with fma=True the same source is compiled with
     multiply-adds contracted into FMA instructions (-mfma -ffp-contract=fast), as nvcc/NVRTC
     contract the reference's kernels by default on a GPU.
The include order makes the generated constants.h win over the one that sits beside
meshdata.cu (-I<tag> -I<kernels> -I-: quote includes search these directories only, in this
order) and oracle/refemu/cuda_runtime.h stand in for the CUDA runtime header.

The reference tree is read from $GS_REFERENCE_ROOT (default /root/reference).  Nothing here runs
where the tree is absent; the fixtures it produces are committed under tests/golden/.
"""
from __future__ import annotations

import hashlib
import os
import re
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
OUT = os.path.join(ORACLE, "_ref", "refemu")


def reference_root() -> str:
    return os.environ.get("GS_REFERENCE_ROOT", "/root/reference")


def kernels_dir() -> str:
    return os.path.join(reference_root(), "src", "kernels")


def available() -> bool:
    return os.path.exists(os.path.join(kernels_dir(), "meshdata.cu"))


def constants_for(case, mnond: int, mnlnd: int) -> dict:
    """Compile-time constants of the reference for one case (placeholder -> value)."""
    p, vg = case.params, case.vgrid
    nbfr = int(case.amig.shape[0])
    return {
        "__USE_LOCALIZED_SIGMA__": "DO_NOT_USE_LOCALIZED_SIGMA", "__USE_FRAMES__": "DO_NOT_USE_FRAMES",
        "__BLOCK_SIZE__": 128, "__N_TRACERS__": case.ntracers, "__N_GPUS__": 1,
        "__ITUR__": 0, "__TURB_SUBMODEL__": -1, "__STABILITY_MODEL__": -1,
        "__NUM_NODES_PER_PARTITION__": case.n_nodes, "__NODE_OFFSET_PER_PARTITION__": 0,
        "__IVCOR__": 2, "__ICS__": 1, "__IMM__": 0, "__INDVEL__": 0, "__IVEG__": 0, "__IHHAT__": int(p.ihhat),
        "__IHYDRAULICS__": 0, "__IBC__": 1, "__IBTP__": 1, "__ICOMPUTE_CPSI3__": 0, "__ISLIP__": 0,
        "__IUPWIND_MOM__": 0, "__IHORCON__": 0, "__HVIS_COEF0__": 0.025,
        # the populate kernel asserts ishapiro == 1 (meshdata.cu:2306); the filter itself is
        # applied only when the driver calls it (schism_step.py:283-286), which it does not
        "__ISHAPIRO__": 1, "__SHAPIRO0__": 0.5, "__NITER_SHAP__": 1,
        "__NCOR__": 0, "__CORICOEF__": repr(float(p.coricoef)), "__SFEA0__": 0, "__NWS__": 0, "__WTIMINC__": 300,
        "__IWIND_FORM__": 1, "__IWINDOFF__": 0, "__DRAMPWIND__": 1, "__IHCONSV__": 0, "__ISCONSV__": 0,
        "__ITR_MET__": 1, "__H_TVD__": -1, "__NCHI__": 0, "__HMIN_MAN__": 1, "__NRAMP_ELEV__": 0,
        "__ILOADTIDE__": 0, "__LOADTIDE_COEF__": 0.1, "__INV_ATM_BND__": 0, "__PRMSL_REF__": 101325,
        "__VEG_LAI__": 1, "__VEG_CW__": 1.5, "__NTIP__": 0, "__TIP_DP__": 40, "__NBFR__": nbfr,
        "__NETTYPE__": 0, "__NFLTYPE__": 0, "__NETTYPE2__": 0, "__NFLTYPE2__": 0, "__NNODE_ET__": 0,
        "__NNODE_FL__": 0, "__IUNDER_DEEP__": 0, "__H1_BCC__": 50, "__H2_BCC__": 100, "__HW_DEPTH__": 1000000,
        "__HW_RATIO__": 0.5, "__NVRT__": vg.nvrt, "__NZLEV__": vg.nz, "__NSIGLEV__": vg.nsiglev,
        "__NOPEN_BOUNDARY_SEGMENTS__": len(case.open_bnd), "__MAX_NODES_PER_OPEN_BOUNDARY_SEGMENT__": mnond,
        "__N_LAND_BOUNDARY_SEGMENTS__": len(case.land_bnd), "__MAX_NODES_PER_LAND_BOUNDARY_SEGMENT__": mnlnd,
        "__REARTH_EQ__": 6378206.4, "__REARTH_POLE__": 6378206.4, "__THETAI__": repr(float(p.thetai)),
        "__RMAXVEL__": repr(float(p.rmaxvel)), "__RHO0__": repr(float(p.rho0)), "__IEOS_TYPE__": 0,
        "__IEOS_PRES__": 0, "__EOS_A__": -0.1, "__EOS_B__": 1001, "__DTB_MIN__": repr(float(p.dtb_min)),
        "__DTB_MAX__": repr(float(p.dtb_max)), "__VELMIN_BTRACK__": repr(float(p.velmin_btrack)), "__NADV__": 1,
        "__DFV0__": repr(float(p.dfv0)), "__DFH0__": repr(float(p.dfh0)), "__XLSC0__": 0.1, "__DZB_MIN__": 0.5,
        "__DT__": repr(float(p.dt)), "__H0__": repr(float(p.h0)),
    }


def _varcodes() -> str:
    """The VarCode enumerators, as the reference's generated constants.h lists them."""
    txt = open(os.path.join(kernels_dir(), "constants.h")).read()
    return re.search(r"enum class VarCode \{([^}]*)\}", txt).group(1)


def build_for(case, mnond: int, mnlnd: int, fma: bool = False) -> str:
    """constants.h + libref_step.so for this case; returns the library path."""
    tmpl = open(os.path.join(kernels_dir(), "constants_template.h")).read()
    vals = constants_for(case, mnond, mnlnd)
    vals["__VARCODES__"] = _varcodes()
    for k, v in vals.items():
        tmpl = tmpl.replace(k, str(v))
    left = sorted(set(re.findall(r"__[A-Z0-9_]+__", tmpl)) - {"__forceinline__", "__device__"})
    if left:
        raise RuntimeError(f"constants template placeholders left unfilled: {left}")
    src = os.path.join(HERE, "ref_step.cpp")
    shim = os.path.join(HERE, "cuda_runtime.h")
    fp = ["-mfma", "-ffp-contract=fast"] if fma else ["-ffp-contract=off"]
    key = hashlib.sha1((tmpl + open(src).read() + open(shim).read() + " ".join(fp)).encode()).hexdigest()[:12]
    d = os.path.join(OUT, key)
    lib = os.path.join(d, "libref_step.so")
    if os.path.exists(lib):
        return lib
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "constants.h"), "w") as f:
        f.write(tmpl)
    tmp = lib + f".tmp{os.getpid()}"
    cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared"] + fp + ["-w",
           "-include", shim, "-I", d, "-I", kernels_dir(), "-I-", "-I", HERE, src, "-o", tmp]
    subprocess.run(cmd, check=True)
    os.replace(tmp, lib)
    return lib
