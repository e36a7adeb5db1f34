"""Build recipes for the oracle (test infrastructure only).

* ``build_oracle()`` compiles the C restatement (oracle/*.c) into oracle/_build/liboracle.so
  with FMA contraction off, so its FP64 arithmetic is plain IEEE mul/add in source order.
* ``build_ref()`` compiles the reference's own grid reader, src/grid/read_and_process_grid.cpp,
  straight from the reference tree into oracle/_ref/ as the Python module ``test`` it defines
  (pybind11, a METIS stand-in header from oracle/metis_stub).  It runs only where the reference
  tree exists; the built module is a checker for connectivity, never part of the product.
* ``build_refemu()`` compiles the reference's step kernels for the host (oracle/refemu/build.py)
  for the 10 km channel case, the library the step fixtures in tests/golden/ come from.

The reference tree is read from $GS_REFERENCE_ROOT (default /root/reference).
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
REFERENCE_ROOT = os.environ.get("GS_REFERENCE_ROOT", "/root/reference")
LIB = os.path.join(BUILD, "liboracle.so")


def _newer(out: str, srcs) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build_oracle(force: bool = False) -> str:
    srcs = sorted(glob.glob(os.path.join(HERE, "*.c")))
    hdrs = sorted(glob.glob(os.path.join(HERE, "*.h")))
    if force or _newer(LIB, srcs + hdrs):
        os.makedirs(BUILD, exist_ok=True)
        tmp = LIB + f".tmp{os.getpid()}"
        cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-fopenmp",
               "-Wall", "-Wno-unused-function", "-o", tmp] + srcs + ["-lm"]
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


def ref_module_path() -> str:
    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    return os.path.join(REF_OUT, "test" + suffix)


def build_ref(force: bool = False) -> str | None:
    """Compile the reference grid reader; returns the module path or None without a tree."""
    src = os.path.join(REFERENCE_ROOT, "src", "grid", "read_and_process_grid.cpp")
    out = ref_module_path()
    if not os.path.exists(src):
        return out if os.path.exists(out) else None
    if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(src):
        return out
    import pybind11
    os.makedirs(REF_OUT, exist_ok=True)
    tmp = out + f".tmp{os.getpid()}"
    # -DNDEBUG: the reference's ArrayOfRows asserts name an undeclared variable
    # (src/include/grid_helper_types.h:189,196) and only compile with asserts off.
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-w", "-DNDEBUG",
           "-I", os.path.join(HERE, "metis_stub"),
           "-I", pybind11.get_include(), "-I", sysconfig.get_paths()["include"],
           src, "-o", tmp]
    subprocess.run(cmd, check=True)
    os.replace(tmp, out)
    return out


def build_refemu() -> str | None:
    """The reference's step kernels compiled for the host for the channel case, or None
    without a reference tree (the fixtures made from it are committed)."""
    from .refemu import build as rb
    if not rb.available() or build_ref() is None:
        return None
    from gschism_b200 import cases
    c = cases.channel()
    return rb.build_for(c, mnond=len(c.open_bnd[0]), mnlnd=len(c.land_bnd[0]))


def load_ref():
    """Import the compiled reference module ``test`` from oracle/_ref (None if absent)."""
    out = ref_module_path()
    if not os.path.exists(out):
        return None
    import importlib.util
    spec = importlib.util.spec_from_file_location("test", out)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_ref(force="--force" in sys.argv))
