"""ctypes bindings of libgschism_b200.so (the C ABI declared in include/gschism_b200.h).

The library is built in-tree (gschism_b200/build.py).  Loading never falls back to anything:
if the shared object is missing the import of any compute entry point raises.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

c_int, c_double, c_void_p, c_size_t = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_size_t
PD = ctypes.POINTER(ctypes.c_double)
PI = ctypes.POINTER(ctypes.c_int32)

GS_OK, GS_ERR_ARG, GS_ERR_CUDA, GS_ERR_OOM, GS_ERR_NOT_CONVERGED, GS_ERR_TIMEOUT, GS_ERR_BAD_MESH, GS_ERR_STATE = range(8)
GS_FP64, GS_FP32_IR = 0, 1
STATUS_NAMES = {0: "GS_OK", 1: "GS_ERR_ARG", 2: "GS_ERR_CUDA", 3: "GS_ERR_OOM", 4: "GS_ERR_NOT_CONVERGED",
                5: "GS_ERR_TIMEOUT", 6: "GS_ERR_BAD_MESH", 7: "GS_ERR_STATE"}

# launch-shape ids of gs_set_launch / gs_get_launch
LAUNCH = dict(BTRACK=0, SIDE_PREP=1, GHAT=2, ASSEMBLE=3, MOMENTUM=4, VVEL=5, NODAL_VEL=6, NODAL_TRACER=7,
              LEVELS=8, JCG_TILES=9)
PHASE = dict(BEGIN=0, BTRACK=1, PREPARE=2, ASSEMBLE=3, SOLVE=4, UPDATE_ELEV=5, MOMENTUM=6, VVEL=7,
             TRANSPORT=8, LEVELS=9, NODAL_VEL=10)

EXPORTS = ["gs_grid_build", "gs_ctx_create", "gs_member_add", "gs_ctx_prepare", "gs_ctx_finalize", "gs_ctx_destroy",
           "gs_last_error", "gs_sync", "gs_set_stream", "gs_step", "gs_phase", "gs_state_get", "gs_state_put", "gs_set_tau",
           "gs_get_stats", "gs_tracer_mass", "gs_set_launch", "gs_get_launch", "gs_member_sizes", "gs_jcg_create", "gs_jcg_buffers", "gs_jcg_solve_csr",
           "gs_jcg_check", "gs_jcg_destroy", "gs_jcg_last_error", "gs_jcg_solve_csr_noalloc",
           "gs_set_vortex", "gs_footprint_bytes", "gs_set_wait_limit", "gs_test_stall_solve", "gs_state_get_async",
           "gs_output_mark", "gs_output_wait", "gs_host_alloc", "gs_host_free", "gs_set_member_start", "gs_get_step"]

GS_MEMBER_PARKED = 2000000000


class GsConfig(ctypes.Structure):
    _fields_ = [("nvrt", c_int), ("ntr", c_int), ("nz", c_int), ("h_s", c_double), ("h_c", c_double),
                ("theta_b", c_double), ("theta_f", c_double), ("ztot", PD), ("sigma", PD),
                ("dt", c_double), ("thetai", c_double), ("h0", c_double), ("dtb_min", c_double),
                ("dtb_max", c_double), ("velmin_btrack", c_double), ("rmaxvel", c_double), ("dfv0", c_double),
                ("coricoef", c_double), ("rho0", c_double), ("grav", c_double), ("dramp", c_double),
                ("ihhat", c_int), ("rtol", c_double), ("maxiter", c_int), ("check_every", c_int),
                ("precision", c_int), ("ir_inner_rtol", c_double), ("ir_inner_maxiter", c_int),
                ("device", c_int), ("itr_met", c_int), ("tvd_limiter", c_int), ("dfh0", c_double)]


class GsMemberDesc(ctypes.Structure):
    _fields_ = [("np", c_int), ("ne", c_int), ("nope", c_int), ("nland", c_int), ("nbfr", c_int),
                ("x", PD), ("y", PD), ("depth", PD), ("drag", PD), ("tau", PD), ("tr_init", PD),
                ("elnode", PI), ("open_start", PI), ("open_nodes", PI), ("land_start", PI), ("land_nodes", PI),
                ("iettype", PI), ("amig", PD), ("ff", PD), ("face", PD), ("emo", PD), ("efa", PD)]


class GsVortex(ctypes.Structure):
    _fields_ = [("x0", c_double), ("y0", c_double), ("heading", c_double), ("speed", c_double),
                ("vmax", c_double), ("rmax", c_double), ("holland_b", c_double), ("rho_air", c_double)]


class GsStats(ctypes.Structure):
    _fields_ = [("jcg_iters", ctypes.c_int64), ("jcg_outer", ctypes.c_int64), ("jcg_relres", c_double),
                ("transport_substeps", ctypes.c_int64), ("walk_cap_hits", ctypes.c_int64),
                ("btrack_stops", ctypes.c_int64), ("error_flags", ctypes.c_int32)]


_lib = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = False):
    """Load the native library; raises if it is not built (no fallback path exists)."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path):
        if build_if_missing:
            _build.build()
        else:
            raise RuntimeError(f"gschism_b200 native library not built: {path} (run gschism_b200/build.py)")
    L = ctypes.CDLL(path)
    I = c_int
    L.gs_grid_build.argtypes = [I, I, PI, PI, PI, PI, PI, PI, PI, PI, PI, PI, PI, PI]
    L.gs_ctx_create.argtypes = [ctypes.POINTER(GsConfig), ctypes.POINTER(c_void_p)]
    L.gs_member_add.argtypes = [c_void_p, ctypes.POINTER(GsMemberDesc), ctypes.POINTER(c_int)]
    L.gs_ctx_prepare.argtypes = [c_void_p]
    L.gs_ctx_finalize.argtypes = [c_void_p]
    L.gs_ctx_destroy.argtypes = [c_void_p]
    L.gs_last_error.argtypes = [c_void_p]
    L.gs_last_error.restype = ctypes.c_char_p
    L.gs_sync.argtypes = [c_void_p]
    L.gs_set_stream.argtypes = [c_void_p, c_void_p]
    L.gs_step.argtypes = [c_void_p, I]
    L.gs_phase.argtypes = [c_void_p, I, I]
    L.gs_state_get.argtypes = [c_void_p, I, I, c_void_p, c_size_t]
    L.gs_state_put.argtypes = [c_void_p, I, I, c_void_p, c_size_t]
    L.gs_set_tau.argtypes = [c_void_p, I, PD]
    L.gs_get_stats.argtypes = [c_void_p, I, ctypes.POINTER(GsStats)]
    L.gs_tracer_mass.argtypes = [c_void_p, I, PD]
    L.gs_set_launch.argtypes = [c_void_p, I, I, I]
    L.gs_get_launch.argtypes = [c_void_p, I, PI, PI]
    L.gs_member_sizes.argtypes = [c_void_p, I] + [ctypes.POINTER(c_int)] * 4
    L.gs_jcg_create.argtypes = [I, I, I, I, ctypes.POINTER(c_void_p)]
    L.gs_jcg_buffers.argtypes = [c_void_p] + [ctypes.POINTER(c_void_p)] * 5
    L.gs_jcg_solve_csr.argtypes = [c_void_p, c_double, I, I, ctypes.POINTER(c_int)]
    L.gs_jcg_check.argtypes = [c_void_p, PD]
    L.gs_jcg_destroy.argtypes = [c_void_p]
    L.gs_jcg_last_error.argtypes = [c_void_p]
    L.gs_jcg_last_error.restype = ctypes.c_char_p
    L.gs_jcg_solve_csr_noalloc.argtypes = [I, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_double, I, I,
                                           c_void_p, ctypes.POINTER(c_int)]
    L.gs_set_vortex.argtypes = [c_void_p, I, ctypes.POINTER(GsVortex)]
    L.gs_set_wait_limit.argtypes = [c_void_p, ctypes.c_longlong]
    L.gs_set_member_start.argtypes = [c_void_p, I, I]
    L.gs_get_step.argtypes = [c_void_p, ctypes.POINTER(c_int)]
    L.gs_test_stall_solve.argtypes = [c_void_p, I]
    L.gs_state_get_async.argtypes = [c_void_p, I, I, c_void_p, c_size_t]
    L.gs_output_mark.argtypes = [c_void_p, ctypes.POINTER(ctypes.c_uint64)]
    L.gs_output_wait.argtypes = [c_void_p, ctypes.c_uint64]
    L.gs_host_alloc.argtypes = [c_size_t]
    L.gs_host_alloc.restype = c_void_p
    L.gs_host_free.argtypes = [c_void_p]
    L.gs_footprint_bytes.argtypes = [I, I, I, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64]
    for name in EXPORTS:
        if name not in ("gs_last_error", "gs_jcg_last_error", "gs_footprint_bytes", "gs_host_alloc"):
            getattr(L, name).restype = c_int
    L.gs_footprint_bytes.restype = c_size_t
    _lib = L
    return L


class GsError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status: int, ctx=None, what: str = "") -> None:
    if status != GS_OK:
        msg = what
        if ctx is not None:
            try:
                msg += ": " + load().gs_last_error(ctx).decode()
            except Exception:
                pass
        raise GsError(status, msg)
