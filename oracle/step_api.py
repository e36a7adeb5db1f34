"""ctypes mirror of oracle/step.h (test infrastructure only)."""
from __future__ import annotations

import ctypes
from typing import Dict

import numpy as np

from . import oracle as _o

c_int, c_double, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
PD = ctypes.POINTER(ctypes.c_double)
PI = ctypes.POINTER(ctypes.c_int32)

# field codes shared with the product (include/gschism_b200.h, GS_F_*)
F = dict(ETA1=0, ETA2=1, NODE_Z=2, NODE_U2=3, NODE_W2=4, NODE_TR=5, NODE_KB=6, NODE_DRY=7, QEL=8, NODE_TAU=9,
         SIDE_U2=10, SIDE_BTU=11, SIDE_ZC=12, SIDE_KB=13, SIDE_DRY=14, SIDE_U=15, SIDE_HHAT=16,
         SIDE_CHI=17, SIDE_QH=18, SIDE_BTELEM=19, SIDE_GRADETA1=20, SIDE_GRADETA2=21,
         ELEM_Z=30, ELEM_W=31, ELEM_QV=32, ELEM_TR=33, ELEM_KB=34, ELEM_DRY=35, ELEM_GHAT=36,
         CSR_DATA=40, CSR_INDPTR=41, CSR_INDICES=42, JCG_X=43, ELBC=44, JCG_X1=45, JCG_X2=46, NODE_RHO=47,
         ELEM_RHO=48)
INT_FIELDS = {"NODE_KB", "NODE_DRY", "SIDE_KB", "SIDE_DRY", "SIDE_BTELEM", "ELEM_KB", "ELEM_DRY",
              "CSR_INDPTR", "CSR_INDICES"}


class OgInput(ctypes.Structure):
    _fields_ = [("np", c_int), ("ne", c_int), ("nvrt", c_int), ("ntr", c_int), ("nope", c_int),
                ("nland", c_int), ("nbfr", c_int),
                ("x", PD), ("y", PD), ("depth", PD), ("drag", PD), ("tau", PD), ("tr_init", PD),
                ("elnode", PI), ("open_start", PI), ("open_nodes", PI), ("land_start", PI),
                ("land_nodes", PI), ("iettype", PI), ("amig", PD), ("ff", PD), ("face", PD),
                ("emo", PD), ("efa", PD),
                ("nz", c_int), ("h_s", c_double), ("h_c", c_double), ("theta_b", c_double),
                ("theta_f", c_double), ("ztot", PD), ("sigma", PD),
                ("dt", c_double), ("thetai", c_double), ("h0", c_double), ("dtb_min", c_double),
                ("dtb_max", c_double), ("velmin_btrack", c_double), ("rmaxvel", c_double),
                ("dfv0", c_double), ("coricoef", c_double), ("rho0", c_double), ("grav", c_double),
                ("dramp", c_double), ("ihhat", c_int), ("itr_met", c_int), ("tvd_limiter", c_int),
                ("dfh0", c_double)]


def declare(L) -> None:
    L.og_model_create.restype = c_void_p
    L.og_model_create.argtypes = [ctypes.POINTER(OgInput), ctypes.POINTER(c_int)]
    L.og_model_free.argtypes = [c_void_p]
    L.og_model_init.argtypes = [c_void_p]
    L.og_model_sizes.argtypes = [c_void_p] + [ctypes.POINTER(c_int)] * 4
    L.og_get.argtypes = [c_void_p, c_int, c_void_p]
    L.og_put.argtypes = [c_void_p, c_int, c_void_p]
    for name in ("og_btrack", "og_essential_bc", "og_update_elevation", "og_vertical_velocity",
                 "og_nodal_velocities"):
        getattr(L, name).argtypes = [c_void_p]
        getattr(L, name).restype = None
    for name in ("og_prepare_elevation", "og_assemble", "og_momentum"):
        getattr(L, name).argtypes = [c_void_p, c_double]
        getattr(L, name).restype = None
    L.og_begin_step.argtypes = [c_void_p, c_int]
    L.og_levels.argtypes = [c_void_p, c_int]
    L.og_transport.argtypes = [c_void_p, c_double]
    L.og_transport.restype = c_int
    L.og_jcg_solve.argtypes = [c_void_p, c_double, c_int, c_int, PD]
    L.og_jcg_solve.restype = c_int
    L.og_step.argtypes = [c_void_p, c_int]
    L.og_step.restype = c_int
    L.og_counters.argtypes = [c_void_p, ctypes.POINTER(ctypes.c_int64)]
    L.og_tracer_mass.argtypes = [c_void_p, PD]
    L.og_set_solver.argtypes = [c_void_p, c_double, c_int, c_int]
    L.og_set_vortex.argtypes = [c_void_p, PD]
    L.og_fct_column.argtypes = [c_int, c_double, PD, PD, PD, PD, PD]
    L.og_fct_column.restype = c_int


def fct_column(dt, q, v, co, cl) -> np.ndarray:
    """The oracle's flux-corrected vertical step of one column (og_fct_column)."""
    L = _o.lib()
    n = len(cl)
    q = np.ascontiguousarray(np.r_[np.asarray(q, float), 0.0][:max(n - 1, 1)])
    v, co, cl = (np.ascontiguousarray(a, dtype=float) for a in (v, co, cl))
    out = np.empty(n)
    if L.og_fct_column(n, float(dt), _pd(q), _pd(v), _pd(co), _pd(cl), _pd(out)) != 0:
        raise ValueError("og_fct_column: empty column")
    return out


def _pd(a):
    return a.ctypes.data_as(PD)


def _pi(a):
    return a.ctypes.data_as(PI)


class OracleModel:
    """One member's step in the CPU oracle, built from a gschism_b200.cases.Case."""

    def __init__(self, case, rtol=None, maxiter=None, check_every=None):
        self.L = _o.lib()
        self.case = case
        p = case.params
        self._keep = []

        def k(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a

        ostart, onodes = _o._flat(case.open_bnd)
        lstart, lnodes = _o._flat(case.land_bnd)
        nbfr = int(case.amig.shape[0])
        emo = np.concatenate(case.emo, axis=0) if case.open_bnd else np.zeros((1, max(nbfr, 1)))
        efa = np.concatenate(case.efa, axis=0) if case.open_bnd else np.zeros((1, max(nbfr, 1)))
        vg = case.vgrid
        inp = OgInput()
        inp.np, inp.ne, inp.nvrt, inp.ntr = case.n_nodes, case.n_elems, vg.nvrt, case.ntracers
        inp.nope, inp.nland, inp.nbfr = len(case.open_bnd), len(case.land_bnd), nbfr
        inp.x, inp.y, inp.depth = _pd(k(case.x, np.float64)), _pd(k(case.y, np.float64)), _pd(k(case.depth, np.float64))
        inp.drag, inp.tau = _pd(k(case.drag, np.float64)), _pd(k(case.tau, np.float64))
        inp.tr_init = _pd(k(case.tr_init, np.float64))
        inp.elnode = _pi(k(case.elnode, np.int32))
        inp.open_start, inp.open_nodes = _pi(k(ostart, np.int32)), _pi(k(onodes if onodes.size else np.zeros(1), np.int32))
        inp.land_start, inp.land_nodes = _pi(k(lstart, np.int32)), _pi(k(lnodes if lnodes.size else np.zeros(1), np.int32))
        inp.iettype = _pi(k(case.iettype, np.int32))
        inp.amig, inp.ff, inp.face = _pd(k(case.amig, np.float64)), _pd(k(case.ff, np.float64)), _pd(k(case.face, np.float64))
        inp.emo, inp.efa = _pd(k(emo, np.float64)), _pd(k(efa, np.float64))
        inp.nz, inp.h_s, inp.h_c, inp.theta_b, inp.theta_f = vg.nz, vg.h_s, vg.h_c, vg.theta_b, vg.theta_f
        inp.ztot, inp.sigma = _pd(k(vg.ztot, np.float64)), _pd(k(vg.sigma, np.float64))
        for name in ("dt", "thetai", "h0", "dtb_min", "dtb_max", "velmin_btrack", "rmaxvel", "dfv0",
                     "coricoef", "rho0", "grav", "dramp"):
            setattr(inp, name, float(getattr(p, name)))
        inp.ihhat = int(p.ihhat)
        inp.itr_met, inp.tvd_limiter, inp.dfh0 = int(p.itr_met), int(p.tvd_limiter), float(p.dfh0)
        st = c_int(0)
        self.h = self.L.og_model_create(ctypes.byref(inp), ctypes.byref(st))
        if st.value != 0:
            raise RuntimeError(f"og_model_create failed: {st.value}")
        self.L.og_model_init(self.h)
        a, b, c, d = c_int(), c_int(), c_int(), c_int()
        self.L.og_model_sizes(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d))
        self.np, self.ne, self.ns, self.nnz = a.value, b.value, c.value, d.value
        self.nvrt, self.ntr = vg.nvrt, case.ntracers
        self.L.og_set_solver(self.h, float(rtol if rtol is not None else p.rtol),
                             int(maxiter if maxiter is not None else p.maxiter),
                             int(check_every if check_every is not None else p.check_every))

    VORTEX_KEYS = ("x0", "y0", "heading", "speed", "vmax", "rmax", "holland_b", "rho_air")

    def set_vortex(self, vortex) -> None:
        """Storm forcing (og_set_vortex), same parameters as the product's gs_vortex; None = off."""
        if vortex is None:
            self.L.og_set_vortex(self.h, None)
            return
        self._vortex = np.array([float(vortex[k]) for k in self.VORTEX_KEYS], dtype=np.float64)
        self.L.og_set_vortex(self.h, _pd(self._vortex))

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.L.og_model_free(self.h)
                self.h = None
        except Exception:
            pass

    # -------------------------------------------------------------- state exchange
    def shape(self, name: str):
        n = {"N": self.np, "S": self.ns, "E": self.ne}
        per = {"ETA1": ("N",), "ETA2": ("N",), "QEL": ("N",), "ELBC": ("N",), "JCG_X": ("N",), "JCG_X1": ("N",), "JCG_X2": ("N",),
               "NODE_KB": ("N",), "NODE_DRY": ("N",), "SIDE_KB": ("S",), "SIDE_DRY": ("S",),
               "SIDE_HHAT": ("S",), "SIDE_CHI": ("S",), "ELEM_KB": ("E",), "ELEM_DRY": ("E",)}
        if name in per:
            return (n[per[name][0]],)
        if name in ("SIDE_U", "SIDE_GRADETA1", "SIDE_GRADETA2"):
            return (self.ns, 2)
        if name == "NODE_TAU":
            return (self.np, 2)
        if name == "ELEM_GHAT":
            return (self.ne, 2)
        if name in ("NODE_Z", "NODE_W2", "NODE_RHO"):
            return (self.nvrt, self.np)
        if name == "NODE_U2":
            return (self.nvrt, self.np, 2)
        if name == "NODE_TR":
            return (self.ntr, self.nvrt, self.np)
        if name in ("SIDE_U2", "SIDE_BTU"):
            return (self.nvrt, self.ns, 2)
        if name in ("SIDE_ZC", "SIDE_QH", "SIDE_BTELEM"):
            return (self.nvrt, self.ns)
        if name in ("ELEM_Z", "ELEM_W", "ELEM_QV", "ELEM_RHO"):
            return (self.nvrt, self.ne)
        if name == "ELEM_TR":
            return (self.ntr, self.nvrt, self.ne)
        if name in ("CSR_DATA", "CSR_INDICES"):
            return (self.nnz,)
        if name == "CSR_INDPTR":
            return (self.np + 1,)
        raise KeyError(name)

    def get(self, name: str) -> np.ndarray:
        out = np.zeros(self.shape(name), dtype=np.int32 if name in INT_FIELDS else np.float64)
        if self.L.og_get(self.h, F[name], out.ctypes.data_as(c_void_p)) != 0:
            raise KeyError(name)
        return out

    def put(self, name: str, value) -> None:
        a = np.ascontiguousarray(value, dtype=np.int32 if name in INT_FIELDS else np.float64)
        assert a.shape == self.shape(name), (name, a.shape, self.shape(name))
        if self.L.og_put(self.h, F[name], a.ctypes.data_as(c_void_p)) != 0:
            raise KeyError(name)

    def snapshot(self, names=None) -> Dict[str, np.ndarray]:
        names = names or [n for n in F if n not in ("CSR_INDPTR", "CSR_INDICES")]
        return {n: self.get(n) for n in names}

    # -------------------------------------------------------------- phases
    def step(self, it: int) -> int:
        return self.L.og_step(self.h, it)

    def run(self, nsteps: int, start: int = 1):
        its = []
        for it in range(start, start + nsteps):
            its.append(self.step(it))
        return its

    def counters(self):
        out = (ctypes.c_int64 * 4)()
        self.L.og_counters(self.h, out)
        return list(out)

    def tracer_mass(self) -> np.ndarray:
        out = np.zeros(max(self.ntr, 1))
        self.L.og_tracer_mass(self.h, _pd(out))
        return out[:self.ntr]

    def begin_step(self, it):
        self.L.og_begin_step(self.h, it)

    def btrack(self):
        self.L.og_btrack(self.h)

    def prepare_elevation(self, time):
        self.L.og_prepare_elevation(self.h, time)

    def assemble(self, time):
        self.L.og_assemble(self.h, time)

    def essential_bc(self):
        self.L.og_essential_bc(self.h)

    def jcg_solve(self, rtol, maxiter, check_every=10):
        rel = c_double(0.0)
        its = self.L.og_jcg_solve(self.h, rtol, maxiter, check_every, ctypes.byref(rel))
        return its, rel.value

    def update_elevation(self):
        self.L.og_update_elevation(self.h)

    def momentum(self, time):
        self.L.og_momentum(self.h, time)

    def vertical_velocity(self):
        self.L.og_vertical_velocity(self.h)

    def transport(self, dt):
        return self.L.og_transport(self.h, dt)

    def levels(self, it):
        self.L.og_levels(self.h, it)

    def nodal_velocities(self):
        self.L.og_nodal_velocities(self.h)
