"""The reference's own step, run on the CPU (test infrastructure only).

`RefStep(case)` writes the case in SCHISM's file formats, reads it back with the reference's own
grid reader (src/grid/read_and_process_grid.cpp readHGrid/readVGrid, compiled by
oracle/build.py:build_ref), builds the reference's mesh with its populate kernels and steps it
with its own kernels in the order of src/python/schism_step.py:95-334 (oracle/refemu/ref_step.cpp
compiled by oracle/refemu/build.py).  Only the elevation solve and the transport sub-step minimum
are restated (pcg_solver.py:1075-1124, meshdata.cu:6842-6863); every other number comes from the
reference's kernels.

One RefStep per process: the reference keeps its mesh in a process-wide global
(`__device__ Mesh* mesh`, meshdata.cu:16), so each library instance holds one mesh.

Inputs the reference takes from its namelist and forcing files are set from the case: M2/S2
constituents on open segments with iettype 3, no wind (nws = 0), drag per node (nchi = 0), the
ramp `dramp` in days, tracers initialised vertically uniform from `tr_init[:, -1]` (the
reference's cold start reads temp.ic/salt.ic per node, main.py:344-372).
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

from . import build as _b
from .. import build as _ob

PD = ctypes.POINTER(ctypes.c_double)
PI = ctypes.POINTER(ctypes.c_int32)

# field codes (oracle/step.h, OGF_*) the reference keeps in its structs
FIELDS = dict(ETA1=0, ETA2=1, NODE_Z=2, NODE_U2=3, NODE_W2=4, NODE_TR=5, NODE_KB=6, NODE_DRY=7, QEL=8,
              NODE_TAU=9, SIDE_U2=10, SIDE_BTU=11, SIDE_ZC=12, SIDE_KB=13, SIDE_DRY=14, SIDE_U=15,
              SIDE_HHAT=16, SIDE_CHI=17, SIDE_QH=18, SIDE_GRADETA1=20, SIDE_GRADETA2=21, ELEM_Z=30,
              ELEM_W=31, ELEM_QV=32, ELEM_TR=33, ELEM_KB=34, ELEM_DRY=35, ELEM_GHAT=36, CSR_DATA=40,
              CSR_INDPTR=41, CSR_INDICES=42, JCG_X=43, ELBC=44, JCG_X1=45, JCG_X2=46, NODE_RHO=47, ELEM_RHO=48)
INT_FIELDS = {"NODE_KB", "NODE_DRY", "SIDE_KB", "SIDE_DRY", "ELEM_KB", "ELEM_DRY", "CSR_INDPTR", "CSR_INDICES"}


class RefInput(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("np", "ne", "ns", "nope", "nland", "mnond", "mnlnd", "nbfr",
                                             "nbnd_nodes", "nbnd_sides")] + \
        [(n, PI) for n in ("i34", "elnode", "elside")] + [("coords", PD)] + \
        [(n, PI) for n in ("isdel", "isidenode", "isbnd", "nond", "nlnd", "iond", "ilnd",
                           "nnp_start", "nnp", "nne_start", "nne")] + \
        [(n, PD) for n in ("drag", "temp", "salt")] + [("kb", PI), ("sigma_lcl", PD)] + \
        [(n, ctypes.c_double) for n in ("h_c", "h_s", "theta_b", "theta_f")] + \
        [(n, PD) for n in ("sigma", "ztot", "cs", "dcs")] + [("n_sigma", ctypes.c_int), ("n_ztot", ctypes.c_int)] + \
        [(n, PD) for n in ("amig", "face", "ff", "emo", "efa", "umo", "ufa", "vmo", "vfa")] + \
        [("ifltype", PI), ("iettype", PI), ("qthcon", PD), ("eth", PD)]


def _quiet(fn):
    """Run fn with the process's stdout sent to /dev/null (the reference prints progress)."""
    import sys
    sys.stdout.flush()
    fd = os.dup(1)
    nul = os.open(os.devnull, os.O_WRONLY)
    os.dup2(nul, 1)
    try:
        return fn()
    finally:
        try:
            ctypes.CDLL(None).fflush(None)
        except Exception:
            pass
        os.dup2(fd, 1)
        os.close(fd)
        os.close(nul)


class RefStep:
    """One case stepped by the reference's kernels on the CPU."""

    def __init__(self, case, rtol=None, maxiter=None, check_every=None, quiet=True, atomic_order=0, dot_order=0,
                 fma=False):
        """atomic_order 1 runs the kernels whose sums are atomic updates (nodal velocities,
        open-boundary velocities, boundary areas) in reversed thread order; dot_order 1 sums the
        solver's dot products in 32-entry blocks added pairwise; fma compiles the kernels with
        contracted multiply-adds.  Each is a choice a GPU run of the reference makes (thread
        order, library reduction order, nvcc's default contraction), so runs that differ in them
        show the reference's own reproducibility."""
        self.case = case
        self.quiet = quiet
        ref = _ob.load_ref() if os.path.exists(_ob.ref_module_path()) else None
        if ref is None:
            _ob.build_ref()
            ref = _ob.load_ref()
        if ref is None:
            raise RuntimeError("the reference grid reader is not available")
        with tempfile.TemporaryDirectory() as d:
            from gschism_b200 import cases as _cases
            _cases.write_case(case, d)
            out = self._run(lambda: ref.readHGrid(os.path.join(d, "hgrid.gr3"), "", 1, 0))
            vg = self._run(lambda: ref.readVGrid(os.path.join(d, "vgrid.in"), case.n_nodes))
        (i34, _pe, _pn, _ps, elnode, elside, coords, _ll, _ic3, isdel, isidenode, isbnd, nond, nlnd, iond,
         ilnd, nne, nnp, _ne, _nn, _ns, nbn, nbs) = out
        nope, mnond = np.asarray(iond).shape
        nland, mnlnd = np.asarray(ilnd).shape
        self.grid = dict(elside=np.asarray(elside), isdel=np.asarray(isdel), isidenode=np.asarray(isidenode))
        lib_path = _b.build_for(case, mnond, mnlnd, fma=fma)
        self.L = L = ctypes.CDLL(lib_path)
        L.rd_create.argtypes = [ctypes.POINTER(RefInput)]
        L.rd_kernel.argtypes = [ctypes.c_char_p, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.rd_time_ramps.argtypes = [ctypes.c_double, ctypes.c_double]
        L.rd_min_transport_dt.restype = ctypes.c_double
        L.rd_transport.argtypes = [ctypes.c_double]
        L.rd_set_solver.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.rd_set_atomic_order.argtypes = [ctypes.c_int]
        L.rd_set_dot_order.argtypes = [ctypes.c_int]
        L.rd_xfer.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        self._keep = []

        def F(a, dt):
            a = np.asfortranarray(np.asarray(a, dtype=dt))
            self._keep.append(a)
            return a

        p = case.params
        nbfr = int(case.amig.shape[0])
        ri = RefInput()
        ri.np, ri.ne, ri.ns = case.n_nodes, case.n_elems, int(np.asarray(isdel).shape[1])
        ri.nope, ri.nland, ri.mnond, ri.mnlnd, ri.nbfr = nope, nland, mnond, mnlnd, nbfr
        ri.nbnd_nodes, ri.nbnd_sides = int(np.asarray(nbn)[0]), int(np.asarray(nbs)[0])
        pi = lambda a: F(a, np.int32).ctypes.data_as(PI)
        pd = lambda a: F(a, np.float64).ctypes.data_as(PD)
        ri.i34, ri.elnode, ri.elside = pi(i34), pi(elnode), pi(elside)
        ri.coords = pd(coords)
        ri.isdel, ri.isidenode, ri.isbnd = pi(isdel), pi(isidenode), pi(isbnd)
        ri.nond, ri.nlnd, ri.iond, ri.ilnd = pi(nond), pi(nlnd), pi(iond), pi(ilnd)
        ri.nnp_start, ri.nnp = pi(nnp[1]), pi(nnp[0])
        ri.nne_start, ri.nne = pi(nne[1]), pi(nne[0])
        tr_top = np.asarray(case.tr_init[:, -1, :], dtype=np.float64)
        ri.drag = pd(case.drag)
        ri.temp = pd(tr_top[0])
        ri.salt = pd(tr_top[1] if case.ntracers > 1 else tr_top[0])
        ri.kb = pi(np.zeros(case.n_nodes, np.int32))
        ri.sigma_lcl = pd(np.zeros(case.n_nodes * case.nvrt))
        ints, ztot, _kb, (h_c, h_s, theta_b, theta_f), _sl, sigma, cs, dcs = vg
        ri.h_c, ri.h_s, ri.theta_b, ri.theta_f = float(h_c), float(h_s), float(theta_b), float(theta_f)
        ri.sigma, ri.ztot, ri.cs, ri.dcs = pd(sigma), pd(ztot), pd(cs), pd(dcs)
        ri.n_sigma, ri.n_ztot = int(np.asarray(sigma).size), int(np.asarray(ztot).size)
        ri.amig, ri.face, ri.ff = pd(case.amig), pd(case.face), pd(case.ff)
        emo = np.zeros((nope, mnond, max(nbfr, 1)))
        efa = np.zeros_like(emo)
        for k, seg in enumerate(case.open_bnd):
            emo[k, :seg.size, :nbfr] = case.emo[k]
            efa[k, :seg.size, :nbfr] = case.efa[k]
        ri.emo, ri.efa = pd(emo), pd(efa)
        z3 = np.zeros_like(emo)
        ri.umo, ri.ufa, ri.vmo, ri.vfa = pd(z3), pd(z3), pd(z3), pd(z3)
        ri.ifltype = pi(np.zeros(nope, np.int32))
        ri.iettype = pi(np.asarray(case.iettype, np.int32))
        ri.qthcon, ri.eth = pd(np.zeros(nope)), pd(np.zeros(nope))
        self._ri = ri
        rc = self._run(lambda: L.rd_create(ctypes.byref(ri)))
        if rc != 0:
            raise RuntimeError(f"rd_create failed: {rc}")
        L.rd_set_solver(float(p.rtol if rtol is None else rtol), int(p.maxiter if maxiter is None else maxiter),
                        int(p.check_every if check_every is None else check_every))
        L.rd_set_atomic_order(int(atomic_order))
        L.rd_set_dot_order(int(dot_order))
        cnt = (ctypes.c_int * 8)()
        L.rd_counts(cnt)
        self.np_, self.ne_, self.ns_, self.nnz = cnt[0], cnt[1], cnt[2], cnt[5]
        # surface stress: with nws = 0 the reference never overwrites Node::tau (setWinds,
        # meshdata.cu:3976, is called only for nws != 0), so a stress set here stays constant
        self.put("NODE_TAU", np.asarray(case.tau, dtype=np.float64))
        self.init()

    def _run(self, fn):
        return _quiet(fn) if self.quiet else fn()

    def k(self, name: str, t: float = 0.0, i1: int = 0, i2: int = 0) -> None:
        rc = self.L.rd_kernel(name.encode(), float(t), int(i1), int(i2))
        if rc != 0:
            raise KeyError(name)

    # ------------------------------------------------------------ cold start / step --------
    def init(self) -> None:
        """schism_init.py:78-103 (inunfl = 0)."""
        def go():
            for n in ("ul0UpdateZCoords", "ul0ComputeDryElements", "ul0ComputeDryNodes"):
                self.k(n)
            self.k("ul0UpdateRewettedNodes", 0, 0, 0)
            self.k("ul0UpdateSides", 0, 0, 0)
            self.k("ul0UpdateSides2")
            self.k("computeNodeDensity")
            self.k("computeElemDensity")
        self._run(go)

    def begin_step(self, it: int) -> float:
        """schism_step.py:95-151: gravity, time ramps, bed deformation, tidal potential, BCs,
        boundary areas, drag, turbulence, horizontal viscosity."""
        time = it * self.case.params.dt

        def go():
            self.k("scaleGravity", 0.1)
            self.L.rd_time_ramps(time, float(self.case.params.dramp))
            self.k("computeBedDeformation")
            self.k("computeTidalPotential", time)
            self.k("getBoundaryConditions", time)
            self.k("resetBoundaryAreas")
            self.k("computeBoundaryAreas")
            self.k("computeFlowBcVelocities", time)
            self.k("computeBottomDragVegetation")
            self.k("computeTurbulence")
            self.k("computeHorizontalViscosity")
        self._run(go)
        return time

    def btrack(self):
        self._run(lambda: self.k("backtrackAllNodes"))

    def prepare_elevation(self, time):
        """schism_step.py:211-234: elevation BCs, U, drag parameters, density gradient,
        baroclinic term, element-averaged ghat."""
        def go():
            self.k("computeElevationBoundaryConditions", time)
            self.k("computeVerticallyIntegratedVelocity")
            self.k("computeVegetationAndDragParameters")
            self.k("computeDensityGradient")
            self.k("computeBaroclinicTerm")
            self.k("computeElemAverageGhat")
        self._run(go)

    def assemble(self, time):
        self._run(lambda: self.k("setupCoefficientMatrixAndRHS", time))

    def essential_bc(self):
        def go():
            self.k("rollUpElevation")
            self.k("setEssentialBC")
        self._run(go)

    def solve(self) -> int:
        return self._run(lambda: self.L.rd_solve())

    def update_elevation(self):
        self._run(lambda: self.k("updateElevation"))

    def momentum(self, time):
        def go():
            self.k("computeHorGradientAtSide")
            self.k("solveMomentumEquations", time)
            self.k("applyMomentumBC")
        self._run(go)

    def vertical_velocity(self):
        self._run(lambda: self.k("computeVerticalVelocity"))

    def transport(self, dt=None) -> int:
        return self._run(lambda: self.L.rd_transport(float(self.case.params.dt if dt is None else dt)))

    def levels(self, it):
        def go():
            self.k("ul0UpdateZCoords")
            self.k("ul0ComputeDryElements")
            self.k("ul0ComputeDryNodes")
            self.k("ul0UpdateRewettedNodes", 0, it, 0)
            self.k("ul0UpdateSides", 0, it, 0)
            self.k("ul0UpdateSides2")
            self.k("computeNodeDensity")
            self.k("computeElemDensity")
        self._run(go)

    def nodal_velocities(self):
        def go():
            for n in ("zeroNodalVelocities", "computeNodalVerticalVelocities1", "computeNodalVerticalVelocities2",
                      "computeNodalHorizontalVelocities1", "computeNodalHorizontalVelocities2",
                      "resetVelocityOpenBndNodes", "setVelocityOpenBndNodes"):
                self.k(n)
        self._run(go)

    def step(self, it: int) -> int:
        """One whole step, schism_step.py:95-334 (ishapiro = 0: no Shapiro filter)."""
        time = self.begin_step(it)
        self.btrack()
        self.prepare_elevation(time)
        self.assemble(time)
        self.essential_bc()
        its = self.solve()
        self.update_elevation()
        self.momentum(time)
        self.vertical_velocity()
        self.transport()
        self.levels(it)
        self.nodal_velocities()
        return its

    def counts(self):
        c = (ctypes.c_int * 8)()
        self.L.rd_counts(c)
        return dict(np=c[0], ne=c[1], ns=c[2], nbp=c[3], nbs=c[4], nnz=c[5], jcg_iters=c[6], substeps=c[7])

    # ------------------------------------------------------------ fields --------
    def shape(self, name):
        nv, nt = self.case.nvrt, self.case.ntracers
        n = {"N": self.np_, "S": self.ns_, "E": self.ne_}[name[0] if name[:4] in ("NODE", "SIDE", "ELEM") else "N"]
        per_level = name in ("NODE_Z", "NODE_U2", "NODE_W2", "SIDE_U2", "SIDE_BTU", "SIDE_ZC", "SIDE_QH",
                             "ELEM_Z", "ELEM_W", "ELEM_QV", "NODE_RHO", "ELEM_RHO")
        vec = name in ("NODE_U2", "SIDE_U2", "SIDE_BTU", "SIDE_U", "SIDE_GRADETA1", "SIDE_GRADETA2",
                       "ELEM_GHAT", "NODE_TAU")
        if name in ("CSR_DATA", "CSR_INDICES"):
            return (self.nnz,)
        if name == "CSR_INDPTR":
            return (self.np_ + 1,)
        if name in ("NODE_TR", "ELEM_TR"):
            return (nt, nv, n)
        shp = ((nv,) if per_level else ()) + (n,) + ((2,) if vec else ())
        return shp

    def get(self, name: str) -> np.ndarray:
        a = np.zeros(self.shape(name), dtype=np.int32 if name in INT_FIELDS else np.float64)
        if self.L.rd_xfer(FIELDS[name], a.ctypes.data_as(ctypes.c_void_p), 1) != 0:
            raise KeyError(name)
        return a

    def put(self, name: str, value) -> None:
        a = np.ascontiguousarray(value, dtype=np.int32 if name in INT_FIELDS else np.float64).reshape(self.shape(name))
        if self.L.rd_xfer(FIELDS[name], a.ctypes.data_as(ctypes.c_void_p), 0) != 0:
            raise KeyError(name)
