"""Host front end of a batch of SCHISM members resident on one B200 (C ABI gs_ctx).

    model = Model([case_a, case_b], precision="fp64")
    model.step(100)                 # every member advances 100 steps, one launch per phase
    eta = model.get(0, "ETA2")      # reference numbering of member 0's own input

Members share the vertical grid and the physics constants; meshes, forcing and initial tracers
are per member.  This mirrors the reference driver loop (src/python/main.py:834-849 calling
schism_step, src/python/schism_step.py:95) with the per-kernel calls replaced by whole-phase
launches over the batch.
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Sequence

import numpy as np

from . import _lib as L
from .cases import Case

FIELDS = dict(ETA1=0, ETA2=1, NODE_Z=2, NODE_U2=3, NODE_W2=4, NODE_TR=5, NODE_KB=6, NODE_DRY=7, QEL=8, NODE_TAU=9,
              SIDE_U2=10, SIDE_BTU=11, SIDE_ZC=12, SIDE_KB=13, SIDE_DRY=14, SIDE_U=15, SIDE_HHAT=16,
              SIDE_CHI=17, SIDE_QH=18, SIDE_BTELEM=19, SIDE_GRADETA1=20, SIDE_GRADETA2=21,
              ELEM_Z=30, ELEM_W=31, ELEM_QV=32, ELEM_TR=33, ELEM_KB=34, ELEM_DRY=35, ELEM_GHAT=36,
              CSR_DATA=40, CSR_INDPTR=41, CSR_INDICES=42, JCG_X=43, ELBC=44, JCG_X1=45, JCG_X2=46, NODE_RHO=47,
              ELEM_RHO=48)
# the fields one step reads from the step before
STATE_FIELDS = ("ETA1", "ETA2", "NODE_Z", "NODE_U2", "NODE_W2", "NODE_TR", "NODE_KB", "NODE_DRY", "SIDE_U2",
                "SIDE_ZC", "SIDE_KB", "SIDE_DRY", "ELEM_Z", "ELEM_TR", "ELEM_KB", "ELEM_DRY", "JCG_X", "JCG_X1",
                "JCG_X2")
INT_FIELDS = {"NODE_KB", "NODE_DRY", "SIDE_KB", "SIDE_DRY", "SIDE_BTELEM", "ELEM_KB", "ELEM_DRY",
              "CSR_INDPTR", "CSR_INDICES"}


def _same_batch(a: Case, b: Case) -> bool:
    """The context takes the vertical grid and the physics constants from its first member."""
    va, vb = a.vgrid, b.vgrid
    same_vg = (va.nvrt == vb.nvrt and va.nz == vb.nz and va.h_s == vb.h_s and va.h_c == vb.h_c
               and va.theta_b == vb.theta_b and va.theta_f == vb.theta_f
               and np.array_equal(va.ztot, vb.ztot) and np.array_equal(va.sigma, vb.sigma))
    return same_vg and a.ntracers == b.ntracers and a.params == b.params


def footprint_bytes(cases: Sequence[Case]) -> int:
    """Upper bound of the device memory a context holding these members allocates
    (gs_footprint_bytes, plus the TVD and vertical-FCT scratch arrays of itr_met 3 and 4).  Side
    and matrix counts follow from the triangulation: a simply connected triangulated domain has
    np + ne - 1 sides and np + 2 ns matrix entries."""
    lib = L.load()
    c0 = cases[0]
    npn = sum(c.n_nodes for c in cases)
    ne = sum(c.n_elems for c in cases)
    ns = sum(c.n_nodes + c.n_elems - 1 for c in cases)
    b = int(lib.gs_footprint_bytes(c0.vgrid.nvrt, c0.ntracers, len(cases), npn, ne, ns, npn + 2 * ns))
    nvrt, ntr, itr = c0.vgrid.nvrt, c0.ntracers, int(c0.params.itr_met)
    if itr >= 3:
        b += ne * nvrt * ntr * 8          # TVD inflow sums
    if itr == 4:
        b += ne * nvrt * 8                # vertical sweep scratch
    return b


def _pd(a):
    return a.ctypes.data_as(L.PD)


def _pi(a):
    return a.ctypes.data_as(L.PI)


def _flat(segs):
    start = np.zeros(len(segs) + 1, dtype=np.int32)
    for k, s in enumerate(segs):
        start[k + 1] = start[k] + len(s)
    nodes = np.concatenate([np.asarray(s, dtype=np.int32) for s in segs]) if segs else np.zeros(1, np.int32)
    return start, np.ascontiguousarray(nodes, dtype=np.int32)


class Model:
    def __init__(self, cases: Sequence[Case], precision: str = "fp64", device: int = 0,
                 rtol: float | None = None, maxiter: int | None = None, check_every: int | None = None,
                 ir_inner_rtol: float = 0.1, ir_inner_maxiter: int = 400, defer_device: bool = False):
        """A batch context of `cases`.  With defer_device the constructor only does the host
        preparation (gs_ctx_prepare, no CUDA call: fit for a worker thread) and finalize() later
        allocates and uploads the device state."""
        self.lib = L.load()
        self.cases: List[Case] = list(cases)
        c0 = self.cases[0]
        vg, p = c0.vgrid, c0.params
        for c in self.cases[1:]:
            if not _same_batch(c, c0):
                raise ValueError("members of one batch share the vertical grid, the tracer count and the "
                                 "physics parameters (Params)")
        self._keep = []
        self._pinned = []
        k = self._k
        cfg = L.GsConfig()
        cfg.nvrt, cfg.ntr, cfg.nz = vg.nvrt, c0.ntracers, vg.nz
        cfg.h_s, cfg.h_c, cfg.theta_b, cfg.theta_f = vg.h_s, vg.h_c, vg.theta_b, vg.theta_f
        cfg.ztot, cfg.sigma = _pd(k(vg.ztot, np.float64)), _pd(k(vg.sigma, np.float64))
        for name in ("dt", "thetai", "h0", "dtb_min", "dtb_max", "velmin_btrack", "rmaxvel", "dfv0", "coricoef",
                     "rho0", "grav", "dramp"):
            setattr(cfg, name, float(getattr(p, name)))
        cfg.ihhat = int(p.ihhat)
        cfg.rtol = float(rtol if rtol is not None else p.rtol)
        cfg.maxiter = int(maxiter if maxiter is not None else p.maxiter)
        cfg.check_every = int(check_every if check_every is not None else p.check_every)
        cfg.precision = {"fp64": L.GS_FP64, "fp32_ir": L.GS_FP32_IR}[precision]
        cfg.ir_inner_rtol, cfg.ir_inner_maxiter = float(ir_inner_rtol), int(ir_inner_maxiter)
        cfg.device = int(device)
        cfg.itr_met, cfg.tvd_limiter, cfg.dfh0 = int(p.itr_met), int(p.tvd_limiter), float(p.dfh0)
        self.precision = precision
        h = ctypes.c_void_p()
        L.check(self.lib.gs_ctx_create(ctypes.byref(cfg), ctypes.byref(h)), None, "gs_ctx_create")
        self.h = h
        for c in self.cases:
            self._add(c)
        self.nvrt, self.ntr = vg.nvrt, c0.ntracers
        self.sizes = None
        if defer_device:
            L.check(self.lib.gs_ctx_prepare(self.h), self.h, "gs_ctx_prepare")
        else:
            self.finalize()

    def finalize(self) -> None:
        """Device half of the set-up (gs_ctx_finalize); a no-op once done."""
        if self.sizes is not None:
            return
        L.check(self.lib.gs_ctx_finalize(self.h), self.h, "gs_ctx_finalize")
        sizes = []
        for m in range(len(self.cases)):
            a, b, cc, d = (ctypes.c_int() for _ in range(4))
            L.check(self.lib.gs_member_sizes(self.h, m, ctypes.byref(a), ctypes.byref(b), ctypes.byref(cc),
                                             ctypes.byref(d)), self.h)
            sizes.append(dict(np=a.value, ne=b.value, ns=cc.value, nnz=d.value))
        self.sizes = sizes

    def _k(self, a, dt):
        a = np.ascontiguousarray(a, dtype=dt)
        self._keep.append(a)
        return a

    def _add(self, c: Case) -> int:
        k = self._k
        d = L.GsMemberDesc()
        d.np, d.ne, d.nope, d.nland, d.nbfr = c.n_nodes, c.n_elems, len(c.open_bnd), len(c.land_bnd), len(c.amig)
        d.x, d.y, d.depth = _pd(k(c.x, np.float64)), _pd(k(c.y, np.float64)), _pd(k(c.depth, np.float64))
        d.drag, d.tau, d.tr_init = _pd(k(c.drag, np.float64)), _pd(k(c.tau, np.float64)), _pd(k(c.tr_init, np.float64))
        d.elnode = _pi(k(c.elnode, np.int32))
        os_, on = _flat(c.open_bnd)
        ls_, ln = _flat(c.land_bnd)
        d.open_start, d.open_nodes = _pi(k(os_, np.int32)), _pi(k(on, np.int32))
        d.land_start, d.land_nodes = _pi(k(ls_, np.int32)), _pi(k(ln, np.int32))
        d.iettype = _pi(k(c.iettype if len(c.iettype) else np.zeros(1), np.int32))
        d.amig, d.ff, d.face = _pd(k(c.amig, np.float64)), _pd(k(c.ff, np.float64)), _pd(k(c.face, np.float64))
        nb = max(len(c.amig), 1)
        emo = np.concatenate(c.emo, axis=0) if c.open_bnd else np.zeros((1, nb))
        efa = np.concatenate(c.efa, axis=0) if c.open_bnd else np.zeros((1, nb))
        d.emo, d.efa = _pd(k(emo, np.float64)), _pd(k(efa, np.float64))
        mid = ctypes.c_int()
        L.check(self.lib.gs_member_add(self.h, ctypes.byref(d), ctypes.byref(mid)), self.h, "gs_member_add")
        return mid.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.gs_ctx_destroy(self.h)
            self.h = None
        for rec in getattr(self, "_pinned", []):
            rec.free()
        self._pinned = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ----------------------------------------------------------------------------- stepping
    def step(self, nsteps: int = 1) -> None:
        L.check(self.lib.gs_step(self.h, int(nsteps)), self.h, "gs_step")

    def phase(self, name: str, arg: int = 0) -> None:
        L.check(self.lib.gs_phase(self.h, L.PHASE[name], int(arg)), self.h, f"gs_phase {name}")

    def set_wait_limit(self, polls: int) -> None:
        """Bound of the device waits in polls (gs_set_wait_limit; 0 = the default, about 2 s)."""
        L.check(self.lib.gs_set_wait_limit(self.h, int(polls)), self.h, "gs_set_wait_limit")

    def test_stall_solve(self, member: int) -> None:
        """Recovery tests only (gs_test_stall_solve): the member's next solves wait for an arrival
        that never comes, so their bounded waits run out; -1 switches it off."""
        L.check(self.lib.gs_test_stall_solve(self.h, int(member)), self.h, "gs_test_stall_solve")

    def set_stream(self, stream_ptr: int | None) -> None:
        """Issue the member work on a caller cudaStream_t (e.g. torch.cuda.Stream().cuda_stream)."""
        L.check(self.lib.gs_set_stream(self.h, ctypes.c_void_p(stream_ptr or None)), self.h, "gs_set_stream")

    def sync(self) -> None:
        L.check(self.lib.gs_sync(self.h), self.h, "gs_sync")

    def stats(self, member: int = 0) -> dict:
        s = L.GsStats()
        L.check(self.lib.gs_get_stats(self.h, member, ctypes.byref(s)), self.h, "gs_get_stats")
        return {f: getattr(s, f) for f, _ in L.GsStats._fields_}

    def set_launch(self, kernel: str, a: int, b: int) -> None:
        """Launch shape of one kernel (gs_set_launch): threads per block and grid cap in blocks
        per SM, or for JCG_TILES the tiles of a large member and the smallest tile in rows."""
        L.check(self.lib.gs_set_launch(self.h, L.LAUNCH[kernel], int(a), int(b)), self.h, f"gs_set_launch {kernel}")

    def get_launch(self, kernel: str):
        a, b = ctypes.c_int(), ctypes.c_int()
        L.check(self.lib.gs_get_launch(self.h, L.LAUNCH[kernel], ctypes.byref(a), ctypes.byref(b)), self.h,
                f"gs_get_launch {kernel}")
        return a.value, b.value

    def launch_table(self) -> dict:
        return {k: self.get_launch(k) for k in L.LAUNCH}

    def tracer_mass(self, member: int = 0) -> np.ndarray:
        """FP64 tracer mass of a member (sum of prism volume x concentration per tracer,
        compensated, deterministic): gs_tracer_mass."""
        out = np.zeros(self.ntr, dtype=np.float64)
        if self.ntr:
            L.check(self.lib.gs_tracer_mass(self.h, member, _pd(out)), self.h, "gs_tracer_mass")
        return out

    # ----------------------------------------------------------------------------- state
    def shape(self, member: int, name: str):
        sz = self.sizes[member]
        n = {"N": sz["np"], "S": sz["ns"], "E": sz["ne"]}
        nv, nt = self.nvrt, self.ntr
        table = {"ETA1": ("N",), "ETA2": ("N",), "QEL": ("N",), "ELBC": ("N",), "JCG_X": ("N",),
                 "JCG_X1": ("N",), "JCG_X2": ("N",), "NODE_KB": ("N",), "NODE_DRY": ("N",),
                 "SIDE_KB": ("S",), "SIDE_DRY": ("S",), "SIDE_HHAT": ("S",), "SIDE_CHI": ("S",),
                 "ELEM_KB": ("E",), "ELEM_DRY": ("E",)}
        if name in table:
            return (n[table[name][0]],)
        if name in ("SIDE_U", "SIDE_GRADETA1", "SIDE_GRADETA2"):
            return (n["S"], 2)
        if name == "NODE_TAU":
            return (n["N"], 2)
        if name == "ELEM_GHAT":
            return (n["E"], 2)
        if name in ("NODE_Z", "NODE_W2", "NODE_RHO"):
            return (nv, n["N"])
        if name == "NODE_U2":
            return (nv, n["N"], 2)
        if name == "NODE_TR":
            return (nt, nv, n["N"])
        if name in ("SIDE_U2", "SIDE_BTU"):
            return (nv, n["S"], 2)
        if name in ("SIDE_ZC", "SIDE_QH", "SIDE_BTELEM"):
            return (nv, n["S"])
        if name in ("ELEM_Z", "ELEM_W", "ELEM_QV", "ELEM_RHO"):
            return (nv, n["E"])
        if name == "ELEM_TR":
            return (nt, nv, n["E"])
        if name in ("CSR_DATA", "CSR_INDICES"):
            return (sz["nnz"],)
        if name == "CSR_INDPTR":
            return (sz["np"] + 1,)
        raise KeyError(name)

    def get(self, member: int, name: str) -> np.ndarray:
        out = np.zeros(self.shape(member, name), dtype=np.int32 if name in INT_FIELDS else np.float64)
        return self.get_into(member, name, out)

    def get_into(self, member: int, name: str, out: np.ndarray) -> np.ndarray:
        """gs_state_get into a caller array of the field's shape and type (page-locked memory
        takes a direct copy)."""
        if out.shape != self.shape(member, name) or out.dtype != (np.int32 if name in INT_FIELDS else np.float64) \
                or not out.flags.c_contiguous:
            raise ValueError(f"{name}: wrong output array")
        L.check(self.lib.gs_state_get(self.h, member, FIELDS[name], out.ctypes.data_as(ctypes.c_void_p),
                                      out.nbytes), self.h, f"gs_state_get {name}")
        return out

    def put(self, member: int, name: str, value) -> None:
        a = np.ascontiguousarray(value, dtype=np.int32 if name in INT_FIELDS else np.float64)
        if a.shape != self.shape(member, name):
            raise ValueError(f"{name}: shape {a.shape} != {self.shape(member, name)}")
        L.check(self.lib.gs_state_put(self.h, member, FIELDS[name], a.ctypes.data_as(ctypes.c_void_p), a.nbytes),
                self.h, f"gs_state_put {name}")

    def set_vortex(self, member: int, vortex) -> None:
        """Storm forcing of a member (gs_set_vortex): a mapping with x0, y0, heading, speed, vmax,
        rmax, holland_b, rho_air, or None to switch it off."""
        if vortex is None:
            L.check(self.lib.gs_set_vortex(self.h, member, None), self.h, "gs_set_vortex")
            return
        v = L.GsVortex(**{k: float(vortex[k]) for k, _ in L.GsVortex._fields_})
        L.check(self.lib.gs_set_vortex(self.h, member, ctypes.byref(v)), self.h, "gs_set_vortex")

    def set_tau(self, member: int, tau) -> None:
        a = np.ascontiguousarray(tau, dtype=np.float64)
        L.check(self.lib.gs_set_tau(self.h, member, _pd(a)), self.h, "gs_set_tau")

    # ----------------------------------------------------------------------------- slots
    def member_state(self, member: int, pinned: bool = False) -> Dict[str, np.ndarray]:
        """The fields a step reads from the step before (every other field is recomputed before
        use), in reference numbering: taken right after construction it is the member's
        cold-start state.  `pinned`: in page-locked buffers owned by this Model (freed by close),
        so that putting the state back is one direct copy per field."""
        if not pinned:
            return {f: self.get(member, f) for f in STATE_FIELDS}
        from .output import _PinnedRecord
        rec = _PinnedRecord(self.lib, {f: self.shape(member, f) for f in STATE_FIELDS},
                            {f: (np.int32 if f in INT_FIELDS else np.float64) for f in STATE_FIELDS})
        self._pinned.append(rec)
        for f in STATE_FIELDS:
            self.get_into(member, f, rec.arrays[f])
        return rec.arrays

    def put_member_state(self, member: int, state: Dict[str, np.ndarray]) -> None:
        for f in STATE_FIELDS:
            self.put(member, f, state[f])

    def set_member_start(self, member: int, start: int) -> None:
        """The member's own step = the context's step - start (gs_set_member_start); a start
        above the context's step parks it (L.GS_MEMBER_PARKED: for good)."""
        L.check(self.lib.gs_set_member_start(self.h, int(member), int(start)), self.h, "gs_set_member_start")

    def current_step(self) -> int:
        s = ctypes.c_int()
        L.check(self.lib.gs_get_step(self.h, ctypes.byref(s)), self.h, "gs_get_step")
        return s.value

    def admit(self, member: int, cold: Dict[str, np.ndarray], tau=None, vortex=None) -> int:
        """Start a new run in a member slot at the next step: its cold-start state, its forcing,
        and its clock from step 1.  Returns the context step the run started after."""
        self.put_member_state(member, cold)
        n = self.shape(member, "NODE_TAU")
        self.set_tau(member, np.zeros(n) if tau is None else tau)
        self.set_vortex(member, vortex)
        start = self.current_step()
        self.set_member_start(member, start)
        return start

    def park(self, member: int, cold: Dict[str, np.ndarray]) -> None:
        """Retire the member's run: back to its cold-start state, no stress, no storm, parked."""
        self.set_member_start(member, L.GS_MEMBER_PARKED)
        self.set_vortex(member, None)
        self.set_tau(member, np.zeros(self.shape(member, "NODE_TAU")))
        self.put_member_state(member, cold)
