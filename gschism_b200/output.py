"""Streamed model output in the reference's NetCDF layout.

Replaces the reference's output path: DeviceToHost (src/iop/deviceToHost.py:37-224), which reads
one field at a time from the device, and writeOutput (src/iop/writeOutput.py:53-375), which
writes every `nspool` steps into files of `ihfskip / nspool` records:

    out2d_<n>.nc              elevation, dryFlagNode, dryFlagElement, dryFlagSide + the 2-D grid
    horizontalVelX_<n>.nc     horizontalVelX  (time, node, layer)
    horizontalVelY_<n>.nc     horizontalVelY
    verticalVelocity_<n>.nc   verticalVelocity
    zCoordinates_<n>.nc       zCoordinates
    verticalVelAtElement_<n>.nc  verticalVelAtElement (time, face, layer)
    temperature_<n>.nc, salinity_<n>.nc   first and second tracer at the nodes

with the reference's dimension and variable names (nSCHISM_hgrid_node/face/edge,
nSCHISM_vgrid_layers, time; SCHISM_hgrid_face_nodes and _edge_nodes 1-based with fill -1; data
in float32).  Files are NetCDF classic with 64-bit offsets (scipy.io.netcdf_file), readable by
the same tools as the reference's NETCDF4 files.  Not written: wind (windSpeedX/Y: this build has
no atmospheric forcing files) and the turbulence/density files (viscosity, turbulentKineticEner,
mixingLength, waterDensity: constant viscosity and no density in the supported physics).

How it streams: after every output step `OutputWriter.step_done` queues, on the context's stream,
one asynchronous read per field (gs_state_get_async: the renumbering runs on the device, one copy
per field into page-locked memory) and a mark (gs_output_mark), then returns; a writer thread
waits for the mark (gs_output_wait) and writes the record while the stepping thread goes on.  A
ring of `ring` page-locked record buffers bounds how far the steps may run ahead of the writer.
"""
from __future__ import annotations

import ctypes
import os
import queue
import threading
from typing import Dict, List, Optional

import numpy as np

from . import _lib as L

# file -> [(variable, model field, component or tracer index, entity)]
FILES = {
    "out2d": [("elevation", "ETA2", None, "node"), ("dryFlagNode", "NODE_DRY", None, "node"),
              ("dryFlagElement", "ELEM_DRY", None, "face"), ("dryFlagSide", "SIDE_DRY", None, "edge")],
    "horizontalVelX": [("horizontalVelX", "NODE_U2", 0, "node")],
    "horizontalVelY": [("horizontalVelY", "NODE_U2", 1, "node")],
    "verticalVelocity": [("verticalVelocity", "NODE_W2", None, "node")],
    "zCoordinates": [("zCoordinates", "NODE_Z", None, "node")],
    "verticalVelAtElement": [("verticalVelAtElement", "ELEM_W", None, "face")],
    "temperature": [("temperature", "NODE_TR", 0, "node")],
    "salinity": [("salinity", "NODE_TR", 1, "node")],
}
DIM = {"node": "nSCHISM_hgrid_node", "face": "nSCHISM_hgrid_face", "edge": "nSCHISM_hgrid_edge"}


def record_to_variables(fields: Dict[str, np.ndarray], ntr: int) -> Dict[str, np.ndarray]:
    """Model fields of one output step -> the reference's variables (float32, per-level fields
    as (entity, layer))."""
    out = {}
    for fname, vars_ in FILES.items():
        for var, field, idx, _ in vars_:
            if field not in fields:
                continue
            if field == "NODE_TR" and (idx is None or idx >= ntr):
                continue
            a = fields[field]
            if field == "NODE_TR":
                a = a[idx].T                      # [nvrt][np] -> (np, nvrt)
            elif field == "NODE_U2":
                a = a[:, :, idx].T                # [nvrt][np][2] -> (np, nvrt)
            elif a.ndim == 2:
                a = a.T                           # [nvrt][n] -> (n, nvrt)
            out[var] = np.ascontiguousarray(a, dtype=np.float32)
    return out


class NetcdfSink:
    """Writes records into the reference's files; no GPU involved (testable on its own)."""

    def __init__(self, out_dir: str, grid: Dict[str, np.ndarray], nvrt: int, ntr: int, dt: float, nspool: int,
                 ihfskip: int, start: str = "2000-01-01T00:00:00+00", files=None):
        self.dir = out_dir
        self.grid = grid
        self.nvrt, self.ntr, self.dt = nvrt, ntr, dt
        self.nspool, self.ihfskip = nspool, ihfskip
        self.per_file = max(1, ihfskip // nspool)
        self.start = start
        self.files = [f for f in (files or FILES) if not (f == "temperature" and ntr < 1)
                      and not (f == "salinity" and ntr < 2)]
        self.open: Dict[str, object] = {}
        self.file_num = 0
        os.makedirs(out_dir, exist_ok=True)

    def _create(self, file_num: int):
        from scipy.io import netcdf_file
        g = self.grid
        npn, ne, ns = g["x"].size, g["face_nodes"].shape[0], g["edge_nodes"].shape[0]
        self.close_files()
        for fname in self.files:
            path = os.path.join(self.dir, f"{fname}_{file_num}.nc")
            f = netcdf_file(path, "w", version=2)
            f.createDimension("time", None)          # the record dimension comes first in this format
            f.createDimension("nSCHISM_hgrid_node", npn)
            f.createDimension("nSCHISM_hgrid_face", ne)
            f.createDimension("nSCHISM_hgrid_edge", ns)
            f.createDimension("nMaxSCHISM_hgrid_face_nodes", 4)
            f.createDimension("nSCHISM_vgrid_layers", self.nvrt)
            f.createDimension("one", 1)
            f.createDimension("two", 2)
            t = f.createVariable("time", "f8", ("time",))
            t.units = f"seconds since {self.start}"
            if fname == "out2d":
                for name, key, dim in (("SCHISM_hgrid_node_x", "x", "node"), ("SCHISM_hgrid_node_y", "y", "node"),
                                       ("SCHISM_hgrid_face_x", "face_x", "face"),
                                       ("SCHISM_hgrid_face_y", "face_y", "face"),
                                       ("SCHISM_hgrid_edge_x", "edge_x", "edge"),
                                       ("SCHISM_hgrid_edge_y", "edge_y", "edge")):
                    v = f.createVariable(name, "f8", (DIM[dim],))
                    v.units = "m"
                    v[:] = g[key]
                v = f.createVariable("depth", "f4", ("nSCHISM_hgrid_node",))
                v.units = "m"
                v[:] = g["depth"]
                v = f.createVariable("bottom_index_node", "i4", ("nSCHISM_hgrid_node",))
                v[:] = g["kb"] + 1
                v = f.createVariable("minimum_depth", "f8", ("one",))
                v[:] = 0.0001
                v = f.createVariable("SCHISM_hgrid_face_nodes", "i4", ("nSCHISM_hgrid_face", "nMaxSCHISM_hgrid_face_nodes"))
                v.start_index = 1
                v.cf_role = "face_node_connectivity"
                v._FillValue = np.int32(-1)
                v[:] = g["face_nodes"]
                v = f.createVariable("SCHISM_hgrid_edge_nodes", "i4", ("nSCHISM_hgrid_edge", "two"))
                v.start_index = 1
                v.cf_role = "edge_node_connectivity"
                v._FillValue = np.int32(-1)
                v[:] = g["edge_nodes"]
            for var, field, idx, ent in FILES[fname]:
                dims = ("time", DIM[ent]) + (("nSCHISM_vgrid_layers",) if field not in
                                             ("ETA2", "NODE_DRY", "ELEM_DRY", "SIDE_DRY") else ())
                f.createVariable(var, "f4", dims)
            self.open[fname] = f
        self.file_num = file_num

    def write(self, it: int, record: Dict[str, np.ndarray]) -> None:
        """Record of step `it` (a multiple of nspool), as record_to_variables returns it."""
        if it % self.nspool:
            return
        k = it // self.nspool - 1                      # output index
        fnum = k // self.per_file + 1
        if fnum != self.file_num:
            self._create(fnum)
        r = k % self.per_file
        for fname, f in self.open.items():
            f.variables["time"][r] = it * self.dt
            for var, _field, _idx, _ent in FILES[fname]:
                if var in record:
                    f.variables[var][r] = record[var]
            f.flush()

    def close_files(self):
        for f in self.open.values():
            f.close()
        self.open = {}

    def close(self):
        self.close_files()


def grid_of(case) -> Dict[str, np.ndarray]:
    """The 2-D grid variables of out2d from a case (reference numbering; 1-based indices)."""
    from . import grid as G
    ne = case.n_elems
    el4 = np.full((ne, 4), -1, np.int32)
    el4[:, :3] = case.elnode
    i34 = np.full(ne, 3, np.int32)
    isb = G._isbnd(case.n_nodes, case.open_bnd, case.land_bnd)
    con = G.build_connectivity(el4, i34, isb, case.n_nodes)
    sn = con["isidenode"]
    fn = np.where(el4 >= 0, el4 + 1, -1).astype(np.int32)
    return {"x": case.x, "y": case.y, "depth": case.depth, "kb": np.zeros(case.n_nodes, np.int32),
            "face_x": case.x[case.elnode].mean(axis=1), "face_y": case.y[case.elnode].mean(axis=1),
            "edge_x": 0.5 * (case.x[sn[:, 0]] + case.x[sn[:, 1]]), "edge_y": 0.5 * (case.y[sn[:, 0]] + case.y[sn[:, 1]]),
            "face_nodes": fn, "edge_nodes": (sn + 1).astype(np.int32)}


class _PinnedRecord:
    """Page-locked buffers for one output record of one member."""

    def __init__(self, lib, shapes: Dict[str, tuple], dtypes: Dict[str, type]):
        self.lib = lib
        self.ptrs, self.arrays = {}, {}
        for f, shp in shapes.items():
            dt = np.dtype(dtypes[f])
            nbytes = int(np.prod(shp)) * dt.itemsize
            p = lib.gs_host_alloc(nbytes)
            if not p:
                self.free()
                raise MemoryError("gs_host_alloc failed")
            self.ptrs[f] = (p, nbytes)
            buf = (ctypes.c_char * nbytes).from_address(p)
            self.arrays[f] = np.frombuffer(buf, dtype=dt).reshape(shp)

    def free(self):
        for p, _ in self.ptrs.values():
            self.lib.gs_host_free(p)
        self.ptrs, self.arrays = {}, {}


class OutputWriter:
    """Streams a member's output every `nspool` steps to the reference's NetCDF files."""

    def __init__(self, model, member: int, out_dir: str, nspool: int, ihfskip: int, ring: int = 3,
                 files=None, grid: Optional[Dict[str, np.ndarray]] = None):
        from .model import FIELDS, INT_FIELDS
        self.m, self.member = model, member
        case = model.cases[member]
        g = grid if grid is not None else grid_of(case)
        g = dict(g)
        g["kb"] = model.get(member, "NODE_KB")
        self.sink = NetcdfSink(out_dir, g, model.nvrt, model.ntr, case.params.dt, nspool, ihfskip, files=files)
        self.nspool = nspool
        wanted = {field for fname in self.sink.files for _, field, _, _ in FILES[fname]}
        self.fields = sorted(wanted)
        shapes = {f: model.shape(member, f) for f in self.fields}
        dtypes = {f: (np.int32 if f in INT_FIELDS else np.float64) for f in self.fields}
        self.codes = {f: FIELDS[f] for f in self.fields}
        self.free: "queue.Queue[_PinnedRecord]" = queue.Queue()
        self.records: List[_PinnedRecord] = [_PinnedRecord(model.lib, shapes, dtypes) for _ in range(ring)]
        for r in self.records:
            self.free.put(r)
        self.work: "queue.Queue" = queue.Queue()
        self.error: Optional[BaseException] = None
        self.written = 0
        self.thread = threading.Thread(target=self._run, name="gschism-output", daemon=True)
        self.thread.start()

    def step_done(self, it: int) -> None:
        """Call after step `it` has been queued (model.step): queues the record's reads."""
        if self.error is not None:
            raise self.error
        if it % self.nspool:
            return
        rec = self.free.get()
        lib, h = self.m.lib, self.m.h
        for f in self.fields:
            p, nbytes = rec.ptrs[f]
            L.check(lib.gs_state_get_async(h, self.member, self.codes[f], ctypes.c_void_p(p), nbytes), h,
                    f"gs_state_get_async {f}")
        t = ctypes.c_uint64(0)
        L.check(lib.gs_output_mark(h, ctypes.byref(t)), h, "gs_output_mark")
        self.work.put((t.value, rec, it))

    def _run(self):
        while True:
            item = self.work.get()
            if item is None:
                return
            ticket, rec, it = item
            try:
                L.check(self.m.lib.gs_output_wait(self.m.h, ticket), self.m.h, "gs_output_wait")
                self.sink.write(it, record_to_variables(rec.arrays, self.m.ntr))
                self.written += 1
            except BaseException as e:  # reported to the stepping thread
                self.error = e
            finally:
                self.free.put(rec)

    def close(self) -> None:
        self.work.put(None)
        self.thread.join()
        self.sink.close()
        for r in self.records:
            r.free()
        self.records = []
        if self.error is not None:
            raise self.error
