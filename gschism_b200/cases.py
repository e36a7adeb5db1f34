"""Seeded synthetic SCHISM cases: jittered-lattice triangulations with an SZ vertical grid.

A case is everything one ensemble member needs: the horizontal grid (node coordinates, depth,
triangles in counter-clockwise order, open and land boundary segments), the SZ vertical grid,
tidal elevation forcing on open segments, bottom drag, wind stress, initial tracers and the
physics parameters of the step.  The same case can be written in SCHISM's own file formats
(`hgrid.gr3`, `vgrid.in`, `drag.gr3`) so that the reference grid readers
(`src/grid/read_and_process_grid.cpp:855` readHGrid, `:1322` readVGrid) parse it too.

No public dataset is involved: every input is drawn from numpy's PCG64 with the seed stored in
the case.  The named workloads follow the five benchmark configurations:

* ``channel``  -- 63x32 lattice over a 10 km x 5 km channel, depth 5->20 m across, 10 sigma
  levels, an M2 tide (0.5 m) on one short side, one Gaussian tracer blob; dt = 100 s.
* ``basin``    -- n x n lattice over 500 km, Gaussian-random-field bathymetry 2..4000 m, 30 SZ
  levels (10 z + 21 sigma), M2+S2 (1.2 m total) on one side, T and S tracers; dt = 120 s.
* ``ensemble`` -- basin-like members with log-uniform sizes, per-member tide amplitude and a
  uniform wind stress; 20 levels, 1 tracer.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import List, Optional

import numpy as np

M2_OMEGA = 2.0 * math.pi / 44712.0      # rad/s (period 12.42 h)
S2_OMEGA = 2.0 * math.pi / 43200.0      # rad/s (period 12.00 h)


@dataclasses.dataclass
class Params:
    """Physics switches and constants of the step (runtime form of the reference's
    compile-time constants, `src/kernels/constants_template.h`)."""
    dt: float = 100.0
    thetai: float = 0.6
    h0: float = 0.01                 # wet/dry threshold [m]
    dtb_min: float = 10.0            # btrack sub-step bounds [s]
    dtb_max: float = 30.0
    velmin_btrack: float = 1e-4      # [m/s]
    rmaxvel: float = 10.0            # velocity clamp, x; y uses 1.013x
    dfv0: float = 1e-2               # constant vertical viscosity (itur = 0)
    coricoef: float = 0.0            # constant Coriolis parameter (ncor = 0)
    rho0: float = 1000.0
    grav: float = 9.81
    dramp: float = 0.5               # ramp time [days] for boundary forcing (0 = off)
    ihhat: int = 1                   # clamp \hat H >= 0 for 3D sides
    rtol: float = 1e-12              # JCG relative tolerance
    maxiter: int = 1500              # JCG iteration cap
    check_every: int = 10            # JCG host/device convergence test period
    itr_met: int = 1                 # tracer transport: 1 upwind (the reference), 3 TVD, 4 TVD + vertical FCT
    tvd_limiter: int = 3             # TVD flux limiter: 0 none, 1 minmod, 2 Osher, 3 van Leer, 4 superbee
    dfh0: float = 0.0                # constant vertical tracer diffusivity [m^2/s] (implicit)


@dataclasses.dataclass
class VGrid:
    """SZ vertical grid (ivcor = 2), as read by readVGrid (read_and_process_grid.cpp:1398-1505)."""
    nvrt: int
    nz: int                      # number of z levels (kz); level nz-1 is -h_s
    h_s: float
    h_c: float
    theta_b: float
    theta_f: float
    ztot: np.ndarray             # [nz]   z levels, ztot[nz-1] = -h_s
    sigma: np.ndarray            # [nsiglev] sigma levels, -1 .. 0

    @property
    def nsiglev(self) -> int:
        return self.nvrt - self.nz + 1

    def cs(self) -> np.ndarray:
        """Song-Haidvogel stretching C(sigma) (read_and_process_grid.cpp:1492-1496)."""
        s, tb, tf = self.sigma, self.theta_b, self.theta_f
        return ((1.0 - tb) * np.sinh(tf * s) / math.sinh(tf)
                + tb * (np.tanh(tf * (s + 0.5)) - math.tanh(tf * 0.5)) / 2.0 / math.tanh(tf * 0.5))


@dataclasses.dataclass
class Case:
    name: str
    seed: int
    x: np.ndarray                # [np] float64
    y: np.ndarray
    depth: np.ndarray
    elnode: np.ndarray           # [ne, 3] int32, 0-based, CCW
    open_bnd: List[np.ndarray]   # node lists along each open segment
    land_bnd: List[np.ndarray]   # node lists along each land segment (endpoints shared with open)
    vgrid: VGrid
    params: Params
    iettype: np.ndarray          # [nope] 0 = none, 3 = tidal harmonics
    # tidal constituents: frequency, nodal factor, equilibrium argument
    amig: np.ndarray             # [nbfr]
    ff: np.ndarray
    face: np.ndarray
    emo: List[np.ndarray]        # per open segment: [nond, nbfr] amplitudes
    efa: List[np.ndarray]        # per open segment: [nond, nbfr] phases (rad)
    drag: np.ndarray             # [np] bottom drag coefficient (nchi = 0)
    tau: np.ndarray              # [np, 2] kinematic surface stress [m^2/s^2]
    tr_init: np.ndarray          # [ntr, nvrt, np] initial nodal tracers
    nsteps: int = 100

    @property
    def n_nodes(self) -> int:
        return int(self.x.shape[0])

    @property
    def n_elems(self) -> int:
        return int(self.elnode.shape[0])

    @property
    def ntracers(self) -> int:
        return int(self.tr_init.shape[0])

    @property
    def nvrt(self) -> int:
        return self.vgrid.nvrt

    def node_z_cold(self) -> np.ndarray:
        """z of every level at eta = 0, level-major [nvrt, np] (used for initial tracers)."""
        return sz_levels(self.vgrid, self.depth, np.zeros_like(self.depth))


# ----------------------------------------------------------------------------------------------
# vertical levels (host copy of the SZ formula, for initial conditions only)
# ----------------------------------------------------------------------------------------------

def sz_kb(vg: VGrid, depth: np.ndarray) -> np.ndarray:
    """Bottom level index of each node (Node::updateKb, meshdata.cu:1676-1718)."""
    kb = np.full(depth.shape, vg.nz - 1, dtype=np.int32)
    deep = depth > vg.h_s
    if np.any(deep):
        # largest L with ztot[L] <= -depth
        idx = np.searchsorted(vg.ztot, -depth[deep], side="right") - 1
        kb[deep] = idx
    return kb


def sz_levels(vg: VGrid, depth: np.ndarray, eta: np.ndarray) -> np.ndarray:
    """z of each level (Node::compZCoord, meshdata.cu:1744-1807), [nvrt, np]; below kb = -depth."""
    nvrt, izlev = vg.nvrt, vg.nz - 1
    kb = sz_kb(vg, depth)
    hmod2 = np.minimum(depth, vg.h_s)
    cs = vg.cs()
    z = np.empty((nvrt, depth.shape[0]))
    for k in range(nvrt):
        if k == nvrt - 1:
            zk = eta.copy()
        elif k == izlev:
            zk = -hmod2
        elif k < izlev:
            zk = np.full(depth.shape, vg.ztot[k]) if k < vg.nz else None
        else:
            ks = k - izlev
            zs = vg.sigma[ks] * (hmod2 + eta) + eta
            zl = eta * (1.0 + vg.sigma[ks]) + vg.h_c * vg.sigma[ks] + (hmod2 - vg.h_c) * cs[ks]
            zk = np.where(hmod2 <= vg.h_c, zs, zl)
        zk = np.where(k == kb, -depth, zk)
        zk = np.where(k < kb, -depth, zk)
        z[k] = zk
    return z


# ----------------------------------------------------------------------------------------------
# lattice triangulation
# ----------------------------------------------------------------------------------------------

def _lattice(nx: int, ny: int, lx: float, ly: float, jitter: float, rng: np.random.Generator):
    """Jittered nx x ny lattice; boundary nodes move only along the boundary, corners stay."""
    dx, dy = lx / (nx - 1), ly / (ny - 1)
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    i, j = i.ravel(), j.ravel()
    x = i * dx
    y = j * dy
    jx = rng.uniform(-jitter, jitter, x.shape) * dx
    jy = rng.uniform(-jitter, jitter, y.shape) * dy
    jx[(i == 0) | (i == nx - 1)] = 0.0
    jy[(j == 0) | (j == ny - 1)] = 0.0
    x = x + jx
    y = y + jy
    # cells (i,j)-(i+1,j+1) split along the same diagonal: interior nodes have 6 neighbours
    ci, cj = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), indexing="xy")
    ci, cj = ci.ravel(), cj.ravel()
    a = ci + cj * nx
    b = a + 1
    c = a + 1 + nx
    d = a + nx
    tri = np.empty((2 * a.size, 3), dtype=np.int64)
    tri[0::2] = np.stack([a, b, c], axis=1)
    tri[1::2] = np.stack([a, c, d], axis=1)
    west = np.arange(ny) * nx                              # i = 0, south -> north
    south = np.arange(nx)                                  # j = 0
    east = np.arange(ny) * nx + nx - 1
    north = (ny - 1) * nx + np.arange(nx)
    return x, y, tri, west, south, east, north


def _boundaries(nx, ny, west, south, east, north):
    """Open boundary: the west side (north -> south, so the domain is on the left).
    Land: south (W->E), east (S->N), north (E->W), sharing end nodes with the open segment."""
    open_seg = west[::-1].copy()
    land = np.concatenate([south, east[1:], north[::-1][1:]])
    return [open_seg], [land]


def _permute(rng, x, y, depth, tri, open_bnd, land_bnd, extra_node_arrays):
    """Seeded random renumbering of nodes and elements (unstructured meshes rarely come
    ordered); keeps each triangle's CCW orientation, rotating its start vertex."""
    n = x.size
    perm = rng.permutation(n)            # new -> old
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n)             # old -> new
    tri = inv[tri]
    ep = rng.permutation(tri.shape[0])
    tri = tri[ep]
    rot = rng.integers(0, 3, tri.shape[0])
    tri = np.stack([tri[np.arange(tri.shape[0]), (rot + s) % 3] for s in range(3)], axis=1)
    out = [a[..., perm] if a is not None else None for a in extra_node_arrays]
    return (x[perm], y[perm], depth[perm], tri, [inv[s] for s in open_bnd],
            [inv[s] for s in land_bnd], out)


def _grf(nx: int, ny: int, lx: float, ly: float, corr: float, rng) -> np.ndarray:
    """Gaussian random field on the lattice with a Gaussian covariance of length `corr`,
    by FFT filtering of white noise; normalised to [0, 1]."""
    w = rng.standard_normal((ny, nx))
    kx = np.fft.fftfreq(nx, d=lx / (nx - 1)) * 2 * np.pi
    ky = np.fft.fftfreq(ny, d=ly / (ny - 1)) * 2 * np.pi
    kk = kx[None, :] ** 2 + ky[:, None] ** 2
    f = np.fft.ifft2(np.fft.fft2(w) * np.exp(-0.25 * kk * corr ** 2)).real
    f = (f - f.min()) / max(f.max() - f.min(), 1e-30)
    return f.ravel()


def _sigma_vgrid(nvrt: int) -> VGrid:
    """Pure-sigma grid: nz = 1 and h_c above every depth, so z = sigma*(h+eta)+eta."""
    return VGrid(nvrt=nvrt, nz=1, h_s=100.0, h_c=30.0, theta_b=0.0, theta_f=1e-4,
                 ztot=np.array([-100.0]), sigma=np.linspace(-1.0, 0.0, nvrt))


def _sz_vgrid(nvrt: int, nz: int, zmax: float, h_s: float = 200.0) -> VGrid:
    ztot = np.concatenate([np.linspace(-zmax, -h_s, nz)])
    ztot[-1] = -h_s
    return VGrid(nvrt=nvrt, nz=nz, h_s=h_s, h_c=10.0, theta_b=0.7, theta_f=5.0,
                 ztot=ztot, sigma=np.linspace(-1.0, 0.0, nvrt - nz + 1))


def _tide_on(open_bnd, comps):
    """emo/efa arrays for every open segment from [(amplitude, phase)] per constituent."""
    emo = [np.tile(np.array([a for a, _ in comps]), (s.size, 1)) for s in open_bnd]
    efa = [np.tile(np.array([p for _, p in comps]), (s.size, 1)) for s in open_bnd]
    return emo, efa


def channel(seed: int = 1, nx: int = 63, ny: int = 32, nvrt: int = 10, shuffle: bool = True,
            nsteps: int = 100) -> Case:
    """Plain FP64 step case: 10 km x 5 km channel, ~2,000 nodes, M2 0.5 m on the west side."""
    rng = np.random.default_rng(seed)
    lx, ly = 10000.0, 5000.0
    x, y, tri, w, s, e, n = _lattice(nx, ny, lx, ly, 0.2, rng)
    depth = 5.0 + 15.0 * (y / ly)
    open_bnd, land_bnd = _boundaries(nx, ny, w, s, e, n)
    if shuffle:
        x, y, depth, tri, open_bnd, land_bnd, _ = _permute(rng, x, y, depth, tri, open_bnd,
                                                           land_bnd, [])
    vg = _sigma_vgrid(nvrt)
    npn = x.size
    r2 = (x - 0.5 * lx) ** 2 + (y - 0.5 * ly) ** 2
    blob = np.exp(-0.5 * r2 / 1000.0 ** 2)
    tr = np.broadcast_to(blob, (1, nvrt, npn)).copy()
    emo, efa = _tide_on(open_bnd, [(0.5, 0.0)])
    return Case(name="channel", seed=seed, x=x, y=y, depth=depth, elnode=tri.astype(np.int32),
                open_bnd=open_bnd, land_bnd=land_bnd, vgrid=vg,
                params=Params(dt=100.0, rtol=1e-12),
                iettype=np.array([3]), amig=np.array([M2_OMEGA]), ff=np.array([1.0]),
                face=np.array([0.0]), emo=emo, efa=efa,
                drag=np.full(npn, 2.5e-3), tau=np.zeros((npn, 2)), tr_init=tr, nsteps=nsteps)


def basin(seed: int = 2, n: int = 1000, nvrt: int = 30, nz: int = 10, ntr: int = 2,
          length: float = 500e3, amp: float = 1.2, tau=(0.0, 0.0), shuffle: bool = True,
          nsteps: int = 200, dt: float = 120.0) -> Case:
    """Single large basin: n x n lattice over `length`, GRF bathymetry 2..4000 m, SZ levels,
    M2 + S2 on the west side (amplitudes split 0.8:0.4 of `amp`), T/S tracers."""
    rng = np.random.default_rng(seed)
    x, y, tri, w, s, e, nn = _lattice(n, n, length, length, 0.2, rng)
    f = _grf(n, n, length, length, 20e3, rng)
    depth = 2.0 + (4000.0 - 2.0) * f
    open_bnd, land_bnd = _boundaries(n, n, w, s, e, nn)
    if shuffle:
        x, y, depth, tri, open_bnd, land_bnd, _ = _permute(rng, x, y, depth, tri, open_bnd,
                                                           land_bnd, [])
    vg = _sz_vgrid(nvrt, nz, 4000.0)
    npn = x.size
    z = sz_levels(vg, depth, np.zeros(npn))
    frac = np.clip(-z / 4000.0, 0.0, 1.0)                  # 0 at surface, 1 at 4000 m
    trs = []
    if ntr >= 1:
        t = 25.0 - 23.0 * frac
        trs.append(t * (1.0 + 0.01 * rng.standard_normal(t.shape)))
    if ntr >= 2:
        sal = 30.0 + 6.0 * frac
        trs.append(sal * (1.0 + 0.01 * rng.standard_normal(sal.shape)))
    for _ in range(2, ntr):
        trs.append(rng.uniform(0.0, 1.0, (nvrt, npn)))
    tr = np.stack(trs[:ntr], axis=0)
    emo, efa = _tide_on(open_bnd, [(amp * 2.0 / 3.0, 0.0), (amp / 3.0, 0.7)])
    tw = np.broadcast_to(np.asarray(tau, dtype=np.float64), (npn, 2)).copy()
    return Case(name="basin", seed=seed, x=x, y=y, depth=depth, elnode=tri.astype(np.int32),
                open_bnd=open_bnd, land_bnd=land_bnd, vgrid=vg,
                params=Params(dt=dt, rtol=1e-12),
                iettype=np.array([3]), amig=np.array([M2_OMEGA, S2_OMEGA]),
                ff=np.array([1.0, 1.0]), face=np.array([0.0, 0.0]), emo=emo, efa=efa,
                drag=np.full(npn, 2.5e-3), tau=tw, tr_init=tr, nsteps=nsteps)


def transport_stress(seed: int = 4, n: int = 2000, nvrt: int = 40, ntr: int = 5, spacing: float = 250.0,
                     tau_mag: float = 0.1, limiter: int = 3, dfh0: float = 1e-4, shuffle: bool = True,
                     nsteps: int = 100, dt: float = 120.0) -> Case:
    """Transport stress case: n x n lattice at `spacing` (2000 x 2000 nodes over 500 km, as the
    single-mesh basin), closed boundaries, GRF bathymetry 2..4000 m, nvrt SZ levels, a uniform wind
    stress of `tau_mag` N/m^2 in a seeded direction, and ntr tracers that each hold a sharp front
    (tanh across a seeded line, 2 km wide) weakening with depth plus two to four Gaussian blobs
    (radius 2-8 km).  TVD horizontal transport (`limiter`) with implicit vertical diffusion
    `dfh0`; with no open boundary the tracer mass changes only through the scheme."""
    rng = np.random.default_rng(seed)
    length = spacing * (n - 1)
    x, y, tri, w, s, e, nn = _lattice(n, n, length, length, 0.2, rng)
    f = _grf(n, n, length, length, 20e3, rng)
    depth = 2.0 + (4000.0 - 2.0) * f
    land = [np.concatenate([s, e[1:], nn[::-1][1:], w[::-1][1:-1]])]
    if shuffle:
        x, y, depth, tri, _, land, _ = _permute(rng, x, y, depth, tri, [], land, [])
    vg = _sz_vgrid(nvrt, max(2, nvrt // 3), 4000.0)
    npn = x.size
    z = sz_levels(vg, depth, np.zeros(npn))
    frac = np.clip(-z / 4000.0, 0.0, 1.0)
    trs = []
    for _ in range(ntr):
        ang = rng.uniform(0.0, 2 * math.pi)
        cx, cy = rng.uniform(0.2, 0.8, 2) * length
        front = 0.5 * (1.0 + np.tanh(((x - cx) * math.cos(ang) + (y - cy) * math.sin(ang)) / 2000.0))
        blobs = np.zeros(npn)
        for _b in range(int(rng.integers(2, 5))):
            bx, by = rng.uniform(0.0, 1.0, 2) * length
            r = rng.uniform(2000.0, 8000.0)
            blobs += rng.uniform(0.3, 1.0) * np.exp(-0.5 * ((x - bx) ** 2 + (y - by) ** 2) / r ** 2)
        trs.append(front[None, :] * (1.0 - 0.5 * frac) + blobs[None, :])
    tr = np.stack(trs, axis=0)
    ang = rng.uniform(0.0, 2 * math.pi)
    tau = np.broadcast_to(np.array([math.cos(ang), math.sin(ang)]) * tau_mag / 1025.0, (npn, 2)).copy()
    return Case(name="transport_stress", seed=seed, x=x, y=y, depth=depth, elnode=tri.astype(np.int32),
                open_bnd=[], land_bnd=land, vgrid=vg,
                params=Params(dt=dt, rtol=1e-12, itr_met=3, tvd_limiter=limiter, dfh0=dfh0),
                iettype=np.zeros(0, dtype=np.int64), amig=np.zeros(0), ff=np.zeros(0), face=np.zeros(0),
                emo=[], efa=[], drag=np.full(npn, 2.5e-3), tau=tau, tr_init=tr, nsteps=nsteps)


def ensemble(n_members: int = 64, seed: int = 3, nmin: int = 20_000, nmax: int = 500_000,
             nvrt: int = 20, shuffle: bool = True, nsteps: int = 100) -> List[Case]:
    """Uneven ensemble: node counts log-uniform in [nmin, nmax] (square-ish lattices),
    per-member seed, tide amplitude U(0.3, 2.0) m and uniform wind stress 0..0.3 N/m^2."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n_members):
        target = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        side = max(8, int(round(math.sqrt(target))))
        amp = rng.uniform(0.3, 2.0)
        mag = rng.uniform(0.0, 0.3)
        ang = rng.uniform(0.0, 2 * math.pi)
        tau = (mag / 1025.0 * math.cos(ang), mag / 1025.0 * math.sin(ang))
        length = 500e3 * side / 1000.0
        c = basin(seed=int(rng.integers(1, 2**31 - 1)), n=side, nvrt=nvrt, nz=max(2, nvrt // 3),
                  ntr=1, length=length, amp=amp, tau=tau, shuffle=shuffle, nsteps=nsteps)
        c.name = f"member{m:02d}"
        out.append(c)
    return out


def storm(seed: int, nmin: int = 10_000, nmax: int = 2_000_000, nvrt: int = 20, dt: float = 150.0,
          hours: float = 48.0, shuffle: bool = True):
    """A storm-surge forecast request: a basin mesh with a node count log-uniform in [nmin, nmax]
    (500 m spacing), 20 levels, 1 tracer, tidal forcing on the west side (0.3-1.0 m), and a radial
    vortex on a straight track crossing the domain: seeded heading, speed 3-8 m/s, maximum wind
    20-60 m/s at a radius of 20-60 km (Holland B 1.2-1.8).  Returns (case, vortex, nsteps) with
    nsteps covering `hours` at `dt`."""
    rng = np.random.default_rng(seed)
    target = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
    side = max(8, int(round(math.sqrt(target))))
    length = 500.0 * side
    amp = rng.uniform(0.3, 1.0)
    c = basin(seed=int(rng.integers(1, 2**31 - 1)), n=side, nvrt=nvrt, nz=max(2, nvrt // 3), ntr=1,
              length=length, amp=amp, shuffle=shuffle, dt=dt)
    c.name = f"storm{seed}"
    return c, _vortex(rng, length), int(round(hours * 3600.0 / dt))


def _vortex(rng, length: float) -> dict:
    heading = rng.uniform(0.0, 2.0 * math.pi)
    # start 3/4 of the domain size behind the centre, so the track crosses the domain
    cx, cy = 0.5 * length, 0.5 * length
    return dict(x0=cx - 0.75 * length * math.cos(heading), y0=cy - 0.75 * length * math.sin(heading),
                heading=heading, speed=rng.uniform(3.0, 8.0), vmax=rng.uniform(20.0, 60.0),
                rmax=rng.uniform(20e3, 60e3), holland_b=rng.uniform(1.2, 1.8), rho_air=1.15)


def storm_on(case: Case, seed: int) -> dict:
    """A seeded storm (the vortex of `storm`) on an existing square storm mesh: a forecast request
    for a region whose mesh is already set up."""
    return _vortex(np.random.default_rng(seed), float(case.x.max() - case.x.min()))


# ----------------------------------------------------------------------------------------------
# SCHISM file formats
# ----------------------------------------------------------------------------------------------

def write_hgrid(case: Case, path: str) -> None:
    """hgrid.gr3 in SCHISM's layout (1-based ids; open and land boundary blocks)."""
    with open(path, "w") as f:
        f.write(f"{case.name} seed={case.seed}\n")
        f.write(f"{case.n_elems} {case.n_nodes}\n")
        for i in range(case.n_nodes):
            f.write(f"{i + 1} {case.x[i]:.17g} {case.y[i]:.17g} {case.depth[i]:.17g}\n")
        for e in range(case.n_elems):
            a, b, c = case.elnode[e] + 1
            f.write(f"{e + 1} 3 {a} {b} {c}\n")
        f.write(f"{len(case.open_bnd)} = Number of open boundaries\n")
        f.write(f"{sum(s.size for s in case.open_bnd)} = Total number of open boundary nodes\n")
        for k, s in enumerate(case.open_bnd):
            f.write(f"{s.size} = Number of nodes for open boundary {k + 1}\n")
            for v in s:
                f.write(f"{v + 1}\n")
        f.write(f"{len(case.land_bnd)} = number of land boundaries\n")
        f.write(f"{sum(s.size for s in case.land_bnd)} = Total number of land boundary nodes\n")
        for k, s in enumerate(case.land_bnd):
            f.write(f"{s.size} 0 = Number of nodes for land boundary {k + 1}\n")
            for v in s:
                f.write(f"{v + 1}\n")


def write_vgrid(case: Case, path: str) -> None:
    """vgrid.in (ivcor = 2).  The level-nz line ("nz -h_s") is written only for nz = 1: the
    reference reader (read_and_process_grid.cpp:1428-1450) skips one line after the z levels
    and reads h_c from the line after "S levels", which holds for these two shapes."""
    vg = case.vgrid
    with open(path, "w") as f:
        f.write("2 !ivcor\n")
        f.write(f"{vg.nvrt} {vg.nz} {vg.h_s:.17g} !nvrt, kz, h_s\n")
        f.write("Z levels\n")
        for k in range(vg.nz - 1):
            f.write(f"{k + 1} {vg.ztot[k]:.17g}\n")
        if vg.nz == 1:
            f.write(f"1 {-vg.h_s:.17g}\n")
        f.write("S levels\n")
        f.write(f"{vg.h_c:.17g} {vg.theta_b:.17g} {vg.theta_f:.17g} !h_c, theta_b, theta_f\n")
        for k in range(vg.nsiglev):
            f.write(f"{k + 1} {vg.sigma[k]:.17g}\n")


def write_gr3_field(case: Case, values: np.ndarray, path: str, label: str) -> None:
    """A node field in .gr3 layout (drag.gr3 and the like)."""
    with open(path, "w") as f:
        f.write(f"{label}\n{case.n_elems} {case.n_nodes}\n")
        for i in range(case.n_nodes):
            f.write(f"{i + 1} {case.x[i]:.17g} {case.y[i]:.17g} {values[i]:.17g}\n")
        for e in range(case.n_elems):
            a, b, c = case.elnode[e] + 1
            f.write(f"{e + 1} 3 {a} {b} {c}\n")


def write_case(case: Case, directory: str) -> None:
    os.makedirs(directory, exist_ok=True)
    write_hgrid(case, os.path.join(directory, "hgrid.gr3"))
    write_vgrid(case, os.path.join(directory, "vgrid.in"))
    write_gr3_field(case, case.drag, os.path.join(directory, "drag.gr3"), "drag")
