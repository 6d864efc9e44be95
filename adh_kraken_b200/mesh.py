"""Meshes, forcing and initial states for the SW2 workloads.

A :class:`SW2Case` holds everything one implicit SW2 run needs, in the reference's
conventions:

* nodes ``xyz`` (x, y, bed elevation z); triangles ``tri`` counter-clockwise;
* boundary segments ``seg`` whose node order gives the outward normal
  (``nrml = (dy, -dx)/len`` for a segment from node 0 to node 1,
  src/structs/selem/selem_1d.c:54-55);
* ``seg_kind`` 0 for a weak velocity boundary ("NB VEL", ``fe_sw2_bc_vel``), 1 for
  a weak depth boundary ("DEPTH", ``fe_sw2_bc_h``), 2 for a discharge string
  (``fe_sw2_bc_discharge``, src/models/sw2/sw2_bc_discharge.c.bk) and 3 for a
  tailwater string (``fe_sw2_bc_tailwater``, sw2_bc_tailwater.c.bk), 4 for an outflow
  string (``fe_sw2_bc_outflow``) and 5 for a flux string (``fe_sw2_bc_flux``);
* the node-major state ``[h, u, v]`` per node (dof = 3*node + var,
  src/structs/sivar_position/sivar_position.c:61-81);
* time series: id 0 = boundary depth (hard-coded in src/models/sw2/sw2_bc_h.c:156),
  ids 1/2 = boundary velocity x/y, id 3 = the discharge string's series value,
  id 4 = the tailwater elevation, id 5 = the flux strings' unit flux (inflow positive); ``bc_conveyance`` and ``bc_rough_height`` are the
  discharge string's conveyance and the boundary strings' roughness height.

The structured flume reproduces the node and triangle layout of the reference's
``create_rectangular_grid`` (src/tools/create_rectangular_grid.c:4-440).  The large
workloads are seeded jittered-Delaunay meshes with synthetic bathymetry and forcing
standing in for field data; their shapes and sizes follow the benchmark configurations.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, Optional, Tuple

import numpy as np

GRAVITY = 9.8  # reference default, src/structs/smodel_super/smodel_super_alloc_init.c


@dataclasses.dataclass
class SW2Case:
    name: str
    xyz: np.ndarray          # (V,3) float64
    tri: np.ndarray          # (T,3) int32
    seg: np.ndarray          # (S,2) int32
    seg_kind: np.ndarray     # (S,) int32: 0 velocity, 1 depth, 2 discharge, 3 tailwater, 4 outflow, 5 flux
    sol0: np.ndarray         # (3V,) float64 initial [h,u,v] per node
    dt: float
    nsteps: int
    series: Dict[int, Tuple[np.ndarray, np.ndarray]]
    t0: float = 0.0
    tol_nonlin: float = 1e-8
    inc_nonlin: float = 1e-6
    max_nonlin_it: int = 10
    gravity: float = GRAVITY
    bc_conveyance: float = 1.0      # discharge string's conveyance (series 3 gives its series value)
    bc_rough_height: float = 0.0    # equivalent roughness height of the boundary strings
    # series ids: 0 depth, 1/2 velocity x/y, 3 discharge series value, 4 tailwater elevation, 5 unit flux

    @property
    def nnodes(self) -> int:
        return int(self.xyz.shape[0])

    @property
    def ntri(self) -> int:
        return int(self.tri.shape[0])

    @property
    def nseg(self) -> int:
        return int(self.seg.shape[0])

    @property
    def ndofs(self) -> int:
        return 3 * self.nnodes


# --------------------------------------------------------------------------- grids

def rectangular_grid(xmin, xmax, ymin, ymax, npx, npy, a0=0.0, ax=0.0):
    """Nodes and triangles laid out as create_rectangular_grid lays them out.

    Nodes run column-major (x outer, y inner; id = i*npy + j), bed ``z = a0 + ax*x``
    evaluated in the reference's term order, and each quad splits into two
    counter-clockwise triangles whose diagonal alternates with the row parity
    (src/tools/create_rectangular_grid.c:141-160, 173-440; theta = 0).
    """
    dx = (xmax - xmin) / float(npx - 1)
    dy = (ymax - ymin) / float(npy - 1)
    i = np.repeat(np.arange(npx, dtype=np.float64), npy)
    j = np.tile(np.arange(npy, dtype=np.float64), npx)
    x = xmin + i * dx
    y = ymin + j * dy
    zero = 0.0
    # a0 + ax*x + ax2*x*x + ay*y + ay2*y*y + axy*x*y + ... with the other terms 0
    z = a0 + ax * x + zero * x * x + zero * y + zero * y * y + zero * x * y \
        + zero * x * x * y + zero * x * y * y + zero * x * x * y * y
    xyz = np.stack([x, y, z], axis=1)
    tris = []
    for ii in range(npx - 1):
        for jj in range(npy - 1):
            n = ii * npy + jj
            if jj % 2 == 0:
                cand = [(n, n + npy, n + npy + 1), (n, n + npy + 1, n + 1)]
            else:
                cand = [(n, n + npy, n + 1), (n + npy, n + npy + 1, n + 1)]
            for a, b, c in cand:
                s1 = xyz[b, :2] - xyz[a, :2]
                s2 = xyz[c, :2] - xyz[a, :2]
                if s1[0] * s2[1] - s1[1] * s2[0] <= 0:
                    b, c = c, b
                tris.append((a, b, c))
    return xyz, np.asarray(tris, dtype=np.int32)


def jittered_delaunay(nx: int, ny: int, lx: float, ly: float, jitter: float, rng,
                      x0: float = 0.0, y0: float = 0.0):
    """Delaunay triangulation of an ``nx`` x ``ny`` grid whose interior nodes are
    jittered uniformly by +-``jitter`` spacings (boundary nodes stay on the hull so
    the domain is the exact rectangle).  Nodes are numbered x-major like the
    structured grid; triangles are oriented counter-clockwise."""
    from scipy.spatial import Delaunay

    dx = lx / (nx - 1)
    dy = ly / (ny - 1)
    ii, jj = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    x = x0 + ii.ravel() * dx
    y = y0 + jj.ravel() * dy
    interior = ((ii > 0) & (ii < nx - 1) & (jj > 0) & (jj < ny - 1)).ravel()
    jx = rng.uniform(-jitter, jitter, size=x.shape) * dx
    jy = rng.uniform(-jitter, jitter, size=y.shape) * dy
    x = np.where(interior, x + jx, x)
    y = np.where(interior, y + jy, y)
    pts = np.stack([x, y], axis=1)
    tri = Delaunay(pts).simplices.astype(np.int64)
    p0, p1, p2 = pts[tri[:, 0]], pts[tri[:, 1]], pts[tri[:, 2]]
    cross = (p1[:, 0] - p0[:, 0]) * (p2[:, 1] - p0[:, 1]) - (p1[:, 1] - p0[:, 1]) * (p2[:, 0] - p0[:, 0])
    flip = cross < 0
    tri[flip, 1], tri[flip, 2] = tri[flip, 2].copy(), tri[flip, 1].copy()
    area = 0.5 * np.abs(cross)
    keep = area > 1e-9 * dx * dy  # drop degenerate slivers on the hull, if any
    tri = tri[keep]
    # element order follows node order (lowest node, then highest) for locality
    order = np.lexsort((tri.max(axis=1), tri.min(axis=1)))
    return x, y, tri[order].astype(np.int32), (ii.ravel(), jj.ravel())


def boundary_segments(node_ids: np.ndarray, outward_sign: int) -> np.ndarray:
    """Consecutive segments along a boundary node chain.  ``node_ids`` run along the
    edge; ``outward_sign`` = +1 keeps that order, -1 reverses it, so the caller picks
    the orientation whose normal (dy, -dx)/len points out of the domain."""
    ids = node_ids if outward_sign > 0 else node_ids[::-1]
    return np.stack([ids[:-1], ids[1:]], axis=1).astype(np.int32)


def _const_series(t0, t1, value):
    return (np.array([t0, t1], dtype=np.float64), np.array([value, value], dtype=np.float64))


# --------------------------------------------------------------------------- configs

def flume_case(nsteps: int = 100, npx: int = 101, npy: int = 11) -> SW2Case:
    """Plain FP64 rectangular flume, CPU-runnable: 1000 m x 100 m, 100 x 10 quads
    split into 2000 triangles (1111 nodes), bed slope 1e-4 falling downstream,
    upstream discharge 50 m^3/s imposed as the velocity 50/(100*2) = 0.25 m/s on the
    x = 0 edge, downstream depth 2.0 m on the x = 1000 edge, h0 = 2 m, u = v = 0,
    dt = 60 s."""
    xyz, tri = rectangular_grid(0.0, 1000.0, 0.0, 100.0, npx, npy, a0=0.0, ax=-1e-4)
    up = np.arange(0, npy)                            # x = 0 edge, j = 0..npy-1
    down = np.arange((npx - 1) * npy, npx * npy)      # x = 1000 edge
    seg_up = boundary_segments(up, -1)                # normal -x
    seg_down = boundary_segments(down, +1)            # normal +x
    seg = np.concatenate([seg_up, seg_down])
    kind = np.concatenate([np.zeros(len(seg_up), np.int32), np.ones(len(seg_down), np.int32)])
    V = xyz.shape[0]
    sol0 = np.zeros(3 * V)
    sol0[0::3] = 2.0
    dt = 60.0
    tf = dt * nsteps
    series = {0: _const_series(0.0, tf, 2.0), 1: _const_series(0.0, tf, 50.0 / (100.0 * 2.0)),
              2: _const_series(0.0, tf, 0.0)}
    return SW2Case("flume", xyz, tri, seg, kind, sol0, dt, nsteps, series)


def bedshstr_drag_coef(depth: float, rough_height: float) -> float:
    """The bed-shear drag coefficient c_f of a roughness height
    (fr_bedshstr_drag_coef, src/friction/fr_bedshstr_drag_coef.c:18-42), for setting
    boundary values on the host."""
    depth = max(depth, 1e-8)
    rough_height = max(rough_height, 1e-8)
    depth_rh = 1.0 / 29.7 if rough_height > 29.7 * depth else depth / rough_height
    bta = 29.7 * depth_rh
    return 2.0 * ((0.4 * bta) / ((bta + 1) * (np.log(bta + 1) - 1) + 1)) ** 2


def flume_structures_case(nsteps: int = 20, npx: int = 21, npy: int = 6, q_unit: float = 0.5,
                          tail_depth: float = 2.0, rough_height: float = 0.05, conveyance: float = 1.0) -> SW2Case:
    """The flume of ``flume_case`` driven by the structure conditions instead of the
    velocity and depth ones: a discharge string on the x = 0 edge
    (sw2_bc_discharge.c.bk: unit inflow q sqrt(2 g / c_f) h^(3/2) / conveyance, with its
    series value q set so that the inflow is ``q_unit`` m^2/s at the initial 2 m depth)
    and a tailwater string on the x = 1000 edge (sw2_bc_tailwater.c.bk: elevation
    z_down + ``tail_depth``).  Boundary roughness height ``rough_height``."""
    base = flume_case(nsteps=nsteps, npx=npx, npy=npy)
    kind = np.where(base.seg_kind == 0, 2, 3).astype(np.int32)
    z_down = float(base.xyz[base.seg[kind == 3][0, 0], 2])
    c_f = bedshstr_drag_coef(2.0, rough_height)
    q_series = q_unit * conveyance / (np.sqrt(2.0 * base.gravity / c_f) * 2.0 ** 1.5)
    tf = base.dt * nsteps
    series = dict(base.series)
    series[3] = _const_series(0.0, tf, float(q_series))
    series[4] = _const_series(0.0, tf, z_down + tail_depth)
    return dataclasses.replace(base, name="flume_structures", seg_kind=kind, series=series,
                               bc_conveyance=conveyance, bc_rough_height=rough_height)


def flume_flux_outflow_case(nsteps: int = 20, npx: int = 21, npy: int = 6, q_unit: float = 0.5) -> SW2Case:
    """The flume of ``flume_case`` with a flux string on the x = 0 edge
    (sw2_bc_flux.c.bk: the series value ``q_unit`` m^2/s carried in as an explicit
    flux) and an outflow string on the x = 1000 edge (sw2_bc_outflow.c.bk: implicit
    flow with the computed depth and velocity)."""
    base = flume_case(nsteps=nsteps, npx=npx, npy=npy)
    kind = np.where(base.seg_kind == 0, 5, 4).astype(np.int32)
    series = dict(base.series)
    series[5] = _const_series(0.0, base.dt * nsteps, float(q_unit))
    return dataclasses.replace(base, name="flume_flux_outflow", seg_kind=kind, series=series)


def still_beach_case(nsteps: int = 1440, npx: int = 16, npy: int = 6, nt: int = 1440) -> SW2Case:
    """Still water on a sloping beach, the reference's wet/dry test
    (src/test/test_sw2_wd.c:40-166): 1000 m x 500 m rectangular grid, bed
    z = 0.0015 x, water level 1 m (h0 = 1 - z, dry where x > 666.7 m), u = v = 0,
    no boundary segments (a closed basin), dt = 864000 s / nt.  The water must stay
    at rest and keep its mass."""
    xyz, tri = rectangular_grid(0.0, 1000.0, 0.0, 500.0, npx, npy, a0=0.0, ax=0.0015)
    V = xyz.shape[0]
    sol0 = np.zeros(3 * V)
    sol0[0::3] = 1.0 - xyz[:, 2]
    dt = 864000.0 / nt
    tf = dt * max(nsteps, 1)
    series = {0: _const_series(0.0, tf, 0.0), 1: _const_series(0.0, tf, 0.0), 2: _const_series(0.0, tf, 0.0)}
    return SW2Case("still_beach", xyz, tri, np.zeros((0, 2), np.int32), np.zeros(0, np.int32), sol0, dt, nsteps,
                   series)


def _edge_chains(ii, jj, nx, ny):
    """Node chains of the four rectangle edges (x-major numbering)."""
    idx = np.arange(nx * ny).reshape(nx, ny)
    return {"west": idx[0, :], "east": idx[nx - 1, :], "south": idx[:, 0], "north": idx[:, ny - 1]}


def basin_case(n: int = 707, seed: int = 2, nsteps: int = 200) -> SW2Case:
    """Fully wet tidal basin: 20 km x 20 km, jittered (+-0.3 spacing) Delaunay of an
    n x n grid (n = 707 gives ~1M triangles), bed at -(10 - sum of 8 Gaussian bumps,
    amplitude U[1,5] m, sigma U[500,2000] m), sinusoidal 1 m / 12.42 h tide as a depth
    boundary on the west edge, dt = 300 s.  The bumps are tapered to zero within
    3 km of the tidal edge so that edge is flat: the reference's depth boundary takes
    one depth for the whole boundary string (src/models/sw2/sw2_bc_h.c:156-159)."""
    rng = np.random.default_rng(seed)
    L = 20000.0
    x, y, tri, (ii, jj) = jittered_delaunay(n, n, L, L, 0.3, rng)
    cx = rng.uniform(0, L, 8); cy = rng.uniform(0, L, 8)
    amp = rng.uniform(1, 5, 8); sig = rng.uniform(500, 2000, 8)
    bump = np.zeros_like(x)
    for k in range(8):
        bump += amp[k] * np.exp(-((x - cx[k]) ** 2 + (y - cy[k]) ** 2) / (2 * sig[k] ** 2))
    taper = np.clip(x / 3000.0, 0.0, 1.0)
    z = -(10.0 - bump * taper)
    xyz = np.stack([x, y, z], axis=1)
    ch = _edge_chains(ii, jj, n, n)
    seg = boundary_segments(ch["west"], -1)
    kind = np.ones(len(seg), np.int32)
    V = xyz.shape[0]
    sol0 = np.zeros(3 * V)
    sol0[0::3] = -z  # still water at eta = 0
    dt = 300.0
    tf = dt * nsteps
    t = np.arange(0.0, tf + dt, dt / 4.0)
    depth = 10.0 + 1.0 * np.sin(2 * np.pi * t / (12.42 * 3600.0))
    series = {0: (t, depth), 1: _const_series(0.0, tf + dt, 0.0), 2: _const_series(0.0, tf + dt, 0.0)}
    return SW2Case("basin", xyz, tri, seg, kind, sol0, dt, nsteps, series)


def beach_case(nx: int = 2828, ny: int = 707, seed: int = 3, nsteps: int = 300, ly: float = 10000.0) -> SW2Case:
    """Wet/dry sloping beach: 40 km x 10 km jittered Delaunay (nx x ny; the default
    2828 x 707 gives ~4M triangles), bed rising linearly from -20 m (x = 0) to +3 m
    (x = 40 km) plus N(0, 0.2 m) noise, still water at eta = 0 so the upper beach is
    dry (h = eta - z <= 0, the reference's wet/dry convention), inflow hydrograph
    Q(t) = 500 + 1500 sin^2(pi t / 6 h) m^3/s imposed as the normal velocity
    Q / (10 km * 20 m) on the deep edge, dt = 120 s.  `ly` < 10 km cuts a strip of
    the same resolution (ny points across ly) that keeps the unit-width discharge,
    i.e. the same inflow velocity."""
    rng = np.random.default_rng(seed)
    LX, LY = 40000.0, float(ly)
    x, y, tri, (ii, jj) = jittered_delaunay(nx, ny, LX, LY, 0.3, rng)
    z = -20.0 + 23.0 * x / LX + rng.normal(0.0, 0.2, size=x.shape)
    west = np.arange(ny)
    z[west] = -20.0  # flat inflow edge
    xyz = np.stack([x, y, z], axis=1)
    ch = _edge_chains(ii, jj, nx, ny)
    seg = boundary_segments(ch["west"], -1)
    kind = np.zeros(len(seg), np.int32)
    V = xyz.shape[0]
    sol0 = np.zeros(3 * V)
    sol0[0::3] = -z
    dt = 120.0
    tf = dt * nsteps
    t = np.arange(0.0, tf + dt, dt / 4.0)
    q = 500.0 + 1500.0 * np.sin(np.pi * t / (6 * 3600.0)) ** 2
    series = {0: _const_series(0.0, tf + dt, 20.0), 1: (t, q / (10000.0 * 20.0)), 2: _const_series(0.0, tf + dt, 0.0)}
    return SW2Case("beach", xyz, tri, seg, kind, sol0, dt, nsteps, series)


def small_delaunay_case(n: int = 24, seed: int = 7, wetdry: bool = True, nsteps: int = 5,
                        dt: float = 30.0) -> SW2Case:
    """A small jittered-Delaunay beach with both boundary kinds and a partly dry
    region, sized for entry-by-entry parity checks against the reference.  Larger
    dt make the Newton solve harder (line-search cuts, then failure)."""
    rng = np.random.default_rng(seed)
    L = 1000.0
    x, y, tri, (ii, jj) = jittered_delaunay(n, n, L, L, 0.3, rng)
    z = -2.0 + (2.6 * x / L if wetdry else 0.0) + rng.normal(0, 0.05, size=x.shape)
    z[np.arange(n)] = -2.0
    z[(n - 1) * n + np.arange(n)] = z[(n - 1) * n + np.arange(n)]  # east edge keeps its noise
    xyz = np.stack([x, y, z], axis=1)
    ch = _edge_chains(ii, jj, n, n)
    seg_w = boundary_segments(ch["west"], -1)
    seg_s = boundary_segments(ch["south"], +1)
    seg = np.concatenate([seg_w, seg_s[: n // 3]])
    kind = np.concatenate([np.zeros(len(seg_w), np.int32), np.ones(n // 3, np.int32)])
    V = xyz.shape[0]
    sol0 = np.zeros(3 * V)
    sol0[0::3] = 0.1 - z
    sol0[1::3] = 0.02 * rng.standard_normal(V)
    sol0[2::3] = 0.02 * rng.standard_normal(V)
    tf = dt * (nsteps + 1)
    series = {0: (np.array([0.0, tf]), np.array([2.1, 2.2])), 1: (np.array([0.0, tf]), np.array([0.05, 0.08])),
              2: _const_series(0.0, tf, 0.01)}
    return SW2Case("delaunay_small", xyz, tri, seg, kind, sol0, dt, nsteps, series)


def basin_hydro_case(hydro_seed: int, n: int = 707, seed: int = 2, nsteps: int = 375, dt: float = 300.0) -> SW2Case:
    """The learned-guess workload: the fully wet tidal basin of :func:`basin_case` (same
    mesh, bathymetry and 1 m / 12.42 h tide on the west edge) with an inflow hydrograph on
    the east edge, Q(t) = 200 + (Q_peak - 200) sin^2(pi t / 24 h) m^3/s, Q_peak drawn from
    U[1000, 3000] by ``hydro_seed``, imposed as the normal velocity Q / (20 km * 10 m)
    (a velocity boundary, like the beach's inflow).  Seeds 40-47 train the network, 48-51
    evaluate it."""
    base = basin_case(n=n, seed=seed, nsteps=nsteps)
    q_peak = float(np.random.default_rng(hydro_seed).uniform(1000.0, 3000.0))
    east = (n - 1) * n + np.arange(n)
    seg_e = boundary_segments(east, +1)
    seg = np.concatenate([base.seg, seg_e])
    kind = np.concatenate([base.seg_kind, np.zeros(len(seg_e), np.int32)])
    tf = dt * (nsteps + 1)
    t = np.arange(0.0, tf + dt, dt / 4.0)
    depth = 10.0 + 1.0 * np.sin(2 * np.pi * t / (12.42 * 3600.0))
    q = 200.0 + (q_peak - 200.0) * np.sin(np.pi * t / (24 * 3600.0)) ** 2
    series = {0: (t, depth), 1: (t, -q / (20000.0 * 10.0)), 2: _const_series(0.0, tf + dt, 0.0)}
    case = SW2Case(f"basin_hydro{hydro_seed}", base.xyz, base.tri, seg, kind, base.sol0, dt, nsteps, series)
    case.q_peak = q_peak
    return case


def estuary_case(nx: int = 4000, ny: int = 2000, seed: int = 5, nsteps: int = 500, dt: float = 180.0) -> SW2Case:
    """Estuary: 80 km x 40 km jittered Delaunay (nx x ny; the default 4000 x 2000 gives
    ~16M triangles), the ocean on the west edge and a river on the east edge.  Depth
    falls from 30 m at the ocean to 2 m at the river end; 32 seeded Gaussian shoals
    (height U[1, 5] m, sigma U[1, 4] km) rise out of the water where the base depth is
    small (partial wet/dry); a meandering channel (centreline 20 km + 5 km sin(2 pi x /
    40 km), 500 m wide) is 2 m deeper.  Forcing: an M2 tide of 1.5 m amplitude (12.42 h)
    as the depth of the flat west edge, and the river's 800 m^3/s as the inflow velocity
    on the east-edge segments inside the channel (800 / (500 m * 4 m)); the rest of the
    boundary is closed.  Still water at eta = 0 to start, dt = 180 s."""
    rng = np.random.default_rng(seed)
    LX, LY = 80000.0, 40000.0
    x, y, tri, (ii, jj) = jittered_delaunay(nx, ny, LX, LY, 0.3, rng)
    depth = 30.0 - 28.0 * x / LX
    cx = rng.uniform(0, LX, 32); cy = rng.uniform(0, LY, 32)
    amp = rng.uniform(1, 5, 32); sig = rng.uniform(1000, 4000, 32)
    for k in range(32):
        depth = depth - amp[k] * np.exp(-((x - cx[k]) ** 2 + (y - cy[k]) ** 2) / (2 * sig[k] ** 2))
    yc = 20000.0 + 5000.0 * np.sin(2 * np.pi * x / 40000.0)
    channel = np.abs(y - yc) < 250.0
    depth = np.where(channel, depth + 2.0, depth)
    west = np.arange(ny)
    depth[west] = 30.0                               # flat tidal edge (one depth for the whole string)
    z = -depth
    xyz = np.stack([x, y, z], axis=1)
    ch = _edge_chains(ii, jj, nx, ny)
    seg_w = boundary_segments(ch["west"], -1)
    east = ch["east"]
    seg_e_all = boundary_segments(east, +1)
    mid = 0.5 * (y[seg_e_all[:, 0]] + y[seg_e_all[:, 1]])
    yce = 20000.0 + 5000.0 * np.sin(2 * np.pi * LX / 40000.0)
    seg_e = seg_e_all[np.abs(mid - yce) < 250.0]
    z[np.unique(seg_e.ravel())] = -4.0               # the river mouth: 4 m deep
    xyz[:, 2] = z
    seg = np.concatenate([seg_w, seg_e])
    kind = np.concatenate([np.ones(len(seg_w), np.int32), np.zeros(len(seg_e), np.int32)])
    V = xyz.shape[0]
    sol0 = np.zeros(3 * V)
    sol0[0::3] = -z
    tf = dt * (nsteps + 1)
    t = np.arange(0.0, tf + dt, dt / 4.0)
    tide = 30.0 + 1.5 * np.sin(2 * np.pi * t / (12.42 * 3600.0))
    series = {0: (t, tide), 1: _const_series(0.0, tf + dt, -800.0 / (500.0 * 4.0)), 2: _const_series(0.0, tf + dt, 0.0)}
    return SW2Case("estuary", xyz, tri, seg, kind, sol0, dt, nsteps, series)
