"""Seeded synthetic problems with the shapes of the benchmark configurations.

No public dataset is involved: meshes are generated (unit square split into
triangles as ``create_rectangle_tris`` does, cf3/Tools/MeshGeneration/
MeshGeneration.cpp:209-253; unit cube split into Kuhn tetrahedra), interior
nodes are jittered from a counter-based hash, initial velocities are sums of
sine modes with seeded phases, and the boundary conditions are those of a
lid-driven cavity.  Every array here is produced identically for the oracle
and the GPU path, so parity tests feed both the same inputs.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import _native as N

DEFAULT_SEED = 20261203


def rectangle_tris(nx: int, ny: int | None = None, jitter: float = 0.2, seed: int = DEFAULT_SEED):
    """(coords (N,2) float64, conn (2*nx*ny, 3) uint32); node = j*(nx+1)+i."""
    ny = nx if ny is None else ny
    coords = np.empty(((nx + 1) * (ny + 1), 2), np.float64)
    conn = np.empty((2 * nx * ny, 3), np.uint32)
    N.check(N.lib().ufem_mesh_rectangle_tris(nx, ny, jitter, seed, N.dptr(coords), N.u32ptr(conn)))
    return coords, conn


def cube_tets(n: int, jitter: float = 0.15, seed: int = DEFAULT_SEED):
    """(coords ((n+1)^3,3) float64, conn (6n^3, 4) uint32); node = (k*(n+1)+j)*(n+1)+i."""
    coords = np.empty(((n + 1) ** 3, 3), np.float64)
    conn = np.empty((6 * n ** 3, 4), np.uint32)
    N.check(N.lib().ufem_mesh_cube_tets(n, jitter, seed, N.dptr(coords), N.u32ptr(conn)))
    return coords, conn


def sine_velocity(coords: np.ndarray, modes: int, seed: int, amplitude: float = 1.0) -> np.ndarray:
    """Sum of `modes` products of sines with seeded integer wavenumbers (1..3)
    and phases per component; each mode carries amplitude/modes."""
    npts, dim = coords.shape
    rng = np.random.default_rng(seed)
    u = np.zeros((npts, dim), np.float64)
    for _ in range(modes):
        for c in range(dim):
            k = rng.integers(1, 4, size=dim)
            ph = rng.uniform(0.0, 2.0 * math.pi, size=dim)
            term = np.ones(npts)
            for a in range(dim):
                term = term * np.sin(math.pi * k[a] * coords[:, a] + ph[a])
            u[:, c] += (amplitude / modes) * term
    return u


def initial_fields(u: np.ndarray, nu: float, p: np.ndarray | None = None):
    """InitialConditions of the NS action (NavierStokes.cpp:194-205):
    navier_stokes_solution = (u, p), linearized_velocity = (u, u, u, u),
    navier_stokes_viscosity = nu.  Returns (up (N,neq), lin (N,4d), nu (N,))."""
    npts, dim = u.shape
    up = np.zeros((npts, dim + 1), np.float64)
    up[:, :dim] = u
    if p is not None:
        up[:, dim] = p
    lin = np.ascontiguousarray(np.tile(u, (1, 4)))
    return up, lin, np.full(npts, nu, np.float64)


def structured_index(dim: int, n: int):
    """Integer lattice indices (i, j[, k]) of the structured generators' nodes."""
    s = n + 1
    idx = np.arange(s ** dim)
    if dim == 2:
        return idx % s, idx // s
    return idx % s, (idx // s) % s, idx // (s * s)


def lid_driven_bcs(dim: int, n: int, lid_velocity: float = 1.0, pin_pressure: bool = True):
    """Ordered Dirichlet list of a lid-driven cavity on the structured mesh of
    `n` cells per side: walls (x=0, x=1, y=0, [y=1, z=0]) get u = 0, then the lid
    (y=1 in 2D, z=1 in 3D) gets u = (lid, 0[, 0]); each region's nodes ascend and
    each node lists its components in turn, as a vector `dirichlet(u) = value`
    does.  Corner nodes appear in several regions (the last value wins for the
    row; the first moves the column).  Pressure is pinned at node 0 last."""
    ijk = structured_index(dim, n)
    if dim == 2:
        regions = [(ijk[0] == 0, 0.0), (ijk[0] == n, 0.0), (ijk[1] == 0, 0.0), (ijk[1] == n, lid_velocity)]
    else:
        regions = [(ijk[0] == 0, 0.0), (ijk[0] == n, 0.0), (ijk[1] == 0, 0.0), (ijk[1] == n, 0.0),
                   (ijk[2] == 0, 0.0), (ijk[2] == n, lid_velocity)]
    nodes, comps, vals = [], [], []
    for mask, lid in regions:
        ids = np.nonzero(mask)[0].astype(np.uint32)
        rep = np.repeat(ids, dim)
        cc = np.tile(np.arange(dim, dtype=np.int32), len(ids))
        vv = np.zeros(len(rep))
        vv[cc == 0] = lid
        nodes.append(rep)
        comps.append(cc)
        vals.append(vv)
    if pin_pressure:
        nodes.append(np.array([0], np.uint32))
        comps.append(np.array([dim], np.int32))
        vals.append(np.array([0.0]))
    return (np.ascontiguousarray(np.concatenate(nodes), dtype=np.uint32),
            np.ascontiguousarray(np.concatenate(comps), dtype=np.int32),
            np.ascontiguousarray(np.concatenate(vals), dtype=np.float64))


@dataclass
class Problem:
    """A complete synthetic NS problem (mesh, fields, BCs, options)."""
    name: str
    dim: int
    n: int
    coords: np.ndarray
    conn: np.ndarray
    up: np.ndarray
    lin: np.ndarray
    nu: np.ndarray
    bc_nodes: np.ndarray
    bc_comps: np.ndarray
    bc_values: np.ndarray
    dt: float
    rho: float = 1.0
    theta: float = 1.0
    steps: int = 1
    extra: dict = field(default_factory=dict)

    @property
    def nb_nodes(self) -> int:
        return self.coords.shape[0]

    @property
    def nb_elems(self) -> int:
        return self.conn.shape[0]


def make_problem(dim: int, n: int, *, jitter: float | None = None, modes: int | None = None, nu: float = 1e-2,
                 dt: float = 0.01, seed: int = DEFAULT_SEED, steps: int = 1, name: str = "custom") -> Problem:
    if dim == 2:
        coords, conn = rectangle_tris(n, n, 0.2 if jitter is None else jitter, seed)
        modes = 4 if modes is None else modes
    else:
        coords, conn = cube_tets(n, 0.15 if jitter is None else jitter, seed)
        modes = 6 if modes is None else modes
    u = sine_velocity(coords, modes, seed + 1)
    up, lin, nuv = initial_fields(u, nu)
    bn, bc, bv = lid_driven_bcs(dim, n)
    return Problem(name, dim, n, coords, conn, up, lin, nuv, bn, bc, bv, dt=dt, steps=steps)


def config(name: str, seed: int = DEFAULT_SEED) -> Problem:
    """The benchmark configurations (sizes exactly as specified):

    cfg1  2D P1 triangles, 64x64 cells x 2 (8,192 tris, 4,225 nodes), jitter 0.2h,
          4 sine modes, nu=1e-2, dt=0.01, 1 step
    cfg2  3D P1 tets, 64^3 cells x 6 (1,572,864 tets, 274,625 nodes), jitter 0.15h,
          6 modes, nu=1e-3, dt=5e-3, 10 steps
    cfg3  3D P1 tets, 128^3 x 6 (12,582,912 tets, 2,146,689 nodes), nu log-uniform
          in [1e-4, 1e-2] drawn from the seed, dt=5e-3
    """
    if name == "cfg1":
        return make_problem(2, 64, nu=1e-2, dt=0.01, seed=seed, steps=1, name=name)
    if name == "cfg2":
        return make_problem(3, 64, nu=1e-3, dt=5e-3, seed=seed, steps=10, name=name)
    if name == "cfg3":
        rng = np.random.default_rng(seed + 3)
        nu = float(10.0 ** rng.uniform(-4.0, -2.0))
        return make_problem(3, 128, nu=nu, dt=5e-3, seed=seed, steps=10, name=name)
    raise KeyError(name)
