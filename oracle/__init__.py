"""FP64 CPU oracle of the UFEM Navier-Stokes step -- TEST INFRASTRUCTURE ONLY.

Python binding of ``liboracle_ufem.so`` (``ufem_oracle.cpp``), the serial FP64
restatement of the reference's assembly, symmetric Dirichlet, solve and update.
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use it, and only as the checker or the timed CPU baseline; the product
package never imports it.  Parity status: see the header of ufem_oracle.cpp.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_ufem.so")

_D = C.POINTER(C.c_double)
_U32 = C.POINTER(C.c_uint32)
_I32 = C.POINTER(C.c_int32)
_I64 = C.POINTER(C.c_int64)


class OrcOptions(C.Structure):
    _fields_ = [("theta", C.c_double), ("dt", C.c_double), ("rho", C.c_double), ("supg_type", C.c_int32),
                ("use_specializations", C.c_int32), ("c1", C.c_double), ("c2", C.c_double),
                ("alpha_ps", C.c_double), ("alpha_su", C.c_double), ("alpha_bu", C.c_double),
                ("u_ref", C.c_double), ("precision", C.c_int32), ("reserved", C.c_int32)]


_SIG = {
    "orc_mesh_rectangle_tris": (None, [C.c_int, C.c_int, C.c_double, C.c_uint64, _D, _U32]),
    "orc_mesh_cube_tets": (None, [C.c_int, C.c_double, C.c_uint64, _D, _U32]),
    "orc_create": (C.c_void_p, [C.c_int, C.c_int64, C.c_int64, _D, _U32, C.POINTER(OrcOptions)]),
    "orc_create_periodic": (C.c_void_p, [C.c_int, C.c_int64, C.c_int64, _D, _U32, C.POINTER(OrcOptions), _U32, _U32,
                                         C.c_int64]),
    "orc_destroy": (None, [C.c_void_p]),
    "orc_create_lss": (C.c_void_p, [C.c_int64, C.c_int, _I64, _U32]),
    "orc_set_row": (None, [C.c_void_p, C.c_int64, C.c_int, C.c_double, C.c_double]),
    "orc_nrows": (C.c_int64, [C.c_void_p]),
    "orc_set_options": (None, [C.c_void_p, C.POINTER(OrcOptions)]),
    "orc_nnz": (C.c_int64, [C.c_void_p]),
    "orc_block_nnz": (C.c_int64, [C.c_void_p]),
    "orc_csr": (None, [C.c_void_p, _I64, _I32]),
    "orc_graph": (None, [C.c_void_p, _I64, _U32]),
    "orc_set_state": (None, [C.c_void_p, _D, _D, _D, _D]),
    "orc_get_state": (None, [C.c_void_p, _D, _D]),
    "orc_set_solution": (None, [C.c_void_p, _D]),
    "orc_get_solution": (None, [C.c_void_p, _D]),
    "orc_clear_dirichlet": (None, [C.c_void_p]),
    "orc_clear_neumann": (None, [C.c_void_p]),
    "orc_add_neumann": (None, [C.c_void_p, _U32, C.c_int64, C.c_int, C.c_double]),
    "orc_add_dirichlet": (None, [C.c_void_p, _U32, C.c_int64, C.c_int, _D]),
    "orc_add_dirichlet_dofs": (None, [C.c_void_p, _U32, _I32, _D, C.c_int64]),
    "orc_assemble": (None, [C.c_void_p, C.c_int]),
    "orc_apply_bcs": (None, [C.c_void_p]),
    "orc_set_system": (None, [C.c_void_p, _D, _D]),
    "orc_dirichlet": (None, [C.c_void_p, C.c_int64, C.c_int, C.c_double]),
    "orc_get_system": (None, [C.c_void_p, _D, _D]),
    "orc_solve": (C.c_int, [C.c_void_p, C.c_double, C.c_int, C.c_int, _I32, _D]),
    "orc_update": (None, [C.c_void_p]),
    "orc_step": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int]),
    "orc_time_assembly": (C.c_double, [C.c_void_p, C.c_int, C.c_int]),
    "orc_time_step_assembly": (C.c_double, [C.c_void_p, C.c_int, C.c_int]),
    "orc_element": (None, [C.c_void_p, C.c_int64, _D, _D, _D]),
    "orc_tau": (None, [C.c_int, C.c_int, _D, _D, C.c_double, C.c_double, C.c_double, C.c_double, _D]),
    "orc_semi_create": (C.c_void_p, [C.c_int, C.c_int64, C.c_int64, _D, _U32, C.POINTER(OrcOptions), C.c_int, _U32,
                                     _U32, C.c_int64]),
    "orc_semi_destroy": (None, [C.c_void_p]),
    "orc_semi_set_state": (None, [C.c_void_p, _D, _D, _D, _D]),
    "orc_semi_get_state": (None, [C.c_void_p, _D, _D]),
    "orc_semi_add_dirichlet": (None, [C.c_void_p, C.c_int, _U32, C.c_int64, C.c_int, _D]),
    "orc_semi_initialize": (None, [C.c_void_p, C.c_int]),
    "orc_semi_clear_dirichlet": (None, [C.c_void_p, C.c_int]),
    "orc_semi_set_fields": (None, [C.c_void_p, _D, _D]),
    "orc_semi_step": (C.c_int, [C.c_void_p, C.c_int, C.c_double, _I32, _D]),
    "orc_semi_velocity_matrix": (None, [C.c_void_p]),
    "orc_semi_rhs": (None, [C.c_void_p, C.c_int, _D, _D, _D, _D, _D, _D]),
    "orc_semi_nnz": (C.c_int64, [C.c_void_p, C.c_int]),
    "orc_semi_get_system": (None, [C.c_void_p, C.c_int, _D, _D, _D]),
    "orc_semi_lumped_inverse": (None, [C.c_void_p, _D]),
}

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        src = os.path.join(HERE, "ufem_oracle.cpp")
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIG.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def options(dt=0.01, rho=1.0, theta=1.0, supg_type=1, use_specializations=True, c1=1.0, c2=16.0,
            alpha_ps=1.0, alpha_su=1.0, alpha_bu=1.0, u_ref=1.0) -> OrcOptions:
    o = OrcOptions()
    o.theta, o.dt, o.rho = theta, dt, rho
    o.supg_type = {"tezduyar": 0, "metric": 1, "cf2": 2}.get(supg_type, supg_type)
    o.use_specializations = 1 if use_specializations else 0
    o.c1, o.c2, o.alpha_ps, o.alpha_su, o.alpha_bu, o.u_ref = c1, c2, alpha_ps, alpha_su, alpha_bu, u_ref
    return o


def mesh_rectangle_tris(nx, ny, jitter, seed):
    coords = np.empty(((nx + 1) * (ny + 1), 2))
    conn = np.empty((2 * nx * ny, 3), np.uint32)
    lib().orc_mesh_rectangle_tris(nx, ny, jitter, seed, _d(coords), conn.ctypes.data_as(_U32))
    return coords, conn


def mesh_cube_tets(n, jitter, seed):
    coords = np.empty(((n + 1) ** 3, 3))
    conn = np.empty((6 * n ** 3, 4), np.uint32)
    lib().orc_mesh_cube_tets(n, jitter, seed, _d(coords), conn.ctypes.data_as(_U32))
    return coords, conn


def tau(dim, supg_type, X, uc, nu, dt, c1=1.0, c2=16.0):
    X = np.ascontiguousarray(X, np.float64)
    uc = np.ascontiguousarray(uc, np.float64)
    out = np.empty(3)
    lib().orc_tau(dim, supg_type, _d(X), _d(uc), nu, dt, c1, c2, _d(out))
    return out  # tau_ps, tau_su, tau_bulk


def lid_driven_problem(dim, n, nu, dt, seed=20261203):
    """The seeded lid-driven cavity of the benchmark, built without the product
    library: the oracle's own mesh generators (bitwise equal to the product's),
    sine-mode initial velocities (4 modes in 2D, 6 in 3D, phases and wavenumbers
    from numpy's default_rng(seed + 1)), the NavierStokes initial conditions and
    the ordered Dirichlet list (walls, then the lid, pressure pinned at node 0).
    Returns a dict of the arrays; tests/test_oracle.py checks it against the
    product's problem generator bitwise."""
    import math
    if dim == 2:
        coords, conn = mesh_rectangle_tris(n, n, 0.2, seed)
        modes = 4
    else:
        coords, conn = mesh_cube_tets(n, 0.15, seed)
        modes = 6
    npts = coords.shape[0]
    rng = np.random.default_rng(seed + 1)
    u = np.zeros((npts, dim))
    for _ in range(modes):
        for c in range(dim):
            k = rng.integers(1, 4, size=dim)
            ph = rng.uniform(0.0, 2.0 * math.pi, size=dim)
            term = np.ones(npts)
            for a in range(dim):
                term = term * np.sin(math.pi * k[a] * coords[:, a] + ph[a])
            u[:, c] += (1.0 / modes) * term
    up = np.zeros((npts, dim + 1))
    up[:, :dim] = u
    lin = np.ascontiguousarray(np.tile(u, (1, 4)))
    nuv = np.full(npts, nu)
    s = n + 1
    idx = np.arange(s ** dim)
    ijk = (idx % s, idx // s) if dim == 2 else (idx % s, (idx // s) % s, idx // (s * s))
    walls = [ijk[0] == 0, ijk[0] == n, ijk[1] == 0] + ([] if dim == 2 else [ijk[1] == n, ijk[2] == 0])
    lid = ijk[1] == n if dim == 2 else ijk[2] == n
    nodes, comps, vals = [], [], []
    for mask, v in [(m, 0.0) for m in walls] + [(lid, 1.0)]:
        ids = np.nonzero(mask)[0].astype(np.uint32)
        cc = np.tile(np.arange(dim, dtype=np.int32), len(ids))
        vv = np.zeros(len(ids) * dim)
        vv[cc == 0] = v
        nodes.append(np.repeat(ids, dim))
        comps.append(cc)
        vals.append(vv)
    nodes.append(np.array([0], np.uint32))
    comps.append(np.array([dim], np.int32))
    vals.append(np.array([0.0]))
    return dict(coords=coords, conn=conn, up=up, lin=lin, nu=nuv, dt=dt,
                bc_nodes=np.concatenate(nodes), bc_comps=np.concatenate(comps), bc_values=np.concatenate(vals))


class LSS:
    """A bare oracle linear system on a node graph (for LSS-level known answers)."""

    def __init__(self, start, adj, neq):
        start = np.ascontiguousarray(start, np.int64)
        adj = np.ascontiguousarray(adj, np.uint32)
        self.N = len(start) - 1
        self.neq = neq
        self._h = lib().orc_create_lss(self.N, neq, start.ctypes.data_as(_I64), adj.ctypes.data_as(_U32))
        self.nnz = lib().orc_nnz(self._h)
        self.nrows = lib().orc_nrows(self._h)

    def set_row(self, blockrow, ieq, diag, offdiag):
        lib().orc_set_row(self._h, blockrow, ieq, diag, offdiag)

    def symmetric_dirichlet(self, blockrow, ieq, value):
        lib().orc_dirichlet(self._h, blockrow, ieq, value)

    def csr(self):
        rp = np.empty(self.nrows + 1, np.int64)
        ci = np.empty(self.nnz, np.int32)
        lib().orc_csr(self._h, rp.ctypes.data_as(_I64), ci.ctypes.data_as(_I32))
        return rp, ci

    def system(self):
        vals = np.empty(self.nnz)
        rhs = np.empty(self.nrows)
        lib().orc_get_system(self._h, _d(vals), _d(rhs))
        return vals, rhs

    def solution(self):
        s = np.empty(self.nrows)
        lib().orc_get_solution(self._h, _d(s))
        return s

    def dense(self):
        rp, ci = self.csr()
        vals, _ = self.system()
        A = np.zeros((self.nrows, self.nrows))
        for r in range(self.nrows):
            A[r, ci[rp[r]:rp[r + 1]]] = vals[rp[r]:rp[r + 1]]
        return A

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None


class Oracle:
    """Serial FP64 restatement of one NavierStokes action + its LSS."""

    def __init__(self, coords, conn, opts: OrcOptions, periodic_links=None):
        """periodic_links: (slaves, masters) node arrays (LSSAction.cpp:245-269)."""
        coords = np.ascontiguousarray(coords, np.float64)
        conn = np.ascontiguousarray(conn, np.uint32)
        self.dim = coords.shape[1]
        self.neq = self.dim + 1
        self.N = coords.shape[0]
        self.E = conn.shape[0]
        self.opts = opts
        if periodic_links is None:
            self._h = lib().orc_create(self.dim, self.N, self.E, _d(coords), conn.ctypes.data_as(_U32), C.byref(opts))
        else:
            sl = np.ascontiguousarray(periodic_links[0], np.uint32)
            ms = np.ascontiguousarray(periodic_links[1], np.uint32)
            self._h = lib().orc_create_periodic(self.dim, self.N, self.E, _d(coords), conn.ctypes.data_as(_U32),
                                                C.byref(opts), sl.ctypes.data_as(_U32), ms.ctypes.data_as(_U32), len(sl))
        if not self._h:
            raise ValueError("oracle: invalid mesh")
        self.nnz = lib().orc_nnz(self._h)
        self.block_nnz = lib().orc_block_nnz(self._h)
        self.nrows = self.N * self.neq

    def set_options(self, opts: OrcOptions):
        self.opts = opts
        lib().orc_set_options(self._h, C.byref(opts))

    def csr(self):
        rp = np.empty(self.nrows + 1, np.int64)
        ci = np.empty(self.nnz, np.int32)
        lib().orc_csr(self._h, rp.ctypes.data_as(_I64), ci.ctypes.data_as(_I32))
        return rp, ci

    def graph(self):
        st = np.empty(self.N + 1, np.int64)
        adj = np.empty(self.block_nnz, np.uint32)
        lib().orc_graph(self._h, st.ctypes.data_as(_I64), adj.ctypes.data_as(_U32))
        return st, adj

    def set_state(self, up, lin, nu, force=None):
        up = np.ascontiguousarray(up, np.float64)
        lin = np.ascontiguousarray(lin, np.float64)
        nu = np.ascontiguousarray(nu, np.float64)
        f = None if force is None else np.ascontiguousarray(force, np.float64)
        lib().orc_set_state(self._h, _d(up), _d(lin), _d(nu), _d(f))

    def state(self):
        up = np.empty((self.N, self.neq))
        lin = np.empty((self.N, 4 * self.dim))
        lib().orc_get_state(self._h, _d(up), _d(lin))
        return up, lin

    def set_solution(self, s):
        lib().orc_set_solution(self._h, _d(np.ascontiguousarray(s, np.float64)))

    def solution(self):
        s = np.empty(self.nrows)
        lib().orc_get_solution(self._h, _d(s))
        return s

    def add_dirichlet(self, nodes, comps, values):
        nodes = np.ascontiguousarray(nodes, np.uint32)
        comps = np.ascontiguousarray(np.broadcast_to(np.asarray(comps, np.int32), nodes.shape))
        values = np.ascontiguousarray(np.broadcast_to(np.asarray(values, np.float64), nodes.shape))
        lib().orc_add_dirichlet_dofs(self._h, nodes.ctypes.data_as(_U32), comps.ctypes.data_as(_I32), _d(values),
                                     len(nodes))

    def clear_dirichlet(self):
        lib().orc_clear_dirichlet(self._h)

    def add_neumann(self, faces, comp: int, flux: float):
        """Constant Neumann condition on Line2D faces (nfaces x 2 node ids)."""
        faces = np.ascontiguousarray(faces, np.uint32)
        lib().orc_add_neumann(self._h, faces.ctypes.data_as(_U32), len(faces), int(comp), float(flux))

    def clear_neumann(self):
        lib().orc_clear_neumann(self._h)

    def assemble(self, nthreads: int = 1):
        lib().orc_assemble(self._h, nthreads)

    def apply_dirichlet(self):
        lib().orc_apply_bcs(self._h)

    def set_system(self, vals, rhs):
        lib().orc_set_system(self._h, _d(np.ascontiguousarray(vals, np.float64)),
                             _d(np.ascontiguousarray(rhs, np.float64)))

    def dirichlet(self, node, comp, value):
        lib().orc_dirichlet(self._h, node, comp, value)

    def system(self):
        vals = np.empty(self.nnz)
        rhs = np.empty(self.nrows)
        lib().orc_get_system(self._h, _d(vals), _d(rhs))
        return vals, rhs

    def solve(self, tol=1e-13, maxit=5000, restart=60):
        it = C.c_int32()
        rr = C.c_double()
        rc = lib().orc_solve(self._h, tol, maxit, restart, C.byref(it), C.byref(rr))
        return {"rc": rc, "iterations": it.value, "rel_residual": rr.value}

    def update(self):
        lib().orc_update(self._h)

    def step(self, nsteps=1, tol=1e-13, maxit=5000, restart=60, nthreads=1):
        return lib().orc_step(self._h, nsteps, tol, maxit, restart, nthreads)

    def time_assembly(self, nthreads=1, reps=1) -> float:
        return lib().orc_time_assembly(self._h, nthreads, reps)

    def time_step_assembly(self, nthreads=1, reps=1) -> float:
        """Seconds for `reps` of ZeroLSS + LinearizeU + assembly + symmetric Dirichlet."""
        return lib().orc_time_step_assembly(self._h, nthreads, reps)

    def element(self, e):
        nd = (self.dim + 1) ** 2
        A = np.empty((nd, nd))
        T = np.empty((nd, nd))
        a = np.empty(nd)
        lib().orc_element(self._h, e, _d(A), _d(T), _d(a))
        return A, T, a

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SemiImplicit:
    """The semi-implicit scheme (NavierStokesSemiImplicit) restated in FP64."""

    def __init__(self, coords, conn, opts: OrcOptions, nb_iterations: int = 2, periodic_links=None):
        self._lib = lib()
        self.coords = np.ascontiguousarray(coords, np.float64)
        self.conn = np.ascontiguousarray(conn, np.uint32)
        self.dim = self.coords.shape[1]
        self.N = self.coords.shape[0]
        sl = ms = None
        n = 0
        if periodic_links is not None:
            sl = np.ascontiguousarray(periodic_links[0], np.uint32)
            ms = np.ascontiguousarray(periodic_links[1], np.uint32)
            n = len(sl)
        self._keep = (sl, ms)
        self._h = self._lib.orc_semi_create(self.dim, self.N, self.conn.shape[0], _d(self.coords),
                                            self.conn.ctypes.data_as(_U32), C.byref(opts), int(nb_iterations),
                                            None if sl is None else sl.ctypes.data_as(_U32),
                                            None if ms is None else ms.ctypes.data_as(_U32), n)
        if not self._h:
            raise RuntimeError("orc_semi_create failed")

    def initial_conditions(self, u, nu, p=None, force=None):
        up = np.zeros((self.N, self.dim + 1))
        up[:, : self.dim] = u
        if p is not None:
            up[:, self.dim] = p
        lin = np.tile(np.asarray(u, np.float64), (1, 4))
        nuv = np.ascontiguousarray(np.broadcast_to(np.asarray(nu, np.float64), (self.N,)))
        self.set_state(up, lin, nuv, force)
        self._lib.orc_semi_initialize(self._h, 1)

    def set_state(self, up, lin, nu, force=None):
        up, lin, nu = (np.ascontiguousarray(a, np.float64) for a in (up, lin, nu))
        f = None if force is None else np.ascontiguousarray(force, np.float64)
        self._lib.orc_semi_set_state(self._h, _d(up), _d(lin), _d(nu), None if f is None else _d(f))

    def initialize(self, reset_history=True):
        self._lib.orc_semi_initialize(self._h, 1 if reset_history else 0)

    def state(self):
        up = np.empty((self.N, self.dim + 1))
        lin = np.empty((self.N, 4 * self.dim))
        self._lib.orc_semi_get_state(self._h, _d(up), _d(lin))
        return up, lin

    def add_velocity_dirichlet(self, nodes, comp, values):
        nodes = np.ascontiguousarray(nodes, np.uint32)
        values = np.ascontiguousarray(np.broadcast_to(np.asarray(values, np.float64), nodes.shape))
        self._lib.orc_semi_add_dirichlet(self._h, 0, nodes.ctypes.data_as(_U32), len(nodes), int(comp), _d(values))

    def add_pressure_dirichlet(self, nodes, values):
        nodes = np.ascontiguousarray(nodes, np.uint32)
        values = np.ascontiguousarray(np.broadcast_to(np.asarray(values, np.float64), nodes.shape))
        self._lib.orc_semi_add_dirichlet(self._h, 1, nodes.ctypes.data_as(_U32), len(nodes), 0, _d(values))

    def clear_dirichlet(self):
        self._lib.orc_semi_clear_dirichlet(self._h, 0)
        self._lib.orc_semi_clear_dirichlet(self._h, 1)

    def set_fields(self, up, lin):
        """Solution and linearised-velocity fields only (viscosity and force kept)."""
        up, lin = (np.ascontiguousarray(a, np.float64) for a in (up, lin))
        self._lib.orc_semi_set_fields(self._h, _d(up), _d(lin))

    def step(self, nsteps=1, tol=1e-13):
        iters = np.zeros(2, np.int32)
        worst = C.c_double()
        rc = self._lib.orc_semi_step(self._h, int(nsteps), tol, iters.ctypes.data_as(_I32), C.byref(worst))
        return rc, (int(iters[0]), int(iters[1])), worst.value

    def velocity_matrix(self):
        self._lib.orc_semi_velocity_matrix(self._h)
        return self.system("velocity")[0]

    def rhs(self, kind: str, uvec, avec, pvec, dpsum, da, dp):
        """Element right-hand side `kind` ("velocity", "pressure", "aup") on the given vectors."""
        arrs = [np.ascontiguousarray(a, np.float64).ravel() for a in (uvec, avec, pvec, dpsum, da, dp)]
        k = {"velocity": 0, "pressure": 1, "aup": 2}[kind]
        self._lib.orc_semi_rhs(self._h, k, *[_d(a) for a in arrs])
        return self.system("pressure" if k == 1 else "velocity")[1]

    def system(self, which: str):
        w = {"velocity": 0, "pressure": 1}[which]
        nnz = self._lib.orc_semi_nnz(self._h, w)
        nrows = self.N * (self.dim if w == 0 else 1)
        v, r, s = np.empty(nnz), np.empty(nrows), np.empty(nrows)
        self._lib.orc_semi_get_system(self._h, w, _d(v), _d(r), _d(s))
        return v, r, s

    def lumped_inverse(self):
        out = np.empty((self.N, self.dim))
        self._lib.orc_semi_lumped_inverse(self._h, _d(out))
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._lib.orc_semi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
