"""Host-side mirror of UFEM's NavierStokes solver action on the B200 library.

``NavierStokes`` follows the reference's ``cf3.UFEM.NavierStokes``
(plugins/UFEM/src/UFEM/ns_implementation/NavierStokes.cpp:49-192), an
``LSSActionUnsteady`` (LSSActionUnsteady.cpp:30-71) whose ``execute`` runs
ZeroLSS -> LinearizeU -> Assembly -> BoundaryConditions -> SolveLSS -> Update.
Option names and meanings are the reference's: ``use_specializations``,
``supg_type`` ("metric" | "tezduyar" | "cf2"), ``theta``, the physics
``density`` and ``dynamic_viscosity`` (the kinematic viscosity is derived as
mu/rho, NavierStokesPhysics.cpp:86-105), and the time step.  Errors raise
``UfemError`` carrying the library's status code.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N

SUPG_TYPES = {"tezduyar": 0, "metric": 1, "cf2": 2}
PRECISIONS = {"fp64": 0, "fp32": 1}


def _stream(stream) -> C.c_void_p | None:
    if stream is None:
        return None
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(int(getattr(stream, "cuda_stream", stream)))


def krylov_options(method: str = "bicgstab", restart: int = 30, max_iters: int = 3000, precond: str = "jacobi",
                   tol: float = 1e-10, mixed: bool | str = False, max_refine: int = 20, inner_tol: float = 1e-3):
    """mixed: False (FP64), True (FP32 inner solves, FP64 residual of the stored
    system) or "matrix_free" (FP32 inner solves on the stored system, FP64
    residual of the FP64 element expressions: with precision="fp32" elements
    the answer is the FP64 system's)."""
    o = N.KrylovOpts()
    o.method = {"gmres": 0, "bicgstab": 1, "cg": 2}[method]
    o.restart = restart
    o.max_iters = max_iters
    o.precond = {"none": 0, "jacobi": 1, "block_jacobi": 2, "two_level": 3, "two_level_coupled": 4}[precond]
    o.tol = tol
    if isinstance(mixed, str):
        if mixed != "matrix_free":
            raise ValueError("mixed must be a bool or 'matrix_free'")
        o.mixed = 2
    else:
        o.mixed = 1 if mixed else 0
    o.max_refine = max_refine
    o.inner_tol = inner_tol
    return o


class NavierStokes:
    """One UFEM NavierStokes action with its linear system on one GPU."""

    def __init__(self, coords: np.ndarray, conn: np.ndarray, *, dt: float, density: float = 1.0,
                 use_specializations: bool = True, supg_type: str = "metric", theta: float = 1.0,
                 c1: float = 1.0, c2: float = 16.0, alpha_ps: float = 1.0, alpha_su: float = 1.0,
                 alpha_bu: float = 1.0, u_ref: float = 1.0, precision: str = "fp64", periodic_links=None):
        """periodic_links: optional (slaves, masters) node arrays; see
        ufem_ns_create_periodic."""
        self._lib = N.lib()
        coords = np.ascontiguousarray(coords, np.float64)
        conn = np.ascontiguousarray(conn, np.uint32)
        self.dim = coords.shape[1]
        self.neq = self.dim + 1
        self.nb_nodes = coords.shape[0]
        self.nb_elems = conn.shape[0]
        if conn.shape[1] != self.dim + 1:
            raise ValueError("connectivity must have dim+1 columns (P1 triangles or tetrahedra)")
        self._opts = N.NSOptions()
        self._lib.ufem_ns_default_options(C.byref(self._opts))
        self._set_fields(dict(dt=dt, density=density, use_specializations=use_specializations,
                              supg_type=supg_type, theta=theta, c1=c1, c2=c2, alpha_ps=alpha_ps,
                              alpha_su=alpha_su, alpha_bu=alpha_bu, u_ref=u_ref, precision=precision))
        mesh = N.Mesh(self.dim, 0, self.nb_nodes, self.nb_elems, N.dptr(coords), N.u32ptr(conn))
        h = C.c_void_p()
        if periodic_links is None:
            N.check(self._lib.ufem_ns_create(C.byref(mesh), C.byref(self._opts), C.byref(h)))
        else:
            sl = np.ascontiguousarray(periodic_links[0], np.uint32)
            ms = np.ascontiguousarray(periodic_links[1], np.uint32)
            if sl.shape != ms.shape:
                raise ValueError("periodic_links: slaves and masters must have the same length")
            N.check(self._lib.ufem_ns_create_periodic(C.byref(mesh), C.byref(self._opts), N.u32ptr(sl), N.u32ptr(ms),
                                                      len(sl), C.byref(h)))
        self._h = h
        nr, nnz, bnnz = C.c_int64(), C.c_int64(), C.c_int64()
        N.check(self._lib.ufem_ns_sizes(self._h, C.byref(nr), C.byref(nnz), C.byref(bnnz)))
        self.nb_rows, self.nnz, self.block_nnz = nr.value, nnz.value, bnnz.value

    # -- options (NavierStokes.cpp:74-98 triggers) ---------------------------
    def _set_fields(self, kw: dict) -> None:
        o = self._opts
        for k, v in kw.items():
            if k == "dt":
                o.dt = float(v)
            elif k == "density":
                o.rho = float(v)
            elif k == "use_specializations":
                o.use_specializations = 1 if v else 0
            elif k == "supg_type":
                if v not in SUPG_TYPES:
                    raise ValueError(f"supg_type must be one of {sorted(SUPG_TYPES)}")
                o.supg_type = SUPG_TYPES[v]
            elif k == "precision":
                o.precision = PRECISIONS[v]
            elif k in ("theta", "c1", "c2", "alpha_ps", "alpha_su", "alpha_bu", "u_ref"):
                setattr(o, k, float(v))
            else:
                raise KeyError(f"unknown option {k}")

    def set_options(self, **kw) -> None:
        self._set_fields(kw)
        N.check(self._lib.ufem_ns_set_options(self._h, C.byref(self._opts)))

    @property
    def options(self) -> dict:
        o = self._opts
        inv = {v: k for k, v in SUPG_TYPES.items()}
        return dict(dt=o.dt, density=o.rho, use_specializations=bool(o.use_specializations),
                    supg_type=inv[o.supg_type], theta=o.theta, c1=o.c1, c2=o.c2, alpha_ps=o.alpha_ps,
                    alpha_su=o.alpha_su, alpha_bu=o.alpha_bu, u_ref=o.u_ref,
                    precision={v: k for k, v in PRECISIONS.items()}[o.precision])

    # -- fields ----------------------------------------------------------------
    def set_state(self, up: np.ndarray, lin: np.ndarray, nu: np.ndarray, force: np.ndarray | None = None) -> None:
        up = np.ascontiguousarray(up, np.float64)
        lin = np.ascontiguousarray(lin, np.float64)
        nu = np.ascontiguousarray(nu, np.float64)
        if up.shape != (self.nb_nodes, self.neq) or lin.shape != (self.nb_nodes, 4 * self.dim) or nu.shape != (self.nb_nodes,):
            raise ValueError("field shapes must be (N, neq), (N, 4*dim), (N,)")
        f = None if force is None else np.ascontiguousarray(force, np.float64)
        N.check(self._lib.ufem_ns_set_state(self._h, N.dptr(up), N.dptr(lin), N.dptr(nu), N.dptr(f)))

    def initial_conditions(self, u: np.ndarray, nu: float | np.ndarray, p: np.ndarray | None = None,
                           force: np.ndarray | None = None) -> None:
        """InitialConditions (NavierStokes.cpp:194-205): u_adv = u1 = u2 = u3 = u, nu_eff = nu."""
        u = np.ascontiguousarray(u, np.float64)
        up = np.zeros((self.nb_nodes, self.neq))
        up[:, : self.dim] = u
        if p is not None:
            up[:, self.dim] = p
        lin = np.tile(u, (1, 4))
        nuv = np.broadcast_to(np.asarray(nu, np.float64), (self.nb_nodes,)).copy()
        self.set_state(up, lin, nuv, force)

    def write_restart(self, path: str, current_time: float | None = None, time_step: float | None = None,
                      iteration: int = 0) -> None:
        """WriteRestartFile (solver/actions/WriteRestartFile.cpp:62-90): the
        device-resident state to `path` (XML) and `path`.bin (tables); the time
        defaults to the handle's."""
        dt = self._opts.dt if time_step is None else time_step
        current_time = self.time if current_time is None else current_time
        N.check(self._lib.ufem_ns_write_restart(self._h, str(path).encode(), float(current_time), float(dt),
                                                int(iteration)))

    def read_restart(self, path: str) -> tuple[float, float, int]:
        """ReadRestartFile (ReadRestartFile.cpp:67-110): restores the state;
        returns (current_time, time_step, iteration)."""
        t, dt, it = C.c_double(), C.c_double(), C.c_int64()
        N.check(self._lib.ufem_ns_read_restart(self._h, str(path).encode(), C.byref(t), C.byref(dt), C.byref(it)))
        return t.value, dt.value, it.value

    def state(self):
        up = np.empty((self.nb_nodes, self.neq))
        lin = np.empty((self.nb_nodes, 4 * self.dim))
        N.check(self._lib.ufem_ns_get_state(self._h, N.dptr(up), N.dptr(lin)))
        return up, lin

    def solution(self) -> np.ndarray:
        s = np.empty(self.nb_rows)
        N.check(self._lib.ufem_ns_get_solution(self._h, N.dptr(s)))
        return s

    def set_solution(self, s: np.ndarray) -> None:
        s = np.ascontiguousarray(s, np.float64)
        N.check(self._lib.ufem_ns_set_solution(self._h, N.dptr(s)))

    # -- boundary conditions -------------------------------------------------
    def clear_dirichlet(self) -> None:
        N.check(self._lib.ufem_ns_clear_dirichlet(self._h))

    def add_dirichlet(self, nodes, comps, values) -> None:
        """Ordered constant Dirichlet conditions; comps may be a scalar."""
        nodes = np.ascontiguousarray(nodes, np.uint32)
        values = np.ascontiguousarray(np.broadcast_to(np.asarray(values, np.float64), nodes.shape))
        comps = np.ascontiguousarray(np.broadcast_to(np.asarray(comps, np.int32), nodes.shape))
        N.check(self._lib.ufem_ns_add_dirichlet_dofs(self._h, N.u32ptr(nodes), N.i32ptr(comps), N.dptr(values),
                                                      len(nodes)))

    # -- actions -------------------------------------------------------------
    # -- overlapped host transfers (ufem_ns_stage_state / commit_state / fetch_rhs) --
    @staticmethod
    def _host_ptr(a):
        """Address of a host buffer: a (pinned) torch tensor or a C-contiguous
        float64 numpy array, which must stay alive until its copy is done."""
        if hasattr(a, "data_ptr"):
            return N.raw_dptr(a.data_ptr())
        if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
            raise ValueError("host buffers must be C-contiguous float64 arrays or tensors")
        return N.dptr(a)

    def stage_state(self, up, lin, nu, copy_stream) -> None:
        """Queue the upload of the next state on `copy_stream` (two staging buffers)."""
        N.check(self._lib.ufem_ns_stage_state(self._h, self._host_ptr(up), self._host_ptr(lin), self._host_ptr(nu),
                                              _stream(copy_stream)))

    def commit_state(self, stream) -> None:
        """Make `stream` wait for the oldest staged state and unpack it into the fields."""
        N.check(self._lib.ufem_ns_commit_state(self._h, _stream(stream)))

    def fetch_rhs(self, out, stream, copy_stream) -> None:
        """Read the RHS back into `out` (nb_rows float64) on `copy_stream`, after `stream`'s work."""
        N.check(self._lib.ufem_ns_fetch_rhs(self._h, self._host_ptr(out), _stream(stream), _stream(copy_stream)))

    def add_dirichlet_function(self, nodes: np.ndarray, comp: int, expr: str) -> None:
        """BCDirichletFunction (BCDirichletFunction.cpp:61-92): component `comp`
        of `nodes` ends at f(x, y, z, t), `expr` evaluated on the device."""
        nodes = np.ascontiguousarray(nodes, np.uint32)
        N.check(self._lib.ufem_ns_add_dirichlet_function(self._h, N.u32ptr(nodes), len(nodes), int(comp),
                                                         str(expr).encode()))

    @property
    def time(self) -> float:
        t = C.c_double()
        N.check(self._lib.ufem_ns_get_time(self._h, C.byref(t)))
        return t.value

    @time.setter
    def time(self, t: float) -> None:
        N.check(self._lib.ufem_ns_set_time(self._h, float(t)))

    def add_neumann(self, faces: np.ndarray, comp: int, flux: float) -> None:
        """BCNeumannConstant (BCNeumannConstant.cpp:54-60) on Line2D faces
        (nfaces x 2 node ids) of a 2D mesh; added before the Dirichlet conditions."""
        faces = np.ascontiguousarray(faces, np.uint32)
        if faces.ndim != 2 or faces.shape[1] != 2:
            raise ValueError("faces must be (nfaces, 2) node ids")
        N.check(self._lib.ufem_ns_add_neumann(self._h, N.u32ptr(faces), len(faces), int(comp), float(flux)))

    def clear_neumann(self) -> None:
        N.check(self._lib.ufem_ns_clear_neumann(self._h))

    def assemble(self, stream=None) -> None:
        """ZeroLSS + LinearizeU + Assembly."""
        N.check(self._lib.ufem_ns_assemble(self._h, _stream(stream)))

    def apply_dirichlet(self, stream=None) -> None:
        N.check(self._lib.ufem_ns_apply_dirichlet(self._h, _stream(stream)))

    def solve(self, stream=None, raise_on_failure: bool = True, **krylov) -> dict:
        st = N.KrylovStatus()
        rc = self._lib.ufem_ns_solve(self._h, C.byref(krylov_options(**krylov)), C.byref(st), _stream(stream))
        if rc != 0 and (raise_on_failure or rc != -7):
            N.check(rc)
        return st.as_dict()

    def update(self, stream=None) -> None:
        N.check(self._lib.ufem_ns_update(self._h, _stream(stream)))

    def execute(self, stream=None, **krylov) -> dict:
        """One time step (LSSAction::execute, LSSAction.cpp:122-135)."""
        self.assemble(stream)
        self.apply_dirichlet(stream)
        st = self.solve(stream, **krylov)
        self.update(stream)
        return st

    def step(self, nsteps: int, stream=None, **krylov) -> dict:
        st = N.KrylovStatus()
        N.check(self._lib.ufem_ns_step(self._h, nsteps, C.byref(krylov_options(**krylov)), C.byref(st),
                                       _stream(stream)))
        return st.as_dict()

    # -- linear system access (LSS::System / Matrix) -------------------------
    def csr(self):
        rowptr = np.empty(self.nb_rows + 1, np.int64)
        colidx = np.empty(self.nnz, np.int32)
        N.check(self._lib.ufem_ns_csr(self._h, N.i64ptr(rowptr), N.i32ptr(colidx)))
        return rowptr, colidx

    def graph(self):
        start = np.empty(self.nb_nodes + 1, np.int64)
        adj = np.empty(self.block_nnz, np.uint32)
        N.check(self._lib.ufem_ns_graph(self._h, N.i64ptr(start), N.u32ptr(adj)))
        return start, adj

    def system(self):
        vals = np.empty(self.nnz)
        rhs = np.empty(self.nb_rows)
        N.check(self._lib.ufem_ns_get_system(self._h, N.dptr(vals), N.dptr(rhs)))
        return vals, rhs

    def prepare_solve(self, batched: bool = False, **krylov) -> None:
        """Allocate the solver workspace and build the preconditioner structure
        ahead of the first solve (optional)."""
        N.check(self._lib.ufem_ns_prepare_solve(self._h, C.byref(krylov_options(**krylov)), 1 if batched else 0))

    def fp64_residual(self, stream=None) -> np.ndarray:
        """b - M x of the FP64 system for the current solution vector, evaluated
        element by element without a matrix (after assemble and apply_dirichlet)."""
        r = np.empty(self.nb_rows)
        N.check(self._lib.ufem_ns_fp64_residual(self._h, N.dptr(r), _stream(stream)))
        return r

    def apply(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty(self.nb_rows)
        N.check(self._lib.ufem_ns_apply(self._h, N.dptr(x), N.dptr(y)))
        return y

    def device_view(self) -> dict:
        v = N.DeviceView()
        N.check(self._lib.ufem_ns_device_view_get(self._h, C.byref(v)))
        return {k: getattr(v, k) for k, _ in v._fields_}

    def device_bytes(self) -> int:
        """Device memory held by this handle (bytes)."""
        v = C.c_int64()
        N.check(self._lib.ufem_ns_device_bytes(self._h, C.byref(v)))
        return v.value

    # -- assembly kernel selection and autotuning -----------------------------
    ASSEMBLY_VARIANTS = {"warp": 0, "chunk": 1, "warp24": 2}

    def set_assembly_kernel(self, variant: str = "warp", warps_per_cta: int = 4) -> None:
        """Pick the assembly kernel: "warp" (warp per group of rows with <= 32 incident elements),
        "warp24" (tetrahedra: groups of <= 24, smaller staging, more resident warps) or "chunk"
        (CTA per row range)."""
        N.check(self._lib.ufem_ns_set_assembly_kernel(self._h, self.ASSEMBLY_VARIANTS[variant], int(warps_per_cta)))

    def assembly_kernel(self) -> tuple[str, int]:
        v, w = C.c_int32(), C.c_int32()
        N.check(self._lib.ufem_ns_get_assembly_kernel(self._h, C.byref(v), C.byref(w)))
        names = {i: k for k, i in self.ASSEMBLY_VARIANTS.items()}
        return names[v.value], w.value

    def tune_assembly(self, reps: int = 5, stream: int = 0) -> dict:
        """Time every assembly kernel candidate on this mesh and keep the fastest."""
        v, w, ms = C.c_int32(), C.c_int32(), C.c_float()
        N.check(self._lib.ufem_ns_tune_assembly(self._h, C.c_void_p(stream), int(reps), C.byref(v), C.byref(w),
                                                C.byref(ms)))
        names = {i: k for k, i in self.ASSEMBLY_VARIANTS.items()}
        return {"variant": names[v.value], "warps_per_cta": w.value, "ms": ms.value}

    # -- timers (component timing of the reference) ----------------------------
    def enable_timing(self, on: bool = True) -> None:
        N.check(self._lib.ufem_ns_enable_timing(self._h, 1 if on else 0))

    def timings(self) -> dict:
        t = N.Timings()
        N.check(self._lib.ufem_ns_get_timings(self._h, C.byref(t)))
        return t.as_dict()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ufem_ns_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class NavierStokesSemiImplicit:
    """UFEM's semi-implicit solver (``cf3.UFEM.NavierStokesSemiImplicit``,
    plugins/UFEM/src/UFEM/ns_semi_implicit/implementation/NavierStokesSemiImplicit.cpp):
    a velocity system and a pressure system, ``nb_iterations`` predictor /
    corrector passes per time step.  Options follow the reference's
    (``theta``, ``nb_iterations``, ``supg_type``, ``alpha_*``, ``c1``, ``c2``,
    ``u_ref``); the body force term is on when a force field is given
    (``enable_body_force``).  Velocity and pressure conditions are added to
    ``VelocityLSS.BC`` / ``PressureLSS.BC`` through ``add_velocity_dirichlet`` and
    ``add_pressure_dirichlet``."""

    def __init__(self, coords: np.ndarray, conn: np.ndarray, *, dt: float, theta: float = 1.0,
                 nb_iterations: int = 2, supg_type: str = "metric", c1: float = 1.0, c2: float = 16.0,
                 alpha_ps: float = 1.0, alpha_su: float = 1.0, alpha_bu: float = 1.0, u_ref: float = 1.0,
                 periodic_links=None):
        self._lib = N.lib()
        coords = np.ascontiguousarray(coords, np.float64)
        conn = np.ascontiguousarray(conn, np.uint32)
        self.dim = coords.shape[1]
        self.nb_nodes = coords.shape[0]
        self.nb_elems = conn.shape[0]
        if conn.shape[1] != self.dim + 1:
            raise ValueError("connectivity must have dim+1 columns (P1 triangles or tetrahedra)")
        o = N.NSOptions()
        self._lib.ufem_ns_default_options(C.byref(o))
        if supg_type not in SUPG_TYPES:
            raise ValueError(f"supg_type must be one of {sorted(SUPG_TYPES)}")
        o.dt, o.theta, o.supg_type = float(dt), float(theta), SUPG_TYPES[supg_type]
        o.c1, o.c2, o.alpha_ps, o.alpha_su, o.alpha_bu, o.u_ref = c1, c2, alpha_ps, alpha_su, alpha_bu, u_ref
        self.dt = float(dt)
        mesh = N.Mesh(self.dim, 0, self.nb_nodes, self.nb_elems, N.dptr(coords), N.u32ptr(conn))
        sl = ms = None
        n = 0
        if periodic_links is not None:
            sl = np.ascontiguousarray(periodic_links[0], np.uint32)
            ms = np.ascontiguousarray(periodic_links[1], np.uint32)
            if sl.shape != ms.shape:
                raise ValueError("periodic_links: slaves and masters must have the same length")
            n = len(sl)
        h = C.c_void_p()
        N.check(self._lib.ufem_nssi_create(C.byref(mesh), C.byref(o), int(nb_iterations),
                                           None if sl is None else N.u32ptr(sl),
                                           None if ms is None else N.u32ptr(ms), n, C.byref(h)))
        self._h = h
        self._keep = (sl, ms)
        vn, pn = C.c_int64(), C.c_int64()
        N.check(self._lib.ufem_nssi_sizes(self._h, C.byref(vn), C.byref(pn)))
        self.velocity_nnz, self.pressure_nnz = vn.value, pn.value
        self.set_krylov()

    def set_krylov(self, velocity: dict | None = None, pressure: dict | None = None) -> None:
        """Krylov options of the two solves (default: CG to 1e-10; point Jacobi
        for the velocity, the two-level preconditioner for the pressure)."""
        kv = krylov_options(**{"method": "cg", **(velocity or {})})
        kp = krylov_options(**{"method": "cg", "precond": "two_level", **(pressure or {})})
        N.check(self._lib.ufem_nssi_set_krylov(self._h, C.byref(kv), C.byref(kp)))

    def initial_conditions(self, u: np.ndarray, nu: float | np.ndarray, p: np.ndarray | None = None,
                           force: np.ndarray | None = None) -> None:
        """Fields and the solver's initial conditions (NavierStokesSemiImplicit.cpp:400-455):
        u_adv = u1 = u2 = u3 = u, nu_eff = nu, the pressure matrix and the lumped mass."""
        u = np.ascontiguousarray(u, np.float64)
        up = np.zeros((self.nb_nodes, self.dim + 1))
        up[:, : self.dim] = u
        if p is not None:
            up[:, self.dim] = p
        lin = np.tile(u, (1, 4))
        nuv = np.ascontiguousarray(np.broadcast_to(np.asarray(nu, np.float64), (self.nb_nodes,)))
        self.set_state(up, lin, nuv, force)
        self.initialize(reset_history=True)

    def set_state(self, up, lin, nu, force=None) -> None:
        up = np.ascontiguousarray(up, np.float64)
        lin = np.ascontiguousarray(lin, np.float64)
        nu = np.ascontiguousarray(nu, np.float64)
        if up.shape != (self.nb_nodes, self.dim + 1) or lin.shape != (self.nb_nodes, 4 * self.dim) or \
                nu.shape != (self.nb_nodes,):
            raise ValueError("field shapes must be (N, dim+1), (N, 4*dim), (N,)")
        f = None if force is None else np.ascontiguousarray(force, np.float64)
        N.check(self._lib.ufem_nssi_set_state(self._h, N.dptr(up), N.dptr(lin), N.dptr(nu), N.dptr(f)))

    def initialize(self, reset_history: bool = True, stream=None) -> None:
        N.check(self._lib.ufem_nssi_initialize(self._h, 1 if reset_history else 0, _stream(stream)))

    @property
    def state(self):
        up = np.empty((self.nb_nodes, self.dim + 1))
        lin = np.empty((self.nb_nodes, 4 * self.dim))
        N.check(self._lib.ufem_nssi_get_state(self._h, N.dptr(up), N.dptr(lin)))
        return up, lin

    @property
    def time(self) -> float:
        t = C.c_double()
        N.check(self._lib.ufem_nssi_get_time(self._h, C.byref(t)))
        return t.value

    def add_velocity_dirichlet(self, nodes, comp: int, values) -> None:
        nodes = np.ascontiguousarray(nodes, np.uint32)
        values = np.ascontiguousarray(np.broadcast_to(np.asarray(values, np.float64), nodes.shape))
        N.check(self._lib.ufem_nssi_add_velocity_dirichlet(self._h, N.u32ptr(nodes), len(nodes), int(comp),
                                                           N.dptr(values)))

    def add_pressure_dirichlet(self, nodes, values) -> None:
        nodes = np.ascontiguousarray(nodes, np.uint32)
        values = np.ascontiguousarray(np.broadcast_to(np.asarray(values, np.float64), nodes.shape))
        N.check(self._lib.ufem_nssi_add_pressure_dirichlet(self._h, N.u32ptr(nodes), len(nodes), N.dptr(values)))

    def add_velocity_dirichlet_function(self, nodes, comp: int, expr: str) -> None:
        nodes = np.ascontiguousarray(nodes, np.uint32)
        N.check(self._lib.ufem_nssi_add_velocity_dirichlet_function(self._h, N.u32ptr(nodes), len(nodes), int(comp),
                                                                    expr.encode()))

    def add_pressure_dirichlet_function(self, nodes, expr: str) -> None:
        nodes = np.ascontiguousarray(nodes, np.uint32)
        N.check(self._lib.ufem_nssi_add_pressure_dirichlet_function(self._h, N.u32ptr(nodes), len(nodes),
                                                                    expr.encode()))

    @time.setter
    def time(self, t: float) -> None:
        N.check(self._lib.ufem_nssi_set_time(self._h, float(t)))

    def write_restart(self, path: str, current_time: float | None = None, time_step: float | None = None,
                      iteration: int = 0) -> None:
        t = self.time if current_time is None else current_time
        N.check(self._lib.ufem_nssi_write_restart(self._h, path.encode(), t,
                                                  self.dt if time_step is None else time_step, int(iteration)))

    def read_restart(self, path: str, initialize: bool = True) -> tuple[float, float, int]:
        """Reads the fields and (by default) reruns the initial-condition assemblies
        without resetting the history; returns (time, time_step, iteration)."""
        t, dt, it = C.c_double(), C.c_double(), C.c_int64()
        N.check(self._lib.ufem_nssi_read_restart(self._h, path.encode(), C.byref(t), C.byref(dt), C.byref(it)))
        if initialize:
            self.initialize(reset_history=False)
        return t.value, dt.value, it.value

    def clear_dirichlet(self) -> None:
        N.check(self._lib.ufem_nssi_clear_dirichlet(self._h))

    def step(self, nsteps: int = 1, stream=None) -> tuple[dict, dict]:
        """nsteps time steps; returns the folded (velocity, pressure) solve statuses."""
        sv, sp = N.KrylovStatus(), N.KrylovStatus()
        N.check(self._lib.ufem_nssi_step(self._h, int(nsteps), C.byref(sv), C.byref(sp), _stream(stream)))
        return sv.as_dict(), sp.as_dict()

    def system(self, which: str):
        """(rowptr, colidx, vals, rhs, sol) of the "velocity" or "pressure" system."""
        w = {"velocity": 0, "pressure": 1}[which]
        nrows = self.nb_nodes * (self.dim if w == 0 else 1)
        nnz = self.velocity_nnz if w == 0 else self.pressure_nnz
        rp, ci = np.empty(nrows + 1, np.int64), np.empty(nnz, np.int32)
        v, r, s = np.empty(nnz), np.empty(nrows), np.empty(nrows)
        N.check(self._lib.ufem_nssi_get_system(self._h, w, N.i64ptr(rp), N.i32ptr(ci), N.dptr(v), N.dptr(r),
                                               N.dptr(s)))
        return rp, ci, v, r, s

    def assemble_velocity_matrix(self, stream=None) -> None:
        N.check(self._lib.ufem_nssi_assemble_velocity_matrix(self._h, _stream(stream)))

    def lumped_inverse(self) -> np.ndarray:
        out = np.empty((self.nb_nodes, self.dim))
        N.check(self._lib.ufem_nssi_get_lumped_inverse(self._h, N.dptr(out)))
        return out

    def device_bytes(self) -> int:
        return int(self._lib.ufem_nssi_device_bytes(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.ufem_nssi_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class Batch:
    """Several NavierStokes handles stepped together: each phase of a time step
    is one launch over all members, and the BiCGStab solve keeps per-member
    scalars, so a member's results are the same alone and in any batch.

    Members must share dim, precision and element form; they stay owned by the
    caller (the batch keeps references) and must not be closed while it lives.
    """

    def __init__(self, members: list, graphs: bool = True, assembly_warps: int | None = None):
        if not members:
            raise ValueError("a batch needs at least one member")
        self._lib = N.lib()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.handle for m in self.members])
        self._b = C.c_void_p()
        N.check(self._lib.ufem_batch_create(arr, len(self.members), C.byref(self._b)))
        self.set_graphs(graphs)
        if assembly_warps is not None:
            N.check(self._lib.ufem_batch_set_assembly_warps(self._b, int(assembly_warps)))

    def __len__(self) -> int:
        return len(self.members)

    def set_graphs(self, on: bool) -> None:
        N.check(self._lib.ufem_batch_set_graphs(self._b, 1 if on else 0))

    def set_active(self, active) -> None:
        """Hold (False) or resume (True) members without rebuilding the batch; a
        held member is neither solved nor updated."""
        arr = (C.c_int32 * len(self.members))(*[1 if a else 0 for a in active])
        N.check(self._lib.ufem_batch_set_active(self._b, arr))

    def tune_assembly(self, reps: int = 5, stream=None) -> dict:
        """Time the batched assembly with 2, 4 and 8 warps per CTA and keep the
        fastest (the members' systems are overwritten; assemble afterwards)."""
        w, ms = C.c_int32(), C.c_float()
        N.check(self._lib.ufem_batch_tune_assembly(self._b, _stream(stream), int(reps), C.byref(w), C.byref(ms)))
        return {"warps_per_cta": w.value, "ms": ms.value}

    def assemble(self, stream=None) -> None:
        N.check(self._lib.ufem_batch_assemble(self._b, _stream(stream)))

    def solve(self, stream=None, **krylov) -> list[dict]:
        sts = (N.KrylovStatus * len(self.members))()
        N.check(self._lib.ufem_batch_solve(self._b, C.byref(krylov_options(**krylov)), sts, _stream(stream)))
        return [s.as_dict() for s in sts]

    def update(self, stream=None) -> None:
        N.check(self._lib.ufem_batch_update(self._b, _stream(stream)))

    def step(self, stream=None, **krylov) -> list[dict]:
        """One time step of every member: assemble, Dirichlet, solve, update."""
        sts = (N.KrylovStatus * len(self.members))()
        N.check(self._lib.ufem_batch_step(self._b, C.byref(krylov_options(**krylov)), sts, _stream(stream)))
        return [s.as_dict() for s in sts]

    def close(self) -> None:
        if getattr(self, "_b", None):
            self._lib.ufem_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
