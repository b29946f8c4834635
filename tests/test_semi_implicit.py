"""Semi-implicit Navier-Stokes (NavierStokesSemiImplicit,
plugins/UFEM/src/UFEM/ns_semi_implicit/): velocity and pressure systems, the
predictor/corrector inner loop, periodic links and the body force.

Pins of the oracle (CPU):
  - the reference's own acceptance case, the periodic body-force channel of
    plugins/UFEM/test/atest-ufem-navier-stokes-semi-implicit-laminar-channel-2d.py
    (10 x 2 domain, 20 x 32 subdivisions, theta 0.5, two inner iterations,
    alpha_su 0, nu 1, force (2, 0), dt 0.5, 50 steps, pressure 10 at the centre):
    |u - y (2 - y)| <= 1e-2 and |v| <= 1e-3, the test's own bounds (the
    reference meshes the blocks with quadrilaterals, here triangles);
  - the same flow in 3D (plane Poiseuille between two walls, periodic in x and z,
    tetrahedra): u = g / (2 nu) y (H - y) to 1e-3, v = w = 0;
  - closed forms: the lumped mass of a node is the sum of |element| / (dim + 1)
    over its elements; the pressure matrix rows sum to zero; both systems are
    symmetric.
GPU parity against the oracle (stated tolerances): velocity matrix, pressure
matrix and lumped inverse within 1e-12 of each row's largest |entry|; three
time steps of a lid-driven cavity (2D and 3D, the three tau types) within 1e-8
of the largest field value with both solvers at 1e-12; the channel case within
1e-7 of the oracle (pressure solves at 1e-10) and inside the reference's bounds; two runs bitwise equal.
"""
import numpy as np
import pytest

import oracle as O
from coolfluid3_b200 import NavierStokesSemiImplicit
from coolfluid3_b200._native import UfemError

from .util import row_scaled_error

TAU = {"tezduyar": 0, "metric": 1, "cf2": 2}


def channel_case():
    """The laminar-channel acceptance case on triangles."""
    c, t = O.mesh_rectangle_tris(20, 32, 0.0, 1)
    c = c.copy()
    c[:, 0] *= 10.0
    c[:, 1] *= 2.0
    right = np.where(np.abs(c[:, 0] - 10) < 1e-9)[0]
    left = np.where(np.abs(c[:, 0]) < 1e-9)[0]
    right, left = right[np.argsort(c[right, 1])], left[np.argsort(c[left, 1])]
    bottom = np.where(np.abs(c[:, 1]) < 1e-9)[0]
    top = np.where(np.abs(c[:, 1] - 2) < 1e-9)[0]
    center = np.where((np.abs(c[:, 0] - 5) < 1e-9) & (np.abs(c[:, 1] - 1) < 1e-9))[0]
    force = np.zeros((c.shape[0], 2))
    force[:, 0] = 2.0
    return c, t, (right, left), (bottom, top), center, force


def setup_channel(S, c, walls, center, force):
    S.initial_conditions(np.zeros((c.shape[0], 2)), 1.0, force=force)
    for nodes in walls:
        S.add_velocity_dirichlet(nodes, 0, 0.0)
        S.add_velocity_dirichlet(nodes, 1, 0.0)
    S.add_pressure_dirichlet(center, 10.0)


def cavity(dim, n, seed=5):
    """Lid-driven cavity: walls at rest, lid u = 1, pressure 0 at node 0;
    a smooth random initial velocity so that every term is exercised."""
    if dim == 2:
        c, t = O.mesh_rectangle_tris(n, n, 0.15, seed)
    else:
        c, t = O.mesh_cube_tets(n, 0.15, seed)
    rng = np.random.default_rng(seed)
    N = c.shape[0]
    u0 = 0.3 * rng.standard_normal((N, dim))
    p0 = 0.1 * rng.standard_normal(N)
    nu = 0.01 * (1.0 + 0.5 * rng.random(N))
    on_wall = np.any((np.abs(c) < 1e-12) | (np.abs(c - 1) < 1e-12), axis=1)
    lid = np.abs(c[:, dim - 1] - 1) < 1e-12
    walls = np.where(on_wall & ~lid)[0]
    lid = np.where(lid)[0]
    u0[on_wall] = 0.0
    u0[lid, 0] = 1.0
    return c, t, u0, p0, nu, walls, lid


def add_cavity_bcs(S, dim, walls, lid):
    for k in range(dim):
        S.add_velocity_dirichlet(walls, k, 0.0)
    S.add_velocity_dirichlet(lid, 0, 1.0)
    for k in range(1, dim):
        S.add_velocity_dirichlet(lid, k, 0.0)
    S.add_pressure_dirichlet(np.array([0]), 0.0)


# ---------------------------------------------------------------------------
# oracle pins (CPU)
# ---------------------------------------------------------------------------
def test_oracle_laminar_channel_acceptance():
    c, t, links, walls, center, force = channel_case()
    S = O.SemiImplicit(c, t, O.options(dt=0.5, theta=0.5, alpha_su=0.0), 2, periodic_links=links)
    setup_channel(S, c, walls, center, force)
    rc, iters, worst = S.step(50)
    assert rc == 0 and worst <= 1e-12
    up, _ = S.state()
    y = c[:, 1]
    assert np.abs(up[:, 0] - y * (2 - y)).max() <= 1e-2
    assert np.abs(up[:, 1]).max() <= 1e-3
    assert np.allclose(up[links[0]], up[links[1]], rtol=0, atol=1e-12)  # slaves carry their masters' values


def test_oracle_plane_poiseuille_3d():
    """The 3D counterpart of the channel case: flow between two walls (y = 0, 2)
    driven by a body force along x, periodic in x and z (edge nodes linked twice,
    chains resolved to the final master), on tetrahedra.  The steady solution is
    u = g / (2 nu) y (H - y), v = w = 0."""
    c, t = O.mesh_cube_tets(8, 0.0, 1)
    c = c.copy()
    H, g, nu = 2.0, 2.0, 1.0
    c[:, 1] *= H
    N = c.shape[0]

    def side(k, v):
        return np.abs(c[:, k] - v) < 1e-9

    key = {tuple(np.round(p, 9)): i for i, p in enumerate(c)}
    sl, ms = [], []
    for i in np.where(side(0, 1.0))[0]:
        sl.append(i)
        ms.append(key[(0.0, round(c[i, 1], 9), round(c[i, 2], 9))])
    for i in np.where(side(2, 1.0) & ~side(0, 1.0))[0]:
        sl.append(i)
        ms.append(key[(round(c[i, 0], 9), round(c[i, 1], 9), 0.0)])
    links = (np.array(sl), np.array(ms))
    S = O.SemiImplicit(c, t, O.options(dt=0.5, theta=0.5, alpha_su=0.0), 2, periodic_links=links)
    force = np.zeros((N, 3))
    force[:, 0] = g
    S.initial_conditions(np.zeros((N, 3)), nu, force=force)
    walls = np.where(side(1, 0.0) | side(1, H))[0]
    for k in range(3):
        S.add_velocity_dirichlet(walls, k, 0.0)
    S.add_pressure_dirichlet(np.array([np.argmin(np.linalg.norm(c - [0.5, 1.0, 0.5], axis=1))]), 10.0)
    rc, _, worst = S.step(40)
    assert rc == 0 and worst <= 1e-12
    up, _ = S.state()
    y = c[:, 1]
    assert np.abs(up[:, 0] - g / (2 * nu) * y * (H - y)).max() <= 1e-3
    assert np.abs(up[:, 1:3]).max() <= 1e-12


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_lumped_mass_closed_form(dim):
    c, t, u0, p0, nu, walls, lid = cavity(dim, 5 if dim == 2 else 3)
    S = O.SemiImplicit(c, t, O.options(dt=0.01), 2)
    S.initial_conditions(u0, nu, p0)
    m = np.zeros(c.shape[0])
    for e in t:
        X = c[e]
        vol = abs(np.linalg.det((X[1:] - X[0]).T)) / (2.0 if dim == 2 else 6.0)
        m[e] += vol / (dim + 1)
    minv = S.lumped_inverse()
    assert np.allclose(minv, (1.0 / m)[:, None], rtol=1e-13, atol=0)


def _dense(rowptr, colidx, vals, n):
    A = np.zeros((n, n))
    for r in range(n):
        A[r, colidx[rowptr[r]:rowptr[r + 1]]] = vals[rowptr[r]:rowptr[r + 1]]
    return A


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_systems_symmetric_and_laplacian(dim):
    c, t, u0, p0, nu, walls, lid = cavity(dim, 4 if dim == 2 else 2)
    S = O.SemiImplicit(c, t, O.options(dt=0.02, theta=0.5), 2)
    S.initial_conditions(u0, nu, p0)
    # the graph is the coupled system's node graph; build the point CSRs here
    G = O.Oracle(c, t, O.options(dt=0.02))
    start, adj = G.graph()
    def csr(neq):
        rp = [0]
        ci = []
        for i in range(len(start) - 1):
            for r in range(neq):
                for k in range(start[i], start[i + 1]):
                    ci.extend(adj[k] * neq + np.arange(neq))
                rp.append(len(ci))
        return np.array(rp), np.array(ci)
    N = c.shape[0]
    Pv, _, _ = S.system("pressure")
    rp, ci = csr(1)
    Ap = _dense(rp, ci, Pv, N)
    assert np.allclose(Ap, Ap.T, rtol=0, atol=1e-14 * np.abs(Ap).max())
    assert np.abs(Ap.sum(axis=1)).max() <= 1e-13 * np.abs(Ap).max()
    Uv = S.velocity_matrix()
    rp, ci = csr(dim)
    Au = _dense(rp, ci, Uv, N * dim)
    assert np.allclose(Au, Au.T, rtol=0, atol=1e-14 * np.abs(Au).max())
    assert np.all(np.linalg.eigvalsh(Au) > 0)


# ---------------------------------------------------------------------------
# GPU parity
# ---------------------------------------------------------------------------
def _pair(c, t, dim, supg="metric", theta=0.5, dt=0.02, nb_iterations=2, links=None, alpha_su=1.0):
    G = NavierStokesSemiImplicit(c, t, dt=dt, theta=theta, nb_iterations=nb_iterations, supg_type=supg,
                                 alpha_su=alpha_su, periodic_links=links)
    S = O.SemiImplicit(c, t, O.options(dt=dt, theta=theta, supg_type=TAU[supg], alpha_su=alpha_su), nb_iterations,
                       periodic_links=links)
    return G, S


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("supg", ["metric", "tezduyar", "cf2"])
def test_matrices_match_oracle(dim, supg):
    c, t, u0, p0, nu, walls, lid = cavity(dim, 9 if dim == 2 else 4)
    G, S = _pair(c, t, dim, supg)
    with G:
        for X in (G, S):
            X.initial_conditions(u0, nu, p0)
        rp, ci, pv, _, _ = G.system("pressure")
        opv, _, _ = S.system("pressure")
        assert row_scaled_error(pv, opv, rp) <= 1e-12
        assert np.allclose(G.lumped_inverse(), S.lumped_inverse(), rtol=1e-13, atol=0)
        # velocity matrix on a non-trivial linearised velocity
        rng = np.random.default_rng(11)
        up = np.zeros((c.shape[0], dim + 1))
        up[:, :dim], up[:, dim] = u0, p0
        lin = np.tile(u0, (1, 4)) + 0.05 * rng.standard_normal((c.shape[0], 4 * dim))
        for X in (G, S):
            X.set_state(up, lin, nu)
        G.assemble_velocity_matrix()
        rp, ci, uv, _, _ = G.system("velocity")
        ouv = S.velocity_matrix()
        assert row_scaled_error(uv, ouv, rp) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("dim,supg,theta,iters", [(2, "metric", 0.5, 2), (2, "tezduyar", 1.0, 3),
                                                   (3, "metric", 0.5, 2), (3, "cf2", 0.7, 1)])
def test_cavity_steps_match_oracle(dim, supg, theta, iters):
    c, t, u0, p0, nu, walls, lid = cavity(dim, 8 if dim == 2 else 4)
    G, S = _pair(c, t, dim, supg, theta=theta, nb_iterations=iters)
    with G:
        G.set_krylov(velocity=dict(tol=1e-12, max_iters=5000), pressure=dict(tol=1e-12, max_iters=5000))
        for X in (G, S):
            X.initial_conditions(u0, nu, p0)
            add_cavity_bcs(X, dim, walls, lid)
        sv, sp = G.step(3)
        assert sv["converged"] and sp["converged"], (sv, sp)
        rc, _, _ = S.step(3)
        assert rc == 0
        gu, gl = G.state
        ou, ol = S.state()
        scale = np.abs(ou).max()
        assert np.abs(gu - ou).max() <= 1e-8 * scale
        assert np.abs(gl - ol).max() <= 1e-8 * np.abs(ol).max()
        assert abs(G.time - 3 * 0.02) < 1e-15


@pytest.mark.gpu
def test_laminar_channel_acceptance_gpu():
    c, t, links, walls, center, force = channel_case()
    G, S = _pair(c, t, 2, "metric", theta=0.5, dt=0.5, nb_iterations=2, links=links, alpha_su=0.0)
    with G:
        # the pressure increments shrink to rounding level as the flow settles:
        # 1e-10 of their norm is the attainable Jacobi-CG accuracy there
        G.set_krylov(velocity=dict(tol=1e-12, max_iters=10000), pressure=dict(tol=1e-10, max_iters=20000))
        for X in (G, S):
            setup_channel(X, c, walls, center, force)
        sv, sp = G.step(50)
        assert sv["converged"] and sp["converged"], (sv, sp)
        S.step(50)
        gu, _ = G.state
        ou, _ = S.state()
        y = c[:, 1]
        assert np.abs(gu[:, 0] - y * (2 - y)).max() <= 1e-2
        assert np.abs(gu[:, 1]).max() <= 1e-3
        assert np.abs(gu - ou).max() <= 1e-7 * np.abs(ou).max()
        assert np.array_equal(gu[links[0]], gu[links[1]])


@pytest.mark.gpu
def test_deterministic_and_errors():
    c, t, u0, p0, nu, walls, lid = cavity(3, 3)
    out = []
    for _ in range(2):
        with NavierStokesSemiImplicit(c, t, dt=0.02, theta=0.5) as G:
            G.initial_conditions(u0, nu, p0)
            add_cavity_bcs(G, 3, walls, lid)
            G.step(2)
            out.append(G.state[0])
    assert np.array_equal(out[0], out[1])
    with NavierStokesSemiImplicit(c, t, dt=0.02) as G:
        with pytest.raises(UfemError):
            G.step(1)  # before the initial conditions
        with pytest.raises(UfemError):
            G.add_velocity_dirichlet(np.array([0]), 3, 0.0)  # component out of range
        assert G.device_bytes() > 0
    with pytest.raises(UfemError):
        NavierStokesSemiImplicit(c, t, dt=0.02, nb_iterations=0)


def _fn_bcs(c, t):
    """Time-dependent conditions of a unit-square flow: lid u = sin(pi x) (1 + t),
    walls at rest, pressure 0.1 t at node 0 (as numpy evaluates the formulas)."""
    return (np.sin(np.pi * c[:, 0]) * (1.0 + t), 0.1 * t)


@pytest.mark.gpu
def test_function_bcs_match_oracle():
    c, tri, u0, p0, nu, walls, lid = cavity(2, 8)
    dt = 0.02
    G, S = _pair(c, tri, 2, "metric", theta=0.5, dt=dt)
    with G:
        G.set_krylov(velocity=dict(tol=1e-12, max_iters=5000), pressure=dict(tol=1e-12, max_iters=5000))
        u0 = u0.copy()
        u0[lid, 0] = np.sin(np.pi * c[lid, 0])
        for X in (G, S):
            X.initial_conditions(u0, nu, p0)
        for k in range(2):
            G.add_velocity_dirichlet(walls, k, 0.0)
        G.add_velocity_dirichlet_function(lid, 0, "sin(pi*x) * (1 + t)")
        G.add_velocity_dirichlet(lid, 1, 0.0)
        G.add_pressure_dirichlet_function(np.array([0]), "0.1 * t")
        for step in range(3):
            tk = step * dt
            ulid, p_pin = _fn_bcs(c[lid], tk)
            S.clear_dirichlet()
            for k in range(2):
                S.add_velocity_dirichlet(walls, k, 0.0)
            S.add_velocity_dirichlet(lid, 0, ulid)
            S.add_velocity_dirichlet(lid, 1, 0.0)
            S.add_pressure_dirichlet(np.array([0]), p_pin)
            S.step(1)
        sv, sp = G.step(3)
        assert sv["converged"] and sp["converged"]
        gu, _ = G.state
        ou, _ = S.state()
        assert np.abs(gu - ou).max() <= 1e-8 * np.abs(ou).max()
        # constrained values come out of the solves (identity rows), to solver accuracy
        assert abs(gu[lid, 0] - np.sin(np.pi * c[lid, 0]) * (1 + 2 * dt)).max() <= 1e-10
        assert abs(gu[0, 2] - 0.1 * 2 * dt) <= 1e-10


@pytest.mark.gpu
def test_restart_continuation(tmp_path):
    """atest-ufem-navier-stokes-restart.py for the semi-implicit solver: six
    steps in one run against three + restart + three.  As in the reference, the
    restarted run rebuilds the pressure matrix from the restarted velocity, so
    the runs agree to solver accuracy, not bitwise (the reference allows 1e9 ulps);
    the restarted run matches the oracle restarted the same way within 1e-8."""
    c, tri, u0, p0, nu, walls, lid = cavity(2, 8)
    kw = dict(velocity=dict(tol=1e-12, max_iters=5000), pressure=dict(tol=1e-12, max_iters=5000))
    path = str(tmp_path / "si.cf3restart")
    with NavierStokesSemiImplicit(c, tri, dt=0.01, theta=0.5) as A:
        A.set_krylov(**kw)
        A.initial_conditions(u0, nu, p0)
        add_cavity_bcs(A, 2, walls, lid)
        A.step(3)
        A.write_restart(path, iteration=3)
        mid_up, mid_lin = A.state
        A.step(3)
        full = A.state[0]
    with NavierStokesSemiImplicit(c, tri, dt=0.01, theta=0.5) as B:
        B.set_krylov(**kw)
        add_cavity_bcs(B, 2, walls, lid)
        t, dt, it = B.read_restart(path)
        assert (it, dt) == (3, 0.01) and abs(t - 0.03) < 1e-15 and abs(B.time - 0.03) < 1e-15
        up, lin = B.state
        assert np.array_equal(up, mid_up) and np.array_equal(lin, mid_lin)
        B.step(3)
        restarted = B.state[0]
    assert np.abs(restarted - full).max() <= 1e-5 * np.abs(full).max()
    S = O.SemiImplicit(c, tri, O.options(dt=0.01, theta=0.5), 2)
    S.set_state(mid_up, mid_lin, np.ascontiguousarray(nu))
    S.initialize(reset_history=False)
    add_cavity_bcs(S, 2, walls, lid)
    S.step(3)
    ou, _ = S.state()
    assert np.abs(restarted - ou).max() <= 1e-8 * np.abs(ou).max()


@pytest.mark.gpu
def test_two_level_pressure_preconditioner():
    """The two-level pressure preconditioner (point Jacobi + Galerkin coarse
    correction on geometric aggregates) gives the point-Jacobi answer to solver
    accuracy with a fraction of the iterations; a pressure system without any
    condition (singular coarse matrix) falls back to point Jacobi and still runs."""
    c, t, u0, p0, nu, walls, lid = cavity(3, 12)
    out = {}
    for pre in ("jacobi", "two_level"):
        with NavierStokesSemiImplicit(c, t, dt=0.01, theta=0.5) as G:
            G.set_krylov(velocity=dict(tol=1e-12, max_iters=5000),
                         pressure=dict(tol=1e-12, max_iters=20000, precond=pre))
            G.initial_conditions(u0, nu, p0)
            add_cavity_bcs(G, 3, walls, lid)
            sv, sp = G.step(2)
            assert sv["converged"] and sp["converged"]
            out[pre] = (G.state[0], sp["iterations"])
    (uj, ij), (ut, it) = out["jacobi"], out["two_level"]
    assert np.abs(ut - uj).max() <= 1e-8 * np.abs(uj).max()
    assert it < 0.6 * ij, (it, ij)  # 27 aggregates on this small mesh; larger meshes gain more
    with NavierStokesSemiImplicit(c, t, dt=0.01, theta=0.5) as G:  # no pressure condition
        G.initial_conditions(u0, nu, p0)
        for k in range(3):
            G.add_velocity_dirichlet(walls, k, 0.0)
        G.step(1)
