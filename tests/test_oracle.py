"""CPU tests that pin the FP64 oracle (no GPU needed).

The reference holds no numeric golden vectors for NS element matrices, so the
oracle is pinned by (a) the reference's own known-answer tests for this path
(symmetric Dirichlet, sparsity structure), (b) closed-form P1 integrals that
the order-2 quadrature must reproduce exactly, (c) structural identities of the
PSPG/SUPG operator, and (d) committed regression fixtures.
"""
import math

import numpy as np
import pytest

import oracle as O
from coolfluid3_b200 import problems as P

from .util import csr_matrix, oracle_for, small_problem


# ---------------------------------------------------------------------------
# structure
# ---------------------------------------------------------------------------
def test_mesh_generators_match_bitwise():
    for nx in (3, 8, 64):
        a = P.rectangle_tris(nx, nx, 0.2, 7)
        b = O.mesh_rectangle_tris(nx, nx, 0.2, 7)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for n in (2, 5, 16):
        a = P.cube_tets(n, 0.15, 11)
        b = O.mesh_cube_tets(n, 0.15, 11)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_generated_elements_positive_and_jitter_bounded():
    c, e = P.cube_tets(6, 0.15, 3)
    X = c[e.astype(np.int64)]
    det = np.linalg.det(X[:, 1:, :] - X[:, :1, :])
    assert (det > 0).all()
    np.testing.assert_allclose(np.abs(det).sum() / 6.0, 1.0, rtol=1e-12)  # volumes tile the cube
    h = 1.0 / 6
    lattice = np.stack(P.structured_index(3, 6), axis=1) * h
    assert np.abs(c - lattice).max() <= 0.15 * h + 1e-15
    c2, e2 = P.rectangle_tris(9, 9, 0.2, 3)
    X = c2[e2.astype(np.int64)]
    det = np.linalg.det(X[:, 1:, :] - X[:, :1, :])
    assert (det > 0).all()
    np.testing.assert_allclose(det.sum() / 2.0, 1.0, rtol=1e-12)


def test_sparsity_sizes_of_the_configs():
    # cfg1: 64x64x2 triangles; small and mid-size tetrahedral cubes
    c, e = P.rectangle_tris(64)
    o = O.Oracle(c, e, O.options())
    assert (o.N, o.E, o.block_nnz, o.nnz) == (4225, 8192, 29057, 261513)
    c, e = P.cube_tets(16)
    o = O.Oracle(c, e, O.options())
    assert (o.N, o.E, o.block_nnz, o.nnz) == (4913, 24576, 66961, 1071376)


def test_sparsity_rows_structured_triangles():
    """Node graph of create_rectangle_tris (SparsityBuilder.cpp:157-189): an
    interior node touches 6 triangles and 7 nodes (self included); the corner
    with both diagonals' ends has 4, the other two corners 3."""
    n = 5
    c, e = P.rectangle_tris(n, n, 0.0, 1)
    o = O.Oracle(c, e, O.options())
    start, adj = o.graph()
    deg = np.diff(start)
    i, j = P.structured_index(2, n)
    interior = (i > 0) & (i < n) & (j > 0) & (j < n)
    assert (deg[interior] == 7).all()
    corner = lambda a, b: int(np.nonzero((i == a) & (j == b))[0][0])
    assert deg[corner(0, 0)] == 4 and deg[corner(n, n)] == 4
    assert deg[corner(n, 0)] == 3 and deg[corner(0, n)] == 3
    # each neighbourhood is sorted, unique and holds the node itself
    for k in range(o.N):
        nb = adj[start[k]:start[k + 1]]
        assert (np.diff(nb.astype(np.int64)) > 0).all() and k in nb


def test_point_csr_expansion():
    """Row node*neq+eq holds adj(node)*neq + c in ascending order (FEVbr point form)."""
    pb = small_problem(3, 3)
    o = oracle_for(pb)
    rp, ci = o.csr()
    st, adj = o.graph()
    neq = 4
    for node in (0, 7, o.N - 1):
        for r in range(neq):
            cols = ci[rp[node * neq + r]:rp[node * neq + r + 1]]
            exp = (adj[st[node]:st[node + 1]].astype(np.int64)[:, None] * neq + np.arange(neq)).ravel()
            assert np.array_equal(cols, exp)


# ---------------------------------------------------------------------------
# symmetric Dirichlet: test/math/utest-lss-symmetric-dirichlet.cpp:146-210
# ---------------------------------------------------------------------------
def test_symmetric_dirichlet_reference_kat():
    """4-node chain, neq = 1, rows set to (diag 2, off-diagonal 1) by set_row,
    symmetric_dirichlet(node 1, eq 0, 10).  The reference checks, over its two
    ranks: A(1,1) = 1, column and row 1 zero elsewhere, A(0,0) = A(2,2) = 2,
    A(2,3) = A(3,2) = 1, rhs = (-10, 10, -10, 0)."""
    start = np.array([0, 2, 5, 8, 10])
    adj = np.array([0, 1, 0, 1, 2, 1, 2, 3, 2, 3], np.uint32)
    s = O.LSS(start, adj, 1)
    for r in range(4):
        s.set_row(r, 0, 2.0, 1.0)
    s.symmetric_dirichlet(1, 0, 10.0)
    A = s.dense()
    _, rhs = s.system()
    expect = np.array([[2, 0, 0, 0], [0, 1, 0, 0], [0, 0, 2, 1], [0, 0, 1, 2]], float)
    assert np.array_equal(A, expect)
    assert np.array_equal(rhs, [-10.0, 10.0, -10.0, 0.0])
    assert s.solution()[1] == 10.0


def test_symmetric_dirichlet_golden_fixture():
    """The same known-answer test, every check taken from the committed
    fixture that tests/golden/make_golden.py extracted from the reference's
    test source (global node ids, the reference's get_value column-first order
    already resolved)."""
    import json
    import os
    kat = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "lss_symmetric_dirichlet_kat.json")))
    n = kat["nodes"]
    start = [0]
    adj = []
    for i in range(n):
        nb = [j for j in (i - 1, i, i + 1) if 0 <= j < n]
        adj += nb
        start.append(len(adj))
    s = O.LSS(np.array(start), np.array(adj, np.uint32), kat["neq"])
    for r in range(n):
        s.set_row(r, 0, kat["set_row"]["diag"], kat["set_row"]["offdiag"])
    d = kat["dirichlet"]
    s.symmetric_dirichlet(d["node"], d["eq"], d["value"])
    A = s.dense()
    _, rhs = s.system()
    assert len(kat["matrix_checks"]) == 10 and len(kat["rhs_checks"]) == 5
    for c in kat["matrix_checks"]:
        assert A[c["row"], c["col"]] == c["value"], c
    for c in kat["rhs_checks"]:
        assert rhs[c["row"]] == c["value"], c


def _parallel_dirichlet(rowptr, colidx, vals, rhs, sol, state_flat, nodes, comps, values, neq):
    """The order-preserving parallel form the GPU applies (see csrc/host.cu)."""
    dof = nodes.astype(np.int64) * neq + comps
    first, last, order = {}, {}, []
    for d, v in zip(dof, values):
        if d not in first:
            first[d] = v
            order.append(d)
        last[d] = v
    rank = {d: k for k, d in enumerate(order)}
    vals, rhs, sol = vals.copy(), rhs.copy(), sol.copy()
    for r in range(len(rowptr) - 1):
        if r in rank:
            continue
        ents = [(rank[c], p) for p in range(rowptr[r], rowptr[r + 1]) for c in [int(colidx[p])] if c in rank]
        for k, p in sorted(ents):
            c = order[k]
            rhs[r] = rhs[r] + (-vals[p]) * (first[c] - state_flat[c])
            vals[p] = 0.0
    for d in order:
        vals[rowptr[d]:rowptr[d + 1]] = 0.0
        p = rowptr[d] + np.nonzero(colidx[rowptr[d]:rowptr[d + 1]] == d)[0][0]
        vals[p] = 1.0
        rhs[d] = sol[d] = last[d] - state_flat[d]
    return vals, rhs, sol


@pytest.mark.parametrize("dim,n", [(2, 4), (3, 2)])
def test_dirichlet_parallel_form_equals_sequential(dim, n):
    """The sequential reference semantics (duplicated corner dofs, last value
    wins for the row, first value moves the column) equal the parallel plan."""
    pb = small_problem(dim, n)
    o = oracle_for(pb, use_specializations=False)
    o.assemble()
    rp, ci = o.csr()
    vals, rhs = o.system()
    sol0 = np.random.default_rng(1).normal(size=o.nrows)
    o.set_solution(sol0)
    state_flat = pb.up.ravel()
    ev, er, es = _parallel_dirichlet(rp, ci, vals, rhs, sol0, state_flat, pb.bc_nodes, pb.bc_comps, pb.bc_values,
                                     dim + 1)
    o.apply_dirichlet()
    gv, gr = o.system()
    assert np.array_equal(gv, ev)
    assert np.array_equal(gr, er)
    assert np.array_equal(o.solution(), es)


# ---------------------------------------------------------------------------
# stabilisation coefficients (SUPG.hpp:140-219)
# ---------------------------------------------------------------------------
def test_tau_metric_unit_triangle():
    X = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]])
    u = np.array([0.3, -0.4])
    nu, dt = 0.01, 0.05
    tps, tsu, tbu = O.tau(2, 1, X, u, nu, dt)
    adv, diff = 0.25, nu * nu * 2.0  # J = I -> g = I: u.g.u = |u|^2, ||g||_F^2 = 2
    assert tsu == pytest.approx(1.0 / math.sqrt(4 / dt ** 2 + adv + 16 * diff), rel=1e-15)
    assert tps == tsu
    assert tbu == pytest.approx(math.sqrt(4 / dt ** 2 + adv + 16 * diff) / 2.0, rel=1e-15)


def test_tau_metric_scaled_tet():
    h = 0.1
    X = np.array([[0, 0, 0], [h, 0, 0], [0, h, 0], [0, 0, h]], float)
    u = np.array([1.0, 2.0, -0.5])
    nu, dt = 1e-3, 5e-3
    tps, tsu, tbu = O.tau(3, 1, X, u, nu, dt, c1=2.0, c2=9.0)
    g = 1 / h ** 2
    adv = g * (u @ u)
    diff = nu * nu * 3 * g * g
    assert tsu == pytest.approx(1 / math.sqrt(4 * 4 / dt ** 2 + adv + 9 * diff), rel=1e-14)
    assert tbu == pytest.approx(math.sqrt(4 / dt ** 2 + adv + 16 * diff) / (3 * g), rel=1e-14)


def test_tau_tezduyar_and_cf2():
    X = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]])
    u = np.array([0.6, 0.8])
    nu, dt = 0.1, 0.01
    tps, tsu, tbu = O.tau(2, 0, X, u, nu, dt)
    exp = 1.0 / (2 * 1.0 / 1.0 + 2 / dt + 4 * nu / 1.0)
    assert tsu == pytest.approx(exp, rel=1e-15) and tps == tsu and tbu == pytest.approx(exp, rel=1e-15)
    tps, tsu, tbu = O.tau(2, 2, X, u, nu, dt)
    he = math.sqrt(4 / 3.141592654 * 0.5)
    ree = he / (2 * nu)
    xi = ree / 3 if ree < 3 else 1.0
    assert tps == pytest.approx(he * xi / 2, rel=1e-14)
    assert tbu == pytest.approx(he / xi, rel=1e-14)
    assert tsu == pytest.approx(dt / 2, rel=1e-9)  # P1: sum_b u.grad N_b is rounding-level


# ---------------------------------------------------------------------------
# element matrices against closed-form P1 integrals
# ---------------------------------------------------------------------------
def _geometry(X):
    d = X.shape[1]
    J = X[1:] - X[0]
    dN = np.hstack([-np.ones((d, 1)), np.eye(d)])
    G = np.linalg.inv(J) @ dN
    V = abs(np.linalg.det(J)) / math.factorial(d)
    return G, V, np.linalg.inv(J)


@pytest.mark.parametrize("dim", [2, 3])
def test_generic_element_closed_form_at_rest(dim):
    """u = u_adv = 0, constant nu: the order-2 quadrature must equal the exact P1
    integrals (mass V(1+d_ab)/((d+1)(d+2)), continuity V/(d+1) G, PSPG
    tau_ps V G.G/rho, viscous nu V G.G, bulk tau_bu V G G)."""
    pb = small_problem(dim, 3)
    pb.up[:] = 0
    pb.lin[:] = 0
    nu, dt, rho = 0.02, 0.01, 1.3
    pb.nu[:] = nu
    o = O.Oracle(pb.coords, pb.conn, O.options(dt=dt, rho=rho, use_specializations=False))
    o.set_state(pb.up, pb.lin, pb.nu)
    n = dim + 1
    for e in (0, 5, pb.nb_elems - 1):
        A, T, a = o.element(e)
        X = pb.coords[pb.conn[e].astype(np.int64)]
        G, V, Ji = _geometry(X)
        g = Ji.T @ Ji
        tps = 1 / math.sqrt(4 / dt ** 2 + 16 * nu * nu * (g * g).sum())
        tbu = math.sqrt(4 / dt ** 2 + 16 * nu * nu * (g * g).sum()) / np.trace(g)
        D = G.T @ G
        M = V * (np.ones((n, n)) + np.eye(n)) / ((dim + 1) * (dim + 2))
        pofs = dim * n
        for i in range(dim):
            ui = slice(i * n, (i + 1) * n)
            np.testing.assert_allclose(T[ui, ui], M, rtol=1e-13, atol=1e-17)
            np.testing.assert_allclose(A[pofs:, ui], V / (dim + 1) * np.tile(G[i], (n, 1)), rtol=1e-12, atol=1e-15)
            np.testing.assert_allclose(T[pofs:, ui], tps * V / (dim + 1) * np.outer(G[i], np.ones(n)),
                                       rtol=1e-12, atol=1e-18)
            np.testing.assert_allclose(A[ui, pofs:], V / (dim + 1) / rho * np.tile(G[i], (n, 1)),
                                       rtol=1e-12, atol=1e-15)
            for j in range(dim):
                uj = slice(j * n, (j + 1) * n)
                exp = tbu * V * np.outer(G[i], G[j]) + (nu * V * D if i == j else 0.0)
                np.testing.assert_allclose(A[ui, uj], exp, rtol=1e-11, atol=1e-13 * np.abs(exp).max())
        np.testing.assert_allclose(A[pofs:, pofs:], tps * V * D / rho, rtol=1e-12, atol=1e-18)
        assert np.all(a == 0)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("spec", [False, True])
def test_element_operator_annihilates_constants(dim, spec):
    """Every A term multiplies a shape-function gradient of the column node, and
    sum_b grad N_b = 0: A applied to a constant (u, p) field vanishes."""
    pb = small_problem(dim, 3)
    o = O.Oracle(pb.coords, pb.conn, O.options(dt=pb.dt, use_specializations=spec, supg_type=1))
    o.set_state(pb.up, pb.lin, pb.nu)
    for e in range(0, pb.nb_elems, 7):
        A, T, _ = o.element(e)
        assert np.abs(A @ np.ones(A.shape[0])).max() <= 1e-11 * np.abs(A).max()


@pytest.mark.parametrize("dim", [2, 3])
def test_specialized_equals_generic_on_shared_terms(dim):
    """With u = u_adv = 0 the closed-form specialised kernels and the generic
    quadrature agree on every term they share (mass, PSPG, continuity, pressure
    gradient); only the viscous/bulk velocity blocks differ by design (4/3 stress
    form, NavierStokesSpecializations.hpp:106-111)."""
    pb = small_problem(dim, 3)
    pb.up[:] = 0
    pb.lin[:] = 0
    n = dim + 1
    pofs = dim * n
    og = O.Oracle(pb.coords, pb.conn, O.options(dt=pb.dt, use_specializations=False))
    os_ = O.Oracle(pb.coords, pb.conn, O.options(dt=pb.dt, use_specializations=True))
    og.set_state(pb.up, pb.lin, pb.nu)
    os_.set_state(pb.up, pb.lin, pb.nu)
    for e in (0, 3, pb.nb_elems - 1):
        Ag, Tg, _ = og.element(e)
        As, Ts, _ = os_.element(e)
        np.testing.assert_allclose(Ts, Tg, rtol=1e-12, atol=1e-14 * np.abs(Tg).max())
        np.testing.assert_allclose(As[pofs:, :], Ag[pofs:, :], rtol=1e-12, atol=1e-12 * np.abs(Ag[pofs:]).max())
        np.testing.assert_allclose(As[:pofs, pofs:], Ag[:pofs, pofs:], rtol=1e-12,
                                   atol=1e-12 * np.abs(Ag[:pofs, pofs:]).max())


def test_body_force_vector():
    """_a[u_i] = int S_a g_i: with u_adv = 0 and a constant force f, a = V/(d+1) f."""
    pb = small_problem(2, 3)
    pb.lin[:] = 0
    f = np.tile([0.7, -1.1], (pb.nb_nodes, 1))
    o = O.Oracle(pb.coords, pb.conn, O.options(dt=pb.dt, use_specializations=False))
    o.set_state(pb.up, pb.lin, pb.nu, f)
    _, _, a = o.element(4)
    X = pb.coords[pb.conn[4].astype(np.int64)]
    _, V, _ = _geometry(X)
    np.testing.assert_allclose(a[:3], V / 3 * 0.7, rtol=1e-13)
    np.testing.assert_allclose(a[3:6], V / 3 * -1.1, rtol=1e-13)
    assert np.all(a[6:] == 0)


# ---------------------------------------------------------------------------
# assembly, solve, time stepping
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("dim,n", [(2, 16), (3, 4)])
def test_multithreaded_assembly_is_bitwise_serial(dim, n):
    pb = small_problem(dim, n)
    o1 = oracle_for(pb, use_specializations=False)
    o4 = oracle_for(pb, use_specializations=False)
    o1.assemble(1)
    o4.assemble(4)
    v1, r1 = o1.system()
    v4, r4 = o4.system()
    assert np.array_equal(v1, v4) and np.array_equal(r1, r4)


def test_oracle_solve_residual():
    pb = small_problem(2, 12)
    o = oracle_for(pb, use_specializations=False)
    o.assemble()
    o.apply_dirichlet()
    st = o.solve(tol=1e-13)
    assert st["rc"] == 0
    rp, ci = o.csr()
    vals, rhs = o.system()
    A = csr_matrix(rp, ci, vals, o.nrows)
    x = o.solution()
    assert np.linalg.norm(rhs - A @ x) <= 1e-12 * np.linalg.norm(rhs)


def test_update_shifts_history():
    pb = small_problem(2, 4)
    o = oracle_for(pb)
    s = np.random.default_rng(0).normal(size=o.nrows)
    o.set_solution(s)
    up0, lin0 = o.state()
    o.update()
    up1, lin1 = o.state()
    d = 2
    np.testing.assert_array_equal(lin1[:, d:2 * d], up0[:, :d])          # u1 = u
    np.testing.assert_array_equal(lin1[:, 2 * d:3 * d], lin0[:, d:2 * d])  # u2 = u1
    np.testing.assert_array_equal(lin1[:, 3 * d:], lin0[:, 2 * d:3 * d])   # u3 = u2
    np.testing.assert_array_equal(up1, up0 + s.reshape(up0.shape))


def test_linearize_first_step_is_u():
    """With u1 = u2 = u3 = u the extrapolation 2.1875u - 2.1875u1 + 1.3125u2 -
    0.3125u3 returns u up to rounding (NavierStokes.cpp:105, ICs :201-204)."""
    pb = small_problem(3, 2)
    o = oracle_for(pb)
    o.assemble()
    _, lin = o.state()
    np.testing.assert_allclose(lin[:, :3], pb.up[:, :3], rtol=0, atol=4e-16)


def test_oracle_problem_builder_matches_product_generator():
    # the reference arm of the benchmark builds its inputs without the product library
    for dim, n in ((2, 8), (3, 4)):
        a = P.make_problem(dim, n, nu=1e-3, dt=5e-3)
        b = O.lid_driven_problem(dim, n, 1e-3, 5e-3)
        for k in ("coords", "conn", "up", "lin", "nu", "bc_nodes", "bc_comps", "bc_values"):
            x, y = getattr(a, k), b[k]
            assert x.dtype == y.dtype and np.array_equal(x, y), k
