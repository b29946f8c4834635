"""GPU parity tests: the sm_100a path through the C ABI against the FP64 oracle.

Tolerances (stated per test): CSR pattern bit-exact; FP64 assembly within
1e-11 of each CSR row's largest |entry| (the two sides evaluate the same
formulas in a different operation order); FP32 element arithmetic within
2e-5 of the row scale; solutions within the Krylov tolerance times a
conditioning margin.
"""
import numpy as np
import pytest

import oracle as O
from coolfluid3_b200 import NavierStokes, UfemError
from coolfluid3_b200 import problems as P

from .util import csr_matrix, oracle_for, row_scaled_error, small_problem, vec_rel_error

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-11
FP32_TOL = 2e-5


def gpu_for(pb, **kw):
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, density=pb.rho, theta=pb.theta, **kw)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    return ns


SUPG = {"tezduyar": 0, "metric": 1, "cf2": 2}


@pytest.mark.parametrize("dim,n", [(2, 4), (2, 64), (3, 2), (3, 8)])
def test_csr_pattern_bitexact(dim, n):
    pb = small_problem(dim, n)
    ns = gpu_for(pb)
    o = oracle_for(pb)
    rp, ci = ns.csr()
    orp, oci = o.csr()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    st, adj = ns.graph()
    ost, oadj = o.graph()
    assert np.array_equal(st, ost) and np.array_equal(adj, oadj)


@pytest.mark.parametrize("dim,n", [(2, 6), (3, 3)])
@pytest.mark.parametrize("spec", [False, True])
@pytest.mark.parametrize("supg", ["metric", "tezduyar", "cf2"])
def test_assembly_fp64_matches_oracle(dim, n, spec, supg):
    if spec and supg != "metric":
        pytest.skip("the specialised kernels always use the default metric tau")
    pb = small_problem(dim, n)
    ns = gpu_for(pb, use_specializations=spec, supg_type=supg)
    o = oracle_for(pb, use_specializations=spec, supg_type=SUPG[supg])
    ns.assemble()
    o.assemble()
    gv, gr = ns.system()
    ov, orr = o.system()
    rp, _ = o.csr()
    assert row_scaled_error(gv, ov, rp) <= FP64_TOL
    assert vec_rel_error(gr, orr) <= 1e-11


@pytest.mark.parametrize("dim,n", [(2, 8), (3, 3)])
def test_assembly_with_body_force_and_theta(dim, n):
    pb = small_problem(dim, n)
    pb.theta = 0.5
    f = np.random.default_rng(5).normal(size=(pb.nb_nodes, dim))
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, theta=0.5, use_specializations=False)
    ns.set_state(pb.up, pb.lin, pb.nu, f)
    o = O.Oracle(pb.coords, pb.conn, O.options(dt=pb.dt, theta=0.5, use_specializations=False))
    o.set_state(pb.up, pb.lin, pb.nu, f)
    ns.assemble()
    o.assemble()
    gv, gr = ns.system()
    ov, orr = o.system()
    rp, _ = o.csr()
    assert row_scaled_error(gv, ov, rp) <= FP64_TOL
    assert vec_rel_error(gr, orr) <= 1e-11


@pytest.mark.parametrize("dim,n", [(2, 16), (3, 6)])
@pytest.mark.parametrize("spec", [False, True])
def test_assembly_fp32_elements_error_bound(dim, n, spec):
    """FP32 element arithmetic + FP64 scatter: error against the FP64 oracle."""
    pb = small_problem(dim, n)
    ns = gpu_for(pb, use_specializations=spec, precision="fp32")
    o = oracle_for(pb, use_specializations=spec)
    ns.assemble()
    o.assemble()
    gv, gr = ns.system()
    ov, orr = o.system()
    rp, _ = o.csr()
    err = row_scaled_error(gv, ov, rp)
    assert err <= FP32_TOL, err
    assert vec_rel_error(gr, orr) <= 1e-4


def test_assembly_is_deterministic():
    pb = small_problem(3, 6)
    ns = gpu_for(pb, use_specializations=False)
    ns.assemble()
    v1, r1 = ns.system()
    ns.assemble()
    v2, r2 = ns.system()
    assert np.array_equal(v1, v2) and np.array_equal(r1, r2)


@pytest.mark.parametrize("dim,n", [(2, 6), (3, 3)])
def test_dirichlet_matches_oracle(dim, n):
    pb = small_problem(dim, n)
    ns = gpu_for(pb, use_specializations=False)
    o = oracle_for(pb, use_specializations=False)
    ns.assemble()
    o.assemble()
    # identical pre-BC systems: start the oracle from the GPU's assembled system
    gv, gr = ns.system()
    o.set_system(gv, gr)
    ns.apply_dirichlet()
    o.apply_dirichlet()
    gv2, gr2 = ns.system()
    ov2, or2 = o.system()
    assert np.array_equal(gv2, ov2)
    assert np.array_equal(gr2, or2)
    assert np.array_equal(ns.solution(), o.solution())


def test_apply_matches_scipy():
    pb = small_problem(3, 4)
    ns = gpu_for(pb)
    ns.assemble()
    rp, ci = ns.csr()
    v, _ = ns.system()
    x = np.random.default_rng(2).normal(size=ns.nb_rows)
    y = ns.apply(x)
    ref = csr_matrix(rp, ci, v, ns.nb_rows) @ x
    assert vec_rel_error(y, ref) <= 1e-13


@pytest.mark.parametrize("case", ["cube20", "fan30"])
def test_apply_matches_scipy_on_long_walks_and_wide_rows(case):
    """The coupled SpMV runs persistent warps that walk several nodes each,
    with the next node's loads in flight: a 20^3 x 6 mesh (9,261 nodes, more
    than the resident warps) takes every warp through that walk; a fan of 60
    tetrahedra around one node gives a row of 33 neighbours, whose column
    pairs past the first 32 each lane loads while it reduces the row."""
    if case == "cube20":
        pb = P.make_problem(3, 20)
        coords, conn, up, lin, nu = pb.coords, pb.conn, pb.up, pb.lin, pb.nu
    else:
        from .test_assembly_kernels import fan_mesh, fan_state
        coords, conn = fan_mesh(3, 30)
        up, lin, nu = fan_state(coords)
    ns = NavierStokes(coords, conn, dt=0.01, use_specializations=False)
    ns.set_state(up, lin, nu)
    ns.assemble()
    rp, ci = ns.csr()
    v, _ = ns.system()
    ref_op = csr_matrix(rp, ci, v, ns.nb_rows)
    rng = np.random.default_rng(5)
    for _ in range(2):  # the same y twice (deterministic)
        x = rng.normal(size=ns.nb_rows)
        y = ns.apply(x)
        assert vec_rel_error(y, ref_op @ x) <= 1e-13
        assert np.array_equal(y, ns.apply(x))
    ns.close()


def fp64_residual(ns) -> float:
    """||b - A x|| / ||b|| of the GPU's solution, evaluated on the host in FP64."""
    rp, ci = ns.csr()
    v, b = ns.system()
    x = ns.solution()
    return vec_rel_error(csr_matrix(rp, ci, v, ns.nb_rows) @ x, b)


@pytest.mark.parametrize("dim,n", [(2, 16), (3, 6)])
@pytest.mark.parametrize("method,precond,mixed", [("gmres", "jacobi", False), ("gmres", "block_jacobi", False),
                                                  ("bicgstab", "jacobi", False), ("bicgstab", "block_jacobi", False),
                                                  ("bicgstab", "jacobi", True), ("gmres", "jacobi", True)])
def test_solve_matches_oracle(dim, n, method, precond, mixed):
    """Solver tolerance 1e-12 on the FP64 residual (also for the FP32 inner
    solve with FP64 refinement).  The solution is compared with the oracle's
    (ILU-GMRES to 1e-13) within 1e-6: these pinned-pressure cavity systems
    have condition numbers near 1e5."""
    pb = small_problem(dim, n)
    ns = gpu_for(pb, use_specializations=False)
    o = oracle_for(pb, use_specializations=False)
    ns.assemble()
    ns.apply_dirichlet()
    o.assemble()
    o.apply_dirichlet()
    st = ns.solve(method=method, precond=precond, mixed=mixed, tol=1e-12, inner_tol=1e-4, max_iters=6000)
    assert st["converged"] == 1, st
    if mixed:
        assert st["refinements"] >= 1
    assert fp64_residual(ns) <= 2e-12
    assert o.solve(tol=1e-13)["rc"] == 0
    assert vec_rel_error(ns.solution(), o.solution()) <= 1e-6


@pytest.mark.parametrize("dim,n,spec", [(2, 16, False), (2, 16, True), (3, 4, False)])
def test_time_steps_match_oracle(dim, n, spec):
    """Three full steps (assemble, BCs, solve, update) against the oracle."""
    pb = small_problem(dim, n)
    ns = gpu_for(pb, use_specializations=spec)
    o = oracle_for(pb, use_specializations=spec)
    for _ in range(3):
        st = ns.execute(tol=1e-12, max_iters=5000)
        assert st["converged"] == 1
        o.assemble()
        o.apply_dirichlet()
        o.solve(tol=1e-13)
        o.update()
    gup, glin = ns.state()
    oup, olin = o.state()
    assert vec_rel_error(gup, oup) <= 1e-6
    assert vec_rel_error(glin, olin) <= 1e-6


def test_cfg1_one_step_plain_and_mixed():
    """cfg1: 1 assembly + 1 linear solve; plain FP64 and the mixed form both
    within 1e-6 of the FP64 oracle's velocity/pressure."""
    pb = P.config("cfg1")
    o = oracle_for(pb, use_specializations=False)
    o.step(1, tol=1e-13)
    oup, _ = o.state()
    for mixed in (False, True):
        ns = gpu_for(pb, use_specializations=False)
        st = ns.execute(tol=1e-12, mixed=mixed, inner_tol=1e-4)
        assert st["converged"] == 1
        gup, _ = ns.state()
        assert vec_rel_error(gup, oup) <= 1e-6
        ns.close()


@pytest.mark.slow
def test_cfg2_assembly_full_size():
    """cfg2 (1,572,864 tets): CSR pattern bit-exact, values and RHS vs the oracle."""
    pb = P.config("cfg2")
    ns = gpu_for(pb, use_specializations=False)
    o = oracle_for(pb, use_specializations=False)
    rp, ci = ns.csr()
    orp, oci = o.csr()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    ns.assemble()
    o.assemble(8)
    gv, gr = ns.system()
    ov, orr = o.system()
    assert row_scaled_error(gv, ov, orp) <= FP64_TOL
    assert vec_rel_error(gr, orr) <= 1e-11
    del o


def test_error_paths_do_not_hang():
    pb = small_problem(2, 4)
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt)
    with pytest.raises(UfemError) as ei:
        ns.assemble()  # before set_state
    assert ei.value.code == -4
    up = pb.up.copy()
    up[3, 0] = np.nan
    ns.set_state(up, pb.lin, pb.nu)
    ns.assemble()
    st = ns.solve(raise_on_failure=False, tol=1e-10)
    assert st["converged"] == 0 and st["status"] == 3


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("spec", [False, True])
def test_single_element_meshes_match_oracle(dim, spec):
    """The smallest inputs: one triangle and one tetrahedron (every node a row
    with a single incidence, one warp group holding all rows), assembled with
    a random state, against the oracle."""
    rng = np.random.default_rng(7 + dim)
    coords = np.array([[0.0, 0.0], [1.0, 0.1], [0.2, 0.9]]) if dim == 2 else \
        np.array([[0.0, 0.0, 0.0], [1.0, 0.1, 0.0], [0.1, 0.9, 0.1], [0.2, 0.1, 1.1]])
    conn = np.arange(dim + 1, dtype=np.uint32)[None, :]
    N = dim + 1
    up = rng.standard_normal((N, dim + 1))
    lin = np.tile(up[:, :dim], (1, 4)) + 0.1 * rng.standard_normal((N, 4 * dim))
    nu = np.full(N, 1e-2)
    ns = NavierStokes(coords, conn, dt=0.01, use_specializations=spec)
    ns.set_state(up, lin, nu)
    o = O.Oracle(coords, conn, O.options(dt=0.01, use_specializations=spec))
    o.set_state(up, lin, nu)
    rp, ci = ns.csr()
    orp, oci = o.csr()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    ns.assemble()
    o.assemble()
    gv, gr = ns.system()
    ov, orr = o.system()
    assert row_scaled_error(gv, ov, orp) <= 1e-11
    assert vec_rel_error(gr, orr) <= 1e-11
    ns.close()
    o.close()
