"""FP32 element matrices with an FP64 answer: the matrix-free FP64 residual.

The FP32-element system differs from the FP64 one by about 2e-5 of each row's
scale, which the incompressible system's conditioning turns into ~3e-4 in the
state: refining against the stored (FP32-element) matrix cannot reach 1e-6.
With mixed = "matrix_free" the refinement residual is b - M x of the FP64
system, evaluated element by element in FP64 (NavierStokesAssembly.hpp:69-71),
and the FP32-element system is only the inner operator.

Tolerances: the residual itself within 1e-12 of ||b|| against the FP64
assembled system; solutions within 1e-6 of the FP64 oracle (ILU-GMRES to 1e-13),
the bound these pinned-pressure cavities allow at a 1e-12 residual.
"""
import numpy as np
import pytest

from coolfluid3_b200 import NavierStokes
from coolfluid3_b200 import problems as P

from .util import csr_matrix, oracle_for, small_problem, vec_rel_error

pytestmark = pytest.mark.gpu


def _free_rows(pb, nrows):
    """Rows without a Dirichlet condition."""
    free = np.ones(nrows, bool)
    free[pb.bc_nodes.astype(np.int64) * (pb.dim + 1) + pb.bc_comps] = False
    return free


def _gpu(pb, precision, spec=False):
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, theta=pb.theta, use_specializations=spec, precision=precision)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    return ns


@pytest.mark.parametrize("dim,n,spec", [(2, 12, False), (2, 12, True), (3, 4, False), (3, 4, True)])
def test_matrix_free_residual_equals_assembled_fp64_residual(dim, n, spec):
    pb = small_problem(dim, n)
    ns = _gpu(pb, "fp64", spec)
    ns.assemble()
    ns.apply_dirichlet()
    rp, ci = ns.csr()
    vals, b = ns.system()
    x = ns.solution()  # constrained entries hold their row values after apply_dirichlet
    rng = np.random.default_rng(5)
    free = _free_rows(pb, ns.nb_rows)
    x = x.copy()
    x[free] = rng.standard_normal(free.sum()) * 1e-2
    ns.set_solution(x)
    r_mf = ns.fp64_residual()
    r_ref = b - csr_matrix(rp, ci, vals, ns.nb_rows) @ x
    assert np.abs(r_mf[~free]).max() == 0.0
    assert np.linalg.norm(r_mf - r_ref) <= 1e-12 * np.linalg.norm(b)
    ns.close()


def test_matrix_free_residual_is_the_fp64_one_for_fp32_elements():
    """The same residual from a precision=fp32 handle (FP32 matrix stored) equals
    the FP64 handle's: it never reads the stored matrix."""
    pb = small_problem(3, 4)
    a, f = _gpu(pb, "fp64"), _gpu(pb, "fp32")
    for ns in (a, f):
        ns.assemble()
        ns.apply_dirichlet()
    x = a.solution().copy()
    free = _free_rows(pb, a.nb_rows)
    x[free] = np.linspace(-1e-2, 1e-2, int(free.sum()))
    for ns in (a, f):
        ns.set_solution(x)
    ra, rf = a.fp64_residual(), f.fp64_residual()
    assert np.linalg.norm(rf - ra) <= 1e-14 * np.linalg.norm(ra)
    a.close()
    f.close()


@pytest.mark.parametrize("name", ["cfg1", "tet6"])
def test_fp32_elements_with_matrix_free_refinement_meet_1e6(name):
    pb = P.config("cfg1") if name == "cfg1" else small_problem(3, 6)
    o = oracle_for(pb, use_specializations=False)
    o.step(1, tol=1e-13)
    oup, _ = o.state()
    errs = {}
    for mixed in (True, "matrix_free"):
        ns = _gpu(pb, "fp32")
        st = ns.execute(tol=1e-12, mixed=mixed, inner_tol=1e-5, max_iters=6000)
        assert st["converged"] == 1, st
        gup, _ = ns.state()
        errs[mixed] = vec_rel_error(gup, oup)
        ns.close()
    assert errs["matrix_free"] <= 1e-6, errs
    assert errs[True] > 10 * errs["matrix_free"], errs  # refinement on the FP32-element matrix stops short


def test_fp32_elements_three_steps_match_oracle():
    pb = small_problem(3, 4)
    ns = _gpu(pb, "fp32")
    o = oracle_for(pb, use_specializations=False)
    for _ in range(3):
        st = ns.execute(tol=1e-12, mixed="matrix_free", inner_tol=1e-5, max_iters=6000)
        assert st["converged"] == 1
        o.assemble()
        o.apply_dirichlet()
        o.solve(tol=1e-13)
        o.update()
    gup, glin = ns.state()
    oup, olin = o.state()
    assert vec_rel_error(gup, oup) <= 1e-6
    assert vec_rel_error(glin, olin) <= 1e-6
    ns.close()
