"""GPU tests of the serving loop (continuous batching under an HBM budget).

Stated tolerances: a request's final state is BITWISE the same when it is
served alone and when it is served in a mix (FP64, mixed-precision solve, FP32
elements); the served mixed-precision form (FP64 elements, FP32 Krylov
operator, FP64 refinement) is within 1e-6 relative of the plain FP64 path
(`run_plain`); with FP32 element arithmetic on the batched path (which
refines against the stored FP32-element system) the served state is within
1e-3 (the perturbation of the system by FP32 element rounding, amplified by the
conditioning of the incompressible system, chiefly in the pressure), and on the
large-request path (refined against the matrix-free FP64 residual) within 1e-6
of the oracle; admission never reserves more than the budget.
"""
import numpy as np
import pytest

import oracle as O
from coolfluid3_b200 import serving as S

from .util import vec_rel_error

pytestmark = pytest.mark.gpu

GB = 1 << 30


def workload(n=8, seed=5, steps=3):
    rng = np.random.default_rng(seed)
    reqs = []
    for k in range(n):
        dim = 2 if k % 2 == 0 else 3
        e = float(np.exp(rng.uniform(np.log(2e3), np.log(2e4))))
        reqs.append(S.make_request(k, dim, e, float(np.exp(rng.uniform(np.log(1e-3), np.log(1e-1)))),
                                   seed * 100 + k, nsteps=steps - (k % 2)))
    return reqs


@pytest.mark.parametrize("precision,mixed", [("fp64", False), ("fp64", True), ("fp32", True)])
def test_results_identical_alone_and_in_the_mix(precision, mixed):
    reqs = workload()
    srv = S.Server(8 * GB, precision=precision, mixed=mixed, realtime=False, mixed_scope="all")
    mix, stats = srv.run(reqs)
    assert stats["requests"] == len(reqs) and stats["rejected"] == 0
    assert srv.max_batch >= 2  # requests really ran together
    for r in mix:
        assert r.ok, r.statuses
    for req in reqs[:4]:
        alone, _ = S.Server(8 * GB, precision=precision, mixed=mixed, realtime=False, mixed_scope="all").run([req])
        assert np.array_equal(alone[0].state, mix[req.rid].state), req.rid


def oracle_state(req):
    o = O.Oracle(req.coords, req.conn, O.options(dt=req.dt, use_specializations=False))
    o.set_state(req.up, req.lin, req.nu)
    o.add_dirichlet(req.bc_nodes, req.bc_comps, req.bc_values)
    o.step(req.nsteps, tol=1e-13)
    return o.state()[0]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-6), ("fp32", 1e-3)])
def test_served_error_against_the_fp64_oracle(precision, tol):
    """Served mixed-precision states against the FP64 oracle (GMRES + ILU to
    1e-13).  The served solve refines with FP64 residuals to 1e-12; the plain
    FP64 path at the reference's 1e-10 is shown beside it (its own error is
    the solver tolerance amplified by the pressure conditioning)."""
    reqs = workload(n=6, seed=9)
    served, sstats = S.Server(8 * GB, precision=precision, mixed=True, realtime=False, mixed_scope="all",
                              krylov=dict(tol=1e-12)).run(reqs)
    plain, pstats = S.run_plain(reqs, realtime=False)
    worst_plain = 0.0
    for a, b, req in zip(served, plain, reqs):
        ref = oracle_state(req)
        assert vec_rel_error(a.state, ref) <= tol, (a.rid, vec_rel_error(a.state, ref))
        worst_plain = max(worst_plain, vec_rel_error(b.state, ref))
    assert worst_plain <= 1e-4
    assert sstats["steps"] == pstats["steps"]
    for k in ("p50", "p99"):
        assert sstats["step_ms"][k] > 0 and pstats["step_ms"][k] > 0


def test_admission_respects_the_hbm_budget():
    reqs = workload(n=6, seed=3)
    need = max(S.estimate_bytes(r) for r in reqs)
    budget = int(2.2 * need)  # at most two of the largest at once
    srv = S.Server(budget, mixed=True, realtime=False)
    res, stats = srv.run(reqs)
    assert stats["requests"] == len(reqs) and all(r.ok for r in res)
    assert srv.peak_bytes <= budget
    with pytest.raises(ValueError):
        S.Server(need // 2, realtime=False).run(reqs)


def test_bad_requests_fail_alone():
    """Host-side fault injection: a degenerate element (rejected at set-up) and
    non-finite initial fields (the member's solve reports status 3); the other
    requests finish with the results they have alone."""
    reqs = workload(n=4, seed=11)
    bad_mesh = S.make_request(100, 2, 2e3, 1e-2, 77, nsteps=2)
    bad_mesh.conn = bad_mesh.conn.copy()
    bad_mesh.conn[0, 2] = bad_mesh.conn[0, 1]  # two equal nodes: zero measure
    bad_state = S.make_request(101, 2, 3e3, 1e-2, 78, nsteps=2)
    bad_state.up = bad_state.up.copy()
    bad_state.up[5, 0] = np.nan
    res, stats = S.Server(8 * GB, precision="fp64", mixed=False, realtime=False).run(reqs + [bad_mesh, bad_state])
    by = {r.rid: r for r in res}
    assert by[100].error is not None
    assert by[101].statuses and by[101].statuses[0]["status"] == 3
    for req in reqs:
        alone, _ = S.Server(8 * GB, precision="fp64", mixed=False, realtime=False).run([req])
        assert np.array_equal(alone[0].state, by[req.rid].state)


def test_poisson_arrivals_realtime():
    reqs = S.poisson_workload(6, rate=200.0, elems=(2e3, 2e4), nsteps=2, seed=4)
    res, stats = S.Server(8 * GB, mixed=True, realtime=True).run(reqs)
    assert stats["requests"] == 6 and all(r.ok for r in res)
    assert stats["steps_per_s"] > 0 and stats["request_s"]["p99"] >= stats["request_s"]["p50"]


def test_large_path_fp32_elements_with_fp64_answers():
    """The mixed form's large-request path (one handle per request on the large
    workers: FP32 element matrices, FP32 inner BiCGStab with the coupled
    two-level preconditioner refined against the matrix-free FP64 residual to
    1e-12): every request within 1e-6 of the FP64 oracle and bitwise the same
    alone and in the mix.  large_rows = 1 sends every request down that path."""
    reqs = workload(n=6, seed=13)
    kw = dict(precision="fp64", mixed=True, realtime=False, krylov=dict(tol=1e-12), large_rows=1,
              large_rows_2d=1, large_precond="two_level_coupled")
    served, stats = S.Server(8 * GB, **kw).run(reqs)
    assert stats["rejected"] == 0 and all(r.ok for r in served)
    for r, req in zip(served, reqs):
        assert vec_rel_error(r.state, oracle_state(req)) <= 1e-6, r.rid
    for req in reqs[:3]:
        alone, _ = S.Server(8 * GB, **kw).run([req])
        assert np.array_equal(alone[0].state, served[req.rid].state), req.rid


def test_fp32_elements_on_every_request_meet_the_fp64_oracle():
    """mixed_scope="elements": the batched small requests also assemble FP32
    element matrices and each member is refined against its own matrix-free
    FP64 residual (the large requests' solve, batched).  Every served state is
    within 1e-6 of the FP64 oracle at a 1e-12 residual, and bitwise the same
    served alone and in the mix."""
    reqs = workload(n=6, seed=9)
    srv = S.Server(8 * GB, precision="fp64", mixed=True, realtime=False, mixed_scope="elements",
                   krylov=dict(tol=1e-12))
    served, _ = srv.run(reqs)
    assert srv.max_batch >= 2
    for a, req in zip(served, reqs):
        assert a.ok, a.statuses
        assert vec_rel_error(a.state, oracle_state(req)) <= 1e-6, a.rid
    for req in reqs[:3]:
        alone, _ = S.Server(8 * GB, precision="fp64", mixed=True, realtime=False, mixed_scope="elements",
                            krylov=dict(tol=1e-12)).run([req])
        assert np.array_equal(alone[0].state, served[req.rid].state), req.rid
