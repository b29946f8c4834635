"""GPU tests of batches: several meshes stepped by one launch per phase.

Stated tolerances: a member's state after batched steps is BITWISE equal to
the same member stepped alone (a batch of one), whatever the other members
are; the batched assembly agrees with the one-mesh kernel to 1e-14 of each
CSR row's largest entry (the same element code compiled into two kernels);
batched solves agree with the one-mesh solver within 1e-6 relative and reach
the FP64 residual tolerance; the mixed batched solve (FP32 operator, FP64
vectors, FP64 residual replacement) meets the same residual and agrees within
1e-6.
"""
import numpy as np
import pytest

from coolfluid3_b200 import Batch, NavierStokes
from coolfluid3_b200 import problems as P

from .util import row_scaled_error, vec_rel_error

pytestmark = pytest.mark.gpu


def member(dim, n, seed, precision="fp64", nu=1e-2, dt=0.01, spec=False):
    pb = P.make_problem(dim, n, nu=nu, dt=dt, seed=seed)
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=spec, precision=precision)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    return ns


SIZES_2D = [(2, 6, 11), (2, 13, 12), (2, 9, 13), (2, 20, 14)]
SIZES_3D = [(3, 3, 21), (3, 5, 22), (3, 4, 23)]


def run_batch(specs, steps, precision="fp64", graphs=True, **krylov):
    ms = [member(*s, precision=precision) for s in specs]
    b = Batch(ms, graphs=graphs)
    sts = []
    for _ in range(steps):
        sts.append(b.step(**krylov))
    states = [m.state()[0] for m in ms]
    b.close()
    return states, sts


@pytest.mark.parametrize("specs", [SIZES_2D, SIZES_3D])
def test_member_results_identical_alone_and_in_the_mix(specs):
    mixed, _ = run_batch(specs, 2)
    for k, s in enumerate(specs):
        alone, _ = run_batch([s], 2)
        assert np.array_equal(alone[0], mixed[k]), s
    # a different mix (reversed order, one member left out)
    sub = list(reversed(specs[1:]))
    other, _ = run_batch(sub, 2)
    for k, s in enumerate(sub):
        assert np.array_equal(other[k], mixed[specs.index(s)]), s


def test_graphs_do_not_change_results():
    a, sa = run_batch(SIZES_2D[:3], 2, graphs=True)
    b, sb = run_batch(SIZES_2D[:3], 2, graphs=False)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert [s["iterations"] for s in sa[-1]] == [s["iterations"] for s in sb[-1]]


@pytest.mark.parametrize("specs", [SIZES_2D, SIZES_3D])
def test_batched_assembly_matches_single_handle(specs):
    ms = [member(*s) for s in specs]
    singles = [member(*s) for s in specs]
    b = Batch(ms)
    b.assemble()
    for m, s in zip(ms, singles):
        s.assemble()
        s.apply_dirichlet()
        v, r = m.system()
        vs, rs = s.system()
        rp, _ = s.csr()
        assert row_scaled_error(v, vs, rp) <= 1e-14
        assert vec_rel_error(r, rs) <= 1e-14
    b.close()


@pytest.mark.parametrize("specs", [SIZES_2D, SIZES_3D])
def test_batched_step_matches_single_handle(specs):
    states, sts = run_batch(specs, 2, tol=1e-12)
    for k, s in enumerate(specs):
        ref = member(*s)
        for _ in range(2):
            ref.execute(tol=1e-12)
        up, _ = ref.state()
        assert vec_rel_error(states[k], up) <= 1e-6, s
        assert sts[-1][k]["converged"] and sts[-1][k]["rel_residual"] <= 1e-12


@pytest.mark.parametrize("specs", [SIZES_2D, SIZES_3D])
def test_mixed_batched_solve(specs):
    """FP32 elements; the mixed solve (FP32 operator, FP64 residual
    replacement) against the FP64-operator solve, both to 1e-12."""
    plain, _ = run_batch(specs, 1, precision="fp32", tol=1e-12)
    mixed, sts = run_batch(specs, 1, precision="fp32", tol=1e-12, mixed=True)
    for k in range(len(specs)):
        assert sts[0][k]["converged"] and sts[0][k]["rel_residual"] <= 1e-12
        assert sts[0][k]["refinements"] >= 1  # convergence is accepted on the FP64 residual
        assert vec_rel_error(mixed[k], plain[k]) <= 1e-6


@pytest.mark.parametrize("specs", [SIZES_2D, SIZES_3D])
def test_mixed_batched_solve_fp64_elements(specs):
    """FP64 element arithmetic, FP32 operator copy for the Krylov iterations,
    FP64 residual replacement: the FP64 residual tolerance is met and the
    state agrees with the plain FP64 batched solve to 1e-7 (both to 1e-12)."""
    plain, _ = run_batch(specs, 2, tol=1e-12)
    mixed, sts = run_batch(specs, 2, tol=1e-12, mixed=True)
    for k in range(len(specs)):
        assert sts[-1][k]["converged"] and sts[-1][k]["rel_residual"] <= 1e-12
        assert vec_rel_error(mixed[k], plain[k]) <= 1e-7


def test_batch_rejects_incompatible_members():
    from coolfluid3_b200 import UfemError
    a = member(2, 4, 1)
    c = member(3, 2, 2)
    with pytest.raises(UfemError):
        Batch([a, c])
    with pytest.raises(UfemError):
        Batch([a, a])


@pytest.mark.parametrize("specs", [SIZES_2D, SIZES_3D])
def test_batch_autotuner(specs):
    """The batch autotuner keeps one of its candidates, and the assembly with
    the chosen width matches the default one to rounding (1e-14 of the row)."""
    ms = [member(*s) for s in specs]
    ref_ms = [member(*s) for s in specs]
    b, ref = Batch(ms), Batch(ref_ms)
    t = b.tune_assembly(reps=2)
    assert t["warps_per_cta"] in (2, 4, 8) and t["ms"] > 0
    b.assemble()
    ref.assemble()
    for m, r in zip(ms, ref_ms):
        v, rhs = m.system()
        vr, rhsr = r.system()
        rp, _ = r.csr()
        assert row_scaled_error(v, vr, rp) <= 1e-14 and vec_rel_error(rhs, rhsr) <= 1e-14
    b.close()
    ref.close()


def test_sixty_four_members_of_mixed_sizes_identical_alone_and_in_the_mix():
    """64 2D members of 4..24 cells a side (log-uniform node counts, seeded
    viscosities): every member's state after two batched steps equals the same
    member stepped alone, bitwise; a held member (set_active) keeps its state."""
    rng = np.random.default_rng(64)
    sides = np.unique(np.round(np.exp(rng.uniform(np.log(4), np.log(24), 64))).astype(int), return_counts=False)
    specs = [(2, int(sides[k % len(sides)]), 100 + k) for k in range(64)]
    mixed, sts = run_batch(specs, 2, tol=1e-10, max_iters=3000)
    assert all(s["converged"] for step in sts for s in step)
    for k in (0, 17, 40, 63):
        alone, _ = run_batch([specs[k]], 2, tol=1e-10, max_iters=3000)
        assert np.array_equal(alone[0], mixed[k]), specs[k]
    # hold every other member after the first step: the others go on exactly as alone
    ms = [member(*s) for s in specs[:8]]
    b = Batch(ms)
    b.step(tol=1e-10, max_iters=3000)
    held = [m.state()[0].copy() for m in ms]
    b.set_active([k % 2 == 0 for k in range(8)])
    st = b.step(tol=1e-10, max_iters=3000)
    for k, m in enumerate(ms):
        if k % 2:
            assert np.array_equal(m.state()[0], held[k]) and st[k]["iterations"] == 0
        else:
            assert np.array_equal(m.state()[0], mixed[k])
    b.close()


def test_batched_two_level_preconditioner():
    """precond "two_level_coupled" in a batch: each member's coarse space is its
    own (aggregates capped at 12 x 12 boxes in 2D); members stay bitwise equal
    alone and in the mix, need fewer iterations than with point Jacobi, and
    agree with the one-handle two-level solve within 1e-6."""
    specs = [(2, 24, 301), (2, 40, 302), (2, 10, 303), (3, 6, 304)]
    specs2 = [s for s in specs if s[0] == 2]
    mixed, sts = run_batch(specs2, 2, tol=1e-12, max_iters=6000, precond="two_level_coupled")
    assert all(s["converged"] for step in sts for s in step)
    for k, s in enumerate(specs2):
        alone, _ = run_batch([s], 2, tol=1e-12, max_iters=6000, precond="two_level_coupled")
        assert np.array_equal(alone[0], mixed[k]), s
        one = member(*s)
        for _ in range(2):
            st = one.execute(tol=1e-12, max_iters=6000, precond="two_level_coupled")
            assert st["converged"]
        assert vec_rel_error(one.state()[0], mixed[k]) <= 1e-6
        one.close()
    _, sj = run_batch(specs2, 1, tol=1e-12, max_iters=6000)
    _, s2 = run_batch(specs2, 1, tol=1e-12, max_iters=6000, precond="two_level_coupled")
    assert sum(s["iterations"] for s in s2[0]) * 2 <= sum(s["iterations"] for s in sj[0])
    mixed3, sts3 = run_batch([specs[3]], 2, tol=1e-12, max_iters=6000, precond="two_level_coupled")
    assert all(s["converged"] for step in sts3 for s in step)


@pytest.mark.parametrize("specs", [SIZES_2D, SIZES_3D])
def test_matrix_free_batched_solve_fp32_elements(specs):
    """FP32 element matrices, each member refined against its own matrix-free
    FP64 residual (mixed = "matrix_free", the one-handle refinement for the
    whole batch): every member reaches the 1e-12 FP64 residual, lands within
    1e-6 of the FP64 oracle after two steps, and is bitwise the same alone and
    in the mix."""
    from .util import oracle_for
    kr = dict(tol=1e-12, mixed="matrix_free", inner_tol=1e-5, max_iters=3000)
    mixed, sts = run_batch(specs, 2, precision="fp32", **kr)
    for k, s in enumerate(specs):
        assert sts[-1][k]["converged"] and sts[-1][k]["rel_residual"] <= 1e-12, sts[-1][k]
        assert sts[-1][k]["refinements"] >= 1
        alone, _ = run_batch([s], 2, precision="fp32", **kr)
        assert np.array_equal(alone[0], mixed[k]), s
        pb = P.make_problem(s[0], s[1], nu=1e-2, dt=0.01, seed=s[2])
        o = oracle_for(pb, use_specializations=False)
        for _ in range(2):
            o.assemble()
            o.apply_dirichlet()
            assert o.solve(tol=1e-13)["rc"] == 0
            o.update()
        assert vec_rel_error(mixed[k], o.state()[0]) <= 1e-6, s
        o.close()
