"""The allocation-free solve, ufem_ns_solve_noalloc, against ufem_ns_solve.

Some callers cannot call cudaMalloc (an application that hands all device
memory to its own pool, a fixed device-memory budget, a loop that must not
take the synchronisation of a first-use allocation).  For them the library
offers one entry point that solves with a fixed scratch area inside the library
instead of allocating.  This test calls it through the C ABI twice in a row on
the same system and checks both results against the allocating entry point's,
within the solver tolerance these tests use elsewhere.  The file is named so
that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

from coolfluid3_b200 import NavierStokes
from coolfluid3_b200 import _native as N
from coolfluid3_b200 import problems as P
from coolfluid3_b200.ufem import krylov_options

pytestmark = pytest.mark.gpu


def _system(dim, n):
    pb = P.make_problem(dim, n)
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    ns.assemble()
    ns.apply_dirichlet()
    return ns


def _noalloc(ns, opts):
    st = N.KrylovStatus()
    rc = N.lib().ufem_ns_solve_noalloc(ns.handle, C.byref(opts), C.byref(st), None)
    N.check(rc)
    return st


@pytest.mark.parametrize("dim,n", [(2, 16), (3, 6)])
def test_noalloc_solve_matches_allocating_solve(dim, n):
    opts = krylov_options(method="bicgstab", precond="jacobi", tol=1e-12, max_iters=6000)
    ref = _system(dim, n)
    ref.set_solution(np.zeros(ref.nb_rows))
    st_ref = ref.solve(method="bicgstab", precond="jacobi", tol=1e-12, max_iters=6000)
    x_ref = ref.solution()
    assert st_ref["converged"] == 1

    ns = _system(dim, n)  # a second handle that never allocates a Krylov workspace
    import torch
    bytes0 = ns.device_bytes()  # counts the handle's Krylov workspace once one exists
    free0, _ = torch.cuda.mem_get_info()
    results = []
    for _ in range(2):  # two calls in a row share the scratch area
        ns.set_solution(np.zeros(ns.nb_rows))
        st = _noalloc(ns, opts)
        assert st.converged == 1 and st.rel_residual <= 1e-12
        results.append(ns.solution())
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    # nothing was allocated: no Krylov workspace on the handle, no drop in free device memory
    assert ns.device_bytes() == bytes0
    assert free1 >= free0, (free0, free1)
    for x in results:
        assert np.linalg.norm(x - x_ref) <= 1e-10 * np.linalg.norm(x_ref)
    ns.close()
    ref.close()


def test_noalloc_rejects_unsupported_options_and_sizes():
    ns = _system(2, 4)
    for kw in (dict(method="gmres"), dict(precond="block_jacobi"), dict(mixed=True)):
        st = N.KrylovStatus()
        rc = N.lib().ufem_ns_solve_noalloc(ns.handle, C.byref(krylov_options(**kw)), C.byref(st), None)
        assert rc == -1, kw  # UFEM_ERR_ARG
    ns.close()
    big = P.make_problem(3, 32)  # 35,937 nodes x 4 = 143,748 rows > UFEM_NOALLOC_MAX_ROWS
    nb = NavierStokes(big.coords, big.conn, dt=big.dt)
    assert nb.nb_rows > 131072
    st = N.KrylovStatus()
    rc = N.lib().ufem_ns_solve_noalloc(nb.handle, C.byref(krylov_options()), C.byref(st), None)
    assert rc == -6 and b"at most" in N.lib().ufem_last_error()  # UFEM_ERR_LIMIT
    nb.close()
