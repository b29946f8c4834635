"""Overlapped host transfers (ufem_ns_stage_state / commit_state / fetch_rhs).

Through the Python wrappers over the C ABI.  Stated tolerance: BITWISE --
pipelined steps on two streams (the upload of
step k+1 queued before step k is assembled, every RHS read back on the copy
stream) give each step exactly the RHS of the sequential path
(ufem_ns_set_state, assembly, Dirichlet, system read).  Misuse (a commit with
nothing staged, a third stage) is refused with UFEM_ERR_STATE.
"""
import numpy as np
import pytest
import torch

from coolfluid3_b200 import NavierStokes, problems as P
from coolfluid3_b200._native import UfemError

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dim,n", [(2, 24), (3, 10)])
def test_pipelined_steps_equal_sequential(dim, n):
    pb = P.make_problem(dim, n, nu=1e-2, dt=0.01)
    rng = np.random.default_rng(11)
    states = []
    for k in range(4):  # four different states of the same mesh
        up = pb.up * (1.0 + 0.1 * k) + 0.01 * rng.normal(size=pb.up.shape)
        lin = pb.lin * (1.0 - 0.05 * k)
        nu = pb.nu * (1.0 + 0.2 * k)
        states.append((up, lin, nu))
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False)
    ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    ref = []
    for up, lin, nu in states:
        ns.set_state(up, lin, nu)
        ns.assemble()
        ns.apply_dirichlet()
        ref.append(ns.system()[1].copy())

    comp, copy = torch.cuda.Stream(), torch.cuda.Stream()
    host = [tuple(torch.from_numpy(np.ascontiguousarray(a)).pin_memory() for a in st) for st in states]
    outs = [torch.empty(ns.nb_rows, dtype=torch.float64).pin_memory() for _ in states]

    def stage(k):
        ns.stage_state(*host[k], copy.cuda_stream)

    stage(0)
    for k in range(len(states)):
        if k + 1 < len(states):
            stage(k + 1)
        ns.commit_state(comp.cuda_stream)
        ns.assemble(comp.cuda_stream)
        ns.apply_dirichlet(comp.cuda_stream)
        ns.fetch_rhs(outs[k], comp.cuda_stream, copy.cuda_stream)
    copy.synchronize()
    comp.synchronize()
    for k in range(len(states)):
        assert np.array_equal(outs[k].numpy(), ref[k]), k

    with pytest.raises(UfemError, match="no staged state"):
        ns.commit_state(comp.cuda_stream)
    stage(0)
    stage(1)
    with pytest.raises(UfemError, match="two staged states"):
        stage(2)
    ns.commit_state(comp.cuda_stream)
    ns.commit_state(comp.cuda_stream)
    comp.synchronize()
    ns.close()
