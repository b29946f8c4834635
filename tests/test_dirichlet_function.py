"""Dirichlet values from a function of coordinates and time (BCDirichletFunction,
plugins/UFEM/src/UFEM/BCDirichletFunction.cpp:61-92), evaluated on the device.

Stated tolerances: the device-evaluated values equal numpy's evaluation of the
same formula to 1e-14 relative (CUDA's and numpy's math functions may differ
in the last bits); the system after the conditions matches the oracle given
numpy's values to 1e-14 of each row's scale; the conditioned components of the
state after a step equal f(x, t) at the step's start time to 1e-14; the time
advances by dt at each update; a batch member applies the same values as its
own handle; malformed formulas are refused with UFEM_ERR_ARG.
"""
import numpy as np
import pytest

import oracle as O
from coolfluid3_b200 import Batch, NavierStokes, problems as P
from coolfluid3_b200._native import UfemError

from .util import row_scaled_error, vec_rel_error

pytestmark = pytest.mark.gpu

EXPR = "sin(pi*x)^2 * (1 + 0.5*cos(3*t)) - 0.25*exp(-y)*sqrt(abs(x - 0.5))"


def f_numpy(x, y, t):
    return np.sin(np.pi * x) ** 2 * (1 + 0.5 * np.cos(3 * t)) - 0.25 * np.exp(-y) * np.sqrt(np.abs(x - 0.5))


def cavity(n):
    pb = P.make_problem(2, n, nu=1e-2, dt=0.01)
    top = np.arange(n * (n + 1), (n + 1) * (n + 1), dtype=np.uint32)
    lid = np.isin(pb.bc_nodes, top) & (pb.bc_comps == 0) & (pb.bc_values == 1.0)
    return pb, top, lid


def handle(pb, lid, top):
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.add_dirichlet(pb.bc_nodes[~lid], pb.bc_comps[~lid], pb.bc_values[~lid])
    ns.add_dirichlet_function(top[1:-1], 0, EXPR)  # the lid's u, corners stay at the walls' 0
    return ns


def test_function_values_and_system_against_oracle():
    n = 14
    pb, top, lid = cavity(n)
    ns = handle(pb, lid, top)
    ns.time = 0.3
    ns.assemble()
    v0, r0 = ns.system()
    ns.apply_dirichlet()
    v1, r1 = ns.system()
    nodes = top[1:-1]
    f = f_numpy(pb.coords[nodes, 0], pb.coords[nodes, 1], 0.3)
    got = r1[nodes.astype(np.int64) * 3 + 0] + pb.up[nodes, 0]  # rhs = f - old on the constrained rows
    assert vec_rel_error(got, f) <= 1e-14
    o = O.Oracle(pb.coords, pb.conn, O.options(dt=pb.dt, use_specializations=False))
    o.set_state(pb.up, pb.lin, pb.nu)
    o.add_dirichlet(pb.bc_nodes[~lid], pb.bc_comps[~lid], pb.bc_values[~lid])
    o.add_dirichlet(nodes, np.zeros(len(nodes), np.int32), f)
    o.set_system(v0, r0)
    o.apply_dirichlet()
    ov, orr = o.system()
    rp, _ = ns.csr()
    assert row_scaled_error(v1, ov, rp) <= 1e-14 and vec_rel_error(r1, orr) <= 1e-14
    ns.close()


def test_time_advances_and_state_takes_the_function_value():
    n = 10
    pb, top, lid = cavity(n)
    ns = handle(pb, lid, top)
    assert ns.time == 0.0
    for k in range(3):
        t = ns.time
        ns.execute(tol=1e-12)
        up, _ = ns.state()
        nodes = top[1:-1]
        f = f_numpy(pb.coords[nodes, 0], pb.coords[nodes, 1], t)
        assert np.max(np.abs(up[nodes, 0] - f)) <= 1e-14 * max(1.0, np.max(np.abs(f)))
        assert abs(ns.time - (k + 1) * pb.dt) <= 1e-15
    ns.close()


def test_batch_member_applies_function_values():
    n = 10
    pb, top, lid = cavity(n)
    a, s = handle(pb, lid, top), handle(pb, lid, top)
    a.time = s.time = 0.7
    b = Batch([a])
    b.assemble()
    s.assemble()
    s.apply_dirichlet()
    v, r = a.system()
    vs, rs = s.system()
    rp, _ = s.csr()
    assert row_scaled_error(v, vs, rp) <= 1e-14 and vec_rel_error(r, rs) <= 1e-14
    b.close()


@pytest.mark.parametrize("bad,msg", [("sin(x", "expected '\\)'"), ("foo(x)", "unknown name"), ("x +* y", "unexpected"),
                                     ("2 x", "trailing")])
def test_malformed_formulas_are_refused(bad, msg):
    pb = P.make_problem(2, 4, nu=1e-2, dt=0.01)
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt)
    with pytest.raises(UfemError, match=msg):
        ns.add_dirichlet_function(np.array([0], np.uint32), 0, bad)
    ns.close()
