"""Constant Neumann condition (BCNeumannConstant, plugins/UFEM/src/UFEM/
BCNeumannConstant.cpp:54-60) on Line2D boundary faces.

Stated tolerances: the oracle's face contribution equals the hand evaluation
of the reference's expression (weight 2 x detJ |dx|/2 x N_i 1/2 x flux x
|normal| |dx|/2 = flux |dx|^2 / 4) to rounding; on the GPU, Neumann + Dirichlet
applied to the same assembled system are BITWISE the oracle's; two time steps
of a shear-driven cavity (traction on the top faces) are within 1e-6 of the
oracle's states; a batch
member applies the same contributions as its own handle (1e-14 of the row
scale, the assembly's rounding).
"""
import numpy as np
import pytest

import oracle as O
from coolfluid3_b200 import Batch, NavierStokes, problems as P

from .util import oracle_for, row_scaled_error, vec_rel_error


def bottom_faces(n):
    """Line2D faces of the y = 0 wall of the structured n x n triangle mesh."""
    nodes = np.arange(n + 1, dtype=np.uint32)  # node = j*(n+1)+i, j = 0
    return np.stack([nodes[:-1], nodes[1:]], axis=1)


def test_oracle_face_contribution_known_answer():
    coords = np.array([[0.0, 0.0], [0.3, 0.4], [0.0, 1.0]])
    conn = np.array([[0, 1, 2]], np.uint32)
    o = O.Oracle(coords, conn, O.options(dt=0.01))
    o.set_state(np.zeros((3, 3)), np.zeros((3, 8)), np.full(3, 1e-2))
    o.set_system(np.zeros(o.nnz), np.zeros(o.nrows))
    o.add_neumann(np.array([[0, 1]]), 2, 3.0)
    o.apply_dirichlet()
    _, rhs = o.system()
    L = 0.5  # |(0.3, 0.4)|
    expect = 3.0 * L * L / 4.0
    assert abs(rhs[0 * 3 + 2] - expect) <= 1e-15 and abs(rhs[1 * 3 + 2] - expect) <= 1e-15
    assert np.count_nonzero(rhs) == 2


@pytest.mark.gpu
def test_neumann_and_dirichlet_bitwise_on_the_same_system():
    pb = P.make_problem(2, 16, nu=1e-2, dt=0.01)
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    faces = bottom_faces(16)
    ns.add_neumann(faces, 2, 0.7)       # pressure rows
    ns.add_neumann(faces[::2], 0, -1.3)  # u rows, overlapping faces add in order
    ns.assemble()
    v0, r0 = ns.system()
    ns.apply_dirichlet()
    v1, r1 = ns.system()
    o = oracle_for(pb)
    o.add_neumann(faces, 2, 0.7)
    o.add_neumann(faces[::2], 0, -1.3)
    o.set_system(v0, r0)
    o.apply_dirichlet()
    ov, orr = o.system()
    assert np.array_equal(v1, ov) and np.array_equal(r1, orr)
    ns.close()


@pytest.mark.gpu
def test_shear_driven_cavity_step_against_oracle():
    """A well-posed use: the lid's u = 1 Dirichlet of the cavity is replaced by
    a constant traction on the u rows of the top faces (v = 0 stays)."""
    n = 12
    pb = P.make_problem(2, n, nu=1e-2, dt=0.01)
    top = np.arange(n * (n + 1), (n + 1) * (n + 1), dtype=np.uint32)
    lid = np.isin(pb.bc_nodes, top) & (pb.bc_comps == 0) & (pb.bc_values == 1.0)
    nodes, comps, values = pb.bc_nodes[~lid], pb.bc_comps[~lid], pb.bc_values[~lid]
    faces = np.stack([top[:-1], top[1:]], axis=1)
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.add_dirichlet(nodes, comps, values)
    ns.add_neumann(faces, 0, 2.0)
    for _ in range(2):
        ns.execute(tol=1e-12)
    up, _ = ns.state()
    o = O.Oracle(pb.coords, pb.conn, O.options(dt=pb.dt, use_specializations=False))
    o.set_state(pb.up, pb.lin, pb.nu)
    o.add_dirichlet(nodes, comps, values)
    o.add_neumann(faces, 0, 2.0)
    o.step(2, tol=1e-13)
    oup, _ = o.state()
    assert np.abs(up[top[1:-1], 0]).min() > 0  # the traction drives the top row
    assert vec_rel_error(up, oup) <= 1e-6
    ns.close()


@pytest.mark.gpu
def test_batch_member_applies_its_neumann_faces():
    pb = P.make_problem(2, 10, nu=1e-2, dt=0.01)
    faces = bottom_faces(10)

    def member():
        m = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False)
        m.set_state(pb.up, pb.lin, pb.nu)
        m.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
        m.add_neumann(faces, 2, 0.9)
        return m

    a, s = member(), member()
    b = Batch([a])
    b.assemble()
    s.assemble()
    s.apply_dirichlet()
    v, r = a.system()
    vs, rs = s.system()
    rp, _ = s.csr()
    assert row_scaled_error(v, vs, rp) <= 1e-14 and vec_rel_error(r, rs) <= 1e-14
    b.close()


@pytest.mark.gpu
def test_neumann_is_two_dimensional_only():
    pb = P.make_problem(3, 2, nu=1e-2, dt=0.01)
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt)
    with pytest.raises(Exception, match="Line2D"):
        ns.add_neumann(np.array([[0, 1]]), 0, 1.0)
    ns.close()
