"""Restart files of the device-resident state (WriteRestartFile /
ReadRestartFile, solver/actions/WriteRestartFile.cpp:62-90,
ReadRestartFile.cpp:67-110).

Stated tolerance: BITWISE -- a handle restored from a restart file steps to
exactly the states of the handle that wrote it (same mesh, options and
boundary conditions).  A corrupted table, a restart of another mesh or a
missing file is refused with UFEM_ERR_IO.
"""
import os

import numpy as np
import pytest

from coolfluid3_b200 import NavierStokes, problems as P
from coolfluid3_b200._native import UfemError

pytestmark = pytest.mark.gpu


def handle(pb, force=None):
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False)
    ns.set_state(pb.up, pb.lin, pb.nu, force)
    ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    return ns


@pytest.mark.parametrize("dim,n,with_force", [(2, 12, False), (3, 6, False), (3, 5, True)])
def test_restart_continues_bitwise(tmp_path, dim, n, with_force):
    pb = P.make_problem(dim, n, nu=1e-2, dt=0.01)
    force = None
    if with_force:
        force = np.random.default_rng(3).normal(size=(pb.nb_nodes, dim))
    a = handle(pb, force)
    for _ in range(2):
        a.execute(tol=1e-12)
    path = os.path.join(tmp_path, "ns.restart.xml")
    a.write_restart(path, current_time=0.02, iteration=2)
    for _ in range(2):
        a.execute(tol=1e-12)
    up_a, lin_a = a.state()

    b = handle(P.make_problem(dim, n, nu=5e-2, dt=0.01))  # other initial fields, overwritten by the restart
    t, dt, it = b.read_restart(path)
    assert (t, dt, it) == (0.02, 0.01, 2)
    for _ in range(2):
        b.execute(tol=1e-12)
    up_b, lin_b = b.state()
    assert np.array_equal(up_a, up_b) and np.array_equal(lin_a, lin_b)
    a.close()
    b.close()


def test_restart_refuses_bad_files(tmp_path):
    pb = P.make_problem(3, 4, nu=1e-2, dt=0.01)
    a = handle(pb)
    path = os.path.join(tmp_path, "ns.restart.xml")
    a.write_restart(path)
    text = open(path).read()
    assert '<restart version="1"' in text and 'path="navier_stokes_solution"' in text

    other = handle(P.make_problem(3, 5, nu=1e-2, dt=0.01))
    with pytest.raises(UfemError, match="another mesh"):
        other.read_restart(path)
    with pytest.raises(UfemError, match="cannot read"):
        a.read_restart(os.path.join(tmp_path, "missing.xml"))

    raw = bytearray(open(path + ".bin", "rb").read())
    raw[100] ^= 0x40
    open(path + ".bin", "wb").write(bytes(raw))
    with pytest.raises(UfemError, match="checksum"):
        a.read_restart(path)
    a.close()
    other.close()
