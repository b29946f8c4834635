"""Parity at the full sizes of the tetrahedral configurations.

cfg2 (64^3 x 6, 1,572,864 tets): ten full time steps on the GPU against the FP64
oracle's ten steps, recorded in tests/golden/cfg2_steps.json by
tests/golden/make_cfg2_steps.py (the oracle's serial solve takes minutes per
step).  cfg3 (128^3 x 6, 12,582,912 tets, 508,839,952 CSR values): the assembled
system against the oracle's (threaded, bitwise equal to serial), FP64 and FP32
element arithmetic.

Tolerances:
 - assembly, FP64 elements: 1e-11 of each CSR row's largest |entry|; RHS 1e-11
   relative (the same bound as the small-mesh parity tests);
 - assembly, FP32 elements: 2e-5 of the row scale, RHS 1e-4 relative (FP32
   rounding of the element arithmetic; measured 1.9e-7 and 4.7e-6);
 - states after each step: velocity within 1e-6 relative; pressure within 1e-4
   relative, and within 1e-6 once the mean offset over the sampled nodes is
   removed: the cavity's pressure is pinned at one corner node, so its constant
   mode is determined far less well than the rest (on this mesh a 1e-12 residual
   moves the pressure by 4e-4 relative, almost all of it a constant offset).  The
   oracle solves to 1e-13 (ILU-GMRES), the GPU to 1e-13 (FP64 refinement of FP32
   inner BiCGStab); measured: velocity 6.3e-9, pressure 4.8e-6, pressure without
   the offset 1.2e-7.
"""
import json
import os

import numpy as np
import pytest

from coolfluid3_b200 import NavierStokes
from coolfluid3_b200 import problems as P

from .util import oracle_for, row_scaled_error, vec_rel_error

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cfg2_steps.json")


def test_cfg2_ten_steps_match_oracle():
    with open(GOLDEN) as f:
        ref = json.load(f)
    pb = P.config("cfg2")
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    nodes = np.asarray(ref["sample_nodes"], np.int64)
    worst = {"velocity": 0.0, "pressure": 0.0}
    for k, rs in enumerate(ref["steps"]):
        st = ns.execute(tol=1e-13, mixed=True, inner_tol=1e-5, max_iters=6000)
        assert st["converged"] == 1, (k, st)
        up, _ = ns.state()
        norms = [float(np.linalg.norm(up[:, c])) for c in range(4)]
        got = up[nodes]
        want = np.asarray(rs["samples"])
        ev = max(vec_rel_error(got[:, :3], want[:, :3]), max(abs(a - b) / b for a, b in zip(norms[:3], rs["norms"][:3])))
        ep = max(vec_rel_error(got[:, 3], want[:, 3]), abs(norms[3] - rs["norms"][3]) / rs["norms"][3])
        dp = got[:, 3] - want[:, 3]
        eo = float(np.linalg.norm(dp - dp.mean()) / np.linalg.norm(want[:, 3]))
        worst["velocity"] = max(worst["velocity"], ev)
        worst["pressure"] = max(worst["pressure"], ep)
        worst["pressure_without_offset"] = max(worst.get("pressure_without_offset", 0.0), eo)
        assert ev <= 1e-6, (k, ev)
        assert ep <= 1e-4, (k, ep)
        assert eo <= 1e-6, (k, eo)
    print("cfg2 ten steps, worst relative error", worst)
    ns.close()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cfg3_assembly_matches_oracle(precision):
    pb = P.config("cfg3")
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False, precision=precision)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    assert ns.nnz == 508_839_952
    o = oracle_for(pb, use_specializations=False)
    rp, ci = ns.csr()
    orp, oci = o.csr()
    assert np.array_equal(rp, orp) and np.array_equal(ci, oci)
    del ci, oci
    ns.assemble()
    o.assemble(os.cpu_count() or 1)
    gv, gr = ns.system()
    ov, orr = o.system()
    err, rerr = row_scaled_error(gv, ov, orp), vec_rel_error(gr, orr)
    print(f"cfg3 {precision}: row-scaled matrix error {err:.3e}, RHS {rerr:.3e}")
    if precision == "fp64":
        assert err <= 1e-11 and rerr <= 1e-11
    else:
        assert err <= 2e-5 and rerr <= 1e-4
    ns.close()
    o.close()


def test_cfg2_specialized_assembly_matches_oracle():
    """The reference's default element form (use_specializations = true, the
    closed-form tetrahedron of NavierStokesSpecializations.hpp) on the full cfg2
    mesh (64^3 x 6 tets).

    The closed form takes the tetrahedron's volume from the 24-term expansion of
    the determinant in absolute coordinates (Tetra3D.cpp:104-128): terms of
    order one cancel down to a volume of order h^3 = n^-3, so either side's
    rounding is of order eps * n^3 relative to the volume, and everything
    divided by it inherits that.  Measured against the oracle: 0.34, 0.45 and
    0.44 eps * n^3 at n = 16, 32, 64 (3.1e-13, 3.3e-12, 2.5e-11).  Bound: 4 eps
    n^3 (2.3e-10 at n = 64) for the row-scaled values and the RHS; the generic
    form, which takes coordinate differences first, stays within 1e-11 at every
    size (the tests above)."""
    pb = P.config("cfg2")
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=True)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    o = oracle_for(pb, use_specializations=True)
    ns.assemble()
    o.assemble(os.cpu_count() or 1)
    gv, gr = ns.system()
    ov, orr = o.system()
    orp, _ = o.csr()
    err, rerr = row_scaled_error(gv, ov, orp), vec_rel_error(gr, orr)
    print(f"cfg2 specialised: row-scaled matrix error {err:.3e}, RHS {rerr:.3e}")
    tol = 4 * np.finfo(np.float64).eps * 64**3
    assert err <= tol and rerr <= tol
    ns.close()
    o.close()
