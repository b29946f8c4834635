"""GPU tests of the assembly kernel variants and the assembly autotuner.

Every variant (warp per row group with 2, 4 or 8 warps per CTA, and the chunk
kernel) sums each CSR value over the same contributions in the same element
order.  The element routines are compiled into each kernel instantiation
separately, so the compiler may contract a different set of multiply-adds:
the variants agree to rounding level (1e-14 of each row's largest entry with
FP64 element arithmetic, 1e-6 with FP32), and each one is deterministic
(bitwise equal results on repeated launches).  Fan meshes put
more than 32 elements around one node, which sends that row to the chunk
kernel inside the warp variant; those systems are also checked against the
FP64 oracle (1e-11 of each row's largest entry).
"""
import numpy as np
import pytest

import oracle as O
from coolfluid3_b200 import NavierStokes
from coolfluid3_b200 import problems as P

from .util import row_scaled_error, small_problem, vec_rel_error

pytestmark = pytest.mark.gpu

VARIANTS = [("warp", 2), ("warp", 4), ("warp", 8), ("chunk", 4)]
VARIANTS_3D = VARIANTS + [("warp24", 2), ("warp24", 4)]


def variants(dim):
    return VARIANTS_3D if dim == 3 else VARIANTS


def fan_mesh(dim: int, m: int):
    """A node surrounded by many elements: 2D, m triangles around node 0;
    3D, 2m tetrahedra around node 0 (a ring of m nodes, an apex above and below)."""
    ang = 2 * np.pi * np.arange(m) / m
    if dim == 2:
        coords = np.vstack([[0.0, 0.0], np.c_[np.cos(ang), np.sin(ang)]])
        conn = np.array([[0, 1 + i, 1 + (i + 1) % m] for i in range(m)], np.uint32)
    else:
        ring = np.c_[np.cos(ang), np.sin(ang), 0.05 * np.sin(3 * ang)]
        coords = np.vstack([[0.0, 0.0, 0.02], ring, [0.1, 0.0, 1.0], [0.0, -0.1, -1.0]])
        top, bot = m + 1, m + 2
        tets = []
        for i in range(m):
            a, b = 1 + i, 1 + (i + 1) % m
            tets += [[0, a, b, top], [0, b, a, bot]]
        conn = np.array(tets, np.uint32)
        for t in conn:  # positive orientation
            x = coords[t]
            if np.linalg.det((x[1:] - x[0])) < 0:
                t[[1, 2]] = t[[2, 1]]
    return coords, conn


def fan_state(coords, seed=3):
    rng = np.random.default_rng(seed)
    npts, dim = coords.shape
    u = np.sin(coords @ rng.normal(size=(dim, dim)) + rng.normal(size=dim))
    up, lin, nu = P.initial_fields(u, 1e-2, rng.normal(size=npts))
    lin[:, dim:] += 0.1 * rng.normal(size=(npts, 3 * dim))  # distinct u1, u2, u3
    return up, lin, nu


def assembled(ns, variant, warps):
    ns.set_assembly_kernel(variant, warps)
    ns.assemble()
    return ns.system()


@pytest.mark.parametrize("dim,n", [(2, 12), (3, 5)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("spec", [False, True])
def test_variants_agree_and_are_deterministic(dim, n, precision, spec):
    pb = small_problem(dim, n)
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=spec, precision=precision)
    ns.set_state(pb.up, pb.lin, pb.nu)
    rp, _ = ns.csr()
    tol = 1e-14 if precision == "fp64" else 1e-6
    ref_v, ref_r = assembled(ns, "warp", 4)
    for variant, warps in variants(dim):
        v, r = assembled(ns, variant, warps)
        assert row_scaled_error(v, ref_v, rp) <= tol, (variant, warps)
        assert vec_rel_error(r, ref_r) <= tol, (variant, warps)
        v2, r2 = assembled(ns, variant, warps)
        assert np.array_equal(v, v2) and np.array_equal(r, r2), (variant, warps)


@pytest.mark.parametrize("dim,m", [(2, 40), (3, 20), (3, 30)])
@pytest.mark.parametrize("spec", [False, True])
def test_fan_mesh_rows_above_32_elements(dim, m, spec):
    coords, conn = fan_mesh(dim, m)
    up, lin, nu = fan_state(coords)
    ns = NavierStokes(coords, conn, dt=0.01, use_specializations=spec)
    ns.set_state(up, lin, nu)
    o = O.Oracle(coords, conn, O.options(dt=0.01, use_specializations=spec))
    o.set_state(up, lin, nu)
    o.assemble()
    ov, orr = o.system()
    rp, _ = o.csr()
    for variant, warps in variants(dim):
        v, r = assembled(ns, variant, warps)
        assert row_scaled_error(v, ov, rp) <= 1e-11, (variant, warps)
        assert vec_rel_error(r, orr) <= 1e-11, (variant, warps)


def test_autotuner_picks_a_candidate_and_keeps_results():
    pb = small_problem(3, 8)
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.assemble()
    v0, r0 = ns.system()
    res = ns.tune_assembly(reps=3)
    assert (res["variant"], res["warps_per_cta"]) in VARIANTS_3D and res["ms"] > 0
    assert ns.assembly_kernel() == (res["variant"], res["warps_per_cta"])
    ns.assemble()
    v1, r1 = ns.system()
    rp, _ = ns.csr()
    assert row_scaled_error(v1, v0, rp) <= 1e-14 and vec_rel_error(r1, r0) <= 1e-14
    ns.assemble()
    v2, r2 = ns.system()
    assert np.array_equal(v1, v2) and np.array_equal(r1, r2)  # deterministic once chosen
