"""CPU tests of the C-ABI library: it loads, exports every declared symbol, and
its host-side validation and fixtures behave -- no kernel is launched here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from coolfluid3_b200 import _native as N
from coolfluid3_b200 import problems as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ufem_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ufem_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    lib = N.lib()
    for n in names:
        assert hasattr(lib, n)
    # the Python binding covers the whole header
    assert set(names) == set(N.SIGNATURES)


@pytest.mark.parametrize("lang,std", [("c", "-std=c99"), ("c++", "-std=c++17")])
def test_header_is_plain_c(tmp_path, lang, std):
    """The boundary header compiles as ISO C99 and as C++ without warnings: plain
    pointers, sizes and status codes, no CUDA or torch types."""
    src = tmp_path / "use_header.c"
    src.write_text('#include "ufem_b200.h"\nint main(void) { ufem_ns_handle* a = 0; ufem_nssi_handle* b = 0; '
                   'ufem_batch* c = 0; (void)a; (void)b; (void)c; return 0; }\n')
    cc = "gcc" if lang == "c" else "g++"
    proc = subprocess.run([cc, std, "-Wall", "-Wextra", "-Werror", "-pedantic", "-x", lang, "-c", str(src),
                           "-I", os.path.dirname(HEADER), "-o", str(tmp_path / "o.o")], capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr
    includes = re.findall(r"#include\s*[<\"]([^>\"]+)", open(HEADER).read())
    assert all(not i.startswith(("cuda", "torch", "ATen")) for i in includes), includes


def test_version_and_defaults():
    lib = N.lib()
    assert b"sm_100a" in lib.ufem_version()
    o = N.NSOptions()
    lib.ufem_ns_default_options(C.byref(o))
    # NavierStokes.cpp:74-98 and SUPG.hpp:94-104 defaults
    assert (o.theta, o.supg_type, o.use_specializations, o.c1, o.c2) == (1.0, 1, 1, 1.0, 16.0)
    assert (o.alpha_ps, o.alpha_su, o.alpha_bu, o.precision) == (1.0, 1.0, 1.0, 0)
    k = N.KrylovOpts()
    lib.ufem_krylov_default_opts(C.byref(k))
    assert (k.method, k.restart, k.max_iters, k.precond, k.tol) == (1, 30, 3000, 1, 1e-10)


def _create(coords, conn, **over):
    lib = N.lib()
    o = N.NSOptions()
    lib.ufem_ns_default_options(C.byref(o))
    for k, v in over.items():
        setattr(o, k, v)
    coords = np.ascontiguousarray(coords, np.float64)
    conn = np.ascontiguousarray(conn, np.uint32)
    mesh = N.Mesh(coords.shape[1], 0, coords.shape[0], conn.shape[0], N.dptr(coords), N.u32ptr(conn))
    h = C.c_void_p()
    rc = lib.ufem_ns_create(C.byref(mesh), C.byref(o), C.byref(h))
    if rc == 0:
        lib.ufem_ns_destroy(h)
    return rc, lib.ufem_last_error().decode()


def test_option_validation_matches_reference_rules():
    c, e = P.rectangle_tris(2)
    rc, msg = _create(c, e, theta=1.5)  # NavierStokesAssembly.hpp:38-40
    assert rc == -1 and "theta" in msg
    rc, msg = _create(c, e, supg_type=7)
    assert rc == -1 and "supg_type" in msg
    rc, msg = _create(c, e, dt=0.0)
    assert rc == -1


def test_mesh_validation():
    c, e = P.rectangle_tris(2)
    bad = e.copy()
    bad[3, 1] = 999
    rc, msg = _create(c, bad)
    assert rc == -3 and "node id" in msg
    deg = e.copy()
    deg[2] = [deg[2, 0], deg[2, 0], deg[2, 1]]  # collapsed element, det J = 0
    rc, msg = _create(c, deg)
    assert rc == -3 and "Jacobian" in msg
    extra = np.vstack([c, [[0.5, 0.5]]])  # a node no element uses
    rc, msg = _create(extra, e)
    assert rc == -3 and "not referenced" in msg


def _gpu_present() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_gpu_present(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback_without_gpu():
    c, e = P.rectangle_tris(3)
    rc, msg = _create(c, e)
    assert rc == -2, msg  # UFEM_ERR_CUDA: there is no CPU path


def test_lid_driven_bc_list_order():
    """Walls then lid, each node listing u, v[, w] in turn; pressure pin last."""
    n = 3
    nodes, comps, vals = P.lid_driven_bcs(2, n)
    i, j = P.structured_index(2, n)
    left = np.nonzero(i == 0)[0]
    assert list(nodes[: 2 * len(left)]) == list(np.repeat(left, 2))
    assert list(comps[:4]) == [0, 1, 0, 1]
    top = np.nonzero(j == n)[0]
    tail = slice(len(nodes) - 1 - 2 * len(top), len(nodes) - 1)
    assert list(nodes[tail]) == list(np.repeat(top, 2))
    assert np.all(vals[tail][comps[tail] == 0] == 1.0) and np.all(vals[tail][comps[tail] == 1] == 0.0)
    assert (nodes[-1], comps[-1], vals[-1]) == (0, 2, 0.0)
    n3, c3, v3 = P.lid_driven_bcs(3, 2)
    assert set(np.unique(c3)) == {0, 1, 2, 3} and c3[-1] == 3


def test_config_shapes():
    pb = P.make_problem(3, 4)
    assert pb.coords.shape == (125, 3) and pb.conn.shape == (384, 4)
    assert pb.up.shape == (125, 4) and pb.lin.shape == (125, 12)
    np.testing.assert_array_equal(pb.lin[:, :3], pb.up[:, :3])
    np.testing.assert_array_equal(pb.lin[:, 9:], pb.up[:, :3])
    assert np.abs(pb.up[:, :3]).max() <= 1.0


def _create_raw(dim, nb_nodes, nb_elems, coords, conn):
    lib = N.lib()
    o = N.NSOptions()
    lib.ufem_ns_default_options(C.byref(o))
    mesh = N.Mesh(dim, 0, nb_nodes, nb_elems, coords, conn)
    h = C.c_void_p()
    rc = lib.ufem_ns_create(C.byref(mesh), C.byref(o), C.byref(h))
    if rc == 0:
        lib.ufem_ns_destroy(h)
    return rc, lib.ufem_last_error().decode()


def test_empty_invalid_and_oversized_meshes_are_refused_before_any_device_work():
    c, e = P.rectangle_tris(2)
    c = np.ascontiguousarray(c, np.float64)
    e = np.ascontiguousarray(e, np.uint32)
    cp, ep = N.dptr(c), N.u32ptr(e)
    rc, msg = _create_raw(2, c.shape[0], 0, cp, ep)  # no elements
    assert rc == -1 and "empty" in msg
    rc, msg = _create_raw(2, 0, e.shape[0], cp, ep)  # no nodes
    assert rc == -1 and "empty" in msg
    rc, msg = _create_raw(4, c.shape[0], e.shape[0], cp, ep)  # only Triag2D and Tetra3D
    assert rc == -1 and "dim" in msg
    rc, msg = _create_raw(2, c.shape[0], e.shape[0], None, ep)
    assert rc == -1 and "NULL" in msg
    # 2^29 tetrahedra: 2^31 incidences overflow the 32-bit incidence and column
    # indices; refused from the sizes alone (the arrays are not read)
    t = np.zeros((1, 4), np.uint32)
    x = np.zeros((4, 3))
    rc, msg = _create_raw(3, 4, 1 << 29, N.dptr(x), N.u32ptr(t))
    assert rc == -6 and "32-bit" in msg
