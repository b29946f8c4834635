"""ctypes binding of ``libufem_b200.so`` (declared in ``include/ufem_b200.h``).

There is no fallback: if the library cannot be loaded, or no sm_100 GPU is
present when a handle is created, the call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libufem_b200.so")

UFEM_OK = 0
ERRORS = {
    -1: "UFEM_ERR_ARG", -2: "UFEM_ERR_CUDA", -3: "UFEM_ERR_MESH", -4: "UFEM_ERR_STATE",
    -5: "UFEM_ERR_NOMEM", -6: "UFEM_ERR_LIMIT", -7: "UFEM_ERR_SOLVE", -8: "UFEM_ERR_IO",
}


class UfemError(RuntimeError):
    """A negative status returned across the C ABI."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, code)}: {message}")
        self.code = code


class Mesh(C.Structure):
    _fields_ = [("dim", C.c_int32), ("reserved", C.c_int32), ("nb_nodes", C.c_int64), ("nb_elems", C.c_int64),
                ("coords", C.POINTER(C.c_double)), ("conn", C.POINTER(C.c_uint32))]


class NSOptions(C.Structure):
    _fields_ = [("theta", C.c_double), ("dt", C.c_double), ("rho", C.c_double), ("supg_type", C.c_int32),
                ("use_specializations", C.c_int32), ("c1", C.c_double), ("c2", C.c_double),
                ("alpha_ps", C.c_double), ("alpha_su", C.c_double), ("alpha_bu", C.c_double),
                ("u_ref", C.c_double), ("precision", C.c_int32), ("reserved", C.c_int32)]


class KrylovOpts(C.Structure):
    _fields_ = [("method", C.c_int32), ("restart", C.c_int32), ("max_iters", C.c_int32), ("precond", C.c_int32),
                ("tol", C.c_double), ("mixed", C.c_int32), ("max_refine", C.c_int32), ("inner_tol", C.c_double)]


class KrylovStatus(C.Structure):
    _fields_ = [("converged", C.c_int32), ("status", C.c_int32), ("iterations", C.c_int32),
                ("refinements", C.c_int32), ("rel_residual", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Timings(C.Structure):
    _fields_ = [("linearize_ms", C.c_double), ("assembly_ms", C.c_double), ("dirichlet_ms", C.c_double),
                ("solve_ms", C.c_double), ("update_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class DeviceView(C.Structure):
    _fields_ = [("rowptr", C.c_void_p), ("colidx", C.c_void_p), ("vals", C.c_void_p), ("rhs", C.c_void_p),
                ("solution", C.c_void_p), ("nb_rows", C.c_int64), ("nnz", C.c_int64)]


_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_I32 = C.POINTER(C.c_int32)
_U32 = C.POINTER(C.c_uint32)

# name -> (restype, argtypes); every symbol declared in include/ufem_b200.h
SIGNATURES = {
    "ufem_last_error": (C.c_char_p, []),
    "ufem_version": (C.c_char_p, []),
    "ufem_mesh_rectangle_tris": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_uint64, _D, _U32]),
    "ufem_mesh_cube_tets": (C.c_int, [C.c_int32, C.c_double, C.c_uint64, _D, _U32]),
    "ufem_ns_default_options": (None, [C.POINTER(NSOptions)]),
    "ufem_krylov_default_opts": (None, [C.POINTER(KrylovOpts)]),
    "ufem_ns_create": (C.c_int, [C.POINTER(Mesh), C.POINTER(NSOptions), C.POINTER(_P)]),
    "ufem_ns_create_periodic": (C.c_int, [C.POINTER(Mesh), C.POINTER(NSOptions), _U32, _U32, C.c_int64,
                                          C.POINTER(_P)]),
    "ufem_ns_set_options": (C.c_int, [_P, C.POINTER(NSOptions)]),
    "ufem_ns_sizes": (C.c_int, [_P, _I64, _I64, _I64]),
    "ufem_ns_csr": (C.c_int, [_P, _I64, _I32]),
    "ufem_ns_graph": (C.c_int, [_P, _I64, _U32]),
    "ufem_ns_set_state": (C.c_int, [_P, _D, _D, _D, _D]),
    "ufem_ns_get_state": (C.c_int, [_P, _D, _D]),
    "ufem_ns_upload_state": (C.c_int, [_P, _D, _D, _D, _D, _P]),
    "ufem_ns_download_state": (C.c_int, [_P, _D, _D, _P]),
    "ufem_ns_set_solution": (C.c_int, [_P, _D]),
    "ufem_ns_get_solution": (C.c_int, [_P, _D]),
    "ufem_ns_clear_dirichlet": (C.c_int, [_P]),
    "ufem_ns_add_dirichlet": (C.c_int, [_P, _U32, C.c_int64, C.c_int32, _D]),
    "ufem_ns_add_dirichlet_dofs": (C.c_int, [_P, _U32, _I32, _D, C.c_int64]),
    "ufem_ns_add_dirichlet_function": (C.c_int, [_P, _U32, C.c_int64, C.c_int32, C.c_char_p]),
    "ufem_ns_set_time": (C.c_int, [_P, C.c_double]),
    "ufem_ns_get_time": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "ufem_ns_add_neumann": (C.c_int, [_P, _U32, C.c_int64, C.c_int32, C.c_double]),
    "ufem_ns_clear_neumann": (C.c_int, [_P]),
    "ufem_ns_assemble": (C.c_int, [_P, _P]),
    "ufem_ns_apply_dirichlet": (C.c_int, [_P, _P]),
    "ufem_ns_solve": (C.c_int, [_P, C.POINTER(KrylovOpts), C.POINTER(KrylovStatus), _P]),
    "ufem_ns_solve_noalloc": (C.c_int, [_P, C.POINTER(KrylovOpts), C.POINTER(KrylovStatus), _P]),
    "ufem_ns_update": (C.c_int, [_P, _P]),
    "ufem_ns_fp64_residual": (C.c_int, [_P, C.POINTER(C.c_double), _P]),
    "ufem_ns_apply_device": (C.c_int, [_P, _P, _P, _P]),
    "ufem_ns_prepare_solve": (C.c_int, [_P, C.POINTER(KrylovOpts), C.c_int32]),
    "ufem_ns_step": (C.c_int, [_P, C.c_int32, C.POINTER(KrylovOpts), C.POINTER(KrylovStatus), _P]),
    "ufem_ns_write_restart": (C.c_int, [_P, C.c_char_p, C.c_double, C.c_double, C.c_int64]),
    "ufem_ns_read_restart": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                       C.POINTER(C.c_int64)]),
    "ufem_ns_stage_state": (C.c_int, [_P, _D, _D, _D, _P]),
    "ufem_ns_commit_state": (C.c_int, [_P, _P]),
    "ufem_ns_fetch_rhs": (C.c_int, [_P, _D, _P, _P]),
    "ufem_ns_get_system": (C.c_int, [_P, _D, _D]),
    "ufem_ns_download_system": (C.c_int, [_P, _D, _D, _P]),
    "ufem_ns_device_view_get": (C.c_int, [_P, C.POINTER(DeviceView)]),
    "ufem_ns_apply": (C.c_int, [_P, _D, _D]),
    "ufem_ns_set_assembly_kernel": (C.c_int, [_P, C.c_int32, C.c_int32]),
    "ufem_ns_get_assembly_kernel": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "ufem_ns_tune_assembly": (C.c_int, [_P, C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                        C.POINTER(C.c_float)]),
    "ufem_ns_device_bytes": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "ufem_batch_create": (C.c_int, [C.POINTER(_P), C.c_int32, C.POINTER(_P)]),
    "ufem_batch_size": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "ufem_batch_set_active": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "ufem_batch_set_graphs": (C.c_int, [_P, C.c_int32]),
    "ufem_batch_set_assembly_warps": (C.c_int, [_P, C.c_int32]),
    "ufem_batch_tune_assembly": (C.c_int, [_P, C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    "ufem_batch_assemble": (C.c_int, [_P, C.c_void_p]),
    "ufem_batch_solve": (C.c_int, [_P, C.POINTER(KrylovOpts), C.POINTER(KrylovStatus), C.c_void_p]),
    "ufem_batch_update": (C.c_int, [_P, C.c_void_p]),
    "ufem_batch_step": (C.c_int, [_P, C.POINTER(KrylovOpts), C.POINTER(KrylovStatus), C.c_void_p]),
    "ufem_batch_destroy": (None, [_P]),
    "ufem_ns_enable_timing": (C.c_int, [_P, C.c_int32]),
    "ufem_ns_get_timings": (C.c_int, [_P, C.POINTER(Timings)]),
    "ufem_ns_destroy": (None, [_P]),
    "ufem_nssi_create": (C.c_int, [C.POINTER(Mesh), C.POINTER(NSOptions), C.c_int32, _U32, _U32, C.c_int64,
                                   C.POINTER(_P)]),
    "ufem_nssi_set_krylov": (C.c_int, [_P, C.POINTER(KrylovOpts), C.POINTER(KrylovOpts)]),
    "ufem_nssi_set_state": (C.c_int, [_P, _D, _D, _D, _D]),
    "ufem_nssi_get_state": (C.c_int, [_P, _D, _D]),
    "ufem_nssi_add_velocity_dirichlet": (C.c_int, [_P, _U32, C.c_int64, C.c_int32, _D]),
    "ufem_nssi_add_pressure_dirichlet": (C.c_int, [_P, _U32, C.c_int64, _D]),
    "ufem_nssi_clear_dirichlet": (C.c_int, [_P]),
    "ufem_nssi_add_velocity_dirichlet_function": (C.c_int, [_P, _U32, C.c_int64, C.c_int32, C.c_char_p]),
    "ufem_nssi_add_pressure_dirichlet_function": (C.c_int, [_P, _U32, C.c_int64, C.c_char_p]),
    "ufem_nssi_set_time": (C.c_int, [_P, C.c_double]),
    "ufem_nssi_write_restart": (C.c_int, [_P, C.c_char_p, C.c_double, C.c_double, C.c_int64]),
    "ufem_nssi_read_restart": (C.c_int, [_P, C.c_char_p, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.POINTER(C.c_int64)]),
    "ufem_nssi_initialize": (C.c_int, [_P, C.c_int32, _P]),
    "ufem_nssi_step": (C.c_int, [_P, C.c_int32, C.POINTER(KrylovStatus), C.POINTER(KrylovStatus), _P]),
    "ufem_nssi_get_time": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "ufem_nssi_sizes": (C.c_int, [_P, _I64, _I64]),
    "ufem_nssi_get_system": (C.c_int, [_P, C.c_int32, _I64, _I32, _D, _D, _D]),
    "ufem_nssi_assemble_velocity_matrix": (C.c_int, [_P, _P]),
    "ufem_nssi_get_lumped_inverse": (C.c_int, [_P, _D]),
    "ufem_nssi_device_bytes": (C.c_int64, [_P]),
    "ufem_nssi_destroy": (None, [_P]),
}

_lib = None


def lib() -> C.CDLL:
    """Load the native library (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing; build it with `python -m coolfluid3_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != UFEM_OK:
        raise UfemError(rc, lib().ufem_last_error().decode())


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, "expected a C-contiguous float64 array"
    return a.ctypes.data_as(_D)


def u32ptr(a: np.ndarray):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(_U32)


def i32ptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I32)


def i64ptr(a: np.ndarray):
    assert a.dtype == np.int64 and a.flags.c_contiguous
    return a.ctypes.data_as(_I64)


def raw_dptr(addr: int):
    """A float64 pointer from a raw address (e.g. a pinned torch tensor's data_ptr())."""
    return C.cast(C.c_void_p(addr), _D)
