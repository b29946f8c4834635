"""Shared helpers of the parity tests."""
from __future__ import annotations

import numpy as np

import oracle as O
from coolfluid3_b200 import problems as P


def row_scaled_error(got: np.ndarray, ref: np.ndarray, rowptr: np.ndarray) -> float:
    """max over entries of |got - ref| / max|ref| of the entry's CSR row."""
    scale = np.maximum.reduceat(np.abs(ref), rowptr[:-1])
    counts = np.diff(rowptr)
    scale = np.repeat(np.where(scale > 0, scale, 1.0), counts)
    return float(np.max(np.abs(got - ref) / scale)) if got.size else 0.0


def vec_rel_error(got: np.ndarray, ref: np.ndarray) -> float:
    n = np.linalg.norm(ref)
    return float(np.linalg.norm(got - ref) / (n if n > 0 else 1.0))


def small_problem(dim: int, n: int, **kw) -> P.Problem:
    return P.make_problem(dim, n, **kw)


def oracle_for(pb: P.Problem, **opt) -> O.Oracle:
    o = O.Oracle(pb.coords, pb.conn, O.options(dt=pb.dt, rho=pb.rho, theta=pb.theta, **opt))
    o.set_state(pb.up, pb.lin, pb.nu)
    o.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    return o


def csr_matrix(rowptr, colidx, vals, n):
    import scipy.sparse as sp
    return sp.csr_matrix((vals, colidx, rowptr), shape=(n, n))
