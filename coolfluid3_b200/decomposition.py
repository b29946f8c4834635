"""One mesh over several GPUs: node partition, one element overlap layer, halo
exchange before each SpMV and all-reduced dot products.

The reference distributes a mesh over MPI ranks: global ids of the nodes across
ranks (SparsityBuilder.cpp:71-155), every rank assembles the elements touching
its nodes and keeps only its own block rows (TrilinosFEVbrMatrix.cpp:242, 280,
301: ``if (idxs[irow] < m_blockrow_size)``), and the ghost values are
synchronised after each loop (common/PE/CommPattern.cpp:567-599).  Here:

* ``partition``: rank r owns a contiguous range of node ids (balanced counts).
  Its local mesh holds every element with at least one owned node (the
  overlap layer); its local nodes are the owned ones (ascending global id)
  followed by the ghosts (ascending global id).  Each owned row of the local
  system then has all its elements, in the same element order, so it equals the
  single-mesh row value for value.  Ghost rows are incomplete and never used.
* The ordered Dirichlet list is filtered to the local nodes (order kept): an
  owned row moves its constrained ghost columns exactly as the single mesh does.
* ``DistributedNS.solve``: BiCGStab with point Jacobi on the owned rows.  Before
  each SpMV the ghost values are fetched from their owners
  (``torch.distributed`` point-to-point: NCCL between GPUs, gloo on CPU; device
  vectors under gloo travel through host copies) into the local vector; dot
  products are local sums all-reduced over the ranks.
* A local engine does the per-rank work.  ``GPUEngine`` is a ``NavierStokes``
  handle on the local mesh whose vectors stay in device memory (the SpMV is the
  library's, ``ufem_ns_apply_device``); any object with the same methods can
  stand in (the CPU tests use the FP64 oracle).  Ghost values arrive in each
  GPU's own memory before the SpMV reads them; no kernel reads another GPU's
  memory.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class LocalPart:
    """One rank's share of a partitioned mesh (all ids are global unless named local)."""
    rank: int
    node_range: tuple[int, int]   # owned nodes [n0, n1)
    elems: np.ndarray             # local elements (global ids, ascending)
    nodes: np.ndarray             # local nodes: owned then ghosts (global ids)
    conn: np.ndarray              # local connectivity (local node ids)
    recv: dict                    # peer -> local positions of the ghosts it owns (in ghost order)
    send: dict                    # peer -> local positions of my owned nodes it needs (in its ghost order)

    @property
    def nb_owned(self) -> int:
        return self.node_range[1] - self.node_range[0]


def node_ranges(nb_nodes: int, world: int) -> list[tuple[int, int]]:
    """Contiguous node ranges of near-equal size, one per rank."""
    cuts = [(nb_nodes * r) // world for r in range(world + 1)]
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def partition(conn: np.ndarray, nb_nodes: int, world: int) -> list[LocalPart]:
    """Partition of the nodes into `world` ranges with one element overlap layer."""
    conn = np.asarray(conn, np.int64)
    ranges = node_ranges(nb_nodes, world)
    owner = np.empty(nb_nodes, np.int64)
    for r, (a, b) in enumerate(ranges):
        owner[a:b] = r
    parts = []
    ghosts_of = []
    for r, (a, b) in enumerate(ranges):
        touch = ((conn >= a) & (conn < b)).any(axis=1)
        elems = np.nonzero(touch)[0]
        used = np.unique(conn[elems])
        ghosts = used[(used < a) | (used >= b)]
        nodes = np.concatenate([np.arange(a, b, dtype=np.int64), ghosts])
        local = np.full(nb_nodes, -1, np.int64)
        local[nodes] = np.arange(len(nodes))
        lconn = local[conn[elems]].astype(np.uint32)
        recv = {}
        for p in np.unique(owner[ghosts]) if len(ghosts) else []:
            recv[int(p)] = (b - a) + np.nonzero(owner[ghosts] == p)[0]
        parts.append(LocalPart(r, (a, b), elems, nodes, np.ascontiguousarray(lconn), recv, {}))
        ghosts_of.append(ghosts)
    for r, (a, b) in enumerate(ranges):  # what each peer needs from r, in that peer's ghost order
        for p in range(world):
            if p == r:
                continue
            g = ghosts_of[p]
            need = g[(g >= a) & (g < b)]
            if len(need):
                parts[r].send[p] = need - a
    return parts


def local_dirichlet(part: LocalPart, nb_nodes: int, nodes, comps, values):
    """The ordered Dirichlet list restricted to the part's local nodes (order kept),
    in local node ids."""
    nodes = np.asarray(nodes, np.int64)
    local = np.full(nb_nodes, -1, np.int64)
    local[part.nodes] = np.arange(len(part.nodes))
    keep = local[nodes] >= 0
    comps = np.broadcast_to(np.asarray(comps, np.int32), nodes.shape)[keep]
    values = np.broadcast_to(np.asarray(values, np.float64), nodes.shape)[keep]
    return local[nodes[keep]].astype(np.uint32), np.ascontiguousarray(comps), np.ascontiguousarray(values)


def _dofs(pos: np.ndarray, neq: int) -> np.ndarray:
    return (np.asarray(pos, np.int64)[:, None] * neq + np.arange(neq)).ravel()


class Halo:
    """Ghost exchange of a local dof vector: every rank sends the owned values its
    peers hold as ghosts and overwrites its ghost rows with its owners' values
    (CommPattern::synchronize)."""

    def __init__(self, part: LocalPart, neq: int, device):
        import torch
        self.send = {p: torch.as_tensor(_dofs(pos, neq), device=device) for p, pos in sorted(part.send.items())}
        self.recv = {p: torch.as_tensor(_dofs(pos, neq), device=device) for p, pos in sorted(part.recv.items())}

    def exchange(self, x) -> None:
        import torch
        import torch.distributed as dist
        if not self.send and not self.recv:
            return
        # gloo moves host memory only: device vectors go through host copies
        wire = torch.device("cpu") if _host_wire(x) else x.device
        ops, inbox, outbox = [], {}, []
        for p, idx in self.send.items():
            buf = x[idx].to(wire).contiguous()
            outbox.append(buf)
            ops.append(dist.P2POp(dist.isend, buf, p))
        for p, idx in self.recv.items():
            buf = torch.empty(len(idx), dtype=x.dtype, device=wire)
            inbox[p] = buf
            ops.append(dist.P2POp(dist.irecv, buf, p))
        for req in dist.batch_isend_irecv(ops):
            req.wait()
        for p, buf in inbox.items():
            x[self.recv[p]] = buf.to(x.device)


def _host_wire(x) -> bool:
    """True when x lives in device memory and the process group is gloo."""
    import torch.distributed as dist
    return x.device.type != "cpu" and dist.is_initialized() and dist.get_backend() == "gloo"


def _allreduce(vals):
    """Sum over the ranks of a few local partial sums (one collective)."""
    import torch
    import torch.distributed as dist
    t = torch.stack([v.reshape(()) for v in vals]).to(torch.float64)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        if _host_wire(t):
            t = t.cpu()
        dist.all_reduce(t)
    return t


class DistributedNS:
    """A NavierStokes action whose mesh is split over the ranks of the default
    process group (rank r of world W holds part r).  engine_factory(coords,
    conn, **options) builds the per-rank engine on the local mesh."""

    def __init__(self, coords, conn, engine_factory, *, rank: int, world: int, **options):
        coords = np.ascontiguousarray(coords, np.float64)
        self.nb_nodes = coords.shape[0]
        self.dim = coords.shape[1]
        self.neq = self.dim + 1
        self.parts = partition(conn, self.nb_nodes, world)
        self.part = self.parts[rank]
        self.engine = engine_factory(np.ascontiguousarray(coords[self.part.nodes]), self.part.conn, **options)
        self.m = self.part.nb_owned * self.neq  # owned rows come first in the local numbering
        self.halo = Halo(self.part, self.neq, self.engine.device)

    # -- inputs (global arrays; each rank keeps its local nodes) ---------------
    def set_state(self, up, lin, nu) -> None:
        n = self.part.nodes
        self.engine.set_state(np.ascontiguousarray(up[n]), np.ascontiguousarray(lin[n]), np.ascontiguousarray(nu[n]))

    def add_dirichlet(self, nodes, comps, values) -> None:
        self.engine.add_dirichlet(*local_dirichlet(self.part, self.nb_nodes, nodes, comps, values))

    # -- one time step ----------------------------------------------------------
    def assemble(self) -> None:
        """ZeroLSS + LinearizeU + assembly + symmetric Dirichlet on the local mesh;
        the owned rows are the single mesh's rows."""
        self.engine.assemble()
        self.engine.apply_dirichlet()

    def _apply(self, v):
        import torch
        xl = torch.zeros(self.engine.nb_rows, dtype=torch.float64, device=self.engine.device)
        xl[: self.m] = v
        self.halo.exchange(xl)
        return self.engine.spmv(xl)[: self.m]

    def _bicgstab(self, x, b, dinv, bnorm, tol, max_iters):
        """One BiCGStab run from x; returns (x, iterations, status)."""
        import torch
        r = b - self._apply(x)
        rhat = r.clone()
        relres = float(_allreduce([r @ r])[0]) ** 0.5 / bnorm
        p = torch.zeros_like(r)
        v = torch.zeros_like(r)
        rho = alpha = omega = 1.0
        it, status = 0, 0
        while relres > tol and it < max_iters:
            rho_new = float(_allreduce([rhat @ r])[0])
            if rho_new == 0.0 or omega == 0.0:
                status = 2  # breakdown: the caller restarts from x
                break
            beta = (rho_new / rho) * (alpha / omega)
            p = r + beta * (p - omega * v)
            ph = dinv * p
            v = self._apply(ph)
            alpha = rho_new / float(_allreduce([rhat @ v])[0])
            s = r - alpha * v
            sh = dinv * s
            t = self._apply(sh)
            ts, tt = _allreduce([t @ s, t @ t]).tolist()
            omega = ts / tt if tt > 0 else 0.0
            x = x + alpha * ph + omega * sh
            r = s - omega * t
            rho = rho_new
            it += 1
            relres = float(_allreduce([r @ r])[0]) ** 0.5 / bnorm
            if not np.isfinite(relres):
                status = 3
                break
        return x, it, status

    def solve(self, tol: float = 1e-10, max_iters: int = 3000, max_restarts: int = 10) -> dict:
        """Point-Jacobi BiCGStab on the owned rows; the initial guess is the
        engine's solution vector (the previous increment, with the condition
        values in the constrained rows).  Convergence is decided on the true
        residual: after a breakdown, or when the recursive residual met the
        tolerance while the true one had drifted above it, BiCGStab restarts
        from its iterate while iterations remain (as the library's solve)."""
        import torch
        m = self.m
        x = self.engine.solution()[:m].clone()
        b = self.engine.rhs()[:m].clone()
        d = self.engine.diag()[:m]
        dinv = torch.where(d != 0, 1.0 / d, torch.ones_like(d))
        bn2 = float(_allreduce([b @ b])[0])
        bnorm = bn2 ** 0.5 if bn2 > 0 else 1.0
        used, status = 0, 0
        for _ in range(max_restarts + 1):
            x, it, status = self._bicgstab(x, b, dinv, bnorm, tol, max_iters - used)
            used += it
            true = b - self._apply(x)
            relres = float(_allreduce([true @ true])[0]) ** 0.5 / bnorm
            if relres <= tol or status == 3 or not np.isfinite(relres) or used >= max_iters:
                break
        xl = torch.zeros(self.engine.nb_rows, dtype=torch.float64, device=self.engine.device)
        xl[:m] = x
        self.halo.exchange(xl)  # ghosts take their owners' increments
        self.engine.set_solution(xl)
        conv = bool(relres <= tol)
        return {"converged": int(conv), "iterations": used, "rel_residual": relres,
                "status": 0 if conv else (status if status else 1)}

    def update(self) -> None:
        self.engine.update()

    def step(self, nsteps: int = 1, **krylov) -> dict:
        st = {}
        for _ in range(nsteps):
            self.assemble()
            st = self.solve(**krylov)
            self.update()
        return st

    # -- results ------------------------------------------------------------------
    def owned_state(self) -> tuple[np.ndarray, np.ndarray]:
        """(global node ids, state rows) of the owned nodes."""
        up = self.engine.state()
        return self.part.nodes[: self.part.nb_owned], up[: self.part.nb_owned]

    def owned_system(self):
        """Owned rows of the assembled system as (global row, global column, value)
        triples and the owned RHS (global row order)."""
        rp, ci, vals, rhs = self.engine.system_csr()
        neq = self.neq
        rows = np.repeat(np.arange(self.m), np.diff(rp[: self.m + 1]))
        gcol_node = self.part.nodes[ci[: rp[self.m]] // neq]
        gcols = gcol_node * neq + ci[: rp[self.m]] % neq
        grow = self.part.nodes[rows // neq] * neq + rows % neq
        return grow, gcols, vals[: rp[self.m]], rhs[: self.m]


class _CudaArray:
    """A device buffer of the library seen by torch without a copy."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (int(ptr), False), "version": 3}


class GPUEngine:
    """The per-rank engine of DistributedNS on a GPU: a NavierStokes handle on the
    local mesh; vectors stay in device memory and the SpMV is the library's."""

    def __init__(self, coords, conn, **options):
        import torch

        from .ufem import NavierStokes
        self.ns = NavierStokes(coords, conn, **options)
        self.device = torch.device("cuda", torch.cuda.current_device())
        self.nb_rows = self.ns.nb_rows
        rp, ci = self.ns.csr()
        rows = np.repeat(np.arange(self.nb_rows), np.diff(rp))
        self.diagpos = torch.as_tensor(np.nonzero(ci == rows)[0], device=self.device)
        view = self.ns.device_view()
        self._vals = torch.as_tensor(_CudaArray(view["vals"], int(rp[-1])), device=self.device)
        self._rhs = torch.as_tensor(_CudaArray(view["rhs"], self.nb_rows), device=self.device)
        self._sol = torch.as_tensor(_CudaArray(view["solution"], self.nb_rows), device=self.device)

    def set_state(self, up, lin, nu):
        self.ns.set_state(up, lin, nu)

    def add_dirichlet(self, nodes, comps, values):
        self.ns.add_dirichlet(nodes, comps, values)

    def assemble(self):
        self.ns.assemble()

    def apply_dirichlet(self):
        self.ns.apply_dirichlet()

    def spmv(self, x):
        import torch

        from . import _native as N
        x = x.contiguous()
        y = torch.empty_like(x)
        N.check(N.lib().ufem_ns_apply_device(self.ns.handle, N.C.c_void_p(x.data_ptr()), N.C.c_void_p(y.data_ptr()),
                                             N.C.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return y

    def rhs(self):
        return self._rhs

    def diag(self):
        return self._vals[self.diagpos]

    def solution(self):
        return self._sol

    def set_solution(self, x):
        self._sol.copy_(x)

    def update(self):
        import torch
        torch.cuda.current_stream().synchronize()
        self.ns.update()

    def state(self):
        return self.ns.state()[0]

    def system_csr(self):
        rp, ci = self.ns.csr()
        vals, rhs = self.ns.system()
        return rp, ci, vals, rhs

    def close(self):
        self.ns.close()
