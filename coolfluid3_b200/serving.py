"""Serving loop: time-stepping solves of different sizes on one GPU.

Requests (a mesh, initial fields, Dirichlet list, time step and a number of
steps) arrive over time.  The server

  * admits them by HBM budget: a request is admitted when a slot is free and
    its estimated device footprint fits the remaining budget (first fit in
    arrival order); the estimate is replaced by the handle's actual footprint
    once it exists, and released when the request completes;
  * builds each admitted request's handle (mesh plan, CSR pattern, fields)
    on a pool of host threads while the GPU keeps stepping the others, and
    keeps mesh, pattern and state resident on the device until the request
    completes;
  * batches continuously: requests below `large_rows` rows are stepped
    together by one worker per mesh dimension every tick (one batched
    assembly launch, one batched BiCGStab with per-request scalars, see
    ``ufem.Batch``); larger requests, whose solves already fill the GPU, run
    one per worker on `large_workers` further workers so that they do not hold
    back the small ones.  Every worker has its own CUDA stream, so the classes
    overlap on the device (the batching workers' streams have the higher
    priority: their kernels are short and latency-bound, the large requests'
    are bandwidth-bound and fill the gaps); requests that arrive while others
    run join at the next tick (the batch is rebuilt with them); finished ones
    are held in place (``Batch.set_active``) and leave at the next rebuild, so
    a finish does not stall the other members;
  * frees the handles of finished requests lazily (when admission waits for
    memory, when no admitted request is left, and at the end): a free
    synchronises the device and would stall the requests still running;
  * in the mixed form, the large requests assemble FP32 element matrices and
    refine their FP32 inner solves against the matrix-free FP64 residual, so
    their answers stay the FP64 system's;
  * reports throughput (time steps per second) beside p50/p99 step latency
    and request latency.

Because a batch member's arithmetic does not depend on the other members, a
request's results are bitwise the same whether it ran alone or in the mix.

``run_plain`` is the reference point: the same requests, one at a time, each
through the plain FP64 one-handle path (``NavierStokes.execute``).
"""
from __future__ import annotations

import math
import threading
import time
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import problems as P
from .ufem import Batch, NavierStokes


@dataclass
class Request:
    rid: int
    coords: np.ndarray
    conn: np.ndarray
    up: np.ndarray
    lin: np.ndarray
    nu: np.ndarray
    bc_nodes: np.ndarray
    bc_comps: np.ndarray
    bc_values: np.ndarray
    dt: float
    nsteps: int
    arrival: float = 0.0  # seconds after the start of the run

    @property
    def dim(self) -> int:
        return self.coords.shape[1]

    @property
    def nb_elems(self) -> int:
        return self.conn.shape[0]


@dataclass
class Result:
    rid: int
    state: np.ndarray | None
    step_ms: list = field(default_factory=list)
    statuses: list = field(default_factory=list)
    arrival: float = 0.0
    admitted: float = 0.0
    ready: float = 0.0     # handle built (device state resident)
    started: float = 0.0   # first time step began
    finished: float = 0.0
    error: str | None = None  # a request rejected at set-up (bad mesh or fields)

    @property
    def ok(self) -> bool:
        return self.error is None and all(s.get("converged", 0) for s in self.statuses)


def estimate_bytes(req: Request, precision: str = "fp64") -> int:
    """Device footprint of a request before its handle exists (P1 meshes:
    about 7 (2D) or 15 (3D) graph neighbours per node, plus 30% margin)."""
    n_nodes, n_elems, dim = len(req.coords), len(req.conn), req.dim
    neq = dim + 1
    bnnz = int(1.3 * n_nodes * (7 if dim == 2 else 15))
    nnz = bnnz * neq * neq
    rows = n_nodes * neq
    per_value = 16  # FP64 values, column indices, FP32 operator copy
    # node records (FP64 state, history, u_adv, coordinates, and the FP32 mirror
    # of FP32 element arithmetic), incidences, graph, values, solver vectors
    return n_nodes * 288 + n_elems * 40 + bnnz * 4 + nnz * per_value + rows * 8 * 16


def make_request(rid: int, dim: int, n_elems: float, nu: float, seed: int, nsteps: int = 10,
                 arrival: float = 0.0) -> Request:
    """A lid-driven cavity request on the structured generators, sized to
    about n_elems elements (2D: 2 s^2 triangles, 3D: 6 s^3 tetrahedra)."""
    if dim == 2:
        s = max(2, int(round(math.sqrt(n_elems / 2.0))))
        dt = 0.01
    else:
        s = max(2, int(round((n_elems / 6.0) ** (1.0 / 3.0))))
        dt = 5e-3
    pb = P.make_problem(dim, s, nu=nu, dt=dt, seed=seed)
    return Request(rid, pb.coords, pb.conn, pb.up, pb.lin, pb.nu, pb.bc_nodes, pb.bc_comps, pb.bc_values, dt,
                   nsteps, arrival)


def poisson_workload(n: int, rate: float, elems=(1e4, 2e6), nu=(1e-4, 1e-1), dims=(2, 3), nsteps: int = 10,
                     seed: int = 20261203) -> list[Request]:
    """Seeded synthetic serving workload: Poisson arrivals at `rate` per second,
    element counts and viscosities log-uniform, dimensions drawn uniformly.
    `elems` is one (low, high) range or a {dim: (low, high)} mapping."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        dim = int(rng.choice(dims))
        lo, hi = elems[dim] if isinstance(elems, dict) else elems
        e = math.exp(rng.uniform(math.log(lo), math.log(hi)))
        v = math.exp(rng.uniform(math.log(nu[0]), math.log(nu[1])))
        out.append(make_request(k, dim, e, v, seed + 7 * k + 1, nsteps, t))
    return out


def _percentiles(xs) -> dict:
    if not xs:
        return {"p50": None, "p99": None, "mean": None}
    a = np.asarray(xs, np.float64)
    return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)), "mean": float(a.mean())}


def summarize(results: list[Result], t_start: float, t_end: float) -> dict:
    steps = sum(len(r.step_ms) for r in results if r.error is None)
    span = max(t_end - t_start, 1e-9)
    return {
        "requests": len(results),
        "steps": steps,
        "seconds": span,
        "steps_per_s": steps / span,
        "step_ms": _percentiles([x for r in results for x in r.step_ms]),
        "request_s": _percentiles([r.finished - r.arrival for r in results if r.error is None]),
        "rejected": sum(1 for r in results if r.error is not None),
    }


def _new_handle(req: Request, precision: str, use_specializations: bool) -> NavierStokes:
    ns = NavierStokes(req.coords, req.conn, dt=req.dt, use_specializations=use_specializations, precision=precision)
    ns.set_state(req.up, req.lin, req.nu)
    ns.add_dirichlet(req.bc_nodes, req.bc_comps, req.bc_values)
    return ns


class _Active:
    def __init__(self, req: Request, ns: NavierStokes, admitted: float, reserved: int):
        self.req = req
        self.ns = ns
        self.reserved = reserved
        self.result = Result(req.rid, None, arrival=req.arrival, admitted=admitted)
        self.done_steps = 0


class Server:
    """Continuous-batching server for one GPU (see the module docstring)."""

    def __init__(self, hbm_budget_bytes: int, max_slots: int = 64, precision: str = "fp64", mixed: bool = True,
                 krylov: dict | None = None, graphs: bool = True, creators: int | None = None,
                 use_specializations: bool = False, realtime: bool = True, large_rows: int = 200_000,
                 large_workers: int = 2, small_priority: bool = True, mixed_scope: str = "elements",
                 large_precond: str = "jacobi", large_rows_2d: int | None = None, small_precond: str = "jacobi"):
        """mixed: the mixed-precision form.  Requests of at least `large_rows`
        rows (stepped one at a time by the large workers; their solves are
        bandwidth-bound) assemble FP32 element matrices and solve with FP32
        inner BiCGStab refined against the matrix-free FP64 residual, so their
        answers are the FP64 system's.  With mixed_scope "elements" (default)
        the batched small requests also assemble FP32 element matrices and every
        member is refined against its own matrix-free FP64 residual (the
        batched form of the large requests' solve); with "large" they keep FP64
        elements and the FP64 operator; with "all" FP64 elements and an FP32
        copy of the operator with FP64 residual replacement.  large_precond: the
        preconditioner of the large requests' one-handle solves ("jacobi" or
        "two_level_coupled"), small_precond that of the batched solves."""
        if mixed_scope not in ("large", "all", "elements"):
            raise ValueError("mixed_scope must be 'large', 'all' or 'elements'")
        if precision not in ("fp32", "fp64"):
            raise ValueError("precision must be fp32 or fp64")
        self.budget = int(hbm_budget_bytes)
        self.max_slots = int(max_slots)
        self.precision = precision
        self.graphs = graphs
        # handle creation (mesh planning on the host) runs on these threads; by
        # default half the host cores, 2 to 8
        import os
        self.creators = int(creators) if creators else max(2, min(8, (os.cpu_count() or 4) // 2))
        self.spec = use_specializations
        self.realtime = realtime
        self.large_rows = int(large_rows)
        # 2D requests go to the one-handle path from a lower size: the batched
        # solve is point-Jacobi BiCGStab, which stalls on fine 2D lid-driven meshes
        self.large_rows_2d = self.large_rows if large_rows_2d is None else int(large_rows_2d)
        self.large_workers = int(large_workers)
        self.small_priority = bool(small_priority)
        self.krylov = dict(method="bicgstab", precond=small_precond, tol=1e-10, max_iters=3000)
        self.krylov.update(krylov or {})
        self.mixed = bool(mixed)
        if not mixed:
            self.krylov_mixed = self.krylov
        elif mixed_scope == "elements":
            self.krylov_mixed = dict(self.krylov, mixed="matrix_free", inner_tol=1e-5, max_refine=30)
        else:
            self.krylov_mixed = dict(self.krylov, mixed=True, inner_tol=1e-6, max_refine=20)
        # large requests of the mixed form: FP32 element matrices, FP32 inner
        # solves refined against the matrix-free FP64 residual
        self.krylov_large = (dict(self.krylov, mixed="matrix_free", inner_tol=1e-5, max_refine=30) if mixed
                             else dict(self.krylov))
        self.krylov_large["precond"] = large_precond  # e.g. "two_level_coupled" (one-handle solves only)
        self.mixed_scope = mixed_scope
        self._starved = False
        self._lock = threading.Condition()
        self._used = 0
        self._slots = 0
        self.peak_bytes = 0
        self.max_batch = 0
        self.errors: list = []

    def _is_large(self, dim: int, rows: int) -> bool:
        return rows >= (self.large_rows_2d if dim == 2 else self.large_rows)

    # -- budget ---------------------------------------------------------------
    def _try_reserve(self, nbytes: int) -> bool:
        with self._lock:
            if self._slots < self.max_slots and self._used + nbytes <= self.budget:
                self._used += nbytes
                self._slots += 1
                self.peak_bytes = max(self.peak_bytes, self._used)
                return True
            return False

    def _adjust(self, old: int, new: int) -> None:
        with self._lock:
            self._used += new - old
            self.peak_bytes = max(self.peak_bytes, self._used)

    def _release(self, nbytes: int) -> None:
        with self._lock:
            self._used -= nbytes
            self._slots -= 1
            self._lock.notify_all()

    # -- run ------------------------------------------------------------------
    def run(self, requests: list[Request]) -> tuple[list[Result], dict]:
        import torch

        reqs = sorted(requests, key=lambda r: r.arrival)
        for r in reqs:
            if estimate_bytes(r, self.precision) > self.budget:
                raise ValueError(f"request {r.rid} alone exceeds the HBM budget")
        # queues: (dim, "small") feeds one batching worker per dimension;
        # (dim, "large") feeds `large_workers` workers that run one request each
        inbox = {(d, c): deque() for d in (2, 3) for c in ("small", "large")}
        results: list[Result] = []
        state = {"open": len(reqs)}
        # the CUDA context exists before the clock starts; the batching workers'
        # streams have the high priority (their kernels are short and latency-bound)
        torch.cuda.init()
        small_streams = {(d, "small"): torch.cuda.Stream(priority=-1 if self.small_priority else 0) for d in (2, 3)}
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0  # noqa: E731

        # Handles and batches of finished requests are freed lazily, on one
        # reclaimer thread.  Freeing device memory synchronises the device, and
        # the library keeps its graph captures apart from such calls, so a free
        # while other requests run stalls all of their work (served throughput
        # then varied from 85 to 160 steps/s between runs, with p99 step
        # latencies up to 760 ms, against ~200 steps/s and 60-105 ms with the
        # frees held back).  They are freed in the order they finished (a batch
        # before its members' handles) when admission waits for memory, when no
        # admitted request is left, and at the end of the run; a request's
        # budget is released once its handle is freed.
        graveyard: deque = deque()
        live = {"n": 0}  # admitted requests that have not finished
        stop = {"flag": False}

        def reap(obj, reserved: int | None) -> None:
            with self._lock:
                graveyard.append((obj, reserved))
                self._lock.notify_all()

        def reclaimer() -> None:
            while True:
                with self._lock:
                    while not (graveyard and (self._starved or live["n"] <= 0 or stop["flag"])):
                        if stop["flag"]:
                            return  # nothing left to free
                        self._lock.wait(0.02)
                    items = list(graveyard)
                    graveyard.clear()
                for obj, reserved in items:
                    try:
                        obj.close()
                    except Exception as e:  # surfaced to the caller; the budget is released all the same
                        with self._lock:
                            self.errors.append(e)
                            self._lock.notify_all()
                    finally:
                        if reserved is not None:
                            self._release(reserved)

        reaper = threading.Thread(target=reclaimer, daemon=True)
        reaper.start()

        def finish(a: _Active, held: bool) -> None:
            a.result.state = a.ns.state()[0]
            a.result.finished = now()
            if not held:  # a held handle is closed (and its budget freed) when its batch is rebuilt
                reap(a.ns, a.reserved)
            with self._lock:
                results.append(a.result)
                state["open"] -= 1
                live["n"] -= 1
                self._lock.notify_all()

        def large_worker(key: tuple):
            # one request at a time through the one-handle path; with the mixed
            # form its element matrices are FP32 and the solve refines against
            # the matrix-free FP64 residual (mixed = "matrix_free")
            stream = torch.cuda.Stream()
            kr = self.krylov_large
            try:
                while True:
                    with self._lock:
                        while not inbox[key] and state["open"] > 0:
                            self._lock.wait(0.05)
                        if not inbox[key]:
                            break
                        a = inbox[key].popleft()
                    a.result.started = time.perf_counter() - t0
                    for _ in range(a.req.nsteps):
                        ts = time.perf_counter()
                        a.ns.assemble(stream)
                        a.ns.apply_dirichlet(stream)
                        st = a.ns.solve(stream, raise_on_failure=False, **kr)
                        a.ns.update(stream)
                        stream.synchronize()
                        a.result.step_ms.append((time.perf_counter() - ts) * 1e3)
                        a.result.statuses.append(st)
                        self.max_batch = max(self.max_batch, 1)
                    finish(a, held=False)
            except Exception as e:  # surface worker failures to the caller
                with self._lock:
                    self.errors.append(e)
                    state["open"] = -10 ** 9
                    self._lock.notify_all()

        def worker(key: tuple, capacity: int):
            # continuous batching of the small requests: newcomers join at the
            # next tick (the batch is rebuilt with them); finished members are
            # held in place (ufem_batch_set_active), so a finish does not stall
            # the others, and leave at the next rebuild -- when newcomers join,
            # when admission waits for memory, or when no member is left
            stream = small_streams[key]
            active: list[_Active] = []
            held: list[_Active] = []
            batch = None

            def drop_batch():
                nonlocal batch
                if batch is not None:
                    stream.synchronize()
                    reap(batch, None)  # before its members' handles (FIFO reaper)
                    batch = None
                for h in held:
                    reap(h.ns, h.reserved)
                held.clear()

            try:
                while True:
                    with self._lock:
                        while not inbox[key] and not active and state["open"] > 0:
                            self._lock.wait(0.05)
                        if not inbox[key] and not active and state["open"] <= 0:
                            break
                        joined = False
                        while inbox[key] and len(active) + len(held) < capacity:
                            active.append(inbox[key].popleft())
                            joined = True
                        starved = self._starved
                    if not active:
                        drop_batch()
                        continue
                    if batch is None or joined or (held and starved):
                        drop_batch()
                        batch = Batch([a.ns for a in active], graphs=self.graphs)
                        members = list(active)
                        self.max_batch = max(self.max_batch, len(active))
                    ts = time.perf_counter()
                    for a in active:
                        if a.done_steps == 0 and a.result.started == 0.0:
                            a.result.started = ts - t0
                    kr = self.krylov_mixed if self.mixed_scope != "large" else self.krylov
                    sts = batch.step(stream, **kr)
                    stream.synchronize()
                    ms = (time.perf_counter() - ts) * 1e3
                    finished = []
                    for a, st in zip(members, sts):
                        if a not in active:
                            continue
                        a.result.step_ms.append(ms)
                        a.result.statuses.append(st)
                        a.done_steps += 1
                        if a.done_steps >= a.req.nsteps:
                            finished.append(a)
                    for a in finished:
                        active.remove(a)
                        held.append(a)
                        finish(a, held=True)
                    if finished and active:
                        batch.set_active([a in active for a in members])
            except Exception as e:  # surface worker failures to the caller
                with self._lock:
                    self.errors.append(e)
                    state["open"] = -10 ** 9
                    self._lock.notify_all()
            finally:
                drop_batch()

        def create(req: Request, est: int, admitted: float):
            ns = None
            try:
                large = self._is_large(req.dim, req.coords.shape[0] * (req.dim + 1))
                fp32_elements = self.mixed and (large or self.mixed_scope == "elements")
                ns = _new_handle(req, "fp32" if fp32_elements else self.precision, self.spec)
                # the one-time work of the first step on this host thread, not on
                # the worker that steps the request: the Dirichlet plan (built by
                # the first conditioning of an assembled system), the solver
                # workspace, the preconditioner structure and, for one handle,
                # the coarse inverse of the first system (which its first solve
                # would otherwise compute first); the state is unchanged
                s = torch.cuda.Stream()
                ns.assemble(s)
                ns.apply_dirichlet(s)
                s.synchronize()
                kr = self.krylov_large if large else (self.krylov_mixed if self.mixed_scope != "large" else self.krylov)
                ns.prepare_solve(batched=not large, **kr)
            except Exception as e:  # the request is rejected; the others go on
                if ns is not None:
                    ns.close()
                self._release(est)
                with self._lock:
                    results.append(Result(req.rid, None, arrival=req.arrival, admitted=admitted, finished=now(),
                                          error=str(e)))
                    state["open"] -= 1
                    live["n"] -= 1
                    self._lock.notify_all()
                return
            actual = ns.device_bytes() + req.coords.shape[0] * (req.dim + 1) * 8 * 14  # + batch vectors
            self._adjust(est, actual)
            a = _Active(req, ns, admitted, actual)
            a.result.ready = now()
            with self._lock:
                cls = "large" if self._is_large(req.dim, ns.nb_rows) else "small"
                inbox[(req.dim, cls)].append(a)
                self._lock.notify_all()

        workers = [threading.Thread(target=worker, args=((d, "small"), self.max_slots), daemon=True) for d in (2, 3)]
        workers += [threading.Thread(target=large_worker, args=((d, "large"),), daemon=True)
                    for d in (2, 3) for _ in range(self.large_workers)]
        for w in workers:
            w.start()
        pool = ThreadPoolExecutor(max_workers=self.creators)
        waiting: deque = deque()
        pending = deque(reqs)
        try:
            while pending or waiting:
                if self.errors:
                    break
                t = now()
                while pending and (pending[0].arrival <= t or not self.realtime):
                    waiting.append(pending.popleft())
                admitted_any = False
                for req in list(waiting):  # first fit in arrival order
                    est = estimate_bytes(req, self.precision)
                    if self._try_reserve(est):
                        waiting.remove(req)
                        with self._lock:
                            live["n"] += 1
                        pool.submit(create, req, est, now())
                        admitted_any = True
                with self._lock:
                    # admission waits for memory: batching workers drop their finished members
                    self._starved = bool(waiting) and not admitted_any
                if not admitted_any:
                    with self._lock:
                        timeout = 0.01
                        if pending and not waiting and self.realtime:
                            timeout = max(0.0, min(0.05, pending[0].arrival - now()))
                        self._lock.wait(timeout)
            with self._lock:
                while state["open"] > 0 and not self.errors:
                    self._lock.wait(0.1)
        finally:
            pool.shutdown(wait=True)
            with self._lock:
                if state["open"] > 0:
                    state["open"] = 0
                self._lock.notify_all()
            for w in workers:
                w.join()
            with self._lock:
                stop["flag"] = True
                self._lock.notify_all()
            reaper.join()  # every handle and batch freed before run() returns
        if self.errors:
            raise self.errors[0]
        t_end = max((r.finished for r in results), default=now())
        t_start = min((r.arrival for r in results), default=0.0) if self.realtime else 0.0
        stats = summarize(results, t_start, t_end)
        stats.update(peak_reserved_bytes=self.peak_bytes, budget_bytes=self.budget, max_batch=self.max_batch)
        return sorted(results, key=lambda r: r.rid), stats


def run_plain(requests: list[Request], krylov: dict | None = None, realtime: bool = True,
              use_specializations: bool = False) -> tuple[list[Result], dict]:
    """The same requests one at a time in arrival order through the plain
    FP64 one-handle path (assemble, Dirichlet, BiCGStab + Jacobi, update)."""
    kr = dict(method="bicgstab", precond="jacobi", tol=1e-10, max_iters=3000)  # as Server
    kr.update(krylov or {})
    reqs = sorted(requests, key=lambda r: r.arrival)
    results = []
    t0 = time.perf_counter()
    for req in reqs:
        if realtime:
            wait = req.arrival - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
        res = Result(req.rid, None, arrival=req.arrival, admitted=time.perf_counter() - t0)
        ns = _new_handle(req, "fp64", use_specializations)
        for _ in range(req.nsteps):
            ts = time.perf_counter()
            ns.assemble()
            ns.apply_dirichlet()
            st = ns.solve(raise_on_failure=False, **kr)  # synchronises (the solve reads its status)
            ns.update()
            res.step_ms.append((time.perf_counter() - ts) * 1e3)
            res.statuses.append(st)
        res.state = ns.state()[0]
        ns.close()
        res.finished = time.perf_counter() - t0
        results.append(res)
    t_end = max(r.finished for r in results)
    t_start = min(r.arrival for r in results) if realtime else 0.0
    return sorted(results, key=lambda r: r.rid), summarize(results, t_start, t_end)
