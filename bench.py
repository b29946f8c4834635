"""Benchmark of the UFEM Navier-Stokes hot path on B200.

Workload (default): the 3D tetrahedral configuration -- unit cube, 64^3 cells x
6 Kuhn tetrahedra (1,572,864 tets, 274,625 nodes, 64,300,048 CSR values),
jitter 0.15h, 6 sine modes, nu = 1e-3, dt = 5e-3 -- with seeded synthetic data.
A step is one full assembly of the linear system of a time step
(LinearizeU + element assembly + scatter into the CSR + symmetric Dirichlet),
inputs resident in HBM; the metric is elements assembled per second (Melem/s).

`e2e` is the same metric through the public C ABI with host buffers: every step
copies its fields from pinned host memory to the device and reads its RHS back.
The value is the pipelined form (ufem_ns_stage_state on an upload stream,
ufem_ns_commit_state + assembly + BCs on the compute stream, ufem_ns_fetch_rhs
on a read-back stream), in which one step's copies overlap each other and
their neighbours' assembly; `e2e.sequential` is upload, assembly and read-back
in turn.

Also reported (extra keys): the roofline of the assembly kernel, the FP64 CPU
oracle timed on this host as the baseline, full time steps per second
(assembly + BCs + Krylov solve + update) of this mesh for the plain FP64 path
and the mixed-precision path, and `serving`: served time steps per second with
p50/p99 step and request latency for a seeded Poisson workload of 2D/3D
requests (continuous batching, mixed-precision solve) against the plain path
that serves the same requests one at a time.  `semi_implicit`: time steps of the
semi-implicit scheme (NavierStokesSemiImplicit) on a 3D cavity beside the FP64
oracle's step on one host core (`--si-only` runs it alone).

Multi-GPU: one mesh is not split across GPUs (one GPU per mesh), so
`--gpus N` (under torchrun) runs N independent replicas; value is the sum over
ranks of the elements assembled divided by the max-over-ranks time.

`--impl reference` times the reference algorithm's CPU restatement (the FP64
oracle, all host threads) on the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Melem/s assembled"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=64, help="cells per cube side (64 = the benchmark configuration)")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--asm-kernel", default="auto", choices=["auto", "warp", "warp24", "chunk"],
                    help="assembly kernel variant; auto = the library's autotuner picks it on this mesh")
    ap.add_argument("--asm-warps", type=int, default=4, choices=[2, 4, 8],
                    help="warps per CTA of the warp assembly kernel when --asm-kernel is given")
    ap.add_argument("--specialized", action="store_true", help="use the closed-form specialised kernels")
    ap.add_argument("--no-extras", action="store_true", help="skip CPU baseline and time-step extras")
    ap.add_argument("--time-steps", type=int, default=2, help="full time steps timed per solver variant")
    ap.add_argument("--serve-requests", type=int, default=24, help="requests of the serving comparison (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="Poisson arrival rate (requests/s)")
    ap.add_argument("--serve-elems-3d", type=float, nargs=2, default=[1e4, 2e6],
                    help="log-uniform element-count range of the served 3D requests")
    ap.add_argument("--serve-elems-2d", type=float, nargs=2, default=[1e4, 3e4],
                    help="log-uniform element-count range of the served 2D requests (point-Jacobi BiCGStab, the "
                         "plain path's solver, stalls on larger 2D lid-driven meshes at dt = 0.01)")
    ap.add_argument("--serve-steps", type=int, default=10, help="time steps per served request")
    ap.add_argument("--serve-nu", type=float, nargs=2, default=[1e-4, 1e-1],
                    help="log-uniform viscosity range of the served requests")
    ap.add_argument("--serve-budget-gb", type=float, default=60.0, help="HBM budget of the server (GB)")
    ap.add_argument("--serve-reps", type=int, default=3, help="served runs per form (the median is reported)")
    ap.add_argument("--serve-sweep", type=float, nargs="*", default=[10.0, 50.0, 200.0, 500.0],
                    help="arrival rates (requests/s) of the sweep (one run per form and rate)")
    ap.add_argument("--serving-only", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--si-n", type=int, default=32, help="cube side of the semi-implicit comparison")
    ap.add_argument("--si-only", action="store_true", help="run only the semi-implicit comparison (one JSON line)")
    ap.add_argument("--cfg3-only", action="store_true", help="run only the 128^3 precision comparison (one JSON line)")
    ap.add_argument("--cfg4-only", action="store_true", help="run only the 256-mesh batch comparison (one JSON line)")
    ap.add_argument("--ts-only", action="store_true",
                    help="after the assembly measurement run only the full time steps (no CPU baseline, cfg3, cfg4, "
                         "semi-implicit or serving)")
    ap.add_argument("--ts-forms", nargs="*", default=None,
                    help="time-step forms to run (plain_fp64, two_level, two_level_1e-12, mixed_two_level_1e-12, "
                         "fp64_1e-13; default all)")
    return ap.parse_args()


def dist_init(ngpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return rank, world, local


def max_over_ranks(x: float, world: int) -> float:
    """Max of a per-rank time over the job (NCCL on GPUs, gloo on CPU)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank: float, ms_max: float, world: int) -> float:
    """Whole-job throughput of N independent replicas: all ranks' units over
    the max-over-ranks time (millions of units per second)."""
    return units_per_rank * world / (ms_max / 1e3) / 1e6


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


class ClockSampler:
    """SM clock and clock-event-reason samples taken DURING the timed region.

    A timed region of K assembly steps lasts only tens of milliseconds, shorter
    than nvidia-smi's 200 ms sampling period, so a thread polls NVML (the
    library behind nvidia-smi) every `interval` seconds while the region runs;
    without NVML it falls back to `nvidia-smi -lms 200`.  Read-only queries.
    """

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index: int, interval: float = 0.002):
        self.gpu = gpu_index
        self.interval = interval
        self.proc = None
        self.thread = None
        self.samples: list[tuple[float, float, int]] = []  # (sm MHz, max sm MHz, reason bits)
        self.path = os.path.join("/tmp", f"ufem_clocks_{os.getpid()}.csv")

    def _nvml_handle(self, nv):
        try:
            import torch
            uuid = str(torch.cuda.get_device_properties(self.gpu).uuid)
            return nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.gpu)

    def __enter__(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._nvml_handle(nv)
            bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop = threading.Event()

            def poll():
                while True:
                    try:
                        sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                        r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
                        self.samples.append((sm, mx, sum(1 << k for k, b in enumerate(bits) if r & b)))
                    except Exception:
                        return
                    if self.stop.wait(self.interval):
                        return

            poll_once = threading.Thread(target=poll, daemon=True)
            self.thread = poll_once
            poll_once.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if self.thread is not None:
            if not self.samples:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "source": "nvml"}
            reasons = sorted({self.NAMES[k] for _, _, r in self.samples for k in range(4) if r >> k & 1})
            return {"sm_mhz": statistics.median(s for s, _, _ in self.samples),
                    "sm_max_mhz": max(m for _, m, _ in self.samples), "reasons": reasons,
                    "samples": len(self.samples), "source": "nvml"}
        try:
            rows = [line.split(",") for line in open(self.path).read().strip().splitlines() if line.strip()]
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        reasons = sorted({self.NAMES[k] for r in rows for k in range(4) if len(r) > 5 + k and "Active" in r[5 + k]
                          and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi"}


def algorithmic_bytes(E, N, nnz, dim):
    """Compulsory HBM bytes of one assembly: connectivity, node data read once
    (coordinates, advection velocity, viscosity, state), each CSR value written
    once, the RHS written once."""
    neq = dim + 1
    return E * (dim + 1) * 4 + N * (8 * dim + 8 * dim + 8 + 8 * neq) + nnz * 8 + N * neq * 8


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    p = os.path.join(ROOT, "profiles", "assembly_traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return None


def cpu_baseline(pb, threads: int, reps: int = 1):
    import oracle as O
    o = O.Oracle(pb.coords, pb.conn, O.options(dt=pb.dt, use_specializations=False))
    o.set_state(pb.up, pb.lin, pb.nu)
    t = o.time_assembly(threads, reps) / reps
    o.close()
    return pb.nb_elems / t / 1e6, t


def bench_config(n, E, Nn, nnz, world):
    """The workload description both arms print (identical strings)."""
    return {"workload": f"3D P1 tets {n}^3x6 ({E} tets, {Nn} nodes, {nnz} CSR values) PSPG/SUPG NS assembly "
                        "(ZeroLSS + LinearizeU + generic element expression + CSR scatter) + symmetric Dirichlet",
            "parallelism": "replicas" if world > 1 else "single device",
            "l2": f"inputs and outputs ({algorithmic_bytes(E, Nn, nnz, 3) / 1e6:.0f} MB per step) larger than L2; "
                  "the GPU arm also writes a 256 MiB buffer between timed steps (flush)"}


def run_reference(args, rank, world):
    """The reference algorithm on the host cores: the FP64 restatement of the
    UFEM step's assembly (ZeroLSS, LinearizeU, per-element Proto expression,
    BlockAccumulator reorder, FEVbr column search) and its symmetric Dirichlet
    conditions, node-partitioned over all host threads like the reference's MPI
    ranks.  The inputs come from the oracle's own generators; this arm never
    loads the product library."""
    if rank != 0:
        return
    import oracle as O
    pb = O.lid_driven_problem(3, args.n, 1e-3, 5e-3)
    threads = os.cpu_count() or 1
    o = O.Oracle(pb["coords"], pb["conn"], O.options(dt=pb["dt"], use_specializations=False))
    o.set_state(pb["up"], pb["lin"], pb["nu"])
    o.add_dirichlet(pb["bc_nodes"], pb["bc_comps"], pb["bc_values"])
    E, Nn = pb["conn"].shape[0], pb["coords"].shape[0]
    for _ in range(args.warmup):
        o.time_step_assembly(threads, 1)
    times = [o.time_step_assembly(threads, 1) for _ in range(args.steps)]
    t = float(np.mean(times))
    value = E / t / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Melem/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(args.n, E, Nn, o.nnz, 1),
        "cpu_baseline": {"value": round(value, 3), "unit": "Melem/s", "cores": threads, "kind": "port",
                         "sample": f"one full step assembly (+ symmetric Dirichlet) of the {E}-tet mesh per step"},
        "e2e": {"value": round(value, 3), "unit": "Melem/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    o.close()
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local):
    import torch

    from coolfluid3_b200 import NavierStokes
    from coolfluid3_b200 import _native as Nat
    from coolfluid3_b200 import problems as P

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pb = P.make_problem(3, args.n, nu=1e-3, dt=5e-3, steps=10)
    E, Nn, dim = pb.nb_elems, pb.nb_nodes, 3
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=args.specialized, precision=args.precision)
    ns.set_state(pb.up, pb.lin, pb.nu)
    ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
    stream = torch.cuda.Stream(device=dev)
    sptr = stream.cuda_stream
    if args.asm_kernel == "auto":
        tuned = ns.tune_assembly(reps=3, stream=sptr)
    else:
        ns.set_assembly_kernel(args.asm_kernel, args.asm_warps)
        tuned = None
    asm_variant, asm_warps = ns.assembly_kernel()
    lanes = 24 if asm_variant == "warp24" else 32  # incidences a warp group holds; longer rows go to the chunk kernel
    big_rows = int((np.bincount(pb.conn.ravel(), minlength=Nn) > lanes).sum())
    asm_launches = 1 if asm_variant == "chunk" else 1 + (1 if big_rows else 0)  # warp kernel + chunk kernel for big rows
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2

    def assemble_step():
        ns.assemble(sptr)
        ns.apply_dirichlet(sptr)

    ns.enable_timing(True)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            flush.zero_()
            assemble_step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    kernel_ms = []
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()
                starts[k].record(stream)
                assemble_step()
                ends[k].record(stream)
                kernel_ms.append(ns.timings()["assembly_ms"])  # events on the launch stream, kernel alone
        torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms = max_over_ranks(float(np.mean(step_ms)), world)
    value = replica_value(E, ms, world)
    kern_ms = float(np.mean(kernel_ms))
    B = algorithmic_bytes(E, Nn, ns.nnz, dim)
    peak, peak_kind = measured_peak()
    achieved = B / (kern_ms / 1e3) / 1e9
    traffic = profiled_traffic()
    traffic_bytes = None
    if traffic and traffic.get("n") == args.n and traffic.get("precision") == args.precision \
            and traffic.get("specialized", False) == args.specialized:
        traffic_bytes = traffic.get("bytes_per_launch")

    # ---- end to end through the C ABI with pinned host buffers ----------------
    # Every step copies its fields from pinned host memory and reads its RHS
    # back.  Sequential form: upload, assemble, read back, one after the other.
    # Pipelined form (the e2e value): ufem_ns_stage_state on an upload stream,
    # commit_state + assembly on the compute stream, fetch_rhs on a read-back
    # stream, so step k+1's upload and step k-1's read-back overlap step k's
    # assembly and each other.
    up_h = torch.from_numpy(pb.up).pin_memory()
    lin_h = torch.from_numpy(pb.lin).pin_memory()
    nu_h = torch.from_numpy(pb.nu).pin_memory()
    rhs_h = [torch.empty(ns.nb_rows, dtype=torch.float64).pin_memory() for _ in range(2)]
    lib = Nat.lib()
    cstream = torch.cuda.Stream(device=dev)  # uploads
    dstream = torch.cuda.Stream(device=dev)  # read-backs: the other direction of the host link
    cptr = Nat.C.c_void_p(cstream.cuda_stream)
    dptr = Nat.C.c_void_p(dstream.cuda_stream)
    P_ = Nat.raw_dptr

    def e2e_step():
        Nat.check(lib.ufem_ns_upload_state(ns.handle, P_(up_h.data_ptr()), P_(lin_h.data_ptr()), P_(nu_h.data_ptr()),
                                           None, Nat.C.c_void_p(sptr)))
        assemble_step()
        Nat.check(lib.ufem_ns_download_system(ns.handle, None, P_(rhs_h[0].data_ptr()), Nat.C.c_void_p(sptr)))
        stream.synchronize()

    def stage():
        Nat.check(lib.ufem_ns_stage_state(ns.handle, P_(up_h.data_ptr()), P_(lin_h.data_ptr()), P_(nu_h.data_ptr()),
                                          cptr))

    def e2e_pipelined(nsteps):
        stage()
        for k in range(nsteps):
            if k + 1 < nsteps:
                stage()
            Nat.check(lib.ufem_ns_commit_state(ns.handle, Nat.C.c_void_p(sptr)))
            assemble_step()
            Nat.check(lib.ufem_ns_fetch_rhs(ns.handle, P_(rhs_h[k % 2].data_ptr()), Nat.C.c_void_p(sptr), dptr))

    for _ in range(args.warmup):
        e2e_step()
    barrier(world)
    seq_ms = []
    for _ in range(args.steps):
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        e2e_step()
        s1.record(stream)
        s1.synchronize()
        seq_ms.append(s0.elapsed_time(s1))
    e2e_pipelined(max(args.warmup, 3))
    torch.cuda.synchronize()
    barrier(world)
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(cstream)  # before the first upload
    e2e_pipelined(args.steps)
    cstream.wait_stream(dstream)
    p1.record(cstream)  # after the last read-back
    p1.synchronize()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(p0.elapsed_time(p1) / args.steps, world)
    e2e_seq_ms = max_over_ranks(float(np.mean(seq_ms)), world)
    h2d = pb.up.nbytes + pb.lin.nbytes + pb.nu.nbytes
    d2h = ns.nb_rows * 8

    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Melem/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32-element/f64-scatter",
        "data": "synthetic",
        "config": bench_config(args.n, E, Nn, ns.nnz, world),
        "kernel": {"element_kernel": "specialized" if args.specialized else "generic (order-2 quadrature)",
                   "precision": args.precision,
                   "assembly_kernel": {"variant": asm_variant, "warps_per_cta": asm_warps,
                                       "autotuned": tuned is not None,
                                       "tuned_ms": None if tuned is None else round(tuned["ms"], 4)}},
        "gpu_launches": (1 + asm_launches + 3) * args.steps,  # linearize, assembly, 3 Dirichlet kernels
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "traffic": traffic_bytes, "algorithmic_bytes": B, "kernel_ms": round(kern_ms, 4)},
        "e2e": {"value": round(E * world / (e2e_ms / 1e3) / 1e6, 3), "unit": "Melem/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_ms, 3),
                "form": "ufem_ns_stage_state (upload stream) / commit_state + assembly + BCs / fetch_rhs (read-back "
                        "stream): uploads and read-backs overlap each other and the neighbouring steps' assembly",
                "sequential": {"value": round(E * world / (e2e_seq_ms / 1e3) / 1e6, 3), "ms_per_step": round(e2e_seq_ms, 3),
                               "form": "ufem_ns_upload_state, assembly + BCs, ufem_ns_download_system, in turn"}},
        "clocks": clk.summary(),
    }

    if rank == 0 and world == 1 and not args.no_extras and args.ts_only:
        line["time_step"] = time_steps(ns, pb, args, stream, sptr)
    elif rank == 0 and world == 1 and not args.no_extras:
        # ---- CPU baseline: the FP64 oracle on this host -------------------------
        v1, t1 = cpu_baseline(pb, 1)
        threads = os.cpu_count() or 1
        vall, tall = cpu_baseline(pb, threads)
        line["cpu_baseline"] = {"value": round(v1, 3), "unit": "Melem/s", "cores": 1, "kind": "port",
                                "sample": f"one full FP64 assembly of the {E}-tet mesh ({t1:.2f} s)",
                                "all_cores": {"value": round(vall, 3), "cores": threads, "seconds": round(tall, 3)}}
        # ---- full time steps: plain FP64 vs mixed precision ---------------------
        line["time_step"] = time_steps(ns, pb, args, stream, sptr)
        # ---- the FP32-element assembly of the same mesh ------------------------
        if args.precision == "fp64":
            try:
                line["fp32_elements"] = fp32_elements(pb, B, peak, stream, sptr, flush)
            except Exception as exc:  # reported, not fatal: the assembly metric above stands
                line["fp32_elements"] = {"error": str(exc)}
        # ---- the precision configuration at its size ------------------------
        try:
            line["cfg3"] = cfg3_precision()
        except Exception as exc:  # reported, not fatal: the assembly metric above stands
            line["cfg3"] = {"error": str(exc)}
        # ---- the batching configuration at its size ------------------------
        try:
            line["cfg4"] = cfg4_batch()
        except Exception as exc:  # reported, not fatal: the assembly metric above stands
            line["cfg4"] = {"error": str(exc)}
        # ---- the semi-implicit scheme, B200 vs the FP64 oracle ------------------
        try:
            line["semi_implicit"] = semi_implicit_compare(args.si_n)
        except Exception as exc:  # reported, not fatal: the assembly metric above stands
            line["semi_implicit"] = {"error": str(exc)}
    ns.close()
    if rank == 0 and world == 1 and not args.no_extras and not args.ts_only and args.serve_requests > 0:
        # ---- served steps/s with p50/p99 vs the plain per-request path ----------
        line["serving"] = serving_in_child()
    if rank == 0:
        print(json.dumps(line), flush=True)


def fp32_elements(pb, B, peak, stream, sptr, flush, reps=10):
    """The same assembly step with FP32 element arithmetic (FP64 accumulation
    into the FP64 CSR values), autotuned on this mesh: the assembly kernel's
    own time (CUDA events on the launch stream, L2 flushed before each step)
    and its fraction of the HBM roofline for the same algorithmic bytes as the
    FP64 form (its outputs are the same FP64 values and RHS)."""
    import torch
    from coolfluid3_b200 import NavierStokes
    ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False, precision="fp32")
    try:
        ns.set_state(pb.up, pb.lin, pb.nu)
        ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
        tuned = ns.tune_assembly(reps=3, stream=sptr)
        variant, warps = ns.assembly_kernel()
        ns.enable_timing(True)
        ms = []
        with torch.cuda.stream(stream):
            for k in range(3 + reps):
                flush.zero_()
                ns.assemble(sptr)
                ns.apply_dirichlet(sptr)
                if k >= 3:
                    ms.append(ns.timings()["assembly_ms"])
        torch.cuda.synchronize()
        kms = float(np.mean(ms))
        achieved = B / (kms / 1e3) / 1e9
        return {"kernel_ms": round(kms, 4), "achieved_gbs": round(achieved, 1), "frac": round(achieved / peak, 4),
                "assembly_kernel": {"variant": variant, "warps_per_cta": warps, "tuned_ms": round(tuned["ms"], 4)},
                "note": "FP32 element arithmetic, FP64 accumulation and FP64 CSR values; row-scaled error against "
                        "the FP64 oracle 1.97e-7 on 128^3 x 6 (tests/test_cfg_parity.py)"}
    finally:
        ns.close()


def time_steps(ns, pb, args, stream, sptr):
    """Full steps (assembly + BCs + Krylov + update), steps/s and per-step latency."""
    import torch
    out = {}
    base_up = pb.up
    results = {}
    # point Jacobi (the reference's drop-in form) and the coupled two-level
    # preconditioner at the reference's 1e-10, the two-level form at 1e-12 (FP64
    # and mixed), and a refined solve to 1e-13: the FP64 answer each form's error
    # is stated against (pressure and velocity apart: the pinned-pressure system
    # determines the pressure far less well than the velocity)
    forms = (("plain_fp64", dict(mixed=False, tol=1e-10)),
             ("two_level", dict(mixed=False, tol=1e-10, precond="two_level_coupled")),
             ("two_level_1e-12", dict(mixed=False, tol=1e-12, precond="two_level_coupled")),
             ("mixed_two_level_1e-12", dict(mixed=True, inner_tol=1e-5, tol=1e-12, precond="two_level_coupled")),
             ("fp64_1e-13", dict(mixed=True, inner_tol=1e-5, tol=1e-13, max_refine=40, precond="two_level_coupled")))
    for label, kw in forms:
        if args.ts_forms is not None and label not in args.ts_forms:
            continue
        ns.set_state(pb.up, pb.lin, pb.nu)
        ns.set_solution(np.zeros(ns.nb_rows))
        lat = []
        iters = []
        st = {"converged": 0}
        try:
            # one untimed step first: the form's one-time set-up (workspace,
            # coarse-space structure, graph captures) is not a step's cost
            for k in range(1 + args.time_steps):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                ns.assemble(sptr)
                ns.apply_dirichlet(sptr)
                st = ns.solve(sptr, raise_on_failure=False, max_iters=6000, **kw)
                ns.update(sptr)
                torch.cuda.synchronize()
                if k:
                    lat.append((time.perf_counter() - t0) * 1e3)
                    iters.append(st["iterations"])
                if not st["converged"]:
                    break
        except Exception as exc:  # reported, not fatal: the assembly metric above stands
            out[label] = {"error": str(exc)}
            continue
        if not lat:
            out[label] = {"error": "the untimed first step did not converge", "status": int(st.get("status", -1))}
            continue
        up, _ = ns.state()
        results[label] = up
        out[label] = {"steps_per_s": round(1e3 / float(np.mean(lat)), 3), "p50_ms": round(float(np.median(lat)), 2),
                      "max_ms": round(float(np.max(lat)), 2), "krylov_iters": iters,
                      "converged": int(st["converged"]), "status": int(st.get("status", -1))}
    if "fp64_1e-13" in results:
        ref = results["fp64_1e-13"]
        for label in ("plain_fp64", "two_level", "two_level_1e-12", "mixed_two_level_1e-12"):
            if label in results:
                d = results[label] - ref
                out[label]["rel_err_vs_fp64_1e-13"] = {
                    "state": float(np.linalg.norm(d) / np.linalg.norm(ref)),
                    "velocity": float(np.linalg.norm(d[:, :-1]) / np.linalg.norm(ref[:, :-1])),
                    "pressure": float(np.linalg.norm(d[:, -1]) / np.linalg.norm(ref[:, -1]))}
    out["steps"] = args.time_steps
    out["note"] = ("each form starts from the same state, takes one untimed step, then the timed steps; errors "
                   "compare the states after those steps")
    ns.set_state(base_up, pb.lin, pb.nu)
    return out


def semi_implicit_compare(n: int, steps: int = 3) -> dict:
    """The semi-implicit scheme (NavierStokesSemiImplicit) on a 3D lid-driven
    cavity of n^3 x 6 tets: ms per time step on the B200 (device-resident, all
    kernels, velocity CG with point Jacobi, pressure CG with the two-level
    preconditioner), and the FP64 oracle's step on one host core
    (ILU(0)-GMRES), both solving to 1e-8."""
    import torch
    from coolfluid3_b200 import NavierStokesSemiImplicit, problems as P
    coords, conn = P.cube_tets(n)
    nodes, comps, vals = P.lid_driven_bcs(3, n, pin_pressure=False)
    u0 = np.zeros((coords.shape[0], 3))
    lid = P.structured_index(3, n)[2] == n
    u0[lid, 0] = 1.0
    dt, theta, nb_it, tol = 0.01, 0.5, 2, 1e-8

    def setup(X):
        X.initial_conditions(u0, 0.01)
        for comp in range(3):
            sel = comps == comp
            X.add_velocity_dirichlet(nodes[sel], comp, vals[sel])
        X.add_pressure_dirichlet(np.array([0], np.uint32), 0.0)

    G = NavierStokesSemiImplicit(coords, conn, dt=dt, theta=theta, nb_iterations=nb_it)
    try:
        G.set_krylov(velocity=dict(tol=tol, max_iters=5000), pressure=dict(tol=tol, max_iters=20000))
        setup(G)
        G.step(1)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sv, sp = G.step(steps)
        torch.cuda.synchronize()
        gpu_ms = (time.perf_counter() - t0) * 1e3 / steps
        gpu_up = G.state[0]
    finally:
        G.close()
    import oracle as O  # CPU baseline leg only
    S = O.SemiImplicit(coords, conn, O.options(dt=dt, theta=theta), nb_it)
    setup(S)
    t0 = time.perf_counter()
    rc, iters, _ = S.step(1, tol=tol)
    cpu_s = time.perf_counter() - t0
    return {"workload": f"3D lid-driven cavity {n}^3x6 ({conn.shape[0]} tets, {coords.shape[0]} nodes), dt {dt}, "
                        f"theta {theta}, {nb_it} inner passes, velocity and pressure solved to {tol}",
            "ms_per_step": round(gpu_ms, 3), "steps_per_s": round(1e3 / gpu_ms, 2),
            "velocity_cg_iters_per_step": round(sv["iterations"] / steps, 1),
            "pressure_cg_iters_per_step": round(sp["iterations"] / steps, 1),
            "converged": bool(sv["converged"] and sp["converged"]),
            "cpu_baseline": {"ms_per_step": round(cpu_s * 1e3, 1), "cores": 1, "kind": "port",
                             "sample": "first time step of the same cavity (FP64 oracle, ILU(0)-GMRES(200))",
                             "gmres_iters": list(iters), "converged": rc == 0}}


def cfg3_precision(steps: int = 2) -> dict:
    """The precision configuration: 128^3 x 6 tets (12,582,912 tets, 2,146,689
    nodes, 508,839,952 CSR values), nu drawn log-uniform in [1e-4, 1e-2] from the
    seed, FP32 element matrices with FP64 scatter.  Two solve forms step from the
    same start: "configured" -- FP32 inner BiCGStab + Jacobi refined to 1e-8
    against the matrix-free FP64 residual (the configuration's Jacobi and 1e-8),
    "configured_gmres30" -- the same with the configuration's GMRES(30) as the
    inner solver (at most 8000 iterations a step) -- and
    "product" -- the same refinement with the coupled two-level preconditioner to
    1e-12.  Each step's state is compared with an FP64-element handle refined to
    1e-13 (velocity, pressure, and pressure without its mean offset: the
    pressure's constant mode is pinned at one node only)."""
    import torch
    from coolfluid3_b200 import NavierStokes, problems as P
    t0 = time.perf_counter()
    pb = P.config("cfg3")
    gen_s = time.perf_counter() - t0
    forms = {"configured": ("fp32", dict(mixed="matrix_free", tol=1e-8, inner_tol=1e-4, max_iters=8000)),
             "configured_gmres30": ("fp32", dict(mixed="matrix_free", method="gmres", restart=30, tol=1e-8,
                                                 inner_tol=1e-4, max_iters=8000)),
             "product": ("fp32", dict(mixed="matrix_free", tol=1e-12, inner_tol=1e-5, max_iters=8000,
                                      precond="two_level_coupled")),
             "fp64_1e-13": ("fp64", dict(mixed=True, tol=1e-13, inner_tol=1e-5, max_iters=8000, max_refine=40,
                                         precond="two_level_coupled"))}
    hs = {}
    for label, (prec, _) in forms.items():
        ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False, precision=prec)
        ns.set_state(pb.up, pb.lin, pb.nu)
        ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
        ns.enable_timing(True)
        hs[label] = ns
    out = {"workload": f"3D P1 tets 128^3x6 ({pb.nb_elems} tets, {pb.nb_nodes} nodes, {hs['product'].nnz} CSR "
                       f"values), nu {pb.nu[0]:.3e}, dt {pb.dt}", "setup_s": round(time.perf_counter() - t0, 1),
           "generate_s": round(gen_s, 1), "steps": []}
    for k in range(steps):
        row = {}
        for label, ns in hs.items():
            torch.cuda.synchronize()
            t = time.perf_counter()
            ns.assemble()
            asm_ms = ns.timings()["assembly_ms"]
            ns.apply_dirichlet()
            st = ns.solve(raise_on_failure=False, **forms[label][1])
            ns.update()
            torch.cuda.synchronize()
            row[label] = {"step_ms": round((time.perf_counter() - t) * 1e3, 1), "assembly_ms": round(asm_ms, 3),
                          "krylov_iters": st["iterations"], "refinements": st.get("refinements", 0),
                          "converged": int(st["converged"]), "rel_residual": st["rel_residual"]}
        ref = hs["fp64_1e-13"].state()[0]
        for label in ("configured", "configured_gmres30", "product"):
            d = hs[label].state()[0] - ref
            dp = d[:, 3] - d[:, 3].mean()
            row[label]["rel_err_vs_fp64"] = {
                "velocity": float(np.linalg.norm(d[:, :3]) / np.linalg.norm(ref[:, :3])),
                "pressure": float(np.linalg.norm(d[:, 3]) / np.linalg.norm(ref[:, 3])),
                "pressure_without_offset": float(np.linalg.norm(dp) / np.linalg.norm(ref[:, 3]))}
        out["steps"].append(row)
    for ns in hs.values():
        ns.close()
    out["form"] = ("FP32 element arithmetic, FP64 scatter; FP32-operator BiCGStab inner solves refined with the "
                   "matrix-free FP64 residual (GMRES(30) inner solves in configured_gmres30); configured: point "
                   "Jacobi to 1e-8; product: coupled two-level "
                   "preconditioner to 1e-12; reference: FP64 elements refined to 1e-13")
    return out


def cfg4_batch(members: int = 256, steps: int = 2, tol: float = 1e-10) -> dict:
    """The batching configuration: 256 independent 2D lid-driven meshes, node
    counts log-uniform in [1e3, 2e5] (square grids, side round(sqrt(N)) - 1,
    jitter 0.2h), nu log-uniform in [1e-3, 1e-1], dt = 0.01, sine-mode initial
    velocities.  Assembled in one persistent launch per phase with the
    autotuned warps per CTA, and stepped as one batch, against the same members
    assembled and stepped one handle at a time.  The batched solve is BiCGStab
    with per-member scalars and the coupled two-level preconditioner (each
    member's own coarse space), solved to `tol`; the one-by-one path solves each
    member with the same preconditioner."""
    import torch
    from coolfluid3_b200 import Batch, NavierStokes, problems as P
    rng = np.random.default_rng(20261203 + 4)
    nodes = np.exp(rng.uniform(np.log(1e3), np.log(2e5), members))
    nus = 10.0 ** rng.uniform(-3.0, -1.0, members)
    t0 = time.perf_counter()
    hs, probs = [], []
    for k in range(members):
        side = max(2, int(round(np.sqrt(nodes[k]))) - 1)
        pb = P.make_problem(2, side, nu=float(nus[k]), dt=0.01, seed=20261203 + 1000 + k)
        ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False)
        ns.set_state(pb.up, pb.lin, pb.nu)
        ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
        hs.append(ns)
        probs.append(pb)
    setup_s = time.perf_counter() - t0
    E = int(sum(p.nb_elems for p in probs))
    b = Batch(hs)
    tuned = b.tune_assembly(reps=3)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def timed(fn, reps=5):
        ts = []
        for _ in range(reps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    ms_batch = timed(b.assemble)
    ms_one = timed(lambda: [h.assemble() for h in hs])

    def reset():
        for h, pb in zip(hs, probs):
            h.set_state(pb.up, pb.lin, pb.nu)
            h.set_solution(np.zeros(h.nb_rows))

    out = {"workload": f"{members} 2D lid-driven meshes, {int(nodes.min())}..{int(nodes.max())} nodes "
                       f"(log-uniform; {E} triangles in all), nu 1e-3..1e-1, dt 0.01", "setup_s": round(setup_s, 1),
           "assembly": {"batched_ms": round(ms_batch, 3), "batched_melem_s": round(E / ms_batch / 1e3, 1),
                        "one_by_one_ms": round(ms_one, 3), "one_by_one_melem_s": round(E / ms_one / 1e3, 1),
                        "speedup": round(ms_one / ms_batch, 2), "warps_per_cta": tuned["warps_per_cta"]}}
    reset()
    torch.cuda.synchronize()
    t = time.perf_counter()
    conv, iters = 0, []
    for _ in range(steps):
        sts = b.step(tol=tol, max_iters=3000, precond="two_level_coupled")
        conv += sum(s["converged"] for s in sts)
        iters.append(int(max(s["iterations"] for s in sts)))
    torch.cuda.synchronize()
    batch_s = time.perf_counter() - t
    reset()
    torch.cuda.synchronize()
    t = time.perf_counter()
    conv1 = 0
    for _ in range(steps):
        for h in hs:
            h.assemble()
            h.apply_dirichlet()
            st = h.solve(tol=tol, max_iters=3000, raise_on_failure=False, precond="two_level_coupled")
            h.update()
            conv1 += int(st["converged"])
    torch.cuda.synchronize()
    one_s = time.perf_counter() - t
    out["time_steps"] = {"tol": tol, "steps": steps,
                         "batched": {"member_steps_per_s": round(members * steps / batch_s, 1),
                                     "seconds": round(batch_s, 2), "converged": f"{conv}/{members * steps}",
                                     "max_iterations_per_step": iters},
                         "one_by_one": {"member_steps_per_s": round(members * steps / one_s, 1),
                                        "seconds": round(one_s, 2), "converged": f"{conv1}/{members * steps}"},
                         "speedup": round(one_s / batch_s, 2)}
    b.close()
    for h in hs:
        h.close()
    # the configuration's element precision: FP32 element arithmetic with FP64
    # accumulation into the FP64 values (assembly only: the batched solve has no
    # matrix-free FP64 refinement, so FP32-element batch solves stop at the
    # FP32-element system's ~3e-4 error)
    hs32 = []
    for pb in probs:
        ns = NavierStokes(pb.coords, pb.conn, dt=pb.dt, use_specializations=False, precision="fp32")
        ns.set_state(pb.up, pb.lin, pb.nu)
        ns.add_dirichlet(pb.bc_nodes, pb.bc_comps, pb.bc_values)
        hs32.append(ns)
    b32 = Batch(hs32)
    tuned32 = b32.tune_assembly(reps=3)
    ms_batch32 = timed(b32.assemble)
    ms_one32 = timed(lambda: [h.assemble() for h in hs32])
    out["assembly_fp32_elements"] = {"batched_ms": round(ms_batch32, 3),
                                     "batched_melem_s": round(E / ms_batch32 / 1e3, 1),
                                     "one_by_one_ms": round(ms_one32, 3),
                                     "one_by_one_melem_s": round(E / ms_one32 / 1e3, 1),
                                     "speedup": round(ms_one32 / ms_batch32, 2),
                                     "warps_per_cta": tuned32["warps_per_cta"]}
    # time steps with the FP32 element matrices, each member refined against its
    # own matrix-free FP64 residual (the FP64 system's answer); inner solves of at
    # most 400 iterations, 8 refinements (about the FP64 form's 3000 iterations)
    kr32 = dict(tol=tol, mixed="matrix_free", inner_tol=1e-5, max_refine=8, max_iters=3000,
                precond="two_level_coupled")

    def reset32():
        for h, pb in zip(hs32, probs):
            h.set_state(pb.up, pb.lin, pb.nu)
            h.set_solution(np.zeros(h.nb_rows))

    reset32()
    torch.cuda.synchronize()
    t = time.perf_counter()
    conv32 = 0
    for _ in range(steps):
        sts = b32.step(**kr32)
        conv32 += sum(s["converged"] for s in sts)
    torch.cuda.synchronize()
    batch32_s = time.perf_counter() - t
    reset32()
    torch.cuda.synchronize()
    t = time.perf_counter()
    conv321 = 0
    for _ in range(steps):
        for h in hs32:
            h.assemble()
            h.apply_dirichlet()
            st = h.solve(raise_on_failure=False, **kr32)
            h.update()
            conv321 += int(st["converged"])
    torch.cuda.synchronize()
    one32_s = time.perf_counter() - t
    out["time_steps_fp32_elements"] = {
        "tol": tol, "steps": steps, "form": "FP32 element matrices, FP32-operator inner BiCGStab refined against "
                                            "each member's matrix-free FP64 residual, two-level preconditioner",
        "batched": {"member_steps_per_s": round(members * steps / batch32_s, 1), "seconds": round(batch32_s, 2),
                    "converged": f"{conv32}/{members * steps}"},
        "one_by_one": {"member_steps_per_s": round(members * steps / one32_s, 1), "seconds": round(one32_s, 2),
                       "converged": f"{conv321}/{members * steps}"},
        "speedup": round(one32_s / batch32_s, 2)}
    b32.close()
    for h in hs32:
        h.close()
    return out


def serving_in_child() -> dict:
    """serving_compare in a fresh process (same arguments): the served makespan
    depends on how host threads and CUDA streams interleave, so it is measured
    apart from the kernel benchmark's process state."""
    cmd = [sys.executable, os.path.abspath(__file__)] + sys.argv[1:] + ["--serving-only"]
    proc = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=sys.stderr, text=True)
    lines = [ln for ln in proc.stdout.strip().splitlines() if ln.startswith("{")]
    if proc.returncode != 0 or not lines:
        return {"error": f"serving run exited with {proc.returncode}"}
    return json.loads(lines[-1])


def serving_compare(args):
    """Continuous batching against the plain FP64 one-request-at-a-time path
    on the same seeded Poisson workload: the served FP64 form and the served
    mixed-precision form (FP32 operator copy, FP64 residual replacement)."""
    from coolfluid3_b200 import serving as S
    t0 = time.perf_counter()
    elems = {2: tuple(args.serve_elems_2d), 3: tuple(args.serve_elems_3d)}
    reqs = S.poisson_workload(args.serve_requests, rate=args.serve_rate, elems=elems, nu=tuple(args.serve_nu),
                              nsteps=args.serve_steps, seed=20261203)
    gen_s = time.perf_counter() - t0
    tol = 1e-12  # both sides at the residual that keeps the state within 1e-6 of the FP64 oracle

    def server(mixed, lpre):
        return S.Server(int(args.serve_budget_gb * 1e9), precision="fp64", mixed=mixed,
                        krylov=dict(tol=tol, max_iters=20000), realtime=True, large_precond=lpre,
                        small_precond=lpre, large_rows_2d=40_000, mixed_scope="elements")

    forms = (("served_fp64", False, "two_level_coupled"), ("served_mixed", True, "two_level_coupled"))
    # untimed warm-up of every form on a few of the requests (first launches of
    # each kernel, graph captures, host thread pools, pinned buffers)
    warm = S.poisson_workload(6, rate=args.serve_rate, elems=elems, nu=tuple(args.serve_nu), nsteps=2, seed=20261202)
    S.run_plain(warm, krylov=dict(tol=tol, max_iters=20000), realtime=False)
    S.run_plain(warm, krylov=dict(tol=tol, max_iters=20000, precond="two_level_coupled"), realtime=False)
    for _, mixed, lpre in forms:
        server(mixed, lpre).run(warm)
    plain, pst = S.run_plain(reqs, krylov=dict(tol=tol, max_iters=20000), realtime=True)
    plain2, pst2 = S.run_plain(reqs, krylov=dict(tol=tol, max_iters=20000, precond="two_level_coupled"), realtime=True)

    def pick(st, res):
        return {"steps_per_s": round(st["steps_per_s"], 3), "seconds": round(st["seconds"], 3),
                "step_ms_p50": round(st["step_ms"]["p50"], 3), "step_ms_p99": round(st["step_ms"]["p99"], 3),
                "request_s_p50": round(st["request_s"]["p50"], 3), "request_s_p99": round(st["request_s"]["p99"], 3),
                "krylov_iterations": int(sum(sum(s["iterations"] for s in r.statuses) for r in res)),
                "converged_requests": int(sum(r.ok for r in res))}

    out = {
        "workload": (f"{len(reqs)} lid-driven requests, Poisson arrivals {args.serve_rate}/s, 3D tets with "
                     f"{elems[3][0]:.0e}..{elems[3][1]:.0e} elements and 2D tris with {elems[2][0]:.0e}.."
                     f"{elems[2][1]:.0e} (log-uniform; total {sum(r.nb_elems for r in reqs)}), nu log-uniform "
                     f"{args.serve_nu[0]:g}..{args.serve_nu[1]:g}, {args.serve_steps} steps each, relative residual "
                     f"{tol:g}"),
        "plain": dict(pick(pst, plain), form="FP64 elements, FP64 BiCGStab + Jacobi, one request at a time"),
        "plain_two_level": dict(pick(pst2, plain2),
                                form="FP64 elements, FP64 BiCGStab + the coupled two-level preconditioner, one request "
                                     "at a time"),
    }
    for label, mixed, lpre in forms:
        # the served makespan depends on how the threads and streams interleave on
        # the device, so each form is served `serve_reps` times and the run with
        # the median throughput is reported (with the range)
        runs = []
        for _ in range(max(1, args.serve_reps)):
            srv = server(mixed, lpre)
            res, st = srv.run(reqs)
            runs.append((st["steps_per_s"], st, res, srv))
        runs.sort(key=lambda x: x[0])
        _, st, res, srv = runs[len(runs) // 2]
        diffs = [float(np.linalg.norm(a.state - b.state) / np.linalg.norm(b.state))
                 for a, b in zip(res, plain) if a.ok and b.ok]
        out[label] = dict(pick(st, res), max_batch=srv.max_batch, peak_reserved_gb=round(srv.peak_bytes / 1e9, 3),
                          speedup_steps_per_s=round(st["steps_per_s"] / pst["steps_per_s"], 3),
                          speedup_vs_plain_two_level=round(st["steps_per_s"] / pst2["steps_per_s"], 3),
                          runs_steps_per_s=[round(r[0], 2) for r in runs],
                          max_rel_diff_vs_plain=max(diffs) if diffs else None,
                          form=(("FP32 element matrices for every request, FP32-operator inner BiCGStab refined "
                                 "against each request's matrix-free FP64 residual (one handle for the large "
                                 "requests, batched for the small ones)"
                                 if mixed else "FP64 elements, FP64 BiCGStab")
                                + "; the coupled two-level preconditioner throughout; continuous batching (small "
                                  "requests batched, large ones concurrent)"))
    out["note"] = ("every form solves to a 1e-12 relative FP64 residual, the tolerance at which the parity tests keep "
                   "the state within 1e-6 of the FP64 oracle (tests/test_serving.py, tests/test_matrix_free.py); "
                   "max_rel_diff_vs_plain is each served request's final state against the plain path's")
    out["workload_gen_s"] = round(gen_s, 2)
    # ---- arrival-rate sweep (one run per form and rate) ----------------------
    sweep = []
    for rate in args.serve_sweep:
        rq = S.poisson_workload(args.serve_requests, rate=rate, elems=elems, nu=tuple(args.serve_nu),
                                nsteps=args.serve_steps, seed=20261203 + int(rate))
        _, ps = S.run_plain(rq, krylov=dict(tol=tol, max_iters=20000), realtime=True)
        row = {"rate_per_s": rate, "plain": {"steps_per_s": round(ps["steps_per_s"], 2),
                                             "step_ms_p50": round(ps["step_ms"]["p50"], 2),
                                             "step_ms_p99": round(ps["step_ms"]["p99"], 2)}}
        for label, mixed, lpre in forms:
            _, st = server(mixed, lpre).run(rq)
            row[label] = {"steps_per_s": round(st["steps_per_s"], 2), "step_ms_p50": round(st["step_ms"]["p50"], 2),
                          "step_ms_p99": round(st["step_ms"]["p99"], 2),
                          "speedup": round(st["steps_per_s"] / ps["steps_per_s"], 2)}
        sweep.append(row)
    out["rate_sweep"] = sweep
    out["workload_gen_s"] = round(gen_s, 2)
    return out


def main():
    args = parse()
    if args.serving_only:
        print(json.dumps(serving_compare(args)), flush=True)
        return
    if args.cfg4_only:
        print(json.dumps({"cfg4": cfg4_batch()}), flush=True)
        return
    if args.cfg3_only:
        print(json.dumps({"cfg3": cfg3_precision()}), flush=True)
        return
    if args.si_only:
        print(json.dumps({"semi_implicit": semi_implicit_compare(args.si_n)}), flush=True)
        return
    rank, world, local = dist_init(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
