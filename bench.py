"""Benchmark of the plain 3D Euler cut-cell solve on B200 (one JSON line on rank 0).

Workload (the largest single-GPU plain configuration the metric is quoted on): the fighter
half model at ~4M cells (stretched grid ~200 x 140 x 140), M0.6, alpha 3 deg, delta 3 deg,
fixed nozzle/intake states from the 1-D cycle (the engine field model sampled as the app's
applyCond does, sea level, full dry throttle; --fix free gives free-stream states instead),
SSP-RK2 with cfl 0.7, MUSCL order 2.  The batched and served legs use the same source of
fixed states.  One *step* is one solve:
reset + ITERS iterations + the FP64 force integral.  Inputs are synthetic in the sense that
the reference publishes no dataset; the geometry is the reference's own parametric fighter.

value  - cell-updates/s with the state resident in HBM (CUDA events on the solver stream);
e2e    - the same through the public solver API with host buffers: each step uploads the
         initial state from pinned memory, solves, reads the full state back and computes
         the forces (CUDA events around the whole sequence on the solver stream).
roofline.achieved - 142 algorithmic bytes per cell-update (stage 1: read Q + metadata 41 B,
         write S1 20 B; stage 2: read S1, Q and metadata 61 B, write B 20 B) x cell-updates/s
         of the stage kernels alone: 71 B x N per RK stage (all of its z-chunk launches) over
         the stage time measured with CUDA events on the solver's stream.

--impl reference times the reference's CPU algorithm instead (the C++ restatement of CfdCPU,
OpenMP over all host cores): the JavaScript original cannot run on this machine.
Multi-GPU (torchrun): each rank solves its own case (weak scaling); timings are the max
over ranks.
"""
import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

ALG_BYTES_PER_CELL_UPDATE = 142
KERNEL_NAMES = {0: "k_stage_cell", 2: "k_stage_tma", 4: "k_stage_pair"}


def measured_traffic(kernel, cells):
    """DRAM bytes per RK stage from the committed ncu summary of the kernel (profiles/), scaled to
    `cells`.

    The summary holds a line `traffic <kernel> <bytes per cell-stage>`: dram__bytes_read.sum +
    dram__bytes_write.sum over whole stages of the 4.13M-cell fighter (k_stage_pair: a range
    capture of 20 iterations, write-backs included; k_stage_tma: per-launch captures)."""
    short = kernel[len("k_stage_"):] if kernel.startswith("k_stage_") else kernel
    path = os.path.join(ROOT, "profiles", f"stage_{short}_fighter4M.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        f = line.strip().strip("`").split()
        if len(f) == 3 and f[0] == "traffic" and f[1] == kernel:
            return float(f[2]) * cells
    return None


WORKLOAD = {"aircraft": "fighter", "cells": 4.0e6, "M": 0.6, "alpha": 3.0, "delta": 3.0, "iters": 2000}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--iters", type=int, default=WORKLOAD["iters"])
    p.add_argument("--cells", type=float, default=WORKLOAD["cells"])
    p.add_argument("--aircraft", default=WORKLOAD["aircraft"], choices=["fighter", "interceptor", "airliner"])
    p.add_argument("--mach", type=float, default=WORKLOAD["M"])
    p.add_argument("--alpha", type=float, default=WORKLOAD["alpha"])
    p.add_argument("--delta", type=float, default=WORKLOAD["delta"])
    p.add_argument("--fix", default="cycle", choices=["cycle", "free"],
                   help="fixed states of the engine cells: the engine field model's (at --altitude, full "
                        "dry throttle) as the app's applyCond samples them, or the free stream")
    p.add_argument("--altitude", type=float, default=0.0, help="altitude [m] of the field-model fixed states")
    p.add_argument("--kernel", type=int, default=4)
    p.add_argument("--kz", type=int, default=0, help="z planes per CTA; 0 picks from the grid size")
    p.add_argument("--cpu-sample-iters", type=int, default=2)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--batch-cases", type=int, default=64)
    p.add_argument("--batch-iters", type=int, default=1000)
    p.add_argument("--serve-requests", type=int, default=200)
    p.add_argument("--serve-rate", type=float, default=20.0)
    p.add_argument("--serve-sequence", type=int, default=0,
                   help="also serve the same arrivals with grid sequencing (coarse case at cells/S first)")
    p.add_argument("--split", type=int, default=0,
                   help="also time the case cut into this many z slabs: on one GPU in one process, or "
                        "under torchrun one slab per rank (halo planes by NCCL send/recv)")
    p.add_argument("--no-batch", action="store_true")
    p.add_argument("--no-serve", action="store_true")
    p.add_argument("--no-c5", action="store_true", help="skip the 120M-cell airliner leg")
    p.add_argument("--c5-iters", type=int, default=200)
    p.add_argument("--profile-range", action="store_true",
                   help="bracket the device-resident timed steps by cudaProfilerStart/Stop, so that a profiler "
                        "in range mode counts their DRAM traffic as a whole (write-backs of earlier launches "
                        "included)")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region (clocks and throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        # raw samples; A3D_BENCH_OUT chooses the folder (default: bench_out/ in the repository)
        out = os.environ.get("A3D_BENCH_OUT", os.path.join(ROOT, "bench_out"))
        self.path = os.path.join(out, f"clocks_rank{index}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if not self.p:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        load = [v for v in sm if smax and v > 0.3 * smax] or sm
        return {"sm_mhz": statistics.median(load) if load else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if (args.impl == "ours" and torch.cuda.is_available()) else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return ws, rank, local


def max_over_ranks(v, ws):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def workload_config(args, g, ws=1):
    """The `config` both arms share, identical in both: the plain solve whose SSP-RK2 iterations
    they time, named by its sizes.  How many iterations one timed step runs is each arm's own
    choice (the metric is a rate) and is stated in its `step` key."""
    return {"workload": f"{args.aircraft} plain solve, {g.NX}x{g.NY}x{g.NZ} = {g.N} cells, "
                        f"M{args.mach} a{args.alpha} d{args.delta}, SSP-RK2 iterations (cfl 0.7, MUSCL order 2)",
            "cells": g.N, "dims": [g.NX, g.NY, g.NZ],
            "fixed_states": args.fix if args.fix == "free" else f"cycle at {args.altitude:g} m",
            "l2": "inputs larger than L2 (three 5-component float32 states of %.0f MB each)" % (20 * g.N / 1e6),
            "parallelism": f"{ws} independent solve(s), one per GPU" if ws > 1 else "one solve"}


def oracle_solver(aero, args, ac, threads):
    """The oracle (C++ CfdCPU restatement, f32 storage / f64 arithmetic) set up on the bench's
    case: same grid, geometry, free stream and fixed states as the GPU arm."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    sh = aero.shape_of(ac)
    g = ref.grid(sh, args.cells)
    geo = ref.geom(sh, g, args.delta)
    s = ref.CfdCPU(g, geo, threads=threads)
    F = aero.cfd.freestream(args.mach, args.alpha)
    s.setFree(F)
    s.setFix(aero.fix_states(ac, args.altitude, args.mach, args.alpha)[1] if args.fix == "cycle" else [F, F, F])
    s.reset()
    return s, g


def cpu_baseline(aero, args, ac, iters, threads):
    """The oracle on a bounded sample of the bench's case: iters timed iterations."""
    s, g = oracle_solver(aero, args, ac, threads)
    s.step(1)  # untimed warm-up iteration
    t0 = time.perf_counter()
    s.step(iters)
    dt = time.perf_counter() - t0
    return g.N * iters / dt, g.N


def bench_c5(aero, args, ws, rank, local):
    """C5: the twin-engine airliner half model at ~120M cells (under-wing nacelle intake-sink,
    bypass and core-jet cells holding the engine field model's 11 km states), M0.78, alpha 2.5,
    delta 0, at a reduced iteration count: cell-updates/s from CUDA events on the solver stream,
    the stage time alone and its HBM roofline (71 algorithmic bytes per cell and stage)."""
    import torch
    case = aero.Case(aircraft_type="airliner", cells=1.2e8, M=0.78, alpha=2.5, delta=0.0, device=local,
                     fixed="cycle", h=11000.0)
    s, g, it = case.solver, case.g, args.c5_iters
    tuning = {"kernel": KERNEL_NAMES[s.kernel()[0]], "march_kz": s.kernel()[1], "z_chunks": s.chunks()}
    stream = torch.cuda.ExternalStream(s.stream, device=torch.device("cuda", local))
    s.step(2)  # warm-up
    s.reset()
    s.sync()
    barrier(ws)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    s.step(it)
    e1.record(stream)
    f = case.forces()
    e2.record(stream)
    e2.synchronize()
    ms_step = max_over_ranks(e0.elapsed_time(e1), ws)
    s.dispose()
    peak, peak_kind = peaks()
    stage_ms = ms_step / (2 * it)
    achieved = ALG_BYTES_PER_CELL_UPDATE / 2 * g.N / (stage_ms * 1e-3) / 1e9
    return {"workload": f"airliner plain solve, {g.NX}x{g.NY}x{g.NZ} = {g.N} cells, M0.78 a2.5 d0, cycle fixed "
                        f"states at 11 km, {it} SSP-RK2 iterations", "cells": g.N,
            "cell_updates_per_s": ws * g.N * it / (ms_step * 1e-3), "ms_per_iteration": ms_step / it,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind, "stage_ms": stage_ms},
            "tuning": tuning, "CL": f["CL"], "CD": f["CD"]}


def bench_batched(aero, args, ws, rank, local):
    """C3: seeded cases of uneven size, all advanced together (concurrent per-case launches or one
    persistent launch per RK stage, in a CUDA graph, mode and schedule autotuned) vs the same cases solved one after another (plain loop).
    The case list is sharded across ranks; solves/s are whole-job values (max time over ranks)."""
    import torch
    serve = importlib.import_module("3d_aero_lab_b200.serve")
    reqs = serve.requests(1, args.batch_cases, fix=args.fix)[rank::ws]
    cases = []
    for r in reqs:
        c = aero.Case(aircraft_type=r["type"], cells=r["cells"], M=r["M"], alpha=r["alpha"], delta=r["delta"],
                      device=local, fixed=r["fix"])
        c.solver.set_kernel(args.kernel, 0)  # plain loop: each lone case's automatic z run and z chunks
        cases.append(c)
    cells = sum(c.g.N for c in cases)
    it = args.batch_iters
    # plain per-case loop
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    plain = []
    for c in cases:
        c.solver.reset()
        c.solver.step(it)
        plain.append(c.forces())
    torch.cuda.synchronize()
    t_plain = max_over_ranks(time.perf_counter() - t0, ws)
    # batched: the cases run concurrently, so each keeps one launch per stage and the 16-plane run
    # (the persistent kernel's z run is the tuner's choice)
    for c in cases:
        c.solver.set_kernel(args.kernel, 16)
        c.solver.set_chunks(1)
    b = aero.Batch([c.solver for c in cases])
    tuned = b.tune(4)
    for c in cases:
        c.solver.reset()
    b.sync()
    torch.cuda.synchronize()
    barrier(ws)
    t0 = time.perf_counter()
    b.step(it)
    b.sync()
    batched = [c.forces() for c in cases]
    t_batch = max_over_ranks(time.perf_counter() - t0, ws)
    dcl = max(abs(x["CL"] - y["CL"]) for x, y in zip(plain, batched))
    b.dispose()
    for c in cases:
        c.solver.dispose()
    n = args.batch_cases
    return {"workload": f"{n} cases (airliner/interceptor/fighter, 20k-2M cells, M 0.3-0.85, alpha -2..8, "
                        f"delta -5..5, seed 1), {it} iterations each", "cells_per_rank": cells,
            "solves_per_s": n / t_batch, "plain_loop_solves_per_s": n / t_plain, "speedup_vs_plain": t_plain / t_batch,
            "cell_updates_per_s": ws * cells * it / t_batch, "schedule": tuned, "max_abs_dCL_batched_vs_plain": dcl}


def bench_served(aero, args, ws, rank, local):
    """C4: Poisson arrivals (seeded) of solve requests into the continuous-batching server, each
    run to a 1e-3 density-residual drop or 3000 iterations, warm starts on repeated geometry,
    150 GB admission budget; vs the same list solved one at a time in arrival order."""
    serve = importlib.import_module("3d_aero_lab_b200.serve")
    reqs = serve.requests(7, args.serve_requests, geometries=max(4, args.serve_requests // 3),
                          fix=args.fix)[rank::ws]
    sv = serve.Server(budget_gb=150.0, residual_drop=1e-3, max_active=64, chunk=50, max_iters=3000, device=local)
    res, wall = serve.poisson_run(sv, reqs, args.serve_rate / ws, seed=7 + rank)
    st = sv.stats()
    sv.close()
    lat = serve.latency_stats(res, 1e-3)
    span = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
    seq = None
    if args.serve_sequence > 1:  # the same arrivals with grid sequencing (coarse case at cells/8 first)
        sq = serve.Server(budget_gb=150.0, residual_drop=1e-3, max_active=64, chunk=50, max_iters=3000, device=local,
                          sequence=args.serve_sequence, sequence_drop=0.05, sequence_max_iters=1500)
        sres, _ = serve.poisson_run(sq, reqs, args.serve_rate / ws, seed=7 + rank)
        sq.close()
        slat = serve.latency_stats(sres)
        sspan = max_over_ranks(max(r["t_done"] for r in sres) - min(r["t_submit"] for r in sres), ws)
        cold = [(a, b) for a, b in zip(res, sres) if not a["warm"] and not b["warm"]]
        seq = {"sequence": args.serve_sequence, "solves_per_s": args.serve_requests / sspan, "p50_s": slat["p50_s"],
               "p99_s": slat["p99_s"], "mean_iterations": float(sum(r["iterations"] for r in sres) / len(sres)),
               "mean_coarse_iterations": float(sum(r["coarse_iterations"] for r in sres) / len(sres)),
               "mean_final_residual_ratio": statistics.fmean([r["residual"] / r["res0"] for r in sres if r["res0"] > 0]),
               "max_abs_dCL_vs_unsequenced": max((abs(a["CL"] - b["CL"]) for a, b in cold), default=None)}
    plain, _ = serve.plain_loop(reqs, args.serve_rate / ws, seed=7 + rank)
    plat = serve.latency_stats(plain, 1e-3)
    pspan = max(r["t_done"] for r in plain) - min(r["t_submit"] for r in plain)
    span = max_over_ranks(span, ws)
    pspan = max_over_ranks(pspan, ws)
    dcl = max(abs(a["CL"] - b["CL"]) for a, b in zip(res, plain) if not a["warm"]) if any(not a["warm"] for a in res) else None
    return {"workload": f"{args.serve_requests} requests, Poisson {args.serve_rate}/s (seed 7), C3 distribution with "
                        f"{max(4, args.serve_requests // 3)} distinct geometries, residual drop 1e-3 or 3000 iterations",
            "solves_per_s": args.serve_requests / span, "p50_s": lat["p50_s"], "p99_s": lat["p99_s"],
            "converged_fraction": lat["converged_fraction"], "latency_converged": lat["converged"],
            "latency_capped": lat["capped"],
            "plain_loop_solves_per_s": args.serve_requests / pspan, "plain_p50_s": plat["p50_s"],
            "plain_p99_s": plat["p99_s"], "plain_converged_fraction": plat["converged_fraction"],
            "speedup_vs_plain": pspan / span,
            "warm_starts": st["warm_starts"], "rounds": st["rounds"],
            "mean_iterations": float(sum(r["iterations"] for r in res) / len(res)),
            "mean_final_residual_ratio": statistics.fmean([r["residual"] / r["res0"] for r in res if r["res0"] > 0]),
            "max_abs_dCL_cold_vs_plain": dcl, "sequenced": seq}


def bench_split(aero, args, ws, rank, local):
    """The plain case cut into z slabs (two halo planes each side, exchanged after every RK stage).

    One process (ws == 1): --split slabs on this GPU, halo copies between them; this measures
    the decomposition's cost against the unsplit solve.  torchrun (ws > 1): one slab per rank,
    halos by NCCL send/recv, forces all-reduced; strong scaling of one case.  Host clock around
    fully synchronised work, max over ranks."""
    import torch
    split = importlib.import_module("3d_aero_lab_b200.split")
    iters = args.iters
    if ws == 1:
        sc = split.SplitCase(args.aircraft, args.cells, args.mach, args.alpha, args.delta, slabs=args.split,
                             devices=(local,), fixed=args.fix, h=args.altitude, kernel=args.kernel, kz=args.kz,
                             align=args.kz)
        N = sc.g.N
        for _ in range(args.warmup):
            sc.step(20)
        sc.sync()
        t0 = time.perf_counter()
        sc.step(iters)
        f = sc.forces()
        sc.sync()
        dt = time.perf_counter() - t0
        sc.dispose()
        return {"workload": f"{args.aircraft} {N} cells in {args.split} z slabs on one GPU, {iters} iterations",
                "cell_updates_per_s": N * iters / dt, "ms_per_iteration": dt / iters * 1e3,
                "slabs": [b["own"] for b in sc.bounds], "CL": f["CL"], "CD": f["CD"]}
    ac = aero.build_aircraft(args.aircraft)
    sh = aero.shape_of(ac)
    g = aero.cfd_grid(sh, args.cells)
    bounds = split.slab_bounds(g.NZ, ws, split.HALO, args.kz)
    b = bounds[rank]
    s = aero.CfdGPU.slab(g, sh, *b["stored"], delta=args.delta, device=local)
    s.set_kernel(args.kernel, args.kz)
    F = aero.freestream(args.mach, args.alpha)
    s.setFree(F)
    s.setFix(aero.fix_states(ac, args.altitude, args.mach, args.alpha)[1] if args.fix == "cycle" else [F, F, F])
    s.set_owned(b["own"][0] - b["stored"][0], b["own"][1] - b["stored"][0])
    s.reset()
    d = split.DistSplit(split.GpuSlab(s, local), b, device=torch.device("cuda", local))
    for _ in range(args.warmup):
        d.step(20)
    s.sync()
    barrier(ws)
    t0 = time.perf_counter()
    d.step(iters)
    f = d.forces(args.alpha, max(args.mach, 0.05), ac.ref, aero.trefftz_x(ac))
    s.sync()
    dt = max_over_ranks(time.perf_counter() - t0, ws)
    barrier(ws)
    s.dispose()
    return {"workload": f"{args.aircraft} {g.N} cells in {ws} z slabs, one per rank, {iters} iterations",
            "cell_updates_per_s": g.N * iters / dt, "ms_per_iteration": dt / iters * 1e3, "scaling": "strong",
            "slabs": [x["own"] for x in bounds], "CL": f["CL"], "CD": f["CD"]}


def run_reference(args, ws, rank):
    """--impl reference: the reference's CPU algorithm (oracle port, all host threads)."""
    if rank != 0:
        return
    aero = importlib.import_module("3d_aero_lab_b200")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    threads = ref.max_threads()
    ac = aero.build_aircraft(args.aircraft)
    s, g = oracle_solver(aero, args, ac, threads)
    per_step = max(1, args.cpu_sample_iters)
    for _ in range(args.warmup):
        s.step(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.step(per_step)
    dt = time.perf_counter() - t0
    v = g.N * per_step * args.steps / dt
    sample = (f"{per_step} iterations per step of the {g.NX}x{g.NY}x{g.NZ} {args.aircraft} case, "
              f"{threads} threads (C++ restatement of CfdCPU; the JavaScript original cannot run here)")
    config = workload_config(args, g, args.gpus)
    out = {"metric": "cell-updates/s", "value": v, "unit": "cell-updates/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "impl": "reference",
           "config": config,
           "step": {"iterations": per_step, "what": "iterations of the oracle on the host cores",
                    "threads": threads},
           "cpu_baseline": {"value": v, "unit": "cell-updates/s", "cores": threads, "kind": "port", "sample": sample},
           "e2e": {"value": v, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, ws, rank)
        return
    import numpy as np
    import torch
    aero = importlib.import_module("3d_aero_lab_b200")
    torch.cuda.set_device(local)
    alpha = args.alpha + 0.25 * rank  # independent case per rank
    ac = aero.build_aircraft(args.aircraft)
    case = aero.Case(ac=ac, cells=args.cells, M=args.mach, alpha=alpha, delta=args.delta, device=local,
                     fixed=args.fix, h=args.altitude)
    s = case.solver
    s.set_kernel(args.kernel, args.kz)
    g = case.g
    N = g.N
    stream = torch.cuda.ExternalStream(s.stream, device=torch.device("cuda", local))
    iters = args.iters
    chunks = s.chunks()  # pipelined z chunks: stage launches per RK stage
    kz_used = s.kernel()[1]
    launches_per_step = 1 + 2 * iters * chunks + 2  # reset fill, stage launches, force reduction

    def solve():
        s.reset()
        s.step(iters)
        return case.forces()

    for _ in range(args.warmup):
        solve()
    s.sync()
    # ---- device-resident timing ----
    clk = Clocks(local)
    barrier(ws)
    torch.cuda.synchronize()
    clk.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if args.profile_range:
        torch.cuda.profiler.start()
    e0.record(stream)
    for _ in range(args.steps):
        f = solve()
    e1.record(stream)
    e1.synchronize()
    if args.profile_range:
        torch.cuda.profiler.stop()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms, ws)
    barrier(ws)
    # ---- stage-kernel time alone (dominant kernel) ----
    k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.reset()
    k0.record(stream)
    s.step(iters)
    k1.record(stream)
    k1.synchronize()
    stage_ms = k0.elapsed_time(k1) / (2 * iters)
    # ---- end to end through the public API with pinned host buffers ----
    Q0 = torch.empty((5, N), dtype=torch.float32, pin_memory=True)
    Q0.numpy()[:] = np.asarray(case.F, np.float32)[:, None]
    Hout = {k: torch.empty(N, dtype=torch.float32, pin_memory=True) for k in ("r", "ru", "rv", "rw", "E")}
    Hnp = {k: v.numpy() for k, v in Hout.items()}
    barrier(ws)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        s.write(Q0.numpy())
        s.step(iters)
        s.read(Hnp)
        fe = case.forces()
    t1.record(stream)
    t1.synchronize()
    e2e_ms = max_over_ranks(t0.elapsed_time(t1) / args.steps, ws)
    s.dispose()
    extra = {}
    if not args.no_c5:
        try:
            extra["c5"] = bench_c5(aero, args, ws, rank, local)
        except Exception as e:  # reported, not hidden
            extra["c5"] = {"error": repr(e)}
    if args.split:
        try:
            extra["split"] = bench_split(aero, args, ws, rank, local)
        except Exception as e:
            extra["split"] = {"error": repr(e)}
    if not args.no_batch:
        try:
            extra["batched"] = bench_batched(aero, args, ws, rank, local)
        except Exception as e:  # reported, not hidden
            extra["batched"] = {"error": repr(e)}
    if not args.no_serve:
        try:
            extra["served"] = bench_served(aero, args, ws, rank, local)
        except Exception as e:
            extra["served"] = {"error": repr(e)}
    cu = N * iters
    value = ws * cu / (ms * 1e-3)
    e2e = ws * cu / (e2e_ms * 1e-3)
    peak, peak_kind = peaks()
    achieved = ALG_BYTES_PER_CELL_UPDATE / 2 * N / (stage_ms * 1e-3) / 1e9
    out = None
    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and ws == 1:
            v, n_cpu = cpu_baseline(aero, args, ac, args.cpu_sample_iters, 1)
            cpu = {"value": v, "unit": "cell-updates/s", "cores": 1, "kind": "port",
                   "sample": f"{args.cpu_sample_iters} iterations of the same {g.NX}x{g.NY}x{g.NZ} grid, 1 thread "
                             "(C++ restatement of CfdCPU; the JavaScript original cannot run here)"}
        out = {"metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": ws,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": workload_config(args, g, ws),
               "step": {"iterations": iters, "what": "reset + iterations + FP64 forces, state resident in HBM"},
               "tuning": {"kernel": KERNEL_NAMES[args.kernel], "march_kz": kz_used, "z_chunks": chunks},
               "e2e": {"value": e2e, "unit": "cell-updates/s", "h2d_bytes_per_step": 20 * N,
                       "d2h_bytes_per_step": 20 * N + 24},
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": measured_traffic(KERNEL_NAMES[args.kernel], N),
                            "peak_source": peak_kind, "kernel": KERNEL_NAMES[args.kernel],
                            "stage_ms": stage_ms},
               "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches_per_step * args.steps,
               "forces": {"CL": f["CL"], "CD": f["CD"], "Cm": f["Cm"], "CL_e2e": fe["CL"]}}
        out.update(extra)
        print(json.dumps(out), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
