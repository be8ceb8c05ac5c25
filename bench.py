#!/usr/bin/env python
"""D'D CG time-to-solution on a 32^3 x 64 Wilson-clover lattice on B200.

One step = one complete D'D conjugate-gradient solve, zero start, to FP64 true
relative residual 1e-10 (benchmark/ddagd_cg/ddagd_cg.jl:587-664 protocol),
mixed precision: int16-storage / FP32-arithmetic inner D'D with FP64 reliable
updates (delta 0.03: 450 iterations as FP64, 7 reliable updates).  The plain FP64 CG (the reference's algorithm and
arithmetic, cg.jl:73-137) is timed in the same run for the "mixed vs FP64"
comparison.  Inputs: SU(3) links exp(0.2 i H), H Gaussian traceless Hermitian
(seed 1), reunitarized; unit-variance complex Gaussian source (seed 2);
kappa 0.1355, cSW 1.0, phases (1,1,1,-1).  Everything synthetic; the links
(1.2 GB) and clover blocks exceed the 126 MB L2, so no flush is needed.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

N > 1 (torchrun): every rank solves its own replica (the path has no data
exchange at one GPU per lattice); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "latticematrices.jl_b200"))

METRIC = ("D†D CG time-to-1e-10 mixed vs FP64, Dslash HBM GB/s; "
          "32³×64 clover, 1 B200")
PHASES = (1, 1, 1, -1)

# Plain FP64 CG iterations this workload needs (32^3x64, kappa 0.1355,
# cSW 1.0, links exp(0.2 i H) seed 1, source seed 2, rtol 1e-10), measured by
# the GPU FP64 solve of this file and by a complete oracle solve; the CPU
# reference arm multiplies its per-iteration time by the count of its own
# complete solve, or by this constant with --no-full-solve or under torchrun.
FP64_ITERATIONS_32x64 = 450

# Algorithmic bytes per lattice site of the two stencil kernels of a CG
# iteration: every operand read once, every output written once, in the
# storage format the kernel reads (links: 12 reals per SU(3) link with the
# third row rebuilt, else 18; clover: two Hermitian 6x6 blocks = 72 reals).
#  K1  tmp = D p  (+|tmp|^2):  links, clover, p, tmp
#  K2  D^+ tmp fused with x += a p, r -= a Ap, |r|^2:  links, clover, tmp,
#      p, r (read+write), x (read+write, FP32 for the mixed solves)
REAL_BYTES = {"double": 8, "single": 4, "half": 2}


def spinor_bytes(prec):
    return 24 * REAL_BYTES[prec] + (4 if prec == "half" else 0)  # + norm


def gauge_bytes(prec, link_reals):
    return (4 * link_reals + 72) * REAL_BYTES[prec]


def x_bytes(prec):
    return 24 * (8 if prec == "double" else 4)


def k1_bytes(prec, link_reals=18):
    return gauge_bytes(prec, link_reals) + 2 * spinor_bytes(prec)


def k2_bytes(prec, link_reals=18):
    return gauge_bytes(prec, link_reals) + 4 * spinor_bytes(prec) + 2 * x_bytes(prec)


# Wilson-clover M: 1320 (hopping) + 504 (clover) + 48 flops per site
FLOPS_PER_SITE_M = 1872


def parse():
    ap = argparse.ArgumentParser(description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["lmb", "reference"], default="lmb")
    ap.add_argument("--lattice", default="32,32,32,64")
    ap.add_argument("--precision", default="half", choices=["single", "half"])
    ap.add_argument("--kappa", type=float, default=0.1355)
    ap.add_argument("--csw", type=float, default=1.0)
    ap.add_argument("--amplitude", type=float, default=0.2)
    ap.add_argument("--rtol", type=float, default=1e-10)
    ap.add_argument("--delta", type=float, default=None,
                    help="reliable-update delta of the mixed solves (default "
                         "0.03 for the clover solve, 0.1 for the sharded one)")
    ap.add_argument("--maxiter", type=int, default=20000)
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--no-full-solve", action="store_true",
                    help="reference arm: skip the complete FP64 oracle solve that fixes the "
                         "iteration count (about two minutes on 16 cores at 32^3x64)")
    ap.add_argument("--workload", default="clover",
                    choices=["clover", "wilson8", "hisq", "hisq_dslash", "batched", "force",
                             "clover_force", "dw", "evenodd", "sharded"],
                    help="clover: 32^3x64 Wilson-clover mixed vs FP64 CG (the "
                         "headline line); wilson8: 8^4 Wilson FP64 CG beside the "
                         "CPU oracle; hisq: 48^3x96 HISQ smearing + CG; batched: "
                         "multi-RHS multi-lattice Wilson CG; force: 24^4 HISQ "
                         "fermion force with a finite-difference check; "
                         "clover_force: 24^4 Wilson-clover fermion force, same check; "
                         "dw: 16^3x32 x L5 12 Mobius domain-wall D5'D5 CG; evenodd: "
                         "32^3x64 clover D x = b, even/odd Schur solve vs the "
                         "D'D CG route; hisq_dslash: one FP64 HISQ D application "
                         "at 8^4 .. 32^4 beside the reference's published table; "
                         "sharded: the clover CG on the native sharded operators "
                         "(lattice split over the ranks; one rank exchanges with itself)")
    ap.add_argument("--l5", type=int, default=12)
    ap.add_argument("--hisq-sizes", default="8,16,24,32",
                    help="hisq_dslash: lattice extents L of the L^4 lattices")
    ap.add_argument("--batched-small", action="store_true",
                    help="batched: 16^4 x8 + 8^4 x4 instead of the benchmark set (profiling)")
    ap.add_argument("--samples", type=int, default=9,
                    help="hisq_dslash: timing samples per size")
    ap.add_argument("--fd-directions", type=int, default=64)
    ap.add_argument("--grid", default="",
                    help="sharded: process grid a,b,c,d (default 1,1,1,N)")
    ap.add_argument("--split", default="",
                    help="sharded: exchanged dimensions as 0/1 flags (default: the grid's "
                         "dimensions with more than one rank; t on one rank)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU)
# ---------------------------------------------------------------------------
def dist_setup(backend):
    import torch.distributed as dist
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws > 1 and not dist.is_initialized():
        from datetime import timedelta
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, local, ws


def max_over_ranks(value, ws, device=None):
    if ws == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle's FP64 CG on the same workload, bounded sample
# ---------------------------------------------------------------------------
def cpu_fp64_cg_seconds_per_iteration(L, kappa, csw, amplitude, budget_s):
    from oracle import oracle as orc
    orc.build()
    threads = os.cpu_count() or 1
    orc.set_num_threads(threads)
    U = orc.random_su3_links(L, amplitude, 1)
    b = orc.gaussian_field(L, 3, 4, 2)
    F = orc.clover_field_strength(U)
    op = orc.Operator(orc.OP_CLOVER, U, L, kappa=kappa, csw=csw, F=F)
    t1 = orc.cg_iterations_seconds(op, b, 1)
    n = max(1, int(budget_s / max(t1, 1e-3)))
    tn = orc.cg_iterations_seconds(op, b, n)
    return tn / n, n, orc.num_threads()


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_per_site():
    """DRAM bytes per site per launch from a committed ncu capture summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "dslash_traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def run_reference(args):
    rank, _, ws = dist_setup("gloo")
    if rank != 0:
        return
    L = tuple(int(v) for v in args.lattice.split(","))
    sites = L[0] * L[1] * L[2] * L[3]
    from oracle import oracle as orc
    orc.build()
    threads = os.cpu_count() or 1
    orc.set_num_threads(threads)
    U = orc.random_su3_links(L, args.amplitude, 1)
    b = orc.gaussian_field(L, 3, 4, 2)
    F = orc.clover_field_strength(U)
    op = orc.Operator(orc.OP_CLOVER, U, L, kappa=args.kappa, csw=args.csw, F=F)
    for _ in range(args.warmup):
        orc.cg_iterations_seconds(op, b, 1)
    per = []
    for _ in range(args.steps):
        per.append(orc.cg_iterations_seconds(op, b, 1))
    t_iter = statistics.mean(per)
    iters = FP64_ITERATIONS_32x64 if L == (32, 32, 32, 64) else None
    full = None
    if ws == 1 and not args.no_full_solve:
        # one complete FP64 solve to the workload's tolerance (not in the
        # per-iteration sample): its iteration count replaces the constant
        import numpy as np
        t0 = time.perf_counter()
        xs, res = orc.cg_ddagd(op, b, rtol=args.rtol, maxiter=args.maxiter)
        t_full = time.perf_counter() - t0
        true_rel = float(np.linalg.norm(b - op.ddagd(xs)) / np.linalg.norm(b))
        full = {"iterations": res["iterations"], "converged": res["converged"],
                "time_s": t_full, "true_rel_residual": true_rel}
        iters = res["iterations"]
    value = t_iter * iters if iters else t_iter
    unit = "s" if iters else "s/iteration"
    sample = (f"{args.steps} FP64 CG iterations (D'D clover + BLAS) on the "
              f"full {L} lattice after {args.warmup} warm-up iterations; "
              f"value = mean seconds per iteration x {iters} iterations "
              + ("(the iteration count of the complete FP64 solve run here)" if full else
                 "(the FP64 iteration count of this workload)")
              if iters else "seconds per FP64 CG iteration")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": unit,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_iter * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "Wilson-clover D'D CG, FP64, CPU oracle port "
                   "of the reference algorithm", "lattice": list(L),
                   "sites": sites, "kappa": args.kappa, "csw": args.csw},
        "cpu_baseline": {"value": value, "unit": unit, "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if full:
        line["full_solve"] = full
    print(json.dumps(line), flush=True)


def run_lmb(args):
    import numpy as np
    import torch

    rank, local, ws = dist_setup("nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import lmb200 as lmb

    L = tuple(int(v) for v in args.lattice.split(","))
    sites = L[0] * L[1] * L[2] * L[3]
    # reliable-update delta: 0.1, 0.05, 0.03, 0.02, 0.01 gave 450, 450, 450,
    # 453, 470 iterations with 10, 8, 7, 6, 6 FP64 updates at 32^3x64
    delta = 0.03 if args.delta is None else args.delta
    U = lmb.random_su3_links(L, args.amplitude, 1, nw=1, device=dev)
    b = lmb.gaussian_fermion(L, 3, 4, 2, nw=1, phases=PHASES, device=dev)
    D = lmb.WilsonDiracCloverOperator4D(U, args.kappa, args.csw)
    A = lmb.DdagDOp(D, b.similar())
    x = b.similar()
    stream = torch.cuda.current_stream()

    def solve(prec, profile=False):
        lmb.clear_matrix_(x)
        return lmb.cg_(x, A, b, rtol=args.rtol, maxiter=args.maxiter,
                       precision=prec, delta=delta, profile=profile)

    def true_rel():
        t1, t2 = b.similar(), b.similar()
        lmb.mul_(t1, D, x)
        lmb.mul_(t2, lmb.adjoint(D), t1)
        r = b.core_view() - t2.core_view()
        return float(torch.linalg.vector_norm(r) / torch.linalg.vector_norm(b.core_view()))

    prec = args.precision
    # warm-up (builds link/clover caches, JIT-free)
    for _ in range(args.warmup):
        solve(prec)
    solve("double")

    # ---- timed: mixed precision solves (value) ----
    results = []
    barrier(ws)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    if args.no_clocks:
        clocks.proc = None
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with (clocks if not args.no_clocks else _Null()):
        start.record(stream)
        # per-kernel CUDA events (for the roofline) on the last timed solve
        # only: recording them costs ~2 % of a solve
        for i in range(args.steps):
            results.append(solve(prec, profile=(i == args.steps - 1)))
        end.record(stream)
        torch.cuda.synchronize()
    barrier(ws)
    t_mixed = start.elapsed_time(end) / 1e3 / args.steps
    t_mixed = max_over_ranks(t_mixed, ws, dev)
    mixed_true = true_rel()
    mixed = results[-1]
    x_mixed = x.core_view().clone()

    # ---- timed: plain FP64 CG (the reference's arithmetic) ----
    r64 = []
    barrier(ws)
    torch.cuda.synchronize()
    start.record(stream)
    for i in range(args.fp64_steps):
        r64.append(solve("double", profile=(i == args.fp64_steps - 1)))
    end.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    t_fp64 = max_over_ranks(start.elapsed_time(end) / 1e3 / args.fp64_steps, ws, dev)
    fp64_true = true_rel()
    res64 = r64[-1]
    # error of the mixed-precision solution against the FP64 solve
    mixed_vs_fp64 = float(torch.linalg.vector_norm(x_mixed - x.core_view())
                          / torch.linalg.vector_norm(x.core_view()))
    del x_mixed

    # ---- e2e: host buffers, copies inside the timed region ----
    b_host = b.A.cpu().pin_memory()
    x_host = torch.empty_like(b_host).pin_memory()
    e2e_t = []
    barrier(ws)
    torch.cuda.synchronize()
    start.record(stream)
    for _ in range(args.steps):
        b.A.copy_(b_host, non_blocking=True)
        lmb.mark_halo_dirty_(b)
        solve(prec)
        x_host.copy_(x.A, non_blocking=True)
    end.record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    t_e2e = max_over_ranks(start.elapsed_time(end) / 1e3 / args.steps, ws, dev)
    nbytes = b_host.numel() * b_host.element_size()

    # ---- per-configuration setup (a new gauge field): link repack, SU(3)
    # check + reconstruct-12 copies, F_mu_nu, clover blocks, their FP32 /
    # int16 copies -- what update_clover! rebuilds per gauge update
    # (WilsonDiracCloverOperator.jl:392-399, 468-479).  Timed as a
    # zero-iteration solve right after the links' epochs change, minus the
    # same call with warm caches.
    def zero_solve():
        lmb.clear_matrix_(x)
        return lmb.cg_(x, A, b, rtol=args.rtol, maxiter=0, precision=prec, delta=delta)

    zero_solve()
    setup_samples = []
    for _ in range(3):
        _, warm = _timed(zero_solve, stream)
        for u in U:
            lmb.mark_halo_dirty_(u)
        _, cold = _timed(zero_solve, stream)
        setup_samples.append(cold - warm)
    setup_ms = statistics.median(setup_samples) * 1e3

    # ---- roofline of the dominant stencil kernel (mixed solve) ----
    k1_ms = sum(r.dslash_ms for r in results)
    k2_ms = sum(r.update_ms for r in results)
    k1_n = sum(r.dslash_launches for r in results)
    k2_n = sum(r.update_launches for r in results)
    peak, peak_kind = measured_peak()
    dominant = "K2 (D^+ tmp fused with the CG update)" if k2_ms >= k1_ms \
        else "K1 (tmp = D p with |tmp|^2)"
    lr, lr64 = mixed.link_reals, res64_link_reals(r64)
    if k2_ms >= k1_ms:
        per_launch_ms, bps = k2_ms / max(k2_n, 1), k2_bytes(prec, lr)
        tkey = f"k2_{prec}"
    else:
        per_launch_ms, bps = k1_ms / max(k1_n, 1), k1_bytes(prec, lr)
        tkey = f"k1_{prec}"
    achieved = bps * sites / (per_launch_ms * 1e-3) / 1e9
    traffic = traffic_per_site().get(tkey)
    k1_gbs = k1_bytes(prec, lr) * sites / (k1_ms / max(k1_n, 1) * 1e-3) / 1e9
    k2_gbs = k2_bytes(prec, lr) * sites / (k2_ms / max(k2_n, 1) * 1e-3) / 1e9
    k1_64 = sum(r.dslash_ms for r in r64) / max(sum(r.dslash_launches for r in r64), 1)
    k2_64 = sum(r.update_ms for r in r64) / max(sum(r.update_launches for r in r64), 1)
    gbs64 = k1_bytes("double", lr64) * sites / (k1_64 * 1e-3) / 1e9
    gbs64_k2 = k2_bytes("double", lr64) * sites / (k2_64 * 1e-3) / 1e9
    gflops = lambda ms: FLOPS_PER_SITE_M * sites / (ms * 1e-3) / 1e9

    line = {
        "metric": METRIC, "value": t_mixed, "unit": "s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_mixed * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 arithmetic on int16 storage, f64 reliable updates"
        if prec == "half" else "f32 inner, f64 reliable updates",
        "data": "synthetic",
        "config": {
            "workload": ("Wilson-clover D'D CG to FP64 true residual "
                         f"{args.rtol:g}, {L[0]}x{L[1]}x{L[2]}x{L[3]}, "
                         f"kappa {args.kappa}, cSW {args.csw}, links "
                         f"exp({args.amplitude} i H) seed 1, Gaussian source "
                         "seed 2, zero start"),
            "lattice": list(L), "sites": sites, "inner_precision": prec,
            "reliable_delta": delta,
            "l2": "inputs larger than L2 (links 1.2 GB + clover), no flush",
            "parallelism": f"replicas x{ws}",
        },
        "mixed": {"time_s": t_mixed, "iterations": mixed.iterations,
                  "reliable_updates": mixed.reliable_updates,
                  "true_rel_residual": mixed_true,
                  "solution_rel_diff_vs_fp64": mixed_vs_fp64},
        "fp64": {"time_s": t_fp64, "iterations": res64.iterations,
                 "true_rel_residual": fp64_true},
        "speedup_mixed_vs_fp64": t_fp64 / t_mixed,
        "dslash": {
            "fp64_k1_gbs": gbs64, "fp64_k2_gbs": gbs64_k2,
            "fp64_k1_gflops_M": gflops(k1_64), "link_reals": lr,
            "fp64_k1_ms": k1_64, "fp64_k2_ms": k2_64,
            f"{prec}_k1_gbs": k1_gbs, f"{prec}_k2_gbs": k2_gbs,
            f"{prec}_k1_ms": k1_ms / max(k1_n, 1),
            f"{prec}_k2_ms": k2_ms / max(k2_n, 1),
            f"{prec}_k1_gflops_M": gflops(k1_ms / max(k1_n, 1)),
        },
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved,
                     "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak,
                     "bytes_per_site": bps,
                     "traffic": traffic * sites if traffic else None,
                     "k1_frac": k1_gbs / peak, "k2_frac": k2_gbs / peak,
                     "fp64_k1_frac": gbs64 / peak, "fp64_k2_frac": gbs64_k2 / peak},
        "setup_ms": setup_ms,
        "e2e": {"value": t_e2e, "unit": "s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes},
        "gpu_launches": int(sum(r.kernel_launches for r in results)),
    }
    if not args.no_clocks:
        line["clocks"] = clocks.summary()
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        t_iter, n, cores = cpu_fp64_cg_seconds_per_iteration(
            L, args.kappa, args.csw, args.amplitude, args.cpu_seconds)
        line["cpu_baseline"] = {
            "value": t_iter * res64.iterations, "unit": "s", "cores": cores,
            "kind": "port",
            "sample": (f"{n} FP64 CG iterations of the oracle on the full "
                       f"lattice ({t_iter:.3f} s each) x {res64.iterations} "
                       "iterations of the FP64 solve")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def res64_link_reals(results):
    return results[-1].link_reals if results else 18


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _timed(fn, stream):
    import torch
    a, b = _events()
    torch.cuda.synchronize()
    a.record(stream)
    out = fn()
    b.record(stream)
    torch.cuda.synchronize()
    return out, a.elapsed_time(b) / 1e3


def run_wilson8(args):
    """Plain Wilson D'D CG, FP64, 8^4, kappa 0.125, links
    exp(0.3 i H) seed 1, source seed 2; GPU solve and the CPU oracle's full
    solve on all host cores."""
    import numpy as np
    import torch
    import lmb200 as lmb
    from oracle import oracle as orc
    L = (8, 8, 8, 8)
    U = lmb.random_su3_links(L, 0.3, 1)
    b = lmb.gaussian_fermion(L, 3, 4, 2, phases=PHASES)
    D = lmb.WilsonDiracOperator4D(U, 0.125)
    A = lmb.DdagDOp(D, b.similar())
    x = b.similar()
    st = torch.cuda.current_stream()
    for _ in range(args.warmup):
        lmb.clear_matrix_(x)
        lmb.cg_(x, A, b, rtol=1e-10)
    ts = []
    for _ in range(args.steps):
        lmb.clear_matrix_(x)
        res, t = _timed(lambda: lmb.cg_(x, A, b, rtol=1e-10), st)
        ts.append(t)
    orc.build()
    orc.set_num_threads(os.cpu_count() or 1)
    Uh = orc.random_su3_links(L, 0.3, 1)
    bh = orc.gaussian_field(L, 3, 4, 2)
    op = orc.Operator(orc.OP_WILSON, Uh, L, kappa=0.125)
    t0 = time.perf_counter()
    xh, rh = orc.cg_ddagd(op, bh, rtol=1e-10)
    t_cpu = time.perf_counter() - t0
    err = float(np.linalg.norm(x.gather_matrix() - xh) / np.linalg.norm(xh))
    print(json.dumps({"workload": "Wilson D'D CG FP64 8^4, kappa 0.125", "gpu_s": statistics.median(ts),
                      "gpu_iterations": res.iterations, "cpu_s": t_cpu, "cpu_iterations": rh["iterations"],
                      "cpu_cores": orc.num_threads(), "solution_rel_diff_vs_oracle": err,
                      "converged": res.converged}), flush=True)


def run_hisq(args):
    """HISQ smearing (fat7+Lepage, U(3), fat7+Naik) on 48^3x96
    links exp(0.25 i H), then staggered D'D CG at mass 0.01 to 1e-10 with FP32
    (and int16) fat/long links and fields, FP64 reliable updates; FP64 CG for
    comparison."""
    import torch
    import lmb200 as lmb
    L = tuple(int(v) for v in (args.lattice if args.lattice != "32,32,32,64"
                                else "48,48,48,96").split(","))
    sites = L[0] * L[1] * L[2] * L[3]
    U = lmb.random_su3_links(L, 0.25, 1, nw=3)
    st = torch.cuda.current_stream()
    links, t_smear = _timed(lambda: lmb.hisq_links_from_thin(U, 0.0), st)
    del links  # the timed call reuses the cached blocks (no cudaMalloc inside)
    links, t_smear = _timed(lambda: lmb.hisq_links_from_thin(U, 0.0), st)
    D = lmb.HISQDiracOperator4D(links, 0.01, 0.0)
    b = lmb.gaussian_fermion(L, 3, 1, 2, nw=3, phases=PHASES)
    A = lmb.DdagDOp(D, b.similar())
    x = b.similar()
    out = {"workload": "HISQ smearing + staggered D'D CG, %dx%dx%dx%d, m 0.01" % L,
           "smear_s": t_smear}
    # algorithmic bytes per site (each link matrix once: 4 fat + 4 Naik x 18
    # reals; K1 links + in + out, K2 links + in + p + r (rw) + x (rw)):
    # FP32 / FP64 156 and 180 reals; int16 links 8 x 36 B, spinor 16 B + 4 B
    # norm, x FP32 24 B
    kbytes = {"single": (156 * 4, 180 * 4), "double": (156 * 8, 180 * 8),
              "half": (288 + 2 * 20, 288 + 4 * 20 + 2 * 24)}
    for prec in ("single", "half", "double"):
        lmb.clear_matrix_(x)
        lmb.cg_(x, A, b, rtol=1e-10, precision=prec, maxiter=args.maxiter)
        lmb.clear_matrix_(x)
        res, t = _timed(lambda: lmb.cg_(x, A, b, rtol=1e-10, precision=prec,
                                         maxiter=args.maxiter, profile=True), st)
        k1 = res.dslash_ms / max(res.dslash_launches, 1)
        k2 = res.update_ms / max(res.update_launches, 1)
        b1, b2 = kbytes[prec]
        out[prec] = {"time_s": t, "iterations": res.iterations, "converged": res.converged,
                     "true_rel_residual": res.true_residual_norm / max(1e-300, float(
                         torch.linalg.vector_norm(b.core_view()))),
                     "reliable_updates": res.reliable_updates,
                     "k1_ms": k1, "k1_gbs": b1 * sites / (k1 * 1e-3) / 1e9,
                     "k2_ms": k2, "k2_gbs": b2 * sites / (k2 * 1e-3) / 1e9}
    out["speedup_single_vs_fp64"] = out["double"]["time_s"] / out["single"]["time_s"]
    out["speedup_half_vs_fp64"] = out["double"]["time_s"] / out["half"]["time_s"]
    print(json.dumps(out), flush=True)


# The reference's published HISQ Dslash table (one H100 NVL, FP64, m 0,
# eps_N -0.083, antiperiodic t; ms per full-lattice application, median):
# LatticeMatrices v1.1.0 and SIMULATeQCD 767a1b1
# (benchmark/HISQ_DIRAC_BENCHMARK_2026-08-17.md:66-69)
HISQ_PUBLISHED_MS = {8: (0.11104, 0.01431), 16: (0.18496, 0.05011),
                     24: (0.64086, 0.24036), 32: (2.56497, 0.70998)}


def run_hisq_dslash(args):
    """One full-lattice HISQ D application, FP64, m 0, eps_N -0.083,
    antiperiodic t, at 8^4, 16^4, 24^4 and 32^4, smearing excluded, with the
    reference's protocol (input and output swapped after every application,
    median of 9 samples; benchmark/HISQ_DIRAC_BENCHMARK_2026-08-17.md:10-40).
    `resident`: the stencil on the library's resident fields (what one Krylov
    iteration pays); `api`: mul! through the public API on padded fields,
    which adds the layout conversion of input and output.  Links exp(0.25 i H)
    seed 1 (deterministic), Gaussian source seed 2.  Algorithmic bytes per
    site: 8 links x 18 reals + in + out = 156 reals (1248 B FP64, 624 B FP32)."""
    import torch
    import lmb200 as lmb
    peak, peak_kind = measured_peak()
    st = torch.cuda.current_stream()
    rows = []
    for n in (int(v) for v in args.hisq_sizes.split(",")):
        L = (n, n, n, n)
        sites = n ** 4
        U = lmb.random_su3_links(L, 0.25, 1, nw=3)
        links = lmb.hisq_links_from_thin(U, -0.083)
        D = lmb.HISQDiracOperator4D(links, 0.0, -0.083)
        psi = lmb.gaussian_fermion(L, 3, 1, 2, nw=3, phases=PHASES)
        out = psi.similar()
        napply = max(20, min(2000, int(2e8 // sites)))
        row = {"L": n, "sites": sites, "napply_per_sample": napply}
        for prec, rb in (("double", 8), ("single", 4)):
            samples = [lmb.operator_timing(D, psi, napply, precision=prec) for _ in range(args.samples)]
            ms = statistics.median(samples)
            gbs = 156 * rb * sites / (ms * 1e-3) / 1e9
            row[prec] = {"resident_ms_median": ms, "resident_ms_min": min(samples),
                         "gbs": gbs, "hbm_frac": gbs / peak}
        # public API, FP64: mul!(out, D, psi), swapping the two fields
        a, b = psi, out
        for _ in range(3):
            lmb.mul_(b, D, a)
            a, b = b, a
        samples = []
        for _ in range(args.samples):
            k = max(5, napply // 4)
            def loop():
                nonlocal a, b
                for _ in range(k):
                    lmb.mul_(b, D, a)
                    a, b = b, a
            _, sec = _timed(loop, st)
            samples.append(sec * 1e3 / k)
        row["double"]["api_ms_median"] = statistics.median(samples)
        if n in HISQ_PUBLISHED_MS:
            lm, sq = HISQ_PUBLISHED_MS[n]
            row["published_h100_ms"] = {"latticematrices_median": lm, "simulateqcd_median": sq}
            row["speedup_vs_latticematrices_h100"] = lm / row["double"]["resident_ms_median"]
        rows.append(row)
        del U, links, D, psi, out, a, b
        torch.cuda.empty_cache()
    print(json.dumps({"workload": "HISQ Dslash FP64, m 0, eps_N -0.083, antiperiodic t, one full-lattice "
                                  "application (smearing excluded)",
                      "peak_gbs": peak, "peak_kind": peak_kind, "rows": rows}), flush=True)


def run_batched(args):
    """16 Gaussian right-hand sides of Wilson D'D on 32^4 plus
    lattices 8^4 x4, 12^4 x4, 16^4 x2, 24^4 x1, in one batched solve (FP32
    arithmetic on FP32 or int16 iterated fields, FP64 reliable updates, CUDA
    graph, autotuned kernel family / group size / tile); compared with
    solving the same systems one right-hand side at a time with the
    single-lattice kernels at the same storage precision."""
    import torch
    import lmb200 as lmb
    shapes = [((32, 32, 32, 32), 16), ((8, 8, 8, 8), 4), ((12, 12, 12, 12), 4),
              ((16, 16, 16, 16), 2), ((24, 24, 24, 24), 1)]
    if args.batched_small:       # a small case of the same kernels (profiling)
        shapes = [((16, 16, 16, 16), 8), ((8, 8, 8, 8), 4)]
    systems = []
    for i, (L, n) in enumerate(shapes):
        U = lmb.random_su3_links(L, 0.2, 10 + i)
        D = lmb.WilsonDiracOperator4D(U, 0.12)
        pairs = []
        for r in range(n):
            b = lmb.gaussian_fermion(L, 3, 4, 100 * i + r, phases=PHASES)
            pairs.append((b.similar(), b))
        systems.append((D, pairs))
    st = torch.cuda.current_stream()
    peak, peak_kind = measured_peak()
    rb = {"single": 96, "half": 52}     # bytes of one stored Wilson spinor (int16: + norm)

    def clear():
        for _, pairs in systems:
            for x, _ in pairs:
                lmb.clear_matrix_(x)

    out = {}
    for prec in ("single", "half"):
        clear()
        lmb.cg_batched_(systems, rtol=1e-10, precision=prec)          # tuning + warm-up
        clear()
        (res, tune), t_batch = _timed(lambda: lmb.cg_batched_(systems, rtol=1e-10, precision=prec), st)

        def sequential():
            rs = []
            for D, pairs in systems:
                A = lmb.DdagDOp(D, pairs[0][1].similar())
                for x, b in pairs:
                    rs.append(lmb.cg_(x, A, b, rtol=1e-10, precision=prec))
            return rs
        clear()
        sequential()
        clear()
        rs, t_seq = _timed(sequential, st)
        # Algorithmic bytes of the two stencil stages of one CG iteration with
        # every system running, what the tuner's ms_stencils times: the
        # reconstruct-12 FP32 links (192 B/site) once per group of NB
        # right-hand sides by each stage, and per right-hand side K1 p + tmp,
        # K2 tmp + p + r rw (spinors S) + x_low rw (FP32, 96 B).
        nb = max(int(tune["rhs_block"]), 1)
        S = rb[prec]
        k12 = sum(L[0] * L[1] * L[2] * L[3] * (384 * (-(-n // nb)) + (6 * S + 192) * n) for L, n in shapes)
        gbs = k12 / (tune["ms_stencils"] * 1e-3) / 1e9
        out[prec] = {"batched_s": t_batch, "sequential_s": t_seq, "speedup": t_seq / t_batch,
                     "all_converged": all(r.converged for r in res),
                     "sequential_converged": all(r.converged for r in rs),
                     "max_iterations": max(r.iterations for r in res),
                     "max_rel_residual": max(r.relative_residual for r in res),
                     "tuning": tune,
                     "roofline": {"kernels": "K1 + K2 of one iteration, every system running",
                                  "bytes": k12, "gbs": gbs, "peak_gbs": peak, "peak_kind": peak_kind,
                                  "hbm_frac": gbs / peak}}
    total_sites_rhs = sum(L[0] * L[1] * L[2] * L[3] * n for L, n in shapes)
    print(json.dumps({"workload": "batched Wilson D'D CG: " + " + ".join(
                          "%d^4 x%d" % (L[0], n) for L, n in shapes),
                      "site_rhs": total_sites_rhs, **out,
                      "speedup_half_batched_vs_single_sequential":
                          out["single"]["sequential_s"] / out["half"]["batched_s"]}), flush=True)


def run_force(args):
    """Fermion force dS/dU, S = phi^+ (D^+D)^-1 phi, HISQ smearing on 24^4
    (mass 0.02, links exp(0.2 i H)), checked by central finite differences
    (eps 1e-5) along random link directions V:
        dS/dt = (S(U + eps V) - S(U - eps V)) / (2 eps).
    S(U') - S(U) is formed as phi^+ d with A' d = phi - A' x0, x0 = A^-1 phi:
    the error of x0 cancels between the two sides, and d is solved to a
    relative tolerance of its own size, so the difference of two nearly
    equal actions never loses digits to cancellation."""
    import numpy as np
    import torch
    import lmb200 as lmb
    L = tuple(int(v) for v in (args.lattice if args.lattice != "32,32,32,64"
                                else "24,24,24,24").split(","))
    U = lmb.random_su3_links(L, 0.2, 1, nw=3)
    phi = lmb.gaussian_fermion(L, 3, 1, 2, nw=3, phases=PHASES)
    cache = lmb.HISQDiracCache4D(U, 0.02, 0.0)
    dU = [u.similar() for u in U]
    st = torch.cuda.current_stream()
    lmb.hisq_fermion_force_(dU, cache, phi, rtol=1e-12)
    for d in dU:
        lmb.clear_matrix_(d)
    res, t_force = _timed(lambda: lmb.hisq_fermion_force_(dU, cache, phi, rtol=1e-12), st)
    G = [d.core_view().clone() for d in dU]
    base = [u.core_view().clone() for u in U]
    gen = torch.Generator(device="cuda").manual_seed(5)
    h = 1e-5
    x0, t, r, d = phi.similar(), phi.similar(), phi.similar(), phi.similar()
    lmb.cg_(x0, lmb.DdagDOp(cache, phi.similar()), phi, rtol=1e-12, maxiter=50000)

    def side(sign, V):
        for u, b, v in zip(U, base, V):
            u.core_view().copy_(b + sign * h * v)
            lmb.mark_halo_dirty_(u)
        A = lmb.DdagDOp(lmb.HISQDiracCache4D(U, 0.02, 0.0), phi.similar())
        A.mul_(t, x0)
        r.core_view().copy_(phi.core_view() - t.core_view())
        lmb.mark_halo_dirty_(r)
        lmb.clear_matrix_(d)
        lmb.cg_(d, A, r, rtol=1e-12, maxiter=50000)
        return lmb.dot(phi, d).real

    ans, fds = [], []
    for k in range(args.fd_directions):
        V = [torch.randn(b.shape, dtype=b.dtype, device=b.device, generator=gen) for b in base]
        fds.append((side(+1, V) - side(-1, V)) / (2 * h))
        ans.append(sum(float((g.conj() * v).sum().real) for g, v in zip(G, V)))
    for u, b in zip(U, base):
        u.core_view().copy_(b)
        lmb.mark_halo_dirty_(u)
    ans, fds = np.array(ans), np.array(fds)
    print(json.dumps({"workload": "HISQ fermion force %dx%dx%dx%d m 0.02" % L,
                      "force_s": t_force, "cg_iterations": res.iterations,
                      "fd_directions": args.fd_directions, "fd_eps": h,
                      "max_rel_diff_vs_fd": float(np.max(np.abs(ans - fds) / np.abs(fds))),
                      "max_diff_over_rms_fd": float(np.max(np.abs(ans - fds)) / np.sqrt(np.mean(fds ** 2))),
                      "rel_diff_norm_vs_fd": float(np.linalg.norm(ans - fds) / np.linalg.norm(fds))}),
          flush=True)


def run_clover_force(args):
    """Wilson-clover fermion force dS/dU, S = phi^+ (D^+D)^-1 phi, on 24^4
    (kappa 0.1355, cSW 1.0, links exp(0.2 i H)), checked by central finite
    differences (eps 1e-5) along random link directions with the
    difference-solve form of run_force."""
    import numpy as np
    import torch
    import lmb200 as lmb
    L = tuple(int(v) for v in (args.lattice if args.lattice != "32,32,32,64"
                                else "24,24,24,24").split(","))
    kappa, csw = args.kappa, args.csw
    U = lmb.random_su3_links(L, 0.2, 1)
    phi = lmb.gaussian_fermion(L, 3, 4, 2, phases=PHASES)
    D = lmb.WilsonDiracCloverOperator4D(U, kappa, csw)
    dU = [u.similar() for u in U]
    st = torch.cuda.current_stream()
    lmb.wilson_clover_fermion_force_(dU, D, phi, rtol=1e-12)
    for d in dU:
        lmb.clear_matrix_(d)
    res, t_force = _timed(lambda: lmb.wilson_clover_fermion_force_(dU, D, phi, rtol=1e-12), st)
    G = [d.core_view().clone() for d in dU]
    base = [u.core_view().clone() for u in U]
    gen = torch.Generator(device="cuda").manual_seed(5)
    h = 1e-5
    x0, t, r, d = phi.similar(), phi.similar(), phi.similar(), phi.similar()
    lmb.cg_(x0, lmb.DdagDOp(D, phi.similar()), phi, rtol=1e-12, maxiter=50000)

    def side(sign, V):
        for u, b, v in zip(U, base, V):
            u.core_view().copy_(b + sign * h * v)
            lmb.mark_halo_dirty_(u)
        A = lmb.DdagDOp(lmb.WilsonDiracCloverOperator4D(U, kappa, csw), phi.similar())
        A.mul_(t, x0)
        r.core_view().copy_(phi.core_view() - t.core_view())
        lmb.mark_halo_dirty_(r)
        lmb.clear_matrix_(d)
        lmb.cg_(d, A, r, rtol=1e-12, maxiter=50000)
        return lmb.dot(phi, d).real

    ans, fds = [], []
    for k in range(args.fd_directions):
        V = [torch.randn(b.shape, dtype=b.dtype, device=b.device, generator=gen) for b in base]
        fds.append((side(+1, V) - side(-1, V)) / (2 * h))
        ans.append(sum(float((g.conj() * v).sum().real) for g, v in zip(G, V)))
    for u, b in zip(U, base):
        u.core_view().copy_(b)
        lmb.mark_halo_dirty_(u)
    ans, fds = np.array(ans), np.array(fds)
    print(json.dumps({"workload": "Wilson-clover fermion force %dx%dx%dx%d kappa %g cSW %g" % (L + (kappa, csw)),
                      "force_s": t_force, "cg_iterations": res.iterations,
                      "fd_directions": args.fd_directions, "fd_eps": h,
                      "max_rel_diff_vs_fd": float(np.max(np.abs(ans - fds) / np.abs(fds))),
                      "max_diff_over_rms_fd": float(np.max(np.abs(ans - fds)) / np.sqrt(np.mean(fds ** 2))),
                      "rel_diff_norm_vs_fd": float(np.linalg.norm(ans - fds) / np.linalg.norm(fds))}),
          flush=True)


def run_dw(args):
    """Mobius domain-wall D5^+ D5 CG (DiracOperators_5D.jl; the Mobius
    example of benchmark/ddagd_cg/README.md): 16^3x32, L5 12, mass 0.1,
    M -1, b 2, c 1, links exp(0.2 i H) seed 1, unit complex Gaussian 5D
    source (torch generator seed 2), phases (1,1,1,-1); FP64 CG and the FP32
    / int16 inner solves with FP64 reliable updates, each to FP64 true
    residual 1e-10, zero start."""
    import contextlib
    import torch
    import lmb200 as lmb
    L = tuple(int(v) for v in (args.lattice if args.lattice != "32,32,32,64"
                                else "16,16,16,32").split(","))
    L5 = args.l5
    V5 = L[0] * L[1] * L[2] * L[3] * L5
    U = lmb.random_su3_links(L, 0.2, 1)
    with contextlib.redirect_stdout(sys.stderr):
        D = lmb.D5DW_MobiusDomainwallOperator5D(U, L5, 0.1, -1.0, 2.0, 1.0)
    b = lmb.LatticeMatrix(3, 4, 5, L + (L5,), phases=PHASES + (1,))
    g = torch.Generator(device="cuda").manual_seed(2)
    b.core_view().copy_(torch.randn(b.core_view().shape, dtype=torch.complex128,
                                    device="cuda", generator=g))
    lmb.mark_halo_dirty_(b)
    A = lmb.DdagDOp(D, b.similar())
    x = b.similar()
    st = torch.cuda.current_stream()
    bn = float(torch.linalg.vector_norm(b.core_view()))
    out = {"workload": "Mobius DW D5'D5 CG %dx%dx%dx%d x L5 %d, m 0.1, M -1, b 2, c 1" % (L + (L5,))}
    for prec in ("double", "single", "half"):
        lmb.clear_matrix_(x)
        lmb.cg_(x, A, b, rtol=args.rtol, precision=prec, maxiter=args.maxiter)
        lmb.clear_matrix_(x)
        res, t = _timed(lambda: lmb.cg_(x, A, b, rtol=args.rtol, precision=prec,
                                         maxiter=args.maxiter, profile=True), st)
        k1 = res.dslash_ms / max(res.dslash_launches, 1)
        k2 = res.update_ms / max(res.update_launches, 1)
        sp, xb = spinor_bytes(prec), x_bytes(prec)
        links = 4 * res.link_reals * REAL_BYTES[prec] / L5  # 4D links shared by L5 slices
        # bytes per 5D site the two-pass kernels move (each operand once):
        #  K1 = D5 p:  Y = B p + C F p (p, Y), stencil (Y, p, out, links)
        #  K2 = D5^+ t + CG update: stencil (t, Z, links), local (t, Z, p,
        #       r rw, x rw)
        k1_b = 5 * sp + links
        k2_b = 7 * sp + 2 * xb + links
        # the operator's compulsory bytes (a one-pass kernel): in, out, links
        k1_min = 2 * sp + links
        k2_min = 4 * sp + 2 * xb + links
        out[prec] = {"time_s": t, "iterations": res.iterations, "converged": res.converged,
                     "true_rel_residual": res.true_residual_norm / bn,
                     "reliable_updates": res.reliable_updates,
                     "k1_ms": k1, "k1_gbs": k1_b * V5 / (k1 * 1e-3) / 1e9,
                     "k1_gbs_compulsory": k1_min * V5 / (k1 * 1e-3) / 1e9,
                     "k2_ms": k2, "k2_gbs": k2_b * V5 / (k2 * 1e-3) / 1e9,
                     "k2_gbs_compulsory": k2_min * V5 / (k2 * 1e-3) / 1e9}
    for prec in ("single", "half"):
        out["speedup_%s_vs_fp64" % prec] = out["double"]["time_s"] / out[prec]["time_s"]
    out["hbm_peak_gbs"] = measured_peak()[0]
    print(json.dumps(out), flush=True)


def run_evenodd(args):
    """D x = b on the headline lattice (32^3x64 Wilson-clover, kappa 0.1355,
    cSW 1.0, links exp(0.2 i H) seed 1, Gaussian source seed 2): the
    even/odd Schur solve (solve_evenodd_) against the reference's route to
    the same x, cg!(x, DdagDOp(D), D'b), both at rtol 1e-10, FP64 and int16
    inner iterations; every solve's |b - D x| / |b| is recomputed in FP64."""
    import torch
    import lmb200 as lmb
    L = tuple(int(v) for v in args.lattice.split(","))
    U = lmb.random_su3_links(L, args.amplitude, 1)
    b = lmb.gaussian_fermion(L, 3, 4, 2, phases=PHASES)
    D = lmb.WilsonDiracCloverOperator4D(U, args.kappa, args.csw)
    Db = b.similar()
    lmb.mul_(Db, lmb.adjoint(D), b)
    A = lmb.DdagDOp(D, b.similar())
    x, t = b.similar(), b.similar()
    st = torch.cuda.current_stream()
    bn = float(torch.linalg.vector_norm(b.core_view()))

    def rel_residual():
        lmb.mul_(t, D, x)
        return float(torch.linalg.vector_norm(b.core_view() - t.core_view())) / bn

    out = {"workload": "Wilson-clover D x = b %dx%dx%dx%d, kappa %g, cSW %g" % (L + (args.kappa, args.csw))}
    for prec in ("double", "half"):
        for route in ("evenodd", "ddagd_cg"):
            if route == "evenodd":
                solve = lambda: lmb.solve_evenodd_(x, D, b, rtol=args.rtol, precision=prec,
                                                   maxiter=args.maxiter)
            else:
                def solve():
                    lmb.clear_matrix_(x)
                    return lmb.cg_(x, A, Db, rtol=args.rtol, precision=prec, maxiter=args.maxiter)
            solve()
            res, sec = _timed(solve, st)
            out["%s_%s" % (route, prec)] = {"time_s": sec, "iterations": res.iterations,
                                            "converged": res.converged,
                                            "rel_residual_b_minus_Dx": rel_residual()}
    for prec in ("double", "half"):
        out["speedup_%s" % prec] = out["ddagd_cg_%s" % prec]["time_s"] / out["evenodd_%s" % prec]["time_s"]
    print(json.dumps(out), flush=True)


def run_sharded(args):
    """The 32^3x64 Wilson-clover D'D CG on the native sharded operators
    (lmb_set_process_grid): the lattice split over a process grid of the
    ranks (--grid, default 1,1,1,N), every rank solving its block with faces
    exchanged over NCCL under the interior sites and every reduction summed
    over the ranks.  One rank with --split (default t) exchanges its faces
    with itself: the sharded machinery on one GPU, timed beside the same
    solve on the unsplit lattice.  Every rank builds the global input (links
    seed 1, source seed 2, as the headline workload) and keeps its padded
    block, halo included; strong scaling (the lattice is fixed)."""
    import ctypes

    import numpy as np
    import torch
    import lmb200 as lmb
    from lmb200._lib import (CGParams, CGResultC, Context, LINKS_THIN, OP_WILSON_CLOVER, PREC)
    from lmb200.distributed import shared_unique_id
    from lmb200._lib import nccl_unique_id

    rank, local, ws = dist_setup("nccl")
    dev = torch.device("cuda", local)
    L = tuple(int(v) for v in args.lattice.split(","))
    grid = tuple(int(v) for v in args.grid.split(",")) if args.grid else (1, 1, 1, ws)
    if int(np.prod(grid)) != ws:
        raise SystemExit(f"--grid {grid} needs {int(np.prod(grid))} ranks, running {ws}")
    if args.split:
        split = tuple(int(v) for v in args.split.split(","))
    else:
        split = tuple(int(p > 1) for p in grid) if ws > 1 else (0, 0, 0, 1)
    PN = tuple(n // p for n, p in zip(L, grid))
    coords = tuple(int(c) for c in np.unravel_index(rank, grid))

    def nb(d, step):
        c = list(coords)
        c[d] = (c[d] + step) % grid[d]
        return int(np.ravel_multi_index(c, grid))

    Ug = lmb.random_su3_links(L, args.amplitude, 1, nw=1, device=dev)
    bg = lmb.gaussian_fermion(L, 3, 4, 2, nw=1, phases=PHASES, device=dev)
    for u in Ug:
        lmb.set_halo_(u)

    def block(A):
        # padded block (halo 1) of a padded global field: storage axis 3 - d
        # is dimension d; global core index g sits at padded index g + 1
        for d in range(4):
            if grid[d] == 1:
                continue
            lo = coords[d] * PN[d]
            idx = (torch.arange(lo - 1, lo + PN[d] + 1, device=dev) % L[d]) + 1
            A = A.index_select(3 - d, idx)
        return A.contiguous()

    U = [block(u.A) for u in Ug]
    b = block(bg.A)
    x = torch.zeros_like(b)
    del Ug, bg
    torch.cuda.empty_cache()
    ctx = Context(local)
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    stream = torch.cuda.current_stream()

    def attach(on):
        if on:
            nid = shared_unique_id() if ws > 1 else nccl_unique_id()
            ctx.set_process_grid(nid, ws, rank, grid, coords, split,
                                 [nb(d, -1) for d in range(4)], [nb(d, +1) for d in range(4)])
        else:
            ctx.set_process_grid(None, 1, 0, (1, 1, 1, 1), (0, 0, 0, 0), (0, 0, 0, 0),
                                 (0, 0, 0, 0), (0, 0, 0, 0))
        ctx.set_geometry(PN, 1, PHASES, coords, 0)
        ctx.upload_links(LINKS_THIN, [u.data_ptr() for u in U], [1, 1, 1, 1], st)

    def solve(prec, profile=False):
        prm = CGParams()
        prm.op = OP_WILSON_CLOVER
        prm.kappa, prm.csw = args.kappa, args.csw
        prm.rtol, prm.atol, prm.maxiter = args.rtol, 0.0, args.maxiter
        prm.precision, prm.delta, prm.profile = PREC[prec], 0.1 if args.delta is None else args.delta, int(profile)
        x.zero_()
        res = CGResultC()
        ctx.check(ctx.lib.lmb_cg_ddagd(ctx.handle, ctypes.byref(prm), x.data_ptr(), b.data_ptr(),
                                       ctypes.byref(res), st))
        return res

    def timed(prec, steps):
        for _ in range(args.warmup if prec == args.precision else 1):
            solve(prec)
        barrier(ws)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        out = [solve(prec, profile=(i == steps - 1)) for i in range(steps)]
        e.record(stream)
        torch.cuda.synchronize()
        barrier(ws)
        sec = max_over_ranks(s.elapsed_time(e) / 1e3 / steps, ws, dev)
        r = out[-1]
        return {"seconds": sec, "iterations": r.iterations, "converged": bool(r.converged),
                "relative_residual": r.relative_residual,
                "k1_ms_per_iteration": r.dslash_ms / max(r.dslash_launches, 1),
                "k2_ms_per_iteration": r.update_ms / max(r.update_launches, 1)}

    attach(True)
    rows = {"sharded": {p: timed(p, s) for p, s in ((args.precision, args.steps), ("double", args.fp64_steps))}}
    if ws == 1:   # the same solves on the unsplit lattice
        attach(False)
        rows["unsplit"] = {p: timed(p, s) for p, s in ((args.precision, args.steps), ("double", args.fp64_steps))}
    if rank == 0:
        print(json.dumps({
            "workload": f"Wilson-clover D'D CG, {'x'.join(map(str, L))}, kappa {args.kappa}, cSW {args.csw}, "
                        f"rtol {args.rtol}, native sharded operators",
            "n_gpus": ws, "grid": grid, "split": split, "block": PN, "scaling": "strong",
            "rows": rows}), flush=True)
    ctx.set_process_grid(None, 1, 0, (1, 1, 1, 1), (0, 0, 0, 0), (0, 0, 0, 0), (0, 0, 0, 0), (0, 0, 0, 0))


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "clover":
        run_lmb(args)
    else:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        {"wilson8": run_wilson8, "hisq": run_hisq, "hisq_dslash": run_hisq_dslash, "batched": run_batched,
         "force": run_force, "clover_force": run_clover_force, "dw": run_dw,
         "evenodd": run_evenodd, "sharded": run_sharded}[args.workload](args)


if __name__ == "__main__":
    main()
