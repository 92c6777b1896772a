#!/usr/bin/env python
"""LS-MPS per-step path on B200: particle-steps/s and PPE solve time at 1M particles.

Workload (one "step" = the whole per-step path on one particle set):
  1,000,000 particles, case `mixed` (80 % jittered bulk lattice +-0.1 l0, 20 % rain on a
  20-degree plate: 3 wall layers, 4-layer film, radius-3 droplets 10-40 l0 above it),
  l0 = 1, re = 2.1 l0, max_neighbors 128; neighbor build + 14-direction classification,
  batched WLS over every particle, WLS-Laplacian PPE over all Interior / NearWall
  particles with p* = sin(0.3x) cos(0.2y) + 0.1z and b = A p*, solved to relative residual
  2e-11 (PPE relative L2 against p* <= 1e-8 for every compared solver, checked). Steps
  cycle through --sets seeded particle sets held on the device (a device-to-device copy
  into the library per step): BiCGStab's stopping iteration on one system moves by +-15 %
  with summation order, so the step time is a mean over systems. Synthetic data, seeded;
  matrices are larger than L2 (126 MB) so no flush is needed.

`value` = particles x GPUs / (device step time, CUDA events on the library's stream, max
over ranks) with the metric's solver (--solver, default `learned_multigrid`: the learned +
mixed-precision solver, i.e. mixed-precision BiCGStab started from the message-passing
network's guess, with the cell-aggregation multigrid V-cycle as its preconditioner; the same
without the network is `multigrid` in ppe_compare). `e2e` = the same
through the C ABI with host buffers: the upload from pinned memory (double-buffered: step
i + 1's copies overlap step i), the step, and the download of the pressure into pinned memory
(asynchronous: step i's result travels while step i + 1 runs; the last download is waited
for), all inside the timed region. The plain FP64 GPU BiCGStab (the reference iteration),
Jacobi FP64, MIXED, LEARNED and both with the multigrid preconditioner are timed on the same
systems beside it (means and per set).
`--impl reference` times the reference's own CPU implementation of the path.

Multi-GPU: replicas only (independent particle sets per rank), `scaling: weak`.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ls-mps_b200"))
# oracle/ (test infrastructure) is imported only by the CPU-baseline leg and the reference arm
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "PPE solve ms & particle-steps/s at 1M, learned+mixed vs plain FP64 @ L2<=1e-8"
UNIT = "particle-steps/s"
L0, RE_RATIO, MAXN = 1.0, 2.1, 128
# bench solver name -> (library solver, preconditioner, launch form). The multigrid solves
# launch eagerly (use_graph 0): with ~27 short kernels per iteration, stream launches keep the
# programmatic-dependent-launch overlap and measured ~5 % faster than the device-driven graph.
SOLVER_SPECS = {"fp64": ("fp64", "jacobi", 1), "jacobi": ("jacobi", "jacobi", 1), "mixed": ("mixed", "jacobi", 1),
                "learned": ("learned", "jacobi", 1), "multigrid": ("mixed", "multigrid", 0),
                "learned_multigrid": ("learned", "multigrid", 0)}
DTYPES = {"fp64": "f64", "jacobi": "f64", "mixed": "f64 vectors + f32 matrix",
          "learned": "f64 vectors + f32 matrix; bf16 network",
          "multigrid": "f64 vectors + f32 matrix; f32 V-cycle, f16 fine A*P",
          "learned_multigrid": "f64 vectors + f32 matrix; f32 V-cycle, f16 fine A*P; bf16 network"}


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mine", choices=["mine", "reference"])
    ap.add_argument("--particles", type=int, default=1_000_000)
    ap.add_argument("--case", default="mixed")
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--sets", type=int, default=4, help="seeded particle sets the steps cycle through")
    ap.add_argument("--solver", default="learned_multigrid", choices=sorted(SOLVER_SPECS))
    ap.add_argument("--weights", default=os.path.join(ROOT, "ls-mps_b200", "weights", "mpnn_rain200k.bin"),
                    help="network weights for the learned solver (trained by ls-mps_b200/train_mpnn.py)")
    ap.add_argument("--tol", type=float, default=2e-11,
                    help="relative residual; 2e-11 brings every compared solver to PPE relative L2 <= 1e-8 "
                         "(at 3e-11 the Jacobi-preconditioned learned solve ended at 1.07e-8 on one set)")
    ap.add_argument("--max-iter", type=int, default=20000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain-FP64 comparison solves")
    ap.add_argument("--cpu-sample-s", type=float, default=8.0, help="CPU BiCGStab sample budget (s)")
    ap.add_argument("--ref-iterations", type=int, default=20,
                    help="reference arm: BiCGStab iterations timed per step (projected to the full count)")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------
# distributed plumbing (replicas only)
# ---------------------------------------------------------------------------------------
class Dist:
    def __init__(self, want_gpu: bool):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            backend = "nccl" if (want_gpu and torch.cuda.is_available()) else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
            dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=300))
            self.pg = dist
            self.backend = backend

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def reduce(self, value: float, op: str) -> float:
        if not self.pg:
            return value
        import torch

        dev = f"cuda:{self.local_rank}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([value], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX if op == "max" else self.pg.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.err_path = self.path + ".err"
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=open(self.err_path, "w"))
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 10:
                rows.append(parts)
        os.unlink(self.path)
        err = open(self.err_path).read().strip()[:200]
        os.unlink(self.err_path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples: " + err]}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        load = [r for r in rows if (num(r[4]) or 0) >= 50] or rows
        sm = [num(r[1]) for r in load if num(r[1]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in load:
            for k, name in enumerate(names):
                if r[6 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": num(rows[0][2]),
                "reasons": sorted(reasons), "samples": len(rows), "samples_under_load": len(load),
                "power_w_max": max((num(r[3]) or 0) for r in rows)}


# ---------------------------------------------------------------------------------------
# the GPU arm
# ---------------------------------------------------------------------------------------
def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def committed_traffic():
    """Per-launch DRAM bytes of the SpMV kernel from the committed ncu summary, if any."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def step(ctx, solver, tol, max_iter, timings, stats=True):
    """One pass of the per-step path on the resident particle set. stats=False (the timed
    steps): the neighbor build, WLS and assembly return no statistics, so the host does not
    wait at the end of each phase (their times come from lsmps_get_timings)."""
    import lsmps_b200 as lib

    re = RE_RATIO * L0
    nst = ctx.build_neighbors(re, MAXN, L0, stats=stats)
    ctx.wls(re, L0, mode=1, stats=False)  # no statistics read-back: the host does not wait here
    pst = ctx.ppe_assemble("wls", 10**12, re, L0, diag_shift=0.0, stats=stats)
    sv, pc, ug = SOLVER_SPECS[solver]
    s = ctx.ppe_solve(sv, max_iter, tol, precond=pc, use_graph=ug)
    t = ctx.timings()
    timings.append({"neighbor_ms": t[1], "wls_ms": t[3], "assembly_ms": t[4], "solve_ms": s.solve_ms,
                    "iterations": s.iterations, "outer": s.outer_iterations})
    return nst, pst, s, lib


def run_mine(args, dist):
    import torch

    import lsmps_b200 as lib

    dev = dist.local_rank
    torch.cuda.set_device(dev)
    # K seeded particle sets of the workload, resident on the device; step i works on set i mod K
    # (one system's BiCGStab iteration count moves by +-15 % with summation order, so the step
    # time is a mean over systems)
    K = max(1, args.sets)
    sets = [lib.generate(None, case=args.case, particles=args.particles, l0=L0, seed=args.seed + dist.rank * K + k)
            for k in range(K)]
    n = len(sets[0][1])
    dsets = [(torch.from_numpy(np.ascontiguousarray(x)).to(f"cuda:{dev}"),
              torch.from_numpy(np.ascontiguousarray(t)).to(f"cuda:{dev}")) for x, t, _ in sets]
    ctx = lib.Context(dev)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    compare = () if args.no_compare else tuple(SOLVER_SPECS)
    if "learned" in args.solver or any("learned" in c for c in compare):
        ctx.mpnn_load(args.weights)
    L = lib.load()

    def put(k):  # device-to-device copy of set k into the context (the inputs stay resident)
        x, t = dsets[k]
        torch.cuda.synchronize()
        ctx._check(L.lsmps_upload_particles_device(ctx.h, C.c_void_p(x.data_ptr()), C.c_void_p(t.data_ptr()),
                                                   len(t)))
        ctx.n = len(t)

    timings = []
    for i in range(max(args.warmup, K)):
        put(i % K)
        nst, pst, s, _ = step(ctx, args.solver, args.tol, args.max_iter, timings)
    timings.clear()

    # ---- device-timed steps (inputs resident) ----
    clocks = ClockSampler(dev)
    launches0 = L.lsmps_launch_count()
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    l2s = []
    for i in range(args.steps):
        put(i % K)
        _, _, s, _ = step(ctx, args.solver, args.tol, args.max_iter, timings, stats=False)
        l2s.append(s.relative_l2_error)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    dist.barrier()
    clk = clocks.stop()
    launches = L.lsmps_launch_count() - launches0
    ms_step = ev0.elapsed_time(ev1) / args.steps
    ms_step_max = dist.reduce(ms_step, "max")
    launches_total = int(dist.reduce(float(launches), "sum"))
    rel_l2 = max(l2s)

    # ---- end to end through the C ABI with host buffers ----
    pins = []
    for x, t, _ in sets:
        px = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
        pt = torch.empty(n, dtype=torch.uint8, pin_memory=True).numpy()
        px[:] = x
        pt[:] = t
        pins.append((px, pt))
    U = max(int(pst.unknowns), 1)
    # two page-locked result buffers, alternated: step i's pressure travels to the host while
    # step i + 1 runs (lsmps_download_pressure_async); the last one is waited for in the region
    pin_ps = [torch.empty(4 * U, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2)]
    d2h = []
    ctx.prefetch(*pins[1 % K])  # untimed: allocates the staging buffers once
    ctx.use_prefetched()
    dist.barrier()
    t0 = time.perf_counter()
    # double-buffered uploads: the copies of step i + 1's particles overlap step i
    ctx.prefetch(*pins[0])
    for i in range(args.steps):
        ctx.use_prefetched()
        if i + 1 < args.steps:
            ctx.prefetch(*pins[(i + 1) % K])
        _, _, s_e, _ = step(ctx, args.solver, args.tol, args.max_iter, [], stats=False)
        u = int(s_e.unknowns)
        ctx.pressure_into_async(pin_ps[i % 2][:u])
        d2h.append(8 * u)
    ctx.download_wait()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    e2e_ms_max = dist.reduce(e2e_ms, "max")

    result = {
        "metric": METRIC, "unit": UNIT, "higher_is_better": True, "n_gpus": dist.world,
        "steps": args.steps, "warmup": max(args.warmup, K), "ms_per_step": ms_step_max,
        "value": n * dist.world / (ms_step_max * 1e-3),
        "scaling": "weak", "vs_baseline": None,
        "dtype": DTYPES[args.solver],
        "data": "synthetic (seeded generator; no dataset)",
        "config": {"workload": f"{args.case} {n} particles, WLS-Laplacian PPE, tol {args.tol:g}",
                   "particles": n, "case": args.case, "particle_sets": K, "seeds": [args.seed + dist.rank * K + k
                                                                                    for k in range(K)],
                   "l0": L0, "re": RE_RATIO * L0, "max_neighbors": MAXN, "solver": args.solver,
                   "ppe_unknowns": int(pst.unknowns), "ppe_nnz": int(pst.nnz), "pairs": int(nst.pairs),
                   "parallelism": f"replicas x{dist.world}", "l2_flush": "inputs larger than L2 (matrix > 126 MB)"},
        "e2e": {"value": n * dist.world / (e2e_ms_max * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": int(pins[0][0].nbytes + pins[0][1].nbytes),
                "d2h_bytes_per_step": int(sum(d2h) / len(d2h)), "ms_per_step": e2e_ms_max},
        "gpu_launches": launches_total,
        "clocks": clk,
        "phases_ms": {k: statistics.mean(t[k] for t in timings) for k in timings[0]},
        "ppe": {"relative_l2_error": rel_l2, "relative_residual": s.relative_residual,
                "iterations": statistics.mean(t["iterations"] for t in timings),
                "outer_iterations": s.outer_iterations, "converged": bool(s.converged),
                "solve_ms": statistics.mean(t["solve_ms"] for t in timings)},
    }

    # ---- the plain FP64 GPU BiCGStab (and the stages between) on the same systems ----
    if not args.no_compare:
        names = compare
        per = {nm: [] for nm in names}
        re = RE_RATIO * L0
        for nm in names:  # first solves: launch-shape autotuning, graph and buffer set-up
            sv, pc, ug = SOLVER_SPECS[nm]
            ctx.ppe_solve(sv, args.max_iter, args.tol, precond=pc, use_graph=ug)
        for k in reversed(range(K)):  # ends on set 0, whose system the CPU baseline reads
            put(k)
            step(ctx, args.solver, args.tol, args.max_iter, [])
            for nm in names:
                # a fresh assembly before each solve, so each solver pays its own set-up (SELL
                # copies, multigrid hierarchy, network graph) as in a step
                ctx.ppe_assemble("wls", 10**12, re, L0, diag_shift=0.0)
                sv, pc, ug = SOLVER_SPECS[nm]
                r = ctx.ppe_solve(sv, args.max_iter, args.tol, precond=pc, use_graph=ug)
                per[nm].append({"solve_ms": r.solve_ms, "iterations": r.iterations, "converged": bool(r.converged),
                                "relative_l2_error": r.relative_l2_error, "relative_residual": r.relative_residual})
        cmp = {nm: {"solve_ms": statistics.mean(x["solve_ms"] for x in v),
                    "iterations": statistics.mean(x["iterations"] for x in v),
                    "converged": all(x["converged"] for x in v),
                    "relative_l2_error": max(x["relative_l2_error"] for x in v),
                    "per_set": list(reversed(v))} for nm, v in per.items()}
        result["ppe_compare"] = cmp
        result["speedup_vs_plain_fp64"] = cmp["fp64"]["solve_ms"] / result["ppe"]["solve_ms"]
        result["l2_target"] = {"bound": 1e-8, "met": bool(rel_l2 <= 1e-8 and all(
            c["converged"] and c["relative_l2_error"] <= 1e-8 for c in cmp.values()))}

    # ---- the precision form's error against FP64, per result (WLS on the reference's quadratic
    # field: gradient and Laplacian RMS; the solvers' PPE relative L2 is in ppe_compare) ----
    if not args.no_compare:
        re = RE_RATIO * L0
        wp = {}
        for name, prec in (("fp64", 0), ("fp32_refined", 1)):
            ctx.wls(re, L0, mode=1, precision=prec)  # warm (autotuning)
            w = ctx.wls(re, L0, mode=1, precision=prec)
            wp[name] = {"ms": ctx.timings()[3], "rms_gradient_error": w.rms_gradient_error,
                        "max_gradient_error": w.max_gradient_error, "rms_laplacian_error": w.rms_laplacian_error,
                        "max_laplacian_error": w.max_laplacian_error, "fp64_fallback": int(w.fp64_fallback)}
        result["wls_precision"] = wp
        ctx.wls(re, L0, mode=1)  # back to the step's FP64 WLS and its system for the kernel benches
        ctx.ppe_assemble("wls", 10**12, re, L0, diag_shift=0.0)

    # ---- roofline of the dominant kernel (the solver's SpMV) and the other kernels ----
    peak, peak_kind = measured_hbm_peak()
    kern = {}
    for name, kid in (("spmv32", lib.KB_SPMV32), ("spmv64", lib.KB_SPMV64), ("nbr_scan", lib.KB_NBR_SCAN),
                      ("nbr_compact", lib.KB_NBR_COMPACT), ("wls", lib.KB_WLS)) + (
                          (("mpnn_layer", lib.KB_MPNN_LAYER),) if "learned" in args.solver else ()) + (
                          (("mg_vcycle", lib.KB_MG_VCYCLE),) if "multigrid" in args.solver else ()):
        ms, nbytes = ctx.kernel_bench(kid, 20)
        gbs = nbytes / (ms * 1e-3) / 1e9
        kern[name] = {"ms": ms, "alg_bytes": nbytes, "achieved_gbs": gbs, "frac": gbs / peak}
    # the all-particle WLS against the measured FP64 peak (its bound): ~170 FLOPs per pair (the
    # moment and right-hand-side passes) and ~800 per particle (9 x 9 Cholesky and two solves)
    pk_ms, pk_flops = ctx.kernel_bench(lib.KB_FP64_PEAK, 5)
    fp64_peak = pk_flops / (pk_ms * 1e-3) / 1e12
    wls_flops = 170.0 * float(nst.pairs) + 800.0 * n
    kern["wls"].update({"fp64_tflops": wls_flops / (kern["wls"]["ms"] * 1e-3) / 1e12, "alg_flops": wls_flops})
    kern["wls"]["fp64_frac"] = kern["wls"]["fp64_tflops"] / fp64_peak
    result["fp64_peak_tflops"] = {"value": fp64_peak, "how": "independent FP64 FMA chains on every SM "
                                  "(lsmps_kernel_bench LSMPS_KB_FP64_PEAK), CUDA events"}
    # the neighbor build as one unit (scan + compaction) against the algorithmic bytes of the
    # build + classification: positions once, row pointers, columns, classes (24 N + 4 (N + 1) + 4 P + N)
    nb_ms = kern["nbr_scan"]["ms"] + kern["nbr_compact"]["ms"]
    nb_bytes = 24.0 * n + 4.0 * (n + 1) + 4.0 * float(nst.pairs) + 1.0 * n
    kern["nbr_build"] = {"ms": nb_ms, "alg_bytes": nb_bytes, "achieved_gbs": nb_bytes / (nb_ms * 1e-3) / 1e9,
                         "frac": nb_bytes / (nb_ms * 1e-3) / 1e9 / peak}
    dom = "spmv64" if args.solver in ("fp64", "jacobi") else "spmv32"
    # the mixed solver's SpMV: FP32 values of A D^-1, FP64 vectors
    traffic = committed_traffic().get(dom)
    result["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": kern[dom]["achieved_gbs"], "peak": peak,
                          "unit": "GB/s", "frac": kern[dom]["frac"], "peak_kind": peak_kind,
                          "traffic": traffic, "kernels": kern}

    # ---- CPU baseline: the reference's own code on a bounded sample (rank 0, N = 1) ----
    if dist.world == 1 and dist.rank == 0 and not args.no_cpu_baseline:
        try:
            plain_it = cmp["fp64"]["per_set"][0]["iterations"] if not args.no_compare else s.iterations
            result["cpu_baseline"] = cpu_baseline(ctx, sets[0][0], sets[0][1], plain_it, args.cpu_sample_s)
        except Exception as e:  # the reference build may be absent on a machine without its sources
            result["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    ctx.close()
    return result


def _ref_case(xyz, types):
    """A reference handle on this particle set with the bench's parameters."""
    from oracle import Ref

    fd, path = tempfile.mkstemp(suffix=".cfg")
    with os.fdopen(fd, "w") as f:
        f.write(f"case=bench\nparticles={len(types)}\nl0={L0}\nre_ratio={RE_RATIO}\nmax_neighbors={MAXN}\n"
                f"wls_samples=4096\nppe_max_unknowns={len(types)}\nppe_max_iter=0\nppe_tol=1e-10\n")
    r = Ref(path)
    os.unlink(path)
    r.set_particles(xyz, types)
    return r


def cpu_baseline(ctx, xyz, types, plain_iterations, sample_s):
    """The reference (oracle/_ref, single-threaded as the reference is) on a bounded sample
    of the same step: its neighbors + classify in full, wls_test on 4096 particles
    extrapolated to all, its assemble_ppe in full, and its BiCGStab iteration on this step's
    WLS matrix for a bounded number of iterations, extrapolated to the iteration count the
    identical FP64 iteration needed on the GPU."""
    from oracle import Ref

    r = _ref_case(xyz, types)
    n = len(types)
    t0 = time.perf_counter()
    r.neighbors()
    t1 = time.perf_counter()
    r.classify()
    t2 = time.perf_counter()
    w = r.wls_test()
    t3 = time.perf_counter()
    _, _, _, _, _, st = r.assemble_ppe()
    t4 = time.perf_counter()
    row, col, val, b, xe, _ = ctx.ppe_reference_numbering()
    # bounded sample of the reference's BiCGStab iteration on this matrix
    probe_x, probe = Ref.bicgstab_csr(row, col, val, b, xe, 3, 0.0)
    per_iter = probe["solve_ms"] / 3.0
    k = int(max(5, min(500, sample_s * 1e3 / max(per_iter, 1e-3))))
    _, info = Ref.bicgstab_csr(row, col, val, b, xe, k, 0.0)
    ms_iter = info["solve_ms"] / max(1, info["iterations"])
    wls_all_ms = (t3 - t2) * 1e3 * n / max(1.0, w["sampled"] + w["failed"])
    step_ms = (t1 - t0) * 1e3 + (t2 - t1) * 1e3 + wls_all_ms + (t4 - t3) * 1e3 + ms_iter * plain_iterations
    return {
        "value": n / (step_ms * 1e-3), "unit": UNIT, "cores": 1, "kind": "reference",
        "sample": (f"reference neighbors+classify+assemble_ppe on all {n} particles, wls_test on "
                   f"{int(w['sampled'])} sampled particles extrapolated to all, and {info['iterations']} "
                   f"reference BiCGStab iterations on this WLS-Laplacian matrix extrapolated to the "
                   f"{plain_iterations} the same FP64 iteration needed"),
        "ms_per_step": step_ms, "bicgstab_ms_per_iteration": ms_iter,
        "phases_ms": {"neighbors": (t1 - t0) * 1e3, "classify": (t2 - t1) * 1e3, "wls_all_est": wls_all_ms,
                      "assemble": (t4 - t3) * 1e3, "solve_est": ms_iter * plain_iterations},
        "host_nproc": os.cpu_count(),
    }


# ---------------------------------------------------------------------------------------
# the reference arm: the reference's CPU implementation of the path
# ---------------------------------------------------------------------------------------
def run_reference(args, dist):
    """Times the reference's own CPU implementation (oracle/_ref, single-threaded as the
    reference is) of this step on the GPU arm's particle sets (same generator, same seeds;
    the oracle's restatement of the generator builds them, so this arm never loads the
    product library). Each step is a bounded sample of the full step, and `value` projects
    it to the full step:
      * timed in full: the reference's neighbors, classify and assemble_ppe on every particle;
      * timed on a sample: its wls_test on its own strided 4,096-particle sample (scaled to
        every particle), and `--ref-iterations` iterations of its BiCGStab on the set's
        WLS-Laplacian system (scaled to the iteration count the same FP64 iteration needs to
        reach the tolerance on that system, found once per set in the warm-up with the
        oracle's multi-threaded FP64 BiCGStab).
    Where the reference lacks a piece (the all-particle WLS behind the WLS-Laplacian rows)
    the oracle's CPU restatement builds the system, outside the timed region."""
    from oracle import Oracle, Ref

    K = max(1, args.sets)
    seeds = [args.seed + k for k in range(K)]
    nt = os.cpu_count() or 1
    re = RE_RATIO * L0
    sets = []
    t_setup = time.perf_counter()
    for sd in seeds:  # inputs and the iteration count to the tolerance, per set
        xyz, types = Oracle.generate(args.case, args.particles, L0, sd)
        n = len(types)
        r = _ref_case(xyz, types)
        row, col, _ = r.neighbors()
        cls = r.classify()
        _, wst, z, ws = Oracle.wls(xyz, cls, row, col, re, L0)
        prow, pcol, pval, pb, pxe, _, _ = Oracle.ppe_assemble(2, xyz, cls, row, col, re, L0, n, 0.0, z, ws, wst)
        _, info = Oracle.bicgstab(prow, pcol, pval, pb, args.max_iter, args.tol, nthreads=nt)
        sets.append((xyz, types, (prow, pcol, pval, pb, pxe), info["iterations"]))
    setup_s = time.perf_counter() - t_setup
    k_it = max(1, args.ref_iterations)
    timed, projected, phases = [], [], []
    for k in range(args.warmup + args.steps):
        xyz, types, (prow, pcol, pval, pb, pxe), iters = sets[k % K]
        n = len(types)
        w0 = time.perf_counter()
        r = _ref_case(xyz, types)
        t0 = time.perf_counter()
        r.neighbors()
        t1 = time.perf_counter()
        r.classify()
        t2 = time.perf_counter()
        w = r.wls_test()
        t3 = time.perf_counter()
        r.assemble_ppe()
        t4 = time.perf_counter()
        _, si = Ref.bicgstab_csr(prow, pcol, pval, pb, pxe, k_it, 0.0)
        t5 = time.perf_counter()
        sampled = max(1.0, w["sampled"] + w["failed"])
        ms_it = si["solve_ms"] / max(1, si["iterations"])
        ph = {"neighbors": (t1 - t0) * 1e3, "classify": (t2 - t1) * 1e3, "wls_test_sample": (t3 - t2) * 1e3,
              "wls_projected": (t3 - t2) * 1e3 * n / sampled, "assemble_ppe": (t4 - t3) * 1e3,
              "bicgstab_sample": (t5 - t4) * 1e3, "bicgstab_projected": ms_it * iters,
              "bicgstab_iterations_projected": iters, "wls_particles_sampled": sampled}
        if k >= args.warmup:
            timed.append((t5 - w0) * 1e3)
            projected.append(ph["neighbors"] + ph["classify"] + ph["wls_projected"] + ph["assemble_ppe"]
                             + ph["bicgstab_projected"])
            phases.append(ph)
    n = args.particles
    ms_timed = statistics.mean(timed)
    ms_proj = statistics.mean(projected)
    value = n / (ms_proj * 1e-3)
    mean_ph = {key: statistics.mean(p[key] for p in phases) for key in phases[0]}
    sample = (f"per step, on set k mod {K}: the reference's neighbors, classify and assemble_ppe on all {n} "
              f"particles (timed in full); its wls_test on {int(mean_ph['wls_particles_sampled'])} strided "
              f"particles, projected to all {n}; {k_it} of its BiCGStab iterations on the set's WLS-Laplacian "
              f"system, projected to the {mean_ph['bicgstab_iterations_projected']:.0f} iterations (mean over "
              f"sets) the same FP64 iteration needs to reach tol {args.tol:g}; single-threaded")
    return {
        "impl": "reference", "metric": METRIC, "unit": UNIT, "higher_is_better": True, "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup,
        # wall time of one timed (sampled) step; `value` is the full step projected from it
        "ms_per_step": ms_timed, "value": value, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator; no dataset)",
        "config": {"workload": f"{args.case} {n} particles, WLS-Laplacian PPE, tol {args.tol:g}", "particles": n,
                   "case": args.case, "particle_sets": K, "seeds": seeds, "l0": L0, "re": re,
                   "max_neighbors": MAXN, "solver": "reference FP64 BiCGStab (CPU)"},
        "projection": {"timed_ms_per_step": ms_timed, "projected_ms_per_full_step": ms_proj,
                       "factor": ms_proj / ms_timed, "phases_ms": mean_ph,
                       "setup_s": setup_s, "note": "value = particles / projected full-step time"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample,
                         "host_nproc": nt},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "product_library_loaded": _product_loaded(),
    }


def _product_loaded():
    """Whether this process mapped the product library (the reference arm must not)."""
    try:
        with open("/proc/self/maps") as f:
            return "liblsmps_b200" in f.read()
    except OSError:
        return None


def main():
    args = parse_args()
    if args.impl == "reference":
        # the reference arm is CPU only: rank 0 measures, the other ranks exit at once
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        os.environ["WORLD_SIZE"] = "1"
    dist = Dist(want_gpu=args.impl == "mine")
    try:
        if args.impl == "reference":
            out = run_reference(args, dist)
        else:
            out = run_mine(args, dist)
        if dist.rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        dist.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
