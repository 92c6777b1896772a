"""Runs one kernel of the path on a named workload, for profilers (ncu) and quick timing.

    python ls-mps_b200/profile_kernels.py --kernel spmv32 --particles 1000000 --reps 3

Builds the workload of bench.py (case `mixed`, l0 = 1, re = 2.1, max_neighbors 128,
WLS-Laplacian PPE) with the library, then launches the chosen kernel `reps` times through
lsmps_kernel_bench and prints its mean time and achieved bandwidth. Under ncu, select the
kernel with -k (spmv32/spmv64: k_bcg_v, nbr_count: k_seg_pass<0>, nbr_fill: k_seg_pass<1>,
nbr_scan: k_seg_scan, nbr_compact: k_slots_compact, wls: k_wls_all, mpnn_layer: k_layer_fwd, mg_vcycle: regex k_mg_). mpnn_layer loads --weights. --autotune prints the
launch shapes the autotuner timed and chose.

    python ls-mps_b200/profile_kernels.py --step-trace learned --precond multigrid

runs the bench's per-step path (neighbor build, WLS, WLS-Laplacian assembly, the solve to
relative residual 2e-11) three times, then once more under the CUDA activity tracer
(torch.profiler, CUPTI) and prints every kernel's share of the step as the time from the
previous kernel's end to its own end. With programmatic dependent launch a kernel starts
before its predecessor ends, so these end-to-end times (which add up to the step) are the
measure of what each kernel costs in the timeline; gaps the host leaves between phases are
charged to the kernel after them.
"""
import argparse
import collections
import json
import os
import sys
import tempfile

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import lsmps_b200 as lib  # noqa: E402

KERNELS = {"spmv32": lib.KB_SPMV32, "spmv64": lib.KB_SPMV64, "nbr_count": lib.KB_NBR_COUNT,
           "nbr_fill": lib.KB_NBR_FILL, "nbr_scan": lib.KB_NBR_SCAN, "nbr_compact": lib.KB_NBR_COMPACT,
           "wls": lib.KB_WLS, "mpnn_layer": lib.KB_MPNN_LAYER, "mg_vcycle": lib.KB_MG_VCYCLE}
WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "mpnn_rain200k.bin")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", choices=sorted(KERNELS), nargs="*", default=["spmv32"])
    ap.add_argument("--particles", type=int, default=1_000_000)
    ap.add_argument("--case", default="mixed")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--solve", choices=["fp64", "jacobi", "mixed", "learned"], default=None,
                    help="also run one PPE solve to relative residual 1e-10")
    ap.add_argument("--precond", choices=["jacobi", "multigrid"], default="jacobi")
    ap.add_argument("--use-graph", type=int, default=1,
                    help="launch form of --solve: 1 device-driven graph, 2 chunk graphs, 0 stream launches "
                         "(0 for ncu, which does not profile kernels inside conditional graph nodes)")
    ap.add_argument("--weights", default=WEIGHTS)
    ap.add_argument("--autotune", type=int, default=1, help="0 off (default shapes), 1 on")
    ap.add_argument("--step-trace", choices=["fp64", "jacobi", "mixed", "learned"], default=None,
                    help="trace one whole step with this solver (with --precond) and print the kernel timeline")
    a = ap.parse_args()
    if a.step_trace:
        step_trace(a)
        return
    xyz, t, _ = lib.generate(None, case=a.case, particles=a.particles, l0=1.0, seed=7)
    with lib.Context(0) as ctx:
        ctx.set_autotune(a.autotune)
        if "mpnn_layer" in a.kernel or a.solve == "learned":
            ctx.mpnn_load(a.weights)
        ctx.upload(xyz, t)
        import time
        for rep in range(3):  # the whole build (host round trips included), warm after the first
            t0 = time.perf_counter()
            nst = ctx.build_neighbors(2.1, 128, 1.0)
            t1 = time.perf_counter()
            print(f"neighbor build {rep}: {(t1 - t0) * 1e3:.2f} ms wall, device phase {ctx.timings()[1]:.3f} ms, "
                  f"pairs {nst.pairs}")
        ctx.wls(2.1, 1.0, mode=1)
        for rep in range(3):  # the whole assembly (rows, scan, pack; host round trips included)
            st = ctx.ppe_assemble("wls", 10**12, 2.1, 1.0, diag_shift=0.0)
            print(f"PPE assembly {rep}: {st.assembly_ms:.3f} ms (device events)")
        print(f"particles {len(t)} unknowns {st.unknowns} nnz {st.nnz}")
        for k in a.kernel:
            ms, nb = ctx.kernel_bench(KERNELS[k], a.reps)
            print(f"{k}: {ms * 1e3:.1f} us per launch, {nb / 1e6:.1f} MB algorithmic, {nb / ms / 1e6:.0f} GB/s")
        if a.solve:
            s = ctx.ppe_solve(a.solve, 20000, 1e-10, precond=a.precond, use_graph=a.use_graph)
            print(f"solve {a.solve}: {s.solve_ms:.2f} ms, {s.iterations} iterations, {s.outer_iterations} sweeps, "
                  f"relative L2 {s.relative_l2_error:.2e}")
        for key, shape, ms, best in ctx.autotune_report():
            print(f"autotune {key} {shape}: {ms * 1e3:.1f} us{'  <- chosen' if best else ''}")


def step_trace(a):
    """Kernel timeline of one bench step (see the module docstring)."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    xyz, t, _ = lib.generate(None, case=a.case, particles=a.particles, l0=1.0, seed=7)
    torch.zeros(1, device="cuda")  # the tracer needs a CUDA context of its own process
    ug = 0 if a.precond == "multigrid" else 1

    def one_step(ctx):
        ctx.build_neighbors(2.1, 128, 1.0)
        ctx.wls(2.1, 1.0, mode=1)
        ctx.ppe_assemble("wls", 10**12, 2.1, 1.0, diag_shift=0.0)
        return ctx.ppe_solve(a.step_trace, 20000, 2e-11, use_graph=ug, precond=a.precond)

    with lib.Context(0) as ctx:
        ctx.set_autotune(a.autotune)
        if a.step_trace == "learned":
            ctx.mpnn_load(a.weights)
        ctx.upload(xyz, t)
        for _ in range(3):
            one_step(ctx)
        ctx.sync()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            s = one_step(ctx)
            ctx.sync()
        tm = ctx.timings()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "trace.json")
        prof.export_chrome_trace(path)
        with open(path) as f:
            ev = json.load(f)["traceEvents"]
    ks = sorted((e for e in ev if e.get("cat") == "kernel"), key=lambda e: e["ts"] + e["dur"])
    if not ks:
        print("no kernels traced")
        return

    def name(e):
        n = e["name"]
        i = n.find("::k_")
        return (n[i + 2:] if i >= 0 else n).split("(")[0]

    cost = collections.defaultdict(list)
    for prev, e in zip(ks, ks[1:]):
        cost[name(e)].append((e["ts"] + e["dur"]) - (prev["ts"] + prev["dur"]))
    span = ks[-1]["ts"] + ks[-1]["dur"] - ks[0]["ts"]
    print(f"step: {len(ks)} kernels over {span / 1e3:.3f} ms (events: neighbors {tm[1]:.3f}, WLS {tm[3]:.3f}, "
          f"assembly {tm[4]:.3f}, solve {s.solve_ms:.3f} ms, {s.iterations} iterations)")
    print(f"{'kernel':58s} {'launches':>8s} {'mean us':>9s} {'total us':>10s} {'share':>7s}")
    for k, v in sorted(cost.items(), key=lambda x: -sum(x[1])):
        print(f"{k[:58]:58s} {len(v):8d} {sum(v) / len(v):9.2f} {sum(v):10.1f} {100 * sum(v) / span:6.1f}%")


if __name__ == "__main__":
    main()
