"""Calibrated synthetic-CSR replay: the GPU solvers and kernels on the statistical proxy that
the reference's calibration tool writes (python/workload_calibration.py:253-301, files
described in WORKLOAD_CALIBRATION.md:26-35).

    python ls-mps_b200/replay_csr.py generate --out calib --particles 1000000
    python ls-mps_b200/replay_csr.py replay --dir calib --out calib/replay.json

`generate` writes the same file set as the reference tool from a profile (this module's
restatement of its published synthesis: row lengths from a four-band mixture with the mean
matched exactly, particle types by ratio, virtual-neighbor counts, ill-conditioned flags,
locality-biased columns i + round(N(0, max(8, sqrt n))) mod n, and a timeline of injections,
deletions, rebuild steps and PPE iteration counts). `replay` loads csr_row_ptr.npy and
csr_col_idx.npy into a context (lsmps_ppe_load_csr: -1 off-diagonals, diagonally dominant
diagonal, b = A 1), solves with each solver to the tolerance (relative L2 against p* = 1),
times the SELL SpMV kernels, and replays the timeline: per step, a solve capped at that
step's ppe_iterations.
"""
import argparse
import csv
import json
import math
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

# rain-on-plate statistics of this repository's generator at 1M particles (the role of the
# reference's calibrated profile)
DEFAULT_PROFILE = dict(particles=1_000_000, neighbor_mean=30.7, neighbor_p90=35, neighbor_p99=40,
                       near_wall_ratio=0.01, free_surface_ratio=0.08, splash_ratio=0.01,
                       virtual_particle_ratio=0.1, wls_ill_conditioned_ratio=0.001, ppe_iterations=60,
                       cnl_rebuild_interval=10, injected_per_step=2000, deleted_per_step=200, timeline_steps=200)


def row_lengths(n, mean, p90, p99, rng):
    """Four bands (50 % low, 40 % mid, 9 % high, 1 % tail), then single-unit changes in a random
    order until the total equals round(mean n)."""
    u = rng.random(n)
    low = max(1.0, 0.55 * mean)
    mid = max(low, min(p90, 1.06 * mean))
    high = max(mid, p90)
    tail = max(high, p99)
    x = np.empty(n)
    bands = [(u < 0.5, 0.75 * low, 1.05 * low), ((u >= 0.5) & (u < 0.9), 0.9 * mid, 1.02 * high),
             ((u >= 0.9) & (u < 0.99), high, max(high + 1.0, 0.98 * tail)), (u >= 0.99, tail, 1.08 * tail)]
    for m, a, b in bands:
        x[m] = rng.uniform(a, b, int(m.sum()))
    x = np.maximum(1, np.rint(x)).astype(np.int64)
    delta = int(round(mean * n)) - int(x.sum())
    order = rng.permutation(n)
    k = 0
    while delta != 0 and k < 100 * n:
        i = order[k % n]
        if delta > 0:
            x[i] += 1
            delta -= 1
        elif x[i] > 1:
            x[i] -= 1
            delta += 1
        k += 1
    return x.astype(np.int32)


def generate(out, profile, seed=0, materialize_csr=True):
    rng = np.random.default_rng(seed)
    n = int(profile["particles"])
    rl = row_lengths(n, profile["neighbor_mean"], profile["neighbor_p90"], profile["neighbor_p99"], rng)
    ratios = [profile.get(k, 0.0) for k in ("near_wall_ratio", "free_surface_ratio", "splash_ratio")]
    s = sum(ratios)
    if s > 0.95:
        ratios = [r * 0.95 / s for r in ratios]
    counts = [int(round(n * r)) for r in ratios]
    ptype = np.concatenate([np.zeros(max(0, n - sum(counts)), np.uint8)] +
                           [np.full(c, t, np.uint8) for c, t in zip(counts, (1, 2, 3))])[:n]
    rng.shuffle(ptype)
    virtual = rng.binomial(np.maximum(rl, 1), min(profile.get("virtual_particle_ratio", 0.0), 0.8)).astype(np.int16)
    bad = rng.random(n) < profile.get("wls_ill_conditioned_ratio", 0.0)
    row_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(rl, out=row_ptr[1:])
    os.makedirs(out, exist_ok=True)
    np.save(os.path.join(out, "particle_type.npy"), ptype)
    np.save(os.path.join(out, "neighbor_row_length.npy"), rl)
    np.save(os.path.join(out, "csr_row_ptr.npy"), row_ptr)
    np.save(os.path.join(out, "virtual_neighbor_count.npy"), virtual)
    np.save(os.path.join(out, "wls_ill_conditioned.npy"), bad)
    if materialize_csr:
        rows = np.repeat(np.arange(n, dtype=np.int64), rl)
        off = np.rint(rng.normal(0.0, max(8.0, math.sqrt(n)), int(row_ptr[-1]))).astype(np.int64)
        np.save(os.path.join(out, "csr_col_idx.npy"), ((rows + off) % n).astype(np.int32))
    steps = int(profile.get("timeline_steps", 200))
    inj, dele = int(profile.get("injected_per_step", 0)), int(profile.get("deleted_per_step", 0))
    rebuild = max(1, int(profile.get("cnl_rebuild_interval", 10)))
    it = profile.get("ppe_iterations", 1)
    with open(os.path.join(out, "timeline.csv"), "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=["step", "injected", "deleted", "cnl_rebuild", "ppe_iterations"])
        w.writeheader()
        for step in range(steps):
            w.writerow({"step": step, "injected": int(rng.poisson(inj)) if inj else 0,
                        "deleted": int(rng.poisson(dele)) if dele else 0, "cnl_rebuild": int(step % rebuild == 0),
                        "ppe_iterations": max(1, int(round(rng.normal(it, max(1.0, 0.05 * it)))))})
    meta = {"particles": n, "neighbor_mean": float(rl.mean()),
            "neighbor_p90": float(np.quantile(rl, 0.9, method="higher")),
            "neighbor_p99": float(np.quantile(rl, 0.99, method="higher")), "csr_nnz": int(row_ptr[-1]),
            "materialized_col_idx": bool(materialize_csr)}
    with open(os.path.join(out, "metadata.json"), "w") as f:
        json.dump(meta, f, indent=2)
    return meta


def replay(d, solvers=("mixed", "fp64"), tol=1e-10, timeline_steps=None, reps=20):
    import lsmps_b200 as lib

    row_ptr = np.load(os.path.join(d, "csr_row_ptr.npy"))
    col = np.load(os.path.join(d, "csr_col_idx.npy"))
    out = {"dir": d, "rows": int(len(row_ptr) - 1), "entries": int(row_ptr[-1]), "solvers": {}, "kernels": {}}
    with lib.Context(0) as ctx:
        t0 = time.perf_counter()
        st = ctx.ppe_load_csr(row_ptr, col)
        out["load_s"] = time.perf_counter() - t0
        out["unknowns"], out["nnz"] = int(st.unknowns), int(st.nnz)
        for name in solvers:
            ctx.ppe_solve(name, 20000, tol)  # warm: SELL copies, graphs
            s = ctx.ppe_solve(name, 20000, tol)
            out["solvers"][name] = {"iterations": s.iterations, "solve_ms": s.solve_ms, "converged": bool(s.converged),
                                    "relative_l2_error": s.relative_l2_error, "relative_residual": s.relative_residual}
        for name, kid in (("spmv32", lib.KB_SPMV32), ("spmv64", lib.KB_SPMV64)):
            ms, nb = ctx.kernel_bench(kid, reps)
            out["kernels"][name] = {"us": ms * 1e3, "alg_bytes": nb, "achieved_gbs": nb / ms / 1e6}
        tl = os.path.join(d, "timeline.csv")
        if os.path.exists(tl):
            steps = list(csv.DictReader(open(tl)))[:timeline_steps]
            ms = []
            for r in steps:  # each step: the solve capped at its iteration count (tolerance out of reach)
                s = ctx.ppe_solve(solvers[0], int(r["ppe_iterations"]), 1e-300)
                ms.append(s.solve_ms)
            out["timeline"] = {"solver": solvers[0], "steps": len(ms), "total_ms": float(sum(ms)),
                               "mean_ms": float(np.mean(ms)) if ms else 0.0,
                               "iterations": int(sum(int(r["ppe_iterations"]) for r in steps))}
    return out


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    g = sub.add_parser("generate")
    g.add_argument("--out", required=True)
    g.add_argument("--particles", type=int, default=DEFAULT_PROFILE["particles"])
    g.add_argument("--profile", default=None, help="JSON with the profile keys (the reference's knobs)")
    g.add_argument("--seed", type=int, default=0)
    r = sub.add_parser("replay")
    r.add_argument("--dir", required=True)
    r.add_argument("--solvers", default="mixed,fp64")
    r.add_argument("--tol", type=float, default=1e-10)
    r.add_argument("--timeline-steps", type=int, default=None)
    r.add_argument("--out", default=None)
    a = ap.parse_args()
    if a.cmd == "generate":
        prof = dict(DEFAULT_PROFILE)
        if a.profile:
            prof.update(json.load(open(a.profile)))
        prof["particles"] = a.particles
        print(json.dumps(generate(a.out, prof, a.seed)))
    else:
        res = replay(a.dir, tuple(a.solvers.split(",")), a.tol, a.timeline_steps)
        print(json.dumps(res))
        if a.out:
            with open(a.out, "w") as f:
                json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
