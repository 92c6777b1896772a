"""Train the learned preconditioner on the GPU and evaluate it against the solver without it.

    python ls-mps_b200/train_mpnn.py --out ls-mps_b200/weights/mpnn_rain200k.bin

Data (the learned-preconditioner workload): rain-on-plate snapshots of --particles (200,000) particles, seeds
1000, 1001, ...; on each, --pairs right-hand sides b = A p* with smooth random fields p*
(the first pair of every snapshot uses the benchmark's p* = sin(0.3x) cos(0.2y) + 0.1z),
solved by the plain FP64 Jacobi-BiCGStab to relative residual 1e-10; the pair
(b / |b|, D p / |b|) is stored on the GPU (--snapshots x --pairs = 2,000 by default).
Training: Adam on the GPU with the library's own forward and backward kernels.
Evaluation: held-out seeds (9000, ...) at 1M of the rain-on-plate case (the training
distribution) and of the bench's `mixed` case: iterations and solve time of LEARNED against
MIXED (the same solver without the network) and plain FP64, and the fallback count.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import lsmps_b200 as lib  # noqa: E402


def random_field(rng):
    modes = []
    for _ in range(3):
        k = rng.normal(size=3)
        k *= rng.uniform(0.05, 0.5) / np.linalg.norm(k)
        modes.append((rng.normal(), k[0], k[1], k[2], rng.uniform(0, 2 * np.pi)))
    return rng.normal(), 0.1 * rng.normal(), modes


BENCH_FIELD = (0.0, 0.1, [(0.5, 0.3, 0.2, 0.0, 0.0), (0.5, 0.3, -0.2, 0.0, 0.0)])  # sin(.3x)cos(.2y)+.1z


def build(ctx, case, n, seed):
    xyz, t, _ = lib.generate(None, case=case, particles=n, l0=1.0, seed=seed)
    ctx.upload(xyz, t)
    ctx.build_neighbors(2.1, 128, 1.0)
    ctx.wls(2.1, 1.0, mode=1)
    return ctx.ppe_assemble("wls", 10**12, 2.1, 1.0, diag_shift=0.0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--particles", type=int, default=200_000)
    ap.add_argument("--snapshots", type=int, default=40)
    ap.add_argument("--pairs", type=int, default=50)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--loss", type=int, default=2, help="0 error, 1 residual |r - A D^-1 y|, 2 both (best measured)")
    ap.add_argument("--eval-cases", default="rain_plate,mixed")
    ap.add_argument("--eval-seeds", type=int, default=3)
    ap.add_argument("--eval-particles", type=int, default=1_000_000)
    ap.add_argument("--eval-tol", type=float, default=3e-11, help="relative residual of the evaluation solves")
    ap.add_argument("--out", default=None)
    ap.add_argument("--load", default=None, help="skip training, evaluate these weights")
    ap.add_argument("--report", default=None, help="write the evaluation as JSON here")
    a = ap.parse_args()
    rng = np.random.default_rng(a.seed)
    report = {"config": vars(a)}
    with lib.Context(0) as ctx:
        ctx.mpnn_init(a.seed)
        if a.load:
            ctx.mpnn_load(a.load)
        else:
            t0 = time.time()
            iters = []
            for s in range(a.snapshots):
                build(ctx, "rain_plate", a.particles, 1000 + s)
                for k in range(a.pairs):
                    ctx.ppe_manufacture(*(BENCH_FIELD if k == 0 else random_field(rng)))
                    st = ctx.ppe_solve("jacobi", 20000, 1e-10)
                    if not st.converged:
                        continue
                    iters.append(st.iterations)
                    ctx.mpnn_add_sample()
            t1 = time.time()
            print(f"data: {ctx.mpnn_sample_count()} pairs in {t1 - t0:.1f} s (mean {np.mean(iters):.0f} "
                  f"plain-solver iterations)", flush=True)
            losses = []
            chunk = max(1, a.steps // 20)
            for done in range(0, a.steps, chunk):
                losses.append(ctx.mpnn_train(steps=min(chunk, a.steps - done), batch=a.batch, lr=a.lr,
                                             seed=a.seed + done, loss=a.loss))
                print(f"step {done + chunk}: loss {losses[-1]:.4f}", flush=True)
            t2 = time.time()
            report["training"] = {"pairs": ctx.mpnn_sample_count(), "data_s": t1 - t0, "train_s": t2 - t1,
                                  "loss_curve": losses}
            if a.out:
                os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
                ctx.mpnn_save(a.out)
            ctx.mpnn_clear_samples()
        evals = []
        for case in a.eval_cases.split(","):
            for k in range(a.eval_seeds):
                build(ctx, case, a.eval_particles, 9000 + k)
                res = {"case": case}
                for name in ("mixed", "learned", "fp64"):
                    ctx.ppe_solve(name, 20000, a.eval_tol)  # warm
                    s = ctx.ppe_solve(name, 20000, a.eval_tol)
                    res[name] = {"iterations": s.iterations, "solve_ms": s.solve_ms, "rel_l2": s.relative_l2_error,
                                 "converged": bool(s.converged), "fallback": s.fallback}
                evals.append(res)
                print(f"{case} seed {9000 + k}: " + ", ".join(
                    f"{n} {r['iterations']} it {r['solve_ms']:.1f} ms" for n, r in res.items() if n != "case"),
                      flush=True)
        report["eval"] = evals
        summary = {}
        for case in a.eval_cases.split(","):
            ev = [e for e in evals if e["case"] == case]
            if not ev:
                continue
            m = np.mean([e["mixed"]["solve_ms"] for e in ev])
            le = np.mean([e["learned"]["solve_ms"] for e in ev])
            p = np.mean([e["fp64"]["solve_ms"] for e in ev])
            summary[case] = {"mixed_ms": m, "learned_ms": le, "plain_fp64_ms": p,
                             "learned_vs_mixed": m / le, "learned_vs_plain_fp64": p / le,
                             "mixed_it": np.mean([e["mixed"]["iterations"] for e in ev]),
                             "learned_it": np.mean([e["learned"]["iterations"] for e in ev]),
                             "fallbacks": int(sum(e["learned"]["fallback"] for e in ev)),
                             "seeds": len(ev),
                             "max_rel_l2": max(e[n]["rel_l2"] for e in ev for n in ("mixed", "learned", "fp64")),
                             "learned_fewer_iterations": int(sum(e["learned"]["iterations"] < e["mixed"]["iterations"]
                                                                 for e in ev))}
        report["summary"] = summary
        print(json.dumps(summary))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1, default=float)


if __name__ == "__main__":
    main()
