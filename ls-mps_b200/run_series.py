"""Rain-on-plate step series: the full per-step path over many steps, per solver.

    python ls-mps_b200/run_series.py --particles 3000000 --steps 200 --out results/series
    python ls-mps_b200/run_series.py --cfg config/industrial_3m_template.cfg --steps 200

Initial particles: the rain_plate generator (20 deg plate, 3 wall layers, 4-layer film with
70 % of the fluid, droplets of radius 3 l0 at 10-40 l0). Each solver (default: mixed precision,
the learned solver, then plain FP64; `mixed+multigrid` adds the multigrid preconditioner,
which does not pay on this warm-started film series) runs the same series from the same
particles and injection seed, so every step has the same particles for every solver. Per
step: neighbor lists (candidate rebuild every --interval steps, refresh in between), WLS,
WLS-Laplacian PPE with the manufactured p* = sin(0.3x) cos(0.2y) + 0.1z, solve warm-started
from the previous pressure; mass balance (device fluid count against initial + injected -
deleted) and PPE relative L2 per step. Writes series_<solver>.csv per solver and summary.json,
and (from the first solver's run; the particles are the same for all) the reference's rain
validation outputs in validation/: metrics.csv, sampling_windows.csv, flow_sections.csv and
mass_conservation.csv with the columns python/validate_outputs.py requires. Lengths are in l0
units scaled by --l0-m (meters per l0) and one step lasts --dt-s seconds.
A .cfg (keys particles, seed, re_ratio, steps, injected_per_step, cnl_rebuild_interval) sets
the defaults of the matching options; the plate and droplets are in units of l0 = 1.
"""
import argparse
import csv
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import lsmps_b200 as lib  # noqa: E402


def read_cfg(path):
    out = {}
    for line in open(path):
        line = line.split("#", 1)[0]
        if "=" in line:
            k, v = line.split("=", 1)
            out[k.strip()] = v.strip()
    return out


def validation_rows(rows, rain, a):
    """The reference's four validation tables (python/rain_plate_cpu.py:326-372) from the
    series statistics and the per-step rain outputs."""
    vol = a.l0_m ** 3
    r0 = rows[0]
    fluid0 = r0["fluid_particles"] - r0["injected_total"] + r0["deleted_total"] - r0["mass_balance"]
    metrics, windows, sections, mass = [], [], [], []
    cumulative = {}
    for r, (win, sec) in zip(rows, rain):
        time = r["step"] * a.dt_s
        injected = fluid0 + r["injected_total"]  # the initial fluid counts as injected at t = 0
        metrics.append({"step": r["step"], "time": time, "particles": r["fluid_particles"],
                        "injected_total": injected, "outflow_total": r["deleted_total"], "invalid_removed_total": 0,
                        "mass_error": injected - r["deleted_total"] - r["fluid_particles"],
                        "pairs": r["pairs"], "unknowns": r["unknowns"], "in_flight": r["in_flight"],
                        "flagged": r["flagged"]})
        for name, (np_, cov, fmean, fp90, fmax) in win.items():
            windows.append({"time": time, "window": name, "particle_count": np_, "fluid_volume_m3": np_ * vol,
                            "coverage_ratio": cov, "film_mean_m": fmean * a.l0_m, "film_p90_m": fp90 * a.l0_m,
                            "film_max_m": fmax * a.l0_m})
        for name, n in sec.items():
            cumulative[name] = cumulative.get(name, 0.0) + n * vol
            sections.append({"time": time, "section": name, "crossing_particle_count": n,
                             "instantaneous_flow_rate_m3s": n * vol / a.dt_s, "crossing_volume_m3": n * vol,
                             "cumulative_volume_m3": cumulative[name]})
        inj_v, rem_v, out_v = injected * vol, r["fluid_particles"] * vol, r["deleted_total"] * vol
        bal = inj_v - rem_v - out_v
        denom = max(inj_v, vol)
        mass.append({"time": time, "injected_volume_m3": inj_v, "remaining_volume_m3": rem_v, "outlet_volume_m3": out_v,
                     "invalid_removed_volume_m3": 0.0, "balance_error_m3": bal, "relative_mass_error": abs(bal) / denom,
                     "invalid_removed_ratio": 0.0})
    return {"metrics.csv": metrics, "sampling_windows.csv": windows, "flow_sections.csv": sections,
            "mass_conservation.csv": mass}


def write_csv(path, rows):
    with open(path, "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=list(rows[0].keys()))
        w.writeheader()
        w.writerows(rows)


def run(ctx, xyz, t, solver, a, rain=None):
    rows = []
    name, _, pc = solver.partition("+")  # e.g. mixed+multigrid: the MIXED solver, multigrid preconditioner
    kw = dict(steps=a.steps, injected_per_step=a.injected, cnl_rebuild_interval=a.interval, solver=name,
              precond=pc or "jacobi", re=a.re, skin=a.skin, tol=a.tol, seed=a.seed)
    with lib.Series(ctx, xyz, t, **kw) as s:
        for _ in range(a.steps):
            st = s.step().as_dict()
            st["solver"] = solver
            rows.append(st)
            if rain is not None:
                rain.append(s.rain_outputs())
            if a.verbose:
                print(f"{solver} step {st['step']}: n {st['particles']} U {st['unknowns']} it {st['iterations']} "
                      f"L2 {st['relative_l2_error']:.2e} solve {st['solve_ms']:.1f} ms step {st['step_ms']:.1f} ms "
                      f"mass {st['mass_balance']}{' rebuild' if st['rebuilt'] else ''}", flush=True)
    return rows


def summarize(rows):
    it = np.array([r["iterations"] for r in rows])
    return {
        "steps": len(rows),
        "total_solve_ms": float(sum(r["solve_ms"] for r in rows)),
        "total_step_ms": float(sum(r["step_ms"] for r in rows)),
        "mean_step_ms": float(np.mean([r["step_ms"] for r in rows])),
        "mean_solve_ms": float(np.mean([r["solve_ms"] for r in rows])),
        "mean_neighbor_ms": float(np.mean([r["neighbor_ms"] for r in rows])),
        "mean_neighbor_ms_rebuild": float(np.mean([r["neighbor_ms"] for r in rows if r["rebuilt"]])),
        "mean_neighbor_ms_refresh": (float(np.mean([r["neighbor_ms"] for r in rows if not r["rebuilt"]]))
                                     if any(not r["rebuilt"] for r in rows) else None),
        "mean_wls_ms": float(np.mean([r["wls_ms"] for r in rows])),
        "mean_assembly_ms": float(np.mean([r["assembly_ms"] for r in rows])),
        "iterations_first": int(it[0]),
        "iterations_mean_warm": float(it[1:].mean()) if len(it) > 1 else None,
        "all_converged": bool(all(r["converged"] for r in rows)),
        "max_relative_l2": float(max(r["relative_l2_error"] for r in rows)),
        "max_abs_mass_balance": int(max(abs(r["mass_balance"]) for r in rows)),
        "rebuilds": int(sum(r["rebuilt"] for r in rows)),
        "forced_rebuilds": int(sum(r["forced_rebuild"] for r in rows)),
        "fallbacks": int(sum(r["fallback"] for r in rows)),
        "particles_first": int(rows[0]["particles"]),
        "particles_last": int(rows[-1]["particles"]),
        "injected_total": int(rows[-1]["injected_total"]),
        "deleted_total": int(rows[-1]["deleted_total"]),
        "unknowns_last": int(rows[-1]["unknowns"]),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cfg", default=None)
    ap.add_argument("--particles", type=int, default=None)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--injected", type=int, default=None)
    ap.add_argument("--interval", type=int, default=None)
    ap.add_argument("--seed", type=int, default=None)
    ap.add_argument("--re", type=float, default=None, help="support radius in l0 (re_ratio)")
    ap.add_argument("--skin", type=float, default=1.0)
    ap.add_argument("--tol", type=float, default=3e-11)
    ap.add_argument("--solvers", default="mixed,learned,fp64",
                    help="comma list of solver names, optionally +multigrid (the preconditioner)")
    ap.add_argument("--weights", default=lib.DEFAULT_WEIGHTS)
    ap.add_argument("--out", default="results/series")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--l0-m", type=float, default=0.004, help="meters per l0 in the validation outputs")
    ap.add_argument("--dt-s", type=float, default=1e-3, help="seconds per step in the validation outputs")
    a = ap.parse_args()
    cfg = read_cfg(a.cfg) if a.cfg else {}
    defaults = {"particles": ("particles", int, 3_000_000), "steps": ("steps", int, 200),
                "injected": ("injected_per_step", int, 2000), "interval": ("cnl_rebuild_interval", int, 10),
                "seed": ("seed", int, 23), "re": ("re_ratio", float, 2.1)}
    for opt, (key, typ, dflt) in defaults.items():
        if getattr(a, opt) is None:
            setattr(a, opt, typ(cfg[key]) if key in cfg else dflt)
    xyz, t, _ = lib.generate(None, case="rain_plate", particles=a.particles, l0=1.0, seed=a.seed)
    os.makedirs(a.out, exist_ok=True)
    summary = {"config": {k: getattr(a, k) for k in ("particles", "steps", "injected", "interval", "seed", "re",
                                                     "skin", "tol", "solvers")}, "solvers": {}}
    with lib.Context(0) as ctx:
        for k, solver in enumerate(a.solvers.split(",")):
            if solver.startswith("learned"):
                ctx.mpnn_load(a.weights)
            rain = [] if k == 0 else None
            rows = run(ctx, xyz, t, solver, a, rain)
            write_csv(os.path.join(a.out, f"series_{solver}.csv"), rows)
            if rain is not None:
                vdir = os.path.join(a.out, "validation")
                os.makedirs(vdir, exist_ok=True)
                for name, tab in validation_rows(rows, rain, a).items():
                    write_csv(os.path.join(vdir, name), tab)
            summary["solvers"][solver] = summarize(rows)
            print(solver, json.dumps(summary["solvers"][solver]), flush=True)
    names = list(summary["solvers"])
    if len(names) > 1:
        base, fast = summary["solvers"][names[-1]], summary["solvers"][names[0]]
        summary["speedup"] = {"solve": base["total_solve_ms"] / fast["total_solve_ms"],
                              "step": base["total_step_ms"] / fast["total_step_ms"],
                              "of": names[0], "over": names[-1]}
        print("speedup", json.dumps(summary["speedup"]))
    with open(os.path.join(a.out, "summary.json"), "w") as f:
        json.dump(summary, f, indent=1)


if __name__ == "__main__":
    main()
