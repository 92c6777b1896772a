"""Writes tests/golden/rain_validation/: the reference's four rain validation tables
(metrics.csv, sampling_windows.csv, flow_sections.csv, mass_conservation.csv, with the columns
python/validate_outputs.py requires) from a small GPU step series, for the tests.

    python tests/golden/make_rain_validation_fixture.py      (needs the GPU library)

The series is the one tests/test_gpu_series.py runs: the rain_plate generator at 60,000
particles (seed 3), 25 steps, 400 particles injected per step (seed 5), candidate rebuild
every 10 steps, plain FP64 solves to 3e-11; tables in meters with l0 = 4 mm and 1 ms steps.
The tables depend only on the particles' motion, injection and deletion, not on the solver.
tests/test_reference_tools.py runs the reference's own validator on these files, and
tests/test_gpu_series.py checks that a fresh GPU run reproduces them.
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "rain_validation")
PLATE = dict(particles=60_000, seed=3)
SERIES = dict(steps=25, injected_per_step=400, cnl_rebuild_interval=10, tol=3e-11, seed=5)
L0_M, DT_S = 0.004, 1e-3


class Units:
    l0_m, dt_s = L0_M, DT_S


def tables(rows, rain):
    """The four tables of a series run (rows: per-step statistics, rain: per-step outputs)."""
    sys.path.insert(0, os.path.join(ROOT, "ls-mps_b200"))
    import run_series

    return run_series.validation_rows([r if isinstance(r, dict) else r.as_dict() for r in rows], rain, Units)


def main():
    sys.path.insert(0, os.path.join(ROOT, "ls-mps_b200"))
    import lsmps_b200 as lib
    import run_series

    xyz, t, _ = lib.generate(None, case="rain_plate", particles=PLATE["particles"], l0=1.0, seed=PLATE["seed"])
    with lib.Context(0) as ctx, lib.Series(ctx, xyz, t, solver="fp64", precond="jacobi", **SERIES) as s:
        rows, rain = [], []
        for _ in range(SERIES["steps"]):
            rows.append(s.step())
            rain.append(s.rain_outputs())
    os.makedirs(OUT, exist_ok=True)
    for name, tab in tables(rows, rain).items():
        run_series.write_csv(os.path.join(OUT, name), tab)
    print("wrote", OUT, sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
