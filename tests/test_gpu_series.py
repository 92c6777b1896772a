"""Rain-on-plate step series and the skin (Verlet) neighbor lists it uses.

* Refreshed lists (candidates of radius re + skin filtered at the current positions) hold
  the same neighbor sets and classes as a fresh build at those positions; the refresh
  refuses once a particle moved more than skin / 2.
* Per-particle warm start: a solve started from its own solution (set per particle) stops
  at once, and the per-particle download puts the unknowns' values at their particles.
* Series: the device fluid count matches initial + injected - deleted at every step (mass
  balance 0); candidate rebuilds at step 1 and every interval steps; every PPE reaches
  relative L2 <= 1e-8 against p*; the warm start needs fewer iterations than the cold first
  solve; the learned, plain FP64 and multigrid-preconditioned series see the same particles.
* Rain validation outputs: the reference's four tables (python/validate_outputs.py columns
  and checks restated: particle identity, coverage in [0, 1], p90 <= max, cumulative flow
  non-decreasing, mass error within the config's 1 %), and the window statistics of the last
  step equal a numpy recomputation from the particle positions.
"""
import math
import os
import sys

import numpy as np
import pytest

import lsmps_b200 as lib

pytestmark = pytest.mark.gpu
SMALL = dict(steps=25, injected_per_step=400, cnl_rebuild_interval=10, tol=3e-11, seed=5)


@pytest.fixture(scope="module")
def plate():
    xyz, t, _ = lib.generate(None, case="rain_plate", particles=60_000, l0=1.0, seed=3)
    return xyz, t


def _rows(row, col):
    return [np.sort(col[row[i]:row[i + 1]]) for i in range(len(row) - 1)]


def _same_lists(a, b):
    (ra, ca), (rb, cb) = a, b
    assert np.array_equal(np.diff(ra), np.diff(rb))
    for x, y in zip(_rows(ra, ca), _rows(rb, cb)):
        assert np.array_equal(x, y)


def test_refresh_equals_fresh_build(built, plate):
    xyz, t = plate
    rng = np.random.default_rng(0)
    with lib.Context(0) as a, lib.Context(0) as b:
        a.upload(xyz, t)
        st = a.build_neighbors_skin(2.1, 0.6, 128, 512, 1.0)
        b.upload(xyz, t)
        sb = b.build_neighbors(2.1, 128, 1.0)
        assert st.pairs == sb.pairs
        _same_lists(a.neighbors(st.pairs), b.neighbors(sb.pairs))
        moved = xyz + rng.uniform(-0.17, 0.17, xyz.shape)  # |d| <= 0.17 sqrt(3) < 0.3 = skin / 2
        a.update_positions(moved)
        assert a.max_displacement() <= 0.3
        st = a.refresh_neighbors()
        b.upload(moved, t)
        sb = b.build_neighbors(2.1, 128, 1.0)
        assert st.pairs == sb.pairs and list(st.type_count) == list(sb.type_count)
        _same_lists(a.neighbors(st.pairs), b.neighbors(sb.pairs))
        assert np.array_equal(a.types(), b.types())
        a.update_positions(xyz + np.array([0.4, 0.0, 0.0]) * (np.arange(len(t)) % 2)[:, None])
        with pytest.raises(lib.LsmpsError) as e:
            a.refresh_neighbors()
        assert e.value.code == lib.ERR_STATE


def test_particle_warm_start(built, plate):
    xyz, t = plate
    with lib.Context(0) as c:
        c.upload(xyz, t)
        c.build_neighbors(2.1, 128, 1.0)
        c.wls(2.1, 1.0, mode=1)
        ps = c.ppe_assemble("wls", 10**12, 2.1, 1.0, diag_shift=0.0)
        cold = c.ppe_solve("fp64", 20000, 3e-11)
        pp = c.pressure_particles(len(t), fill=-7.0)
        row, col, val, b, xe, part = c.ppe(ps.unknowns, ps.nnz)
        p_ref = c.pressure(ps.unknowns)
        assert np.array_equal(pp[part], p_ref)  # unknown rank -> its particle
        others = np.ones(len(t), bool)
        others[part] = False
        assert np.all(pp[others] == -7.0)
        c.ppe_assemble("wls", 10**12, 2.1, 1.0, diag_shift=0.0)
        c.set_initial_pressure(pp)
        warm = c.ppe_solve("fp64", 20000, 3e-11, warm_start=True)
        assert warm.converged and warm.iterations <= 2 < cold.iterations


@pytest.fixture(scope="module")
def series_runs(built, plate):
    xyz, t = plate
    out = {}
    with lib.Context(0) as ctx:
        ctx.mpnn_load(lib.DEFAULT_WEIGHTS)
        for key, solver, pc in (("learned", "learned", "jacobi"), ("fp64", "fp64", "jacobi"),
                                ("multigrid", "mixed", "multigrid")):
            with lib.Series(ctx, xyz, t, solver=solver, precond=pc, **SMALL) as s:
                rows, rain = [], []
                for _ in range(SMALL["steps"]):
                    rows.append(s.step())
                    rain.append(s.rain_outputs())
                out[key] = (rows, s.particles())
                out[key + "_rain"] = rain
    return out


def test_series_mass_balance_and_cadence(series_runs):
    rows, _ = series_runs["fp64"]
    for r in rows:
        assert r.mass_balance == 0
        assert r.injected_total == SMALL["injected_per_step"] * r.step
        assert r.forced_rebuild == 0
        assert bool(r.rebuilt) == (r.step == 1 or r.step % SMALL["cnl_rebuild_interval"] == 0)
        if r.rebuilt:
            assert r.in_flight == 0  # injected droplets join at rebuilds
        else:
            assert r.max_displacement <= 0.5 * 1.0
    assert rows[-1].deleted_total > 0  # the film reaches the outflow edge


def test_series_accuracy_and_warm_start(series_runs):
    for solver in ("learned", "fp64", "multigrid"):
        rows, _ = series_runs[solver]
        for r in rows:
            assert r.converged, (solver, r.step)
            assert r.relative_l2_error <= 1e-8, (solver, r.step, r.relative_l2_error)
        warm = np.mean([r.iterations for r in rows[1:]])
        assert warm < rows[0].iterations, (solver, warm, rows[0].iterations)


def test_series_same_particles_for_both_solvers(series_runs):
    (ra, (xa, ma, _)), (rb, (xb, mb, _)) = series_runs["learned"], series_runs["fp64"]
    assert [r.particles for r in ra] == [r.particles for r in rb]
    assert [r.unknowns for r in ra] == [r.unknowns for r in rb]
    assert np.array_equal(xa, xb) and np.array_equal(ma, mb)
    rm, (xm, mm, _) = series_runs["multigrid"]
    assert [r.unknowns for r in rm] == [r.unknowns for r in rb]
    assert np.array_equal(xm, xb) and np.array_equal(mm, mb)
    # the preconditioner cuts the iterations of every step
    assert sum(r.iterations for r in rm) * 3 < sum(r.iterations for r in rb)


REQUIRED = {
    "metrics.csv": {"step", "time", "particles", "injected_total", "outflow_total", "invalid_removed_total",
                    "mass_error"},
    "sampling_windows.csv": {"time", "window", "particle_count", "fluid_volume_m3", "coverage_ratio", "film_mean_m",
                             "film_p90_m", "film_max_m"},
    "flow_sections.csv": {"time", "section", "crossing_particle_count", "instantaneous_flow_rate_m3s",
                          "crossing_volume_m3", "cumulative_volume_m3"},
    "mass_conservation.csv": {"time", "injected_volume_m3", "remaining_volume_m3", "outlet_volume_m3",
                              "invalid_removed_volume_m3", "balance_error_m3", "relative_mass_error",
                              "invalid_removed_ratio"},
}


def test_rain_validation_outputs(series_runs):
    sys.path.insert(0, os.path.dirname(lib.__file__))
    import run_series

    rows, (xyz, mat, _) = series_runs["fp64"]
    rain = series_runs["fp64_rain"]

    class A:
        l0_m, dt_s = 0.004, 1e-3

    tabs = run_series.validation_rows([r.as_dict() for r in rows], rain, A)
    for name, cols in REQUIRED.items():
        tab = tabs[name]
        assert tab and cols <= set(tab[0])
        assert all(math.isfinite(float(v)) for r in tab for k, v in r.items() if k not in ("window", "section"))
    m = tabs["metrics.csv"]
    assert all(b["time"] > a["time"] for a, b in zip(m, m[1:]))
    for r in m:
        assert r["injected_total"] - r["outflow_total"] - r["invalid_removed_total"] - r["particles"] == r["mass_error"]
        assert r["mass_error"] == 0
    for r in tabs["sampling_windows.csv"]:
        assert 0 <= r["coverage_ratio"] <= 1 and r["film_p90_m"] <= r["film_max_m"] + 1e-15
    by = {}
    for r in tabs["flow_sections.csv"]:
        by.setdefault(r["section"], []).append(r["cumulative_volume_m3"])
    assert all(all(b >= a for a, b in zip(v, v[1:])) for v in by.values())
    assert max(r["relative_mass_error"] for r in tabs["mass_conservation.csv"]) <= 0.01
    # the last step's windows from the positions (numpy), the same definitions
    a = math.radians(20.0)
    t1 = np.array([math.cos(a), 0, math.sin(a)])
    nrm = np.array([-math.sin(a), 0, math.cos(a)])
    plate_len = max((xyz[mat == 0] @ t1).max(), 1.0)
    fluid = mat != 0
    u = 1 - (xyz[fluid] @ t1) / plate_len
    d = xyz[fluid] @ nrm
    win, _ = rain[-1]
    for name, lo, hi in lib.RAIN_WINDOWS:
        sel = (u >= lo) & (u < hi) & (d >= 0) & (d <= 3.0)
        cell = np.minimum(31, ((u[sel] - lo) / (hi - lo) * 32).astype(int))
        cnt = np.bincount(cell, minlength=32)
        thick = np.array([d[sel][cell == c].max() + 1.0 for c in range(32) if cnt[c]])
        np_, cov, fmean, fp90, fmax = win[name]
        assert np_ == sel.sum() and cov == (cnt >= 1).sum() / 32
        if len(thick):
            assert abs(fmean - thick.mean()) <= 1e-12 and abs(fp90 - np.quantile(thick, 0.9)) <= 1e-12
            assert abs(fmax - thick.max()) <= 1e-12  # d = x n_x + z n_z: FMA on the GPU


def test_rain_tables_reproduce_the_validated_fixture(series_runs):
    """A fresh run reproduces tests/golden/rain_validation, the tables on which the reference's
    own python/validate_outputs.py passes (tests/test_reference_tools.py)."""
    import csv

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_rain_validation_fixture as fx

    assert fx.SERIES == SMALL and fx.PLATE == {"particles": 60_000, "seed": 3}
    rows, _ = series_runs["fp64"]
    tabs = fx.tables(rows, series_runs["fp64_rain"])
    for name, tab in tabs.items():
        ref = list(csv.DictReader(open(os.path.join(fx.OUT, name))))
        assert len(ref) == len(tab), name
        for got, want in zip(tab, ref):
            assert set(want) == {str(k) for k in got}, name
            for k, v in got.items():
                if k in ("window", "section"):
                    assert str(v) == want[k]
                else:
                    assert math.isclose(float(v), float(want[k]), rel_tol=1e-12, abs_tol=1e-300), (name, k, v, want[k])
