"""The reference's own Python tools run on this repository's files (CPU, where the reference
tree is present; the LSMPS_REFERENCE environment variable names it):

* python/validate_outputs.py, unmodified, on the rain validation tables that the GPU step
  series wrote (tests/golden/rain_validation, made by tests/golden/make_rain_validation_fixture.py;
  tests/test_gpu_series.py checks that a fresh GPU run reproduces them): it must pass with the
  reference's config/rain_plate_validation.json.
* the calibration fixture (tests/golden/calibration) is the file set python/workload_calibration.py
  wrote (tests/golden/make_calibration_fixture.py ran it): its arrays are consistent with one
  another and with the tool's own metadata.json; tests/test_replay_csr.py replays it on the GPU.
"""
import csv
import json
import os
import subprocess
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
REF_ROOT = os.environ.get("LSMPS_REFERENCE", "/root/reference")


def test_reference_validator_passes_the_gpu_tables(tmp_path):
    tool = os.path.join(REF_ROOT, "python", "validate_outputs.py")
    if not os.path.exists(tool):
        pytest.skip("the reference tree is not present")
    report = tmp_path / "report.json"
    p = subprocess.run([sys.executable, tool, "--output", os.path.join(GOLDEN, "rain_validation"), "--config",
                        os.path.join(REF_ROOT, "config", "rain_plate_validation.json"), "--report", str(report)],
                       capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    summary = json.loads(report.read_text())
    assert summary["passed"] and not summary["errors"]
    assert {c["check"] for c in summary["checks"]} >= {"particle_identity", "mass_conservation", "invalid_removal"}


def test_rain_tables_are_nontrivial():
    d = os.path.join(GOLDEN, "rain_validation")
    rows = {n: list(csv.DictReader(open(os.path.join(d, n)))) for n in
            ("metrics.csv", "sampling_windows.csv", "flow_sections.csv", "mass_conservation.csv")}
    assert len(rows["metrics.csv"]) == 25
    assert int(rows["metrics.csv"][-1]["outflow_total"]) > 0  # the film reaches the outflow edge
    assert any(float(r["coverage_ratio"]) > 0 for r in rows["sampling_windows.csv"])
    assert any(int(r["crossing_particle_count"]) > 0 for r in rows["flow_sections.csv"])


def test_calibration_fixture_is_the_tool_output():
    d = os.path.join(GOLDEN, "calibration")
    meta = json.load(open(os.path.join(d, "metadata.json")))
    rl = np.load(os.path.join(d, "neighbor_row_length.npy"))
    rp = np.load(os.path.join(d, "csr_row_ptr.npy"))
    col = np.load(os.path.join(d, "csr_col_idx.npy"))
    pt = np.load(os.path.join(d, "particle_type.npy"))
    n = meta["particles"]
    assert rl.dtype == np.int32 and rp.dtype == np.int64 and col.dtype == np.int32 and pt.dtype == np.uint8
    assert len(rl) == len(pt) == n and rp[0] == 0 and np.array_equal(np.diff(rp), rl)
    assert meta["csr_nnz"] == int(rp[-1]) == len(col) and meta["materialized_col_idx"]
    assert col.min() >= 0 and col.max() < n
    assert meta["neighbor_mean"] == float(rl.mean())
    assert meta["neighbor_p90"] == float(np.quantile(rl, 0.9, method="higher"))
    assert meta["neighbor_p99"] == float(np.quantile(rl, 0.99, method="higher"))
    # the tool's type codes: 0 interior, 1 near wall, 2 free surface, 3 splash
    for code, key in ((1, "near_wall_ratio"), (2, "free_surface_ratio"), (3, "splash_ratio")):
        assert meta[key] == float(np.mean(pt == code))
    tl = list(csv.DictReader(open(os.path.join(d, "timeline.csv"))))
    assert len(tl) == 200 and set(tl[0]) == {"step", "injected", "deleted", "cnl_rebuild", "ppe_iterations"}
