"""The lsmps-bench CLI is a drop-in: same JSON / CSV bytes and summary as the reference's
CLI on the reference's cases, timing fields aside."""
import json
import subprocess

import pytest

import lsmps_b200 as lib
from _util import strip_csv_timings, strip_json_timings

pytestmark = pytest.mark.gpu
CASES = ["smoke", "bulk_uniform", "wall_film", "rain_injection", "narrow_gap"]


@pytest.mark.parametrize("name", CASES)
def test_cli_outputs_match_reference(built, golden, cfg_dir, tmp_path, name):
    g = golden["cases"][name]["cli"]
    r = subprocess.run([lib.CLI_PATH, str(cfg_dir / f"{name}.cfg"), str(tmp_path)], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == g["exit_code"], r.stderr
    case = json.loads(g["json"])["case"]
    mine = (tmp_path / f"{case}.json").read_text()
    assert strip_json_timings(mine) == strip_json_timings(g["json"])
    assert strip_csv_timings((tmp_path / f"{case}.csv").read_text()) == strip_csv_timings(g["csv"])
    # the summary lines before the timing / output lines are identical too
    assert r.stdout.splitlines()[:6] == g["stdout"].splitlines()[:6]
    ext = json.loads((tmp_path / f"{case}.gpu.json").read_text())
    assert ext["iterations"] == json.loads(g["json"])["ppe"]["iterations"]


def test_cli_missing_config(built, tmp_path):
    r = subprocess.run([lib.CLI_PATH, str(tmp_path / "nope.cfg"), str(tmp_path)], capture_output=True, text=True)
    assert r.returncode == 1 and "cannot open config" in r.stderr


def test_cli_multigrid_solver(built, golden, tmp_path):
    """The .cfg keys solver=mixed, precond=multigrid on the reference's bulk case with the
    WLS-Laplacian rows over all unknowns (l0 = 0.01, so the FP16 A*P scaling is exercised
    away from l0 = 1): converged to the manufactured solution in far fewer iterations."""
    base = golden["cases"]["bulk_uniform"]["cfg_text"].replace("ppe_max_unknowns = 6000",
                                                               "ppe_max_unknowns = 1000000")
    out = {}
    for pc in ("jacobi", "multigrid"):
        cfg = tmp_path / f"{pc}.cfg"
        cfg.write_text(base.replace("case=bulk_uniform", f"case=bulk_{pc}") +
                       f"\nppe_variant=wls\nwls_mode=all\nsolver=mixed\nprecond={pc}\nppe_tol=3e-11\n"
                       "ppe_max_iter=20000\n")
        r = subprocess.run([lib.CLI_PATH, str(cfg), str(tmp_path)], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        out[pc] = json.loads((tmp_path / f"bulk_{pc}.gpu.json").read_text())
    mg = out["multigrid"]
    assert mg["precond"] == "multigrid" and mg["relative_l2_error"] <= 1e-8
    assert mg["iterations"] * 3 <= out["jacobi"]["iterations"], (mg["iterations"], out["jacobi"]["iterations"])
