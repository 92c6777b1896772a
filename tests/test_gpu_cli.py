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
