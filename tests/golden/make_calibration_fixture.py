"""Writes tests/golden/calibration/: the synthetic CSR workload of the reference's own
calibration tool (python/workload_calibration.py, run unmodified from the reference tree with
--materialize-csr), for the replay tests.

    LSMPS_REFERENCE=/path/to/LS-MPS python tests/golden/make_calibration_fixture.py

The tool runs on the reference's shipped profiles (config/customer_car_rain_profile.example.json
as the target, config/plate_rain_baseline_profile.json as the baseline) with the target's
particle count scaled down to PARTICLES so that the fixture stays small; every other metric
(neighbor mean / P90 / P99, type ratios, timeline) is the profile's. The files are copied as
the tool wrote them (npy arrays, timeline.csv, metadata.json); source.json records the command.
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("LSMPS_REFERENCE", "/root/reference")  # the reference source tree
OUT = os.path.join(HERE, "calibration")
PARTICLES = 6000
SEED = 42


def main():
    tool = os.path.join(REF_ROOT, "python", "workload_calibration.py")
    target = json.load(open(os.path.join(REF_ROOT, "config", "customer_car_rain_profile.example.json")))
    target["metrics"]["particles"] = PARTICLES
    with tempfile.TemporaryDirectory() as tmp:
        tpath = os.path.join(tmp, "target.json")
        json.dump(target, open(tpath, "w"), indent=1)
        cmd = [sys.executable, tool, "--target", tpath, "--baseline",
               os.path.join(REF_ROOT, "config", "plate_rain_baseline_profile.json"), "--out",
               os.path.join(tmp, "out"), "--seed", str(SEED), "--iterations", "2000", "--materialize-csr"]
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
        src = os.path.join(tmp, "out", "synthetic_workload")
        if os.path.isdir(OUT):
            shutil.rmtree(OUT)
        shutil.copytree(src, OUT)
    cmd_rec = ["python/workload_calibration.py"] + [os.path.basename(c) if os.path.sep in c else c for c in cmd[2:]]
    json.dump({"tool": "python/workload_calibration.py (reference, unmodified)", "command": " ".join(cmd_rec),
               "target": "config/customer_car_rain_profile.example.json with particles = %d" % PARTICLES,
               "baseline": "config/plate_rain_baseline_profile.json", "seed": SEED},
              open(os.path.join(OUT, "source.json"), "w"), indent=1)
    print("wrote", OUT, sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
