"""Generates tests/golden/reference_cases.json from the reference implementation.

Runs the reference (lilux618/LS-MPS, compiled from its own sources into
oracle/_ref/libref.so by oracle/Makefile) on each of its shipped .cfg inputs and records,
per case, the values the GPU path must reproduce: particle-set and neighbor-CSR hashes,
class counts, neighbor statistics, the wls_test statistics, the assembled PPE (sizes and a
hash of its CSR bytes) and the BiCGStab outcome. Floating-point values are stored both as
numbers and as float.hex() strings so that tests can demand bit equality.

Usage (where the reference sources exist): python tests/golden/make_golden.py
The .cfg files are read from the reference's config/ directory and their text is stored in
the fixture, so the GPU tests need nothing from the reference at run time.
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from oracle import REF_BIN, Ref, build  # noqa: E402

REF_ROOT = os.environ.get("LSMPS_REFERENCE", "/root/reference")  # the reference source tree
CASES = ["smoke", "bulk_uniform", "wall_film", "rain_injection", "narrow_gap"]


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def fl(x: float):
    return {"value": float(x), "hex": float(x).hex()}


def case_record(name: str) -> dict:
    cfg = os.path.join(REF_ROOT, "config", f"{name}.cfg")
    text = open(cfg).read()
    r = Ref(cfg)
    xyz, t_in, _ = r.generate()
    row, col, trunc = r.neighbors()
    types = r.classify()
    wls = r.wls_test()
    prow, pcol, pval, pb, pxe, pst = r.assemble_ppe()
    sol = r.solve_ppe()
    counts = np.diff(row)
    srt = np.sort(counts)
    n = len(counts)
    pct = {q: int(srt[int(q * (n - 1))]) for q in (0.5, 0.9, 0.99)}
    with tempfile.TemporaryDirectory() as td:
        cli = subprocess.run([REF_BIN, cfg, td], capture_output=True, text=True)
        cfg_case = r.cfg("case")
        json_text = open(os.path.join(td, f"{cfg_case}.json")).read()
        csv_text = open(os.path.join(td, f"{cfg_case}.csv")).read()
    return {
        "cli": {"exit_code": cli.returncode, "stdout": cli.stdout, "json": json_text, "csv": csv_text},
        "cfg_text": text,
        "particles": int(n),
        "positions_sha256": digest(xyz, t_in),
        "neighbors": {
            "pairs": int(len(col)), "truncated": int(trunc), "csr_sha256": digest(row, col),
            "mean": fl(len(col) / n), "p50": pct[0.5], "p90": pct[0.9], "p99": pct[0.99],
        },
        "types": {"counts": np.bincount(types, minlength=5).tolist(), "sha256": digest(types)},
        "wls": {k: (int(v) if k in ("sampled", "ok", "regularized", "failed", "virtual_points") else fl(v))
                for k, v in wls.items()},
        "ppe": {
            **{k: int(v) for k, v in pst.items()},
            "csr_sha256": digest(prow, pcol, pval), "b_sha256": digest(pb), "x_exact_sha256": digest(pxe),
        },
        "solve": {
            "iterations": int(sol["iterations"]), "converged": bool(sol["converged"]),
            "initial_residual": fl(sol["initial_residual"]), "final_residual": fl(sol["final_residual"]),
            "relative_l2_error": fl(sol["relative_l2_error"]), "max_error": fl(sol["max_error"]),
        },
    }


def main():
    build()
    out = {
        "source": "reference lilux618/LS-MPS src/lsmps.cpp compiled with g++ -O3 -std=c++17",
        # Published v0.2 table (reference README.md:54-57): unknowns, nnz, iterations, rel L2
        "readme_table": {
            "bulk_uniform": [6000, 160953, 265, 3.72e-5],
            "wall_film": [6000, 76247, 394, 1.75e-5],
            "rain_injection": [6000, 76157, 351, 1.31e-5],
            "narrow_gap": [6000, 76251, 359, 2.08e-5],
        },
        "cases": {name: case_record(name) for name in CASES},
    }
    with open(os.path.join(HERE, "reference_cases.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "reference_cases.json"))


if __name__ == "__main__":
    main()
