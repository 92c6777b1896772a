"""Calibrated synthetic CSR (the reference's python/workload_calibration.py file set) and its
GPU replay.

CPU: the generator writes the reference tool's files and dtypes, the row lengths sum to
round(mean n), the reported quantiles are the realized ones, columns are in range.
GPU: lsmps_ppe_load_csr installs the system as documented (diagonal last, -1 off-diagonals,
b = A 1), rejects bad input, refuses the learned solver; the replay's solvers reach p* = 1.
"""
import json
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ls-mps_b200"))
import lsmps_b200 as lib  # noqa: E402
import replay_csr  # noqa: E402

FILES = {"particle_type.npy": np.uint8, "neighbor_row_length.npy": np.int32, "csr_row_ptr.npy": np.int64,
         "csr_col_idx.npy": np.int32, "virtual_neighbor_count.npy": np.int16, "wls_ill_conditioned.npy": np.bool_}


def _profile(n):
    p = dict(replay_csr.DEFAULT_PROFILE)
    p.update(particles=n, timeline_steps=12)
    return p


def test_generator_writes_the_reference_file_set(tmp_path):
    n = 20000
    meta = replay_csr.generate(str(tmp_path), _profile(n), seed=3)
    for name, dt in FILES.items():
        a = np.load(tmp_path / name)
        assert a.dtype == dt, name
    rl = np.load(tmp_path / "neighbor_row_length.npy")
    rp = np.load(tmp_path / "csr_row_ptr.npy")
    col = np.load(tmp_path / "csr_col_idx.npy")
    assert len(rl) == n and rp[0] == 0 and np.array_equal(np.diff(rp), rl)
    assert rl.sum() == round(_profile(n)["neighbor_mean"] * n) and rl.min() >= 1
    # the exact-mean adjustment moves the quantiles off the profile's (as in the reference tool,
    # which reports the realized ones): check the ordering and the reported values
    p90, p99 = np.quantile(rl, 0.9, method="higher"), np.quantile(rl, 0.99, method="higher")
    assert rl.mean() <= p90 <= p99 and meta["neighbor_p90"] == p90 and meta["neighbor_p99"] == p99
    assert col.min() >= 0 and col.max() < n and len(col) == rp[-1]
    t = (tmp_path / "timeline.csv").read_text().splitlines()
    assert t[0] == "step,injected,deleted,cnl_rebuild,ppe_iterations" and len(t) == 13
    assert json.loads((tmp_path / "metadata.json").read_text())["csr_nnz"] == int(rp[-1]) == meta["csr_nnz"]


@pytest.mark.gpu
def test_load_csr_and_replay(built, tmp_path):
    n = 60000
    replay_csr.generate(str(tmp_path), _profile(n), seed=5)
    rp = np.load(tmp_path / "csr_row_ptr.npy")
    col = np.load(tmp_path / "csr_col_idx.npy")
    with lib.Context(0) as c:
        st = c.ppe_load_csr(rp, col)
        row, acol, val, b, xe, part = c.ppe(st.unknowns, st.nnz)
        assert st.unknowns == n and np.array_equal(part, np.arange(n)) and np.all(xe == 1.0)
        for i in (0, 1, n // 2, n - 1):  # off-diagonals -1 in input order, the diagonal last
            cols = col[rp[i]:rp[i + 1]]
            off = cols[cols != i]
            assert np.array_equal(acol[row[i]:row[i + 1] - 1], off) and np.all(val[row[i]:row[i + 1] - 1] == -1.0)
            assert acol[row[i + 1] - 1] == i and val[row[i + 1] - 1] == max(1.0, len(off) * (1 + 1e-3))
        rows = np.repeat(np.arange(n), np.diff(row))
        assert np.allclose(b, np.bincount(rows, weights=val, minlength=n), rtol=1e-14, atol=0)
        bad = col.copy()
        bad[7] = n
        with pytest.raises(lib.LsmpsError) as e:
            c.ppe_load_csr(rp, bad)
        assert e.value.code == lib.ERR_ARG
        c.ppe_load_csr(rp, col)
        c.mpnn_init(0)
        with pytest.raises(lib.LsmpsError) as e:
            c.ppe_solve("learned", 100, 1e-10)
        assert e.value.code == lib.ERR_STATE
    res = replay_csr.replay(str(tmp_path), ("mixed", "fp64"), tol=1e-11)
    for name, s in res["solvers"].items():
        assert s["converged"] and s["relative_l2_error"] <= 1e-8, (name, s)
    assert all(k["achieved_gbs"] > 0 for k in res["kernels"].values())
    assert res["timeline"]["steps"] == 12


@pytest.mark.gpu
def test_replay_the_reference_tool_output(built):
    """The replay on the file set the reference's python/workload_calibration.py wrote
    (tests/golden/calibration): every solver reaches p* = 1, the SpMV kernels run, and the
    tool's 200-step timeline replays."""
    d = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "calibration")
    res = replay_csr.replay(d, ("mixed", "fp64", "jacobi"), tol=1e-11)
    meta = json.load(open(os.path.join(d, "metadata.json")))
    assert res["rows"] == meta["particles"] and res["entries"] == meta["csr_nnz"]
    for name, s in res["solvers"].items():
        assert s["converged"] and s["relative_l2_error"] <= 1e-8, (name, s)
    assert all(k["achieved_gbs"] > 0 for k in res["kernels"].values())
    assert res["timeline"]["steps"] == 200
