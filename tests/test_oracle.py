"""The CPU oracle pinned against the reference (CPU only).

The restatement in oracle/lsmps_oracle.cpp must equal the reference compiled from its own
sources (oracle/_ref/libref.so) bit for bit on the reference's own inputs, and both must
reproduce the committed golden fixture and the reference README's published table.
"""
import hashlib

import numpy as np
import pytest

from oracle import Oracle, Ref, REF_QUADRATIC

CASES = ["smoke", "bulk_uniform", "wall_film", "rain_injection", "narrow_gap"]


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.fixture(scope="module")
def ref_runs(built, have_ref, cfg_dir):
    if not have_ref:
        pytest.skip("oracle/_ref/libref.so not built here")
    runs = {}
    for name in CASES:
        r = Ref(str(cfg_dir / f"{name}.cfg"))
        xyz, t, _ = r.generate()
        runs[name] = (r, xyz, t)
    return runs


@pytest.mark.parametrize("name", CASES)
def test_reference_matches_golden(ref_runs, golden, name):
    r, xyz, t = ref_runs[name]
    g = golden["cases"][name]
    assert sha(xyz, t) == g["positions_sha256"]
    row, col, trunc = r.neighbors()
    assert sha(row, col) == g["neighbors"]["csr_sha256"]
    assert trunc == g["neighbors"]["truncated"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_neighbors_and_types_bit_exact(ref_runs, golden, name):
    r, xyz, t = ref_runs[name]
    re = r.cfg("re_ratio") * r.cfg("l0")
    row, col, trunc = Oracle.neighbors(xyz, re, int(r.cfg("max_neighbors")))
    g = golden["cases"][name]
    assert sha(row, col) == g["neighbors"]["csr_sha256"]
    assert trunc == g["neighbors"]["truncated"]
    types = Oracle.classify(xyz, t, row, col, r.cfg("l0"))
    assert sha(types) == g["types"]["sha256"]
    assert np.bincount(types, minlength=5).tolist() == g["types"]["counts"]


@pytest.mark.parametrize("name", ["smoke", "bulk_uniform", "rain_injection"])
def test_oracle_wls_bit_exact(ref_runs, name):
    r, xyz, t = ref_runs[name]
    r.neighbors()
    types = r.classify()
    re, l0 = r.cfg("re_ratio") * r.cfg("l0"), r.cfg("l0")
    row, col, _ = Oracle.neighbors(xyz, re, int(r.cfg("max_neighbors")))
    x, st, z, ws = Oracle.wls(xyz, types, row, col, re, l0, coef=REF_QUADRATIC)
    checked = 0
    for i in range(0, len(types), 53):
        code, xr = r.wls_particle(i)
        if types[i] in (2, 4):
            assert st[i] == 2
            continue
        if code < 0:
            assert st[i] in (3, 4)
            continue
        assert st[i] == code
        assert np.array_equal(x[i, 0], xr)
        checked += 1
    assert checked > 50


@pytest.mark.parametrize("name", CASES)
def test_oracle_ppe_and_bicgstab_bit_exact(ref_runs, golden, name):
    r, xyz, t = ref_runs[name]
    r.neighbors()
    types = r.classify()
    g = golden["cases"][name]
    re, l0 = r.cfg("re_ratio") * r.cfg("l0"), r.cfg("l0")
    row, col, _ = Oracle.neighbors(xyz, re, int(r.cfg("max_neighbors")))
    prow, pcol, val, b, xe, up, stats = Oracle.ppe_assemble(0, xyz, types, row, col, re, l0,
                                                            int(r.cfg("ppe_max_unknowns")))
    assert sha(prow, pcol, val) == g["ppe"]["csr_sha256"]
    assert sha(b) == g["ppe"]["b_sha256"] and sha(xe) == g["ppe"]["x_exact_sha256"]
    for k in ("unknowns", "nnz", "dirichlet", "neumann", "failed_rows"):
        assert stats[k] == g["ppe"][k]
    x, info = Oracle.bicgstab(prow, pcol, val, b, int(r.cfg("ppe_max_iter")), r.cfg("ppe_tol"))
    assert info["iterations"] == g["solve"]["iterations"]
    assert info["converged"] == g["solve"]["converged"]
    assert float(info["final_residual"]).hex() == g["solve"]["final_residual"]["hex"]
    e = x - xe
    rel = np.sqrt(np.sum(e * e) / max(np.sum(xe * xe), 1e-30))
    assert rel == pytest.approx(g["solve"]["relative_l2_error"]["value"], rel=1e-12)


def test_readme_table(golden):
    """The fixture reproduces the reference README's published v0.2 table (README.md:54-57)."""
    for name, (unk, nnz, iters, rel) in golden["readme_table"].items():
        g = golden["cases"][name]
        assert g["ppe"]["unknowns"] == unk and g["ppe"]["nnz"] == nnz
        assert g["solve"]["iterations"] == iters
        assert round(g["solve"]["relative_l2_error"]["value"], 7) == pytest.approx(rel, rel=5e-3)


def test_oracle_wls_reproduces_quadratics():
    """Second-order WLS reproduces gradients and Laplacians of quadratics to rounding."""
    rng = np.random.default_rng(3)
    nx = 12
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(nx), np.arange(nx), indexing="ij"), -1).reshape(-1, 3)
    xyz = (g + 0.5 + rng.uniform(-0.1, 0.1, g.shape)).astype(np.float64)
    t = np.zeros(len(xyz), np.uint8)
    row, col, _ = Oracle.neighbors(xyz, 2.1, 128)
    types = Oracle.classify(xyz, t, row, col, 1.0)
    coef = rng.normal(size=(3, 10))
    x, st, z, ws = Oracle.wls(xyz, types, row, col, 2.1, 1.0, coef=coef)
    ok = (st == 0) | (st == 1)
    assert ok.sum() > 0.9 * len(xyz)
    for f in range(3):
        c = coef[f]
        gx = c[1] + 2 * c[4] * xyz[:, 0] + c[7] * xyz[:, 1] + c[8] * xyz[:, 2]
        lap = 2 * (c[4] + c[5] + c[6])
        assert np.max(np.abs(x[ok, f, 0] - gx[ok])) < 1e-9
        assert np.max(np.abs(x[ok, f, 3:6].sum(1) - lap)) < 1e-8


def test_oracle_wls_ppe_converges():
    """The WLS-Laplacian PPE rows (negative coefficients clipped) give a solvable system."""
    rng = np.random.default_rng(5)
    nx = 16
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(nx), np.arange(nx), indexing="ij"), -1).reshape(-1, 3)
    xyz = (g + 0.5 + rng.uniform(-0.1, 0.1, g.shape)).astype(np.float64)
    t = np.zeros(len(xyz), np.uint8)
    row, col, _ = Oracle.neighbors(xyz, 2.1, 128)
    types = Oracle.classify(xyz, t, row, col, 1.0)
    x, st, z, ws = Oracle.wls(xyz, types, row, col, 2.1, 1.0)
    prow, pcol, val, b, xe, up, stats = Oracle.ppe_assemble(2, xyz, types, row, col, 2.1, 1.0, 10**9, 0.0,
                                                            z, ws, st)
    assert np.all(val[prow[1:] - 1] > 0)  # diagonal last and positive
    off = np.ones(len(val), bool)
    off[prow[1:] - 1] = False
    assert np.all(val[off] < 0)
    for pc in (0, 1):
        xs, info = Oracle.bicgstab(prow, pcol, val, b, 5000, 1e-10, precond=pc)
        assert info["converged"]
        assert np.linalg.norm(xs - xe) / np.linalg.norm(xe) < 1e-8
