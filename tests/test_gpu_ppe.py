"""GPU PPE assembly: the reference variant bit for bit; shifted and WLS variants against
the oracle (values within 1e-12 relative)."""
import numpy as np
import pytest
import scipy.sparse as sp

import lsmps_b200 as lib
from _util import cfg_params, jittered_lattice, sha
from oracle import Oracle

pytestmark = pytest.mark.gpu
CASES = ["smoke", "bulk_uniform", "wall_film", "rain_injection", "narrow_gap"]


@pytest.fixture(scope="module")
def ctx(built):
    c = lib.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", CASES)
def test_reference_variant_bit_exact(ctx, golden, cfg_dir, name):
    g = golden["cases"][name]
    p = cfg_params(g["cfg_text"])
    xyz, t, _ = lib.generate(str(cfg_dir / f"{name}.cfg"))
    ctx.upload(xyz, t)
    ctx.build_neighbors(p["re"], p["max_neighbors"], p["l0"])
    st = ctx.ppe_assemble("reference", p["ppe_max_unknowns"], p["re"], p["l0"])
    for k in ("unknowns", "nnz", "dirichlet", "neumann", "failed_rows"):
        assert getattr(st, k) == g["ppe"][k], k
    row, col, val, b, xe, part = ctx.ppe(st.unknowns, st.nnz)
    assert sha(row, col, val) == g["ppe"]["csr_sha256"]
    assert sha(b) == g["ppe"]["b_sha256"]
    assert sha(xe) == g["ppe"]["x_exact_sha256"]


def _csr(row, col, val, n):
    # copies: scipy sorts indices in place when it canonicalises a matrix
    return sp.csr_matrix((val.copy(), col.copy(), row.copy()), shape=(n, n))


@pytest.mark.parametrize("variant", ["shifted", "wls"])
@pytest.mark.parametrize("case", ["lattice", "rain_plate"])
def test_variants_match_oracle(ctx, variant, case):
    if case == "lattice":
        xyz = jittered_lattice(18, 0.1, seed=7)
        t = np.zeros(len(xyz), np.uint8)
    else:
        xyz, t, _ = lib.generate(None, case="rain_plate", particles=40_000, l0=1.0, seed=9)
    ctx.upload(xyz, t)
    ctx.build_neighbors(2.1, 128, 1.0)
    types = ctx.types()
    row, col, _ = Oracle.neighbors(xyz, 2.1, 128)
    z = ws = wst = None
    if variant == "wls":
        ctx.wls(2.1, 1.0, mode=1)
        _, wst, z, ws = ctx.wls_result()
        _, so, zo, wo = Oracle.wls(xyz, types, row, col, 2.1, 1.0)
        assert np.array_equal(wst, so)
        z, ws = zo, wo  # the oracle assembles from its own WLS vectors
    cap = 10**9
    st = ctx.ppe_assemble(variant, cap, 2.1, 1.0, diag_shift=1e-3)
    prow, pcol, pval, b, xe, part = ctx.ppe(st.unknowns, st.nnz)
    vid = lib.VARIANTS[variant]
    orow, ocol, oval, ob, oxe, oup, ost = Oracle.ppe_assemble(vid, xyz, types, row, col, 2.1, 1.0, cap, 1e-3,
                                                              z, ws, wst)
    assert st.unknowns == ost["unknowns"]
    assert np.array_equal(part, oup)
    assert np.allclose(xe, oxe, rtol=1e-14, atol=1e-14)
    n = st.unknowns
    if variant == "shifted":
        # same operations in the same order as the oracle: identical CSR
        assert np.array_equal(prow, orow) and np.array_equal(pcol, ocol)
        assert np.array_equal(pval, oval)
        assert np.allclose(b, ob, rtol=1e-13, atol=1e-13 * np.abs(ob).max())
    else:
        # the GPU rows use the GPU's WLS vectors (FP64, different rounding order than the
        # oracle's); clipping may differ only for coefficients within rounding of zero
        assert abs(st.nnz - ost["nnz"]) <= max(2, st.nnz // 100000)
        A, O = _csr(prow, pcol, pval, n), _csr(orow, ocol, oval, n)
        assert abs(A - O).max() <= 1e-8 * abs(O).max()
        assert np.allclose(b, ob, rtol=1e-8, atol=1e-8 * np.abs(ob).max())


def test_cap_and_empty(ctx):
    xyz = jittered_lattice(10, 0.1, seed=3)
    ctx.upload(xyz, np.zeros(len(xyz), np.uint8))
    ctx.build_neighbors(2.1, 96, 1.0)
    st = ctx.ppe_assemble("reference", 100, 2.1, 1.0)
    assert st.unknowns == 100
    st = ctx.ppe_assemble("reference", 0, 2.1, 1.0)
    assert st.unknowns == 0 and st.nnz == 0
    s = ctx.ppe_solve("reference", 10, 1e-7)
    assert s.iterations == 0 and s.converged == 0


def test_neighbors_and_assembly_without_statistics(ctx):
    """A neighbor build and an assembly called without statistics (out = NULL) return without
    waiting for their last kernels, leave the same lists and system as with statistics, and
    their phase times are read by lsmps_get_timings (the assembly's also by the next solve)."""
    xyz, t, _ = lib.generate(None, case="mixed", particles=50_000, l0=1.0, seed=4)
    ctx.upload(xyz, t)
    nst = ctx.build_neighbors(2.1, 128, 1.0)
    row, col = ctx.neighbors(nst.pairs)
    ctx.wls(2.1, 1.0, mode=1)
    pst = ctx.ppe_assemble("wls", 10**12, 2.1, 1.0, diag_shift=0.0)
    ref = ctx.ppe(pst.unknowns, pst.nnz)
    assert ctx.build_neighbors(2.1, 128, 1.0, stats=False) is None
    tm = ctx.timings()
    assert tm[1] > 0.0
    row2, col2 = ctx.neighbors(nst.pairs)
    assert np.array_equal(row, row2) and np.array_equal(col, col2)
    ctx.wls(2.1, 1.0, mode=1, stats=False)
    assert ctx.ppe_assemble("wls", 10**12, 2.1, 1.0, diag_shift=0.0, stats=False) is None
    s = ctx.ppe_solve("mixed", 5000, 1e-10, precond="multigrid")
    assert s.converged and s.assembly_ms > 0.0
    assert s.unknowns == pst.unknowns and s.nnz == pst.nnz
    assert ctx.timings()[4] == s.assembly_ms
    got = ctx.ppe(pst.unknowns, pst.nnz)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
