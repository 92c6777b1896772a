"""GPU multigrid preconditioner (ls-mps_b200/csrc/multigrid.cu).

* The hierarchy and the V-cycle equal the FP64 restatement in oracle/multigrid_oracle.py:
  same level sizes, and D M z within FP32 rounding.
* MIXED and LEARNED with precond="multigrid" reach the manufactured solution (relative L2
  <= 1e-8 at residual tolerance 3e-11) in a fraction of the Jacobi iterations. The result
  is deterministic and identical across the three launch forms.
* The preconditioner is refused where it does not apply.
"""
import numpy as np
import pytest

import lsmps_b200 as lib
import multigrid_oracle as mgo

pytestmark = pytest.mark.gpu
RE, L0 = 2.1, 1.0


@pytest.fixture(scope="module")
def ctx(built):
    c = lib.Context(0)
    yield c
    c.close()


def _setup(ctx, case="mixed", n=60_000, seed=5):
    xyz, t, _ = lib.generate(None, case=case, particles=n, l0=L0, seed=seed)
    ctx.upload(xyz, t)
    ctx.build_neighbors(RE, 128, L0)
    ctx.wls(RE, L0, mode=1)
    st = ctx.ppe_assemble("wls", 10**9, RE, L0, diag_shift=0.0)
    return xyz, st


@pytest.mark.parametrize("case", ["mixed", "rain_plate"])
def test_vcycle_matches_restatement(ctx, case):
    import scipy.sparse as sp

    xyz, st = _setup(ctx, case, 60_000, 5)
    row, col, val, b, xe, part = ctx.ppe(st.unknowns, st.nnz)
    A = sp.csr_matrix((val, col, row), shape=(st.unknowns, st.unknowns))
    H = mgo.Hierarchy(A, mgo.cells_of(xyz, xyz[part], RE))
    z = np.random.default_rng(1).standard_normal(st.unknowns)
    out = ctx.mg_apply(z)
    rows, setup_ms = ctx.mg_info()
    assert list(rows) == H.sizes
    assert setup_ms > 0
    ref = H.apply(z)
    # FP32 inside the V-cycle, FP16 AP in both: agreement to single-precision rounding of its
    # levels plus the odd half-precision entry rounded the other way (FP32 vs FP64 sums)
    assert np.linalg.norm(out - ref) <= 1e-4 * np.linalg.norm(ref)
    assert np.array_equal(ctx.mg_apply(z), out)  # deterministic


def test_single_level_hierarchy(ctx):
    """A system with at most 256 cells: level 1 is the coarsest (one block solves it)."""
    import scipy.sparse as sp
    from _util import jittered_lattice

    xyz = jittered_lattice(12, 0.1, seed=4)
    ctx.upload(xyz, np.zeros(len(xyz), np.uint8))
    ctx.build_neighbors(RE, 128, L0)
    ctx.wls(RE, L0, mode=1)
    st = ctx.ppe_assemble("wls", 10**9, RE, L0, diag_shift=0.0)
    row, col, val, b, xe, part = ctx.ppe(st.unknowns, st.nnz)
    A = sp.csr_matrix((val, col, row), shape=(st.unknowns, st.unknowns))
    H = mgo.Hierarchy(A, mgo.cells_of(xyz, xyz[part], RE))
    assert H.levels == 1
    z = np.random.default_rng(2).standard_normal(st.unknowns)
    out = ctx.mg_apply(z)
    rows, _ = ctx.mg_info()
    assert list(rows) == H.sizes
    ref = H.apply(z)
    assert np.linalg.norm(out - ref) <= 1e-4 * np.linalg.norm(ref)
    s = ctx.ppe_solve("mixed", 5000, 3e-11, precond="multigrid")
    assert s.converged and s.relative_l2_error <= 1e-8


def test_multigrid_solves_to_target(ctx):
    _setup(ctx, "mixed", 200_000, 7)
    jac = ctx.ppe_solve("mixed", 20000, 3e-11)
    mg = ctx.ppe_solve("mixed", 20000, 3e-11, precond="multigrid")
    assert jac.converged and mg.converged
    assert mg.relative_l2_error <= 1e-8
    assert mg.final_residual <= 3e-11 * max(1.0, mg.initial_residual) * 1.01
    assert mg.iterations * 4 <= jac.iterations, (mg.iterations, jac.iterations)
    p1 = ctx.pressure(mg.unknowns)
    again = ctx.ppe_solve("mixed", 20000, 3e-11, precond="multigrid")
    assert again.iterations == mg.iterations
    assert np.array_equal(ctx.pressure(mg.unknowns), p1)


def test_launch_forms_agree(ctx):
    _setup(ctx, "rain_plate", 80_000, 2)
    out = []
    for g in (1, 2, 0):
        st = ctx.ppe_solve("mixed", 20000, 3e-11, use_graph=g, precond="multigrid")
        assert st.converged
        out.append((st.iterations, ctx.pressure(st.unknowns)))
    for it, p in out[1:]:
        assert it == out[0][0]
        assert np.array_equal(p, out[0][1])


def test_learned_with_multigrid(ctx):
    _setup(ctx, "mixed", 100_000, 11)
    ctx.mpnn_load(lib.DEFAULT_WEIGHTS)
    st = ctx.ppe_solve("learned", 20000, 3e-11, precond="multigrid")
    assert st.converged and st.relative_l2_error <= 1e-8


def test_learned_multigrid_setup_beside_network_is_deterministic(ctx):
    """After each assembly the LEARNED solver with the multigrid builds the hierarchy on a second
    stream while the network runs; the two read the same system and write disjoint buffers, so
    every fresh assembly + solve gives the same bits, in every launch form."""
    _setup(ctx, "mixed", 80_000, 13)
    ctx.mpnn_load(lib.DEFAULT_WEIGHTS)
    out = []
    for g in (0, 1, 2, 0):
        ctx.ppe_assemble("wls", 10**9, RE, L0, diag_shift=0.0)  # a new hierarchy per solve
        st = ctx.ppe_solve("learned", 20000, 3e-11, use_graph=g, precond="multigrid")
        assert st.converged and st.relative_l2_error <= 1e-8
        out.append((st.iterations, ctx.pressure(st.unknowns)))
    for it, p in out[1:]:
        assert it == out[0][0]
        assert np.array_equal(p, out[0][1])


def test_warm_start_with_multigrid(ctx):
    _setup(ctx, "mixed", 60_000, 12)
    cold = ctx.ppe_solve("mixed", 20000, 3e-11, precond="multigrid")
    warm = ctx.ppe_solve("mixed", 20000, 3e-11, warm_start=True, precond="multigrid")
    assert warm.converged and warm.iterations <= 2
    assert warm.relative_l2_error <= 1e-8
    assert cold.iterations > warm.iterations


def test_refusals(ctx):
    _setup(ctx, "mixed", 20_000, 1)
    with pytest.raises(lib.LsmpsError) as e:
        ctx.ppe_solve("fp64", 100, 1e-10, precond="multigrid")
    assert e.value.code == lib.ERR_ARG
    n = 1000
    row = np.arange(0, 2 * n + 1, 2, dtype=np.int64)
    col = np.stack([np.arange(n), (np.arange(n) + 1) % n], 1).reshape(-1).astype(np.int32)
    ctx.ppe_load_csr(row, col)
    with pytest.raises(lib.LsmpsError) as e:
        ctx.ppe_solve("mixed", 100, 1e-10, precond="multigrid")
    assert e.value.code == lib.ERR_STATE
