"""CPU checks of the multigrid restatement (oracle/multigrid_oracle.py) on oracle-assembled
WLS-Laplacian systems: the hierarchy's coarse operators are 27-slot stencils, and the V-cycle
as BiCGStab's right preconditioner needs far fewer iterations than Jacobi."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import lsmps_b200 as lib
import multigrid_oracle as mgo
from oracle import Oracle

RE, L0 = 2.1, 1.0


@pytest.fixture(scope="module")
def system(built):
    xyz, t, _ = lib.generate(None, case="mixed", particles=30_000, l0=L0, seed=3)
    row, col, _ = Oracle.neighbors(xyz, RE, 128)
    cls = Oracle.classify(xyz, t, row, col, L0)
    _, wst, z, ws = Oracle.wls(xyz, cls, row, col, RE, L0)
    prow, pcol, pval, b, xe, up, _ = Oracle.ppe_assemble(2, xyz, cls, row, col, RE, L0, len(t), 0.0, z, ws, wst)
    A = sp.csr_matrix((pval, pcol, prow), shape=(len(b), len(b)))
    H = mgo.Hierarchy(A, mgo.cells_of(xyz, xyz[up], RE))
    return A, b, xe, H


def test_coarse_operators_are_27_slot_stencils(system):
    A, _, _, H = system
    assert H.sizes[0] == A.shape[0] and mgo.is_coarsest(H.sizes[-1], H.levels)
    assert all(a > b for a, b in zip(H.sizes, H.sizes[1:]))
    for M in H.Al:
        assert np.diff(M.indptr).max() <= 27
        # Galerkin products of an M-matrix with nonnegative row sums keep both properties
        off = M - sp.diags(M.diagonal())
        assert off.data.max(initial=0.0) <= 1e-12 * abs(M.diagonal()).max()
        assert (M @ np.ones(M.shape[0])).min() >= -1e-9 * abs(M.diagonal()).max()


def test_vcycle_is_linear(system):
    A, b, _, H = system
    rng = np.random.default_rng(0)
    u, v = rng.standard_normal((2, A.shape[0]))
    lhs = H.apply(2.0 * u - 3.0 * v)
    rhs = 2.0 * H.apply(u) - 3.0 * H.apply(v)
    assert np.linalg.norm(lhs - rhs) <= 1e-12 * np.linalg.norm(rhs)


def _iterations(A, b, M):
    it = [0]
    x, info = spla.bicgstab(A, b, rtol=3e-11, atol=0.0, maxiter=5000, M=M,
                            callback=lambda _: it.__setitem__(0, it[0] + 1))
    return x, info, it[0]


def test_vcycle_preconditions(system):
    A, b, xe, H = system
    d = A.diagonal()
    n = A.shape[0]
    mg = spla.LinearOperator((n, n), matvec=lambda z: H.apply(z) / d)
    x, info, it_mg = _iterations(A, b, mg)
    assert info == 0 and np.linalg.norm(x - xe) <= 1e-8 * np.linalg.norm(xe)
    _, info_j, it_j = _iterations(A, b, sp.diags(1.0 / d))
    assert info_j == 0
    assert it_mg * 4 <= it_j, (it_mg, it_j)


def test_restatement_matches_dense_two_level_cycle(built):
    """The restatement on a system small enough for one coarse level, against the V-cycle
    written out with dense matrices: P from the cells, A1 = P^T A P, the coarsest level's
    Jacobi sweeps, alpha P e1, one fine Jacobi sweep, times D (FP16 A P / a_ii included)."""
    from _util import jittered_lattice

    xyz = jittered_lattice(10, 0.1, seed=3)
    t = np.zeros(len(xyz), np.uint8)
    row, col, _ = Oracle.neighbors(xyz, RE, 128)
    cls = Oracle.classify(xyz, t, row, col, L0)
    _, wst, z, ws = Oracle.wls(xyz, cls, row, col, RE, L0)
    prow, pcol, pval, b, xe, up, _ = Oracle.ppe_assemble(2, xyz, cls, row, col, RE, L0, len(t), 0.0, z, ws, wst)
    A = sp.csr_matrix((pval, pcol, prow), shape=(len(b), len(b))).toarray()
    cells = mgo.cells_of(xyz, xyz[up], RE)
    H = mgo.Hierarchy(sp.csr_matrix(A), cells)
    assert H.levels == 1 and len(b) > 100
    _, agg = np.unique(cells[:, 0] + 1000 * cells[:, 1] + 10 ** 6 * cells[:, 2], return_inverse=True)
    P = np.zeros((len(b), agg.max() + 1))
    P[np.arange(len(b)), agg] = 1.0
    A1 = P.T @ A @ P
    d, d1 = np.diag(A), np.diag(A1)
    aps = (A @ P) / d[:, None]
    aps = np.where(aps != 0, aps.astype(np.float16).astype(np.float64), 0.0)
    zv = np.random.default_rng(5).standard_normal(len(b))
    r1 = P.T @ zv
    e = mgo.OMEGA * r1 / d1
    for _ in range(mgo.SWEEPS - 1):
        e = e + mgo.OMEGA * (r1 - A1 @ e) / d1
    want = mgo.OMEGA * zv + mgo.ALPHA * d * (P @ e - mgo.OMEGA * (aps @ e))
    got = H.apply(zv)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
