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
    assert H.sizes[0] == A.shape[0] and H.sizes[-1] <= mgo.COARSE_MAX
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
