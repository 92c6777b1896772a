"""ORACLE — test infrastructure, not product code.

FP64 restatement of the library's cell-aggregation multigrid preconditioner
(``ls-mps_b200/csrc/multigrid.cu``), for checking the GPU V-cycle. It has no reference
counterpart: the reference's BiCGStab (``src/lsmps.cpp:67``) runs unpreconditioned. The
multigrid only changes how fast the solvers converge; the system they solve is still the
reference's.

The hierarchy is built from the unknowns' cells, floor(x / re) per axis, offset by the
minimum over all particles. That is the neighbor grid of ``src/lsmps.cpp:16-18,26``.
Level 1 has one aggregate per cell; level l + 1 groups the 2x2x2 blocks of level l
((c - cmin) >> l). Coarsening stops at the first level that ``is_coarsest`` accepts: at most
``COARSE_SMALL`` rows, or at most ``COARSE_MAX`` rows from level ``COARSE_DEEP`` on.
Each coarse operator is the Galerkin product P^T A P with piecewise-constant P. The V-cycle
(OMEGA, ALPHA, SWEEPS) is documented in ``multigrid.cu``. ``apply`` returns D M z, the
operator the solvers apply while iterating on y = D x. Its fine-level sweep uses the same
FP16 rounding of AP / a_ii as the library.

Only tests import this module.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

COARSE_MAX = 640
COARSE_SMALL = 256
COARSE_DEEP = 3


def is_coarsest(n, level):
    """The multigrid.cu rule: a level of at most COARSE_SMALL rows, or of at most COARSE_MAX
    rows at level COARSE_DEEP or deeper, is the coarsest."""
    return n <= COARSE_SMALL or (n <= COARSE_MAX and level >= COARSE_DEEP)
SWEEPS = 10
OMEGA = 1.0
ALPHA = 1.5


def _inv_diag(A):
    d = A.diagonal()
    out = np.zeros_like(d)
    ok = (d > 0) & np.isfinite(d)
    out[ok] = 1.0 / d[ok]
    return out


def _groups(keys):
    """Aggregate index of each row: distinct keys numbered in ascending key order."""
    _, inv = np.unique(keys, return_inverse=True)
    return inv.reshape(-1)


class Hierarchy:
    """Levels of one assembled system. A: CSR (U x U) in any unknown numbering; cells: U x 3
    integer cell coordinates of the unknowns' particles relative to the grid minimum."""

    def __init__(self, A, cells):
        self.A = sp.csr_matrix(A)
        c = np.asarray(cells, dtype=np.int64)
        self.P = []     # P[l]: rows of level l -> rows of level l + 1 (level 0 = unknowns)
        self.Al = []    # Al[l - 1]: operator of level l >= 1
        self.sizes = [self.A.shape[0]]
        key = (c[:, 2] << 42) | (c[:, 1] << 21) | c[:, 0]
        agg = _groups(key)
        coord = np.zeros((agg.max() + 1, 3), np.int64)
        coord[agg] = c
        Acur = self.A
        while True:
            n = Acur.shape[0]
            nc = int(agg.max()) + 1
            P = sp.csr_matrix((np.ones(n), (np.arange(n), agg)), shape=(n, nc))
            self.P.append(P)
            Acur = sp.csr_matrix(P.T @ Acur @ P)
            self.Al.append(Acur)
            self.sizes.append(nc)
            if is_coarsest(nc, len(self.Al)):
                break
            coord = coord >> 1
            key = (coord[:, 2] << 42) | (coord[:, 1] << 21) | coord[:, 0]
            agg = _groups(key)
            ncoord = np.zeros((agg.max() + 1, 3), np.int64)
            ncoord[agg] = coord
            coord = ncoord
        self.Dinv = [_inv_diag(M) for M in self.Al]
        self.d0 = self.A.diagonal()

    @property
    def levels(self):
        return len(self.Al)

    def _cycle(self, l, r):
        A, Di = self.Al[l - 1], self.Dinv[l - 1]
        if l == self.levels:
            e = OMEGA * Di * r
            for _ in range(SWEEPS - 1):
                e = e + OMEGA * Di * (r - A @ e)
            return e
        x = OMEGA * Di * r
        P = self.P[l]
        ec = self._cycle(l + 1, P.T @ (r - A @ x))
        x = x + ALPHA * (P @ ec)
        return x + OMEGA * Di * (r - A @ x)

    def apply(self, z):
        """D M z for one vector of U values. The fine smoothing sweep uses AP / a_ii rounded to
        FP16, as the library stores it: d (P e1 - omega fl16(D^-1 A P) e1)."""
        P0 = self.P[0]
        if not hasattr(self, "_aps"):
            aps = sp.csr_matrix(sp.diags(1.0 / self.d0) @ (self.A @ P0))
            aps.data = aps.data.astype(np.float16).astype(np.float64)
            self._aps = aps
        e1 = self._cycle(1, P0.T @ z)
        return OMEGA * z + ALPHA * self.d0 * (P0 @ e1 - OMEGA * (self._aps @ e1))


def cells_of(xyz_all, xyz_unknowns, re):
    """Cell coordinates of the unknowns relative to the minimum cell over all particles."""
    cmin = np.floor(np.asarray(xyz_all) / re).astype(np.int64).min(axis=0)
    return np.floor(np.asarray(xyz_unknowns) / re).astype(np.int64) - cmin
