"""The oracle's restatement of the pressure projection with Neumann walls (CPU): on a lattice
block standing on three wall layers, Dirichlet walls (WLS rows, variant 2) leave the layer next
to the wall with more divergence than before the projection, while Neumann walls (variant 3
rows, wall neighbors taking the particle's own value in every WLS derivative, the mirrored
wall value of the reference's python/rain_plate_lsmps_cpu.py:90-100,179) remove it there as
well. The same statistics are asserted on the GPU by tests/test_gpu_projection.py."""
import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from _util import jittered_lattice
from oracle import Oracle

RE, L0 = 2.1, 1.0
WALL, FREE, SPLASH = 4, 1, 2


def _hops(row, col, seed, depth=3):
    """Neighbor-hop distance from the seed particles, exact up to depth (99 beyond)."""
    h = np.where(seed, 0, 99)
    nonempty = np.diff(row) > 0
    for _ in range(depth):
        best = np.full(len(h), 99)
        best[nonempty] = np.minimum.reduceat(h[col] + 1, row[:-1][nonempty])
        h = np.minimum(h, best)
    return h


def _project(xyz, cls, row, col, ustar, variant, mirror, dt=0.01, rho=1000.0):
    _, wst, z, ws = Oracle.wls(xyz, cls, row, col, RE, L0)
    G, _ = Oracle.wls_fields(xyz, cls, row, col, RE, L0, ustar, mirror_walls=mirror)
    div = G[:, 0, 0] + G[:, 1, 1] + G[:, 2, 2]
    prow, pcol, pval, _, _, up, _ = Oracle.ppe_assemble(variant, xyz, cls, row, col, RE, L0, len(cls), 0.0, z, ws, wst)
    A = sp.csr_matrix((pval, pcol, prow), shape=(len(up), len(up)))
    p = np.zeros(len(cls))
    p[up] = spla.spsolve(A.tocsc(), -rho / dt * div[up])
    Gp, _ = Oracle.wls_fields(xyz, cls, row, col, RE, L0, p, mirror_walls=mirror)
    u = ustar - dt / rho * Gp[:, 0, :3]
    u[cls == WALL] = ustar[cls == WALL]
    G2, _ = Oracle.wls_fields(xyz, cls, row, col, RE, L0, u, mirror_walls=mirror)
    unk = np.zeros(len(cls), bool)
    unk[up] = True
    return div, G2[:, 0, 0] + G2[:, 1, 1] + G2[:, 2, 2], unk


def test_neumann_walls_remove_the_divergence_next_to_the_wall(built):
    xyz = jittered_lattice(20, 0.1, seed=4)
    t = np.zeros(len(xyz), np.uint8)
    t[xyz[:, 2] < 3.0] = WALL
    row, col, _ = Oracle.neighbors(xyz, RE, 128)
    cls = Oracle.classify(xyz, t, row, col, L0)
    x, y, zz = xyz.T
    ustar = np.stack([0.2 * np.cos(0.2 * x) * np.cos(0.15 * y) + np.sin(0.1 * y),
                      -0.15 * np.sin(0.2 * x) * np.sin(0.15 * y) + np.sin(0.1 * zz), 0.04 * (zz - 3.0)], 1)
    hs = _hops(row, col, (cls == FREE) | (cls == SPLASH))
    hw = _hops(row, col, cls == WALL)
    rms = lambda d, m: float(np.sqrt(np.mean(d[m] ** 2)))
    out = {}
    for variant, mirror in ((2, False), (3, True)):
        before, after, unk = _project(xyz, cls, row, col, ustar, variant, mirror)
        band1 = unk & (hs >= 3) & (hw == 1)
        band2 = unk & (hs >= 3) & (hw == 2)
        assert band1.sum() > 100 and band2.sum() > 100
        out[variant] = (rms(before, band1), rms(after, band1), rms(before, band2), rms(after, band2))
    d1b, d1a, _, _ = out[2]
    n1b, n1a, n2b, n2a = out[3]
    assert d1a > 0.5 * d1b
    assert n1a <= 0.25 * n1b and n2a <= 0.05 * n2b


def test_predictor_reproduces_a_quadratic_laplacian(built):
    """The oracle's predictor (python/rain_plate_lsmps_cpu.py:184-196, in 3-D): deep in the fluid
    the WLS Laplacian of a quadratic velocity is exact (the second-order basis reproduces it), so
    u* - u = dt (nu lap u + g) to round-off; wall particles keep u; with Dirichlet walls the
    predictor differs next to the wall from the mirrored (Neumann) one."""
    xyz = jittered_lattice(16, jitter=0.1, seed=11)
    t = np.zeros(len(xyz), np.uint8)
    t[xyz[:, 2] < 3.0] = WALL
    row, col, _ = Oracle.neighbors(xyz, RE, 128)
    cls = Oracle.classify(xyz, t, row, col, L0)
    x, y, z = xyz.T
    u = np.stack([0.1 * x * x + 0.05 * y * z, 0.03 * y * y - 0.02 * x * z, 0.04 * z * z + 0.01 * x * y], 1)
    dt, nu, g = 0.01, 0.5, np.array([0.0, 0.0, -9.81])
    us = {m: Oracle.predict_velocity(xyz, cls, row, col, RE, L0, u, dt, nu, g, mirror_walls=m) for m in (False, True)}
    walls = cls == WALL
    lo, hi = xyz.min(0), xyz.max(0)
    deep = (~walls) & np.all(xyz > lo + np.array([3, 3, 6]), 1) & np.all(xyz < hi - 3, 1)
    assert deep.sum() > 50 and walls.sum() == 16 * 16 * 3
    for m in (False, True):
        assert np.array_equal(us[m][walls], u[walls])
        lap = ((us[m][deep] - u[deep]) / dt - g) / nu
        assert np.abs(lap - np.array([0.2, 0.06, 0.08])).max() < 1e-9
    near = (~walls) & (xyz[:, 2] < 4.5)
    assert np.abs(us[False][near] - us[True][near]).max() > 1e-4
    assert np.array_equal(us[False][deep], us[True][deep])
