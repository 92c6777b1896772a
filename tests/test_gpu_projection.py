"""WLS of caller fields and the pressure projection step (the reference's 2-D
python/rain_plate_lsmps_cpu.py:202-260, in 3-D).

* lsmps_wls_fields equals the oracle's restatement (orc_wls_fields) per particle to 1e-8
  relative, with the same statuses.
* The projection of u* = grad(phi) + w (div w = 0) on a jittered lattice block with a free
  surface: the pressure equals the CPU solution of the downloaded system (spsolve) to 1e-6,
  the corrected velocity equals u* - dt/rho grad p with the oracle's gradients to 1e-6, and
  the divergence over the core (unknowns three or more neighbor hops inside the free
  surface) drops at least 20x.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import lsmps_b200 as lib
from _util import jittered_lattice
from oracle import Oracle

pytestmark = pytest.mark.gpu
RE, L0 = 2.1, 1.0


@pytest.fixture(scope="module")
def block(built):
    torch = pytest.importorskip("torch")
    xyz = jittered_lattice(36, jitter=0.1, seed=4)
    t = np.zeros(len(xyz), np.uint8)
    ctx = lib.Context(0)
    ctx.upload(xyz, t)
    ctx.build_neighbors(RE, 128, L0)
    ctx.wls(RE, L0, mode=1)
    ps = ctx.ppe_assemble("wls", 10**12, RE, L0, diag_shift=0.0)
    row, col, _ = Oracle.neighbors(xyz, RE, 128)
    cls = Oracle.classify(xyz, t, row, col, L0)
    assert np.array_equal(cls, ctx.types())
    yield torch, ctx, xyz, cls, row, col, ps
    ctx.close()


def _fields(xyz):
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    # grad of phi = sin(0.2x) cos(0.15y) + 0.02 z^2, plus w = (sin(0.1y), sin(0.1z), sin(0.1x)) (div w = 0)
    gx = 0.2 * np.cos(0.2 * x) * np.cos(0.15 * y) + np.sin(0.1 * y)
    gy = -0.15 * np.sin(0.2 * x) * np.sin(0.15 * y) + np.sin(0.1 * z)
    gz = 0.04 * z + np.sin(0.1 * x)
    return np.stack([gx, gy, gz], 1)


def test_wls_fields_match_oracle(block):
    torch, ctx, xyz, cls, row, col, _ = block
    f = _fields(xyz)
    g = ctx.wls_fields(f).cpu().numpy()
    x, st = Oracle.wls_fields(xyz, cls, row, col, RE, L0, f)
    ok = (st == 0) | (st == 1)
    assert ok.sum() > 0.9 * len(st)
    assert np.all(g[~ok] == 0)
    scale = np.abs(x[ok]).max(axis=(1, 2))[:, None, None] + 1e-30
    assert np.abs(g[ok] - x[ok]).max() <= 1e-8 * scale.max()
    assert np.all(np.abs(g[ok] - x[ok]) <= 1e-8 * scale)


def test_projection_step(block):
    torch, ctx, xyz, cls, row, col, ps = block
    dt, rho = 0.01, 1000.0
    ustar = _fields(xyz)
    u, p, st = ctx.projection_step(ustar, dt, rho, solver="fp64", tol=1e-12)
    u, p = u.cpu().numpy(), p.cpu().numpy()
    assert st.converged and st.unknowns == ps.unknowns
    # the pressure against a direct solve of the same system (downloaded, b = -rho/dt div u*)
    prow, pcol, val, b, _, part = ctx.ppe(ps.unknowns, ps.nnz)
    A = sp.csr_matrix((val, pcol, prow), shape=(ps.unknowns, ps.unknowns))
    pref = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(p[part] - pref) <= 1e-6 * np.linalg.norm(pref)
    others = np.ones(len(p), bool)
    others[part] = False
    assert np.all(p[others] == 0)
    # the divergence the right-hand side came from, with the oracle's gradients
    x, st_w = Oracle.wls_fields(xyz, cls, row, col, RE, L0, ustar)
    div = x[:, 0, 0] + x[:, 1, 1] + x[:, 2, 2]
    assert np.allclose(b, -rho / dt * div[part], rtol=1e-8, atol=1e-8 * np.abs(b).max())
    # u = u* - dt/rho grad p (walls keep u*: there are none here)
    xp, _ = Oracle.wls_fields(xyz, cls, row, col, RE, L0, p)
    uref = ustar - dt / rho * xp[:, 0, :3]
    assert np.linalg.norm(u - uref) <= 1e-6 * np.linalg.norm(uref)
    # the projection removes the divergence away from the boundary (measured on the CPU with
    # the same operators: 80x at three or more neighbor hops from free-surface and near-wall
    # particles; the first two layers keep a residual from the one-sided stencils)
    assert st.measured == ps.unknowns and 0 < st.core < st.measured
    assert st.div_core_after_rms <= 0.05 * st.div_core_before_rms, (st.div_core_before_rms, st.div_core_after_rms)
    assert np.isfinite(st.div_after_rms)


def _wall_fields(xyz):
    """u* = grad(phi) + w with phi = sin(0.2x) cos(0.15y) + 0.02 (z - 3)^2 and w = (sin(0.1y),
    sin(0.1z), 0): div w = 0, and the normal component vanishes on the wall plane z = 3."""
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    gx = 0.2 * np.cos(0.2 * x) * np.cos(0.15 * y) + np.sin(0.1 * y)
    gy = -0.15 * np.sin(0.2 * x) * np.sin(0.15 * y) + np.sin(0.1 * z)
    gz = 0.04 * (z - 3.0)
    return np.stack([gx, gy, gz], 1)


def test_projection_neumann_walls(built):
    """A lattice block on three wall layers (z < 3) with a free surface elsewhere. With Dirichlet
    walls (p = 0 at the wall particles) the band next to the wall keeps its divergence; with
    Neumann walls (LSMPS_PPE_WALL_NEUMANN: wall neighbors take the particle's own value, as the
    reference's mirrored virtual points) the divergence drops next to the wall too, and two hops
    in as much as in the core. The Neumann system and the corrected velocity equal the oracle's
    (variant 3, mirrored wall values)."""
    pytest.importorskip("torch")
    xyz = jittered_lattice(26, jitter=0.1, seed=4)
    t = np.zeros(len(xyz), np.uint8)
    t[xyz[:, 2] < 3.0] = lib.WALL
    ustar = _wall_fields(xyz)
    dt, rho = 0.01, 1000.0
    res = {}
    with lib.Context(0) as ctx:
        ctx.upload(xyz, t)
        ctx.build_neighbors(RE, 128, L0)
        ctx.wls(RE, L0, mode=1)
        cls = ctx.types()
        for neumann in (False, True):
            ps = ctx.ppe_assemble("wls", 10**12, RE, L0, diag_shift=0.0, wall_neumann=neumann)
            u, p, st = ctx.projection_step(ustar, dt, rho, solver="fp64", tol=1e-12)
            system = ctx.ppe(ps.unknowns, ps.nnz)  # b = -rho / dt div u* after the step
            res[neumann] = (ps, system, u.cpu().numpy(), p.cpu().numpy(), st)
    d, nm = res[False][4], res[True][4]
    assert nm.converged and nm.wall_band1 > 300 and nm.wall_band2 > 300 and nm.core > 300
    assert d.div_wall1_after_rms > 0.5 * d.div_wall1_before_rms, (d.div_wall1_before_rms, d.div_wall1_after_rms)
    assert nm.div_wall1_after_rms <= 0.25 * nm.div_wall1_before_rms, (nm.div_wall1_before_rms, nm.div_wall1_after_rms)
    assert nm.div_wall2_after_rms <= 0.05 * nm.div_wall2_before_rms, (nm.div_wall2_before_rms, nm.div_wall2_after_rms)
    assert nm.div_core_after_rms <= 0.05 * nm.div_core_before_rms
    # the Neumann rows against the oracle's variant 3 (built from the oracle's own WLS vectors)
    ps, (prow, pcol, val, b, _, part), u, p, _ = res[True]
    row, col, _ = Oracle.neighbors(xyz, RE, 128)
    _, wst, z, ws = Oracle.wls(xyz, cls, row, col, RE, L0)
    orow, ocol, oval, _, _, oup, ost = Oracle.ppe_assemble(3, xyz, cls, row, col, RE, L0, len(t), 0.0, z, ws, wst)
    assert np.array_equal(part, oup) and abs(ps.nnz - ost["nnz"]) <= max(2, ps.nnz // 100000)
    A = sp.csr_matrix((val.copy(), pcol.copy(), prow.copy()), shape=(ps.unknowns, ps.unknowns))
    O = sp.csr_matrix((oval, ocol, orow), shape=(ps.unknowns, ps.unknowns))
    assert abs(A - O).max() <= 1e-8 * abs(O).max()
    pref = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(p[part] - pref) <= 1e-6 * np.linalg.norm(pref)
    xp, _ = Oracle.wls_fields(xyz, cls, row, col, RE, L0, p, mirror_walls=True)
    uref = ustar - dt / rho * xp[:, 0, :3]
    walls = cls == lib.WALL
    uref[walls] = ustar[walls]
    assert np.linalg.norm(u - uref) <= 1e-6 * np.linalg.norm(uref)


def _quadratic_velocity(xyz):
    """A quadratic velocity field: lap u = (0.2, 0.06, 0.08) everywhere."""
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    return np.stack([0.1 * x * x + 0.05 * y * z, 0.03 * y * y - 0.02 * x * z, 0.04 * z * z + 0.01 * x * y], 1)


@pytest.mark.parametrize("neumann", [False, True])
def test_predict_velocity(built, neumann):
    """lsmps_predict_velocity (the reference's provisional_velocity, in 3-D) on a lattice block on
    three wall layers: equals the oracle's u + dt (nu lap u + g) to 1e-12 of |u*|, walls keep u,
    and deep inside the fluid the WLS Laplacian of the quadratic field is the exact one."""
    pytest.importorskip("torch")
    xyz = jittered_lattice(20, jitter=0.1, seed=11)
    t = np.zeros(len(xyz), np.uint8)
    t[xyz[:, 2] < 3.0] = lib.WALL
    u = _quadratic_velocity(xyz)
    dt, nu, g = 0.01, 0.5, (0.0, 0.0, -9.81)
    with lib.Context(0) as ctx:
        ctx.upload(xyz, t)
        ctx.build_neighbors(RE, 128, L0)
        cls = ctx.types()
        us = ctx.predict_velocity(u, dt, nu, g, wall_neumann=neumann).cpu().numpy()
    row, col, _ = Oracle.neighbors(xyz, RE, 128)
    ref = Oracle.predict_velocity(xyz, cls, row, col, RE, L0, u, dt, nu, g, mirror_walls=neumann)
    assert np.abs(us - ref).max() <= 1e-12 * np.abs(ref).max()
    walls = cls == lib.WALL
    assert walls.sum() > 1000 and np.array_equal(us[walls], u[walls])
    # interior particles whose support lies inside the fluid: the quadratic is reproduced
    lo, hi = xyz.min(0), xyz.max(0)
    deep = (~walls) & np.all(xyz > lo + np.array([3, 3, 6]), 1) & np.all(xyz < hi - 3, 1)
    assert deep.sum() > 100
    lap = (us[deep] - u[deep]) / dt - np.array(g)
    assert np.abs(lap / nu - np.array([0.2, 0.06, 0.08])).max() < 1e-5
