"""GPU WLS: the reference's sampled test bit for bit; the batched all-particle WLS against
the oracle (FP64 tolerance 1e-9 absolute on solutions of O(1)); FP32 + refinement
against FP64."""
import numpy as np
import pytest

import lsmps_b200 as lib
from _util import cfg_params, jittered_lattice
from oracle import Oracle

pytestmark = pytest.mark.gpu
CASES = ["smoke", "bulk_uniform", "wall_film", "rain_injection", "narrow_gap"]


@pytest.fixture(scope="module")
def ctx(built):
    c = lib.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", CASES)
def test_sampled_wls_bit_exact(ctx, golden, cfg_dir, name):
    g = golden["cases"][name]
    p = cfg_params(g["cfg_text"])
    xyz, t, _ = lib.generate(str(cfg_dir / f"{name}.cfg"))
    ctx.upload(xyz, t)
    ctx.build_neighbors(p["re"], p["max_neighbors"], p["l0"])
    st = ctx.wls(p["re"], p["l0"], mode=0, wls_samples=p["wls_samples"])
    for k in ("sampled", "ok", "regularized", "failed", "virtual_points"):
        assert getattr(st, k) == g["wls"][k], k
    for k in ("max_gradient_error", "rms_gradient_error", "max_laplacian_error", "rms_laplacian_error"):
        assert float(getattr(st, k)).hex() == g["wls"][k]["hex"], k


def _setup(ctx, xyz, t, re, l0, maxn=128):
    ctx.upload(xyz, t)
    ctx.build_neighbors(re, maxn, l0)
    types = ctx.types()
    row, col, _ = Oracle.neighbors(xyz, re, maxn)
    return types, row, col


@pytest.mark.parametrize("case", ["lattice", "rain_plate"])
def test_all_particle_wls_matches_oracle(ctx, case):
    rng = np.random.default_rng(11)
    if case == "lattice":
        xyz = jittered_lattice(20, 0.1, seed=1)
        t = np.zeros(len(xyz), np.uint8)
    else:
        xyz, t, _ = lib.generate(None, case="rain_plate", particles=60_000, l0=1.0, seed=5)
    coef = rng.normal(size=(3, 10))
    types, row, col = _setup(ctx, xyz, t, 2.1, 1.0)
    st = ctx.wls(2.1, 1.0, mode=1, coef=coef, store=True)
    x, status, z, ws = ctx.wls_result(nrhs=3, with_x=True)
    xo, so, zo, wo = Oracle.wls(xyz, types, row, col, 2.1, 1.0, coef=coef)
    assert np.array_equal(status, so)
    ok = (so == 0) | (so == 1)
    assert np.allclose(ws, wo, rtol=1e-13, atol=0)
    # per particle: |x - x_oracle| <= 1e-8 |x_oracle| + 1e-10 (FP64, different summation order)
    err = np.linalg.norm((x - xo)[ok], axis=-1)
    assert np.all(err <= 1e-8 * np.linalg.norm(xo[ok], axis=-1) + 1e-10)
    zerr = np.linalg.norm((z - zo)[ok], axis=-1)
    assert np.all(zerr <= 1e-8 * np.linalg.norm(zo[ok], axis=-1) + 1e-10)
    assert st.sampled == ok.sum()
    # quadratics are reproduced to rounding; droplet-edge stencils are ill-conditioned
    assert st.rms_gradient_error < 1e-8 and st.rms_laplacian_error < 1e-6


def test_all_particle_wls_without_statistics(ctx):
    """A mode-1 WLS call without statistics (out = NULL) returns without waiting, leaves the
    same results, and its phase time is read by lsmps_get_timings."""
    xyz, t, _ = lib.generate(None, case="rain_plate", particles=40_000, l0=1.0, seed=6)
    _setup(ctx, xyz, t, 2.1, 1.0)
    ctx.wls(2.1, 1.0, mode=1, store=True)
    ref = ctx.wls_result(nrhs=1, with_x=True)
    assert ctx.wls(2.1, 1.0, mode=1, store=True, stats=False) is None
    assert ctx.timings()[3] > 0.0
    got = ctx.wls_result(nrhs=1, with_x=True)
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
    st = ctx.ppe_assemble("wls", 10**9, 2.1, 1.0, diag_shift=0.0)  # the WLS state is set
    assert st.unknowns > 0


def test_mixed_precision_wls_refines_to_fp64(ctx):
    xyz = jittered_lattice(24, 0.1, seed=2)
    t = np.zeros(len(xyz), np.uint8)
    coef = np.random.default_rng(3).normal(size=(3, 10))
    _setup(ctx, xyz, t, 2.1, 1.0)
    st64 = ctx.wls(2.1, 1.0, mode=1, coef=coef, store=True, precision=0)
    x64, s64, z64, _ = ctx.wls_result(nrhs=3, with_x=True)
    st32 = ctx.wls(2.1, 1.0, mode=1, coef=coef, store=True, precision=1)
    x32, s32, z32, _ = ctx.wls_result(nrhs=3, with_x=True)
    ok = (s64 == 0) & (s32 == 0)
    assert ok.mean() > 0.95
    # FP64-residual refinement sweeps bring the FP32 factor to FP64 accuracy (per particle,
    # relative to the solution's norm)
    err = np.linalg.norm((x32 - x64)[ok], axis=-1)
    assert np.all(err <= 1e-8 * np.linalg.norm(x64[ok], axis=-1) + 1e-10)
    zerr = np.linalg.norm((z32 - z64)[ok], axis=-1)
    assert np.all(zerr <= 1e-8 * np.linalg.norm(z64[ok], axis=-1) + 1e-10)
    assert st32.rms_gradient_error < 1e-8 and st32.rms_laplacian_error < 1e-6
