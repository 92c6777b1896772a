"""lsmps_ppe_residual_static: the residual check whose reduction scratch is a static device
array (no allocation), against the existing entry points on the same assembled system.

* |b| (zero vector) equals lsmps_ppe_solve's initial residual and the assembled b of
  lsmps_download_ppe; |b - A q| for a random q equals the FP64 CSR product of the
  downloaded system; |b - A p| of the solver's own solution equals its final residual
  within the rounding bound of that (cancelling) difference.
* Two calls in a row give the same bits (the ticket word is cleared between calls) and the
  device's free memory does not change across them.
* nvec outside 1..8 and ld < U are rejected with LSMPS_ERR_ARG.

This file is collected last so that it also runs after every other test in one session.
"""
import ctypes as C

import numpy as np
import pytest

import lsmps_b200 as lib

pytestmark = pytest.mark.gpu
EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def system(built):
    torch = pytest.importorskip("torch")
    ctx = lib.Context(0)
    xyz, t, _ = lib.generate(None, case="rain_plate", particles=60_000, l0=1.0, seed=11)
    ctx.upload(xyz, t)
    ctx.build_neighbors(2.1, 128, 1.0)
    ctx.wls(2.1, 1.0, mode=1)
    ps = ctx.ppe_assemble("wls", 10**12, 2.1, 1.0, diag_shift=0.0)
    U = ps.unknowns
    st = ctx.ppe_solve("fp64", 20000, 1e-10)
    assert st.converged
    p = ctx.pressure(U)
    row, col, val, b, xe, _ = ctx.ppe(U, ps.nnz)
    yield torch, ctx, U, st, p, (row, col, val, b)
    ctx.close()


def _call(torch, ctx, vecs, ld=None, nvec=None):
    P = torch.from_numpy(np.ascontiguousarray(vecs)).cuda()
    nv = len(vecs) if nvec is None else nvec
    out = torch.full((max(nv, 1) + 1,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = ctx.L.lsmps_ppe_residual_static(ctx.h, C.c_void_p(P.data_ptr()), vecs.shape[1] if ld is None else ld,
                                         nv, C.c_void_p(out.data_ptr()))
    if rc == lib.OK:
        ctx.sync()
    return rc, out.cpu().numpy()


def _csr_times(row, col, val, x):
    y = np.zeros(len(row) - 1)
    rows = np.repeat(np.arange(len(row) - 1), np.diff(row))
    np.add.at(y, rows, val * x[col])
    return y


def test_matches_existing_entry_points(system):
    torch, ctx, U, st, p, (row, col, val, b) = system
    rng = np.random.default_rng(5)
    q = rng.standard_normal(U)
    vecs = np.stack([np.zeros(U), q, p])
    rc, out = _call(torch, ctx, vecs)
    assert rc == lib.OK, ctx.L.lsmps_last_error(ctx.h)
    bnorm = out[3]
    # zero vector: r = b exactly, accumulated in the same order as |b|
    assert out[0] == bnorm
    assert abs(bnorm - np.linalg.norm(b)) <= 1e-13 * np.linalg.norm(b)
    assert abs(bnorm - st.initial_residual) <= 1e-13 * st.initial_residual
    # random vector against the downloaded CSR in FP64
    ref_q = np.linalg.norm(b - _csr_times(row, col, val, q))
    assert abs(out[1] - ref_q) <= 1e-12 * ref_q
    # the solver's own solution: |b - A p| cancels, so compare within its rounding bound
    bound = 64 * EPS * np.linalg.norm(_csr_times(row, col, np.abs(val), np.abs(p)) + np.abs(b))
    assert abs(out[2] - st.final_residual) <= bound


def test_two_calls_in_a_row_identical_without_allocation(system):
    torch, ctx, U, st, p, _ = system
    q = np.random.default_rng(6).standard_normal(U)
    vecs = np.stack([p, q])
    rc1, out1 = _call(torch, ctx, vecs)
    assert rc1 == lib.OK, ctx.L.lsmps_last_error(ctx.h)
    P = torch.from_numpy(vecs).cuda()
    outs = [torch.full((3,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for o in outs:
        assert ctx.L.lsmps_ppe_residual_static(ctx.h, C.c_void_p(P.data_ptr()), U, 2,
                                               C.c_void_p(o.data_ptr())) == lib.OK
    ctx.sync()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    a, b2 = (o.cpu().numpy() for o in outs)
    assert a.tobytes() == b2.tobytes() == out1.tobytes()
    assert np.all(np.isfinite(a))


def test_rejects_sizes_beyond_the_static_scratch(system):
    torch, ctx, U, st, p, _ = system
    vecs = np.zeros((9, U))
    rc, _ = _call(torch, ctx, vecs)
    assert rc == lib.ERR_ARG
    assert b"at most 8 vectors" in ctx.L.lsmps_last_error(ctx.h)
    rc, _ = _call(torch, ctx, vecs[:1], nvec=0)
    assert rc == lib.ERR_ARG
    rc, _ = _call(torch, ctx, np.zeros((2, U)), ld=U - 1)
    assert rc == lib.ERR_ARG
    # a valid call still works after the rejected ones
    rc, out = _call(torch, ctx, np.stack([p]))
    assert rc == lib.OK and np.all(np.isfinite(out))
