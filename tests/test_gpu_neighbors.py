"""GPU neighbor build + classification: bit-exact with the reference and the oracle."""
import numpy as np
import pytest

import lsmps_b200 as lib
from _util import cfg_params, sha
from oracle import Oracle

pytestmark = pytest.mark.gpu
CASES = ["smoke", "bulk_uniform", "wall_film", "rain_injection", "narrow_gap"]


@pytest.fixture(scope="module")
def ctx(built):
    c = lib.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", CASES)
def test_reference_cases_bit_exact(ctx, golden, cfg_dir, name):
    g = golden["cases"][name]
    p = cfg_params(g["cfg_text"])
    xyz, t, _ = lib.generate(str(cfg_dir / f"{name}.cfg"))
    ctx.upload(xyz, t)
    st = ctx.build_neighbors(p["re"], p["max_neighbors"], p["l0"])
    assert st.pairs == g["neighbors"]["pairs"]
    assert st.truncated == g["neighbors"]["truncated"]
    assert float(st.mean).hex() == g["neighbors"]["mean"]["hex"]
    assert (st.p50, st.p90, st.p99) == (g["neighbors"]["p50"], g["neighbors"]["p90"], g["neighbors"]["p99"])
    assert list(st.type_count) == g["types"]["counts"]
    row, col = ctx.neighbors(st.pairs)
    assert sha(row, col) == g["neighbors"]["csr_sha256"]
    assert sha(ctx.types()) == g["types"]["sha256"]


def check_against_oracle(ctx, xyz, t, re, maxn, l0):
    ctx.upload(xyz, t)
    st = ctx.build_neighbors(re, maxn, l0)
    row_o, col_o, tr_o = Oracle.neighbors(xyz, re, maxn)
    row, col = ctx.neighbors(st.pairs)
    assert np.array_equal(row, row_o)
    assert np.array_equal(col, col_o)
    assert st.truncated == tr_o
    types_o = Oracle.classify(xyz, t, row_o, col_o, l0)
    assert np.array_equal(ctx.types(), types_o)
    return st


@pytest.mark.parametrize("case,n", [("rain_plate", 100_000), ("mixed", 200_000)])
def test_new_generators_bit_exact(ctx, case, n):
    xyz, t, _ = lib.generate(None, case=case, particles=n, l0=1.0, seed=3)
    check_against_oracle(ctx, xyz, t, 2.1, 128, 1.0)


def test_truncation(ctx):
    xyz, t, _ = lib.generate(None, case="bulk_uniform", particles=8000, l0=1.0, jitter=0.1, seed=1)
    st = check_against_oracle(ctx, xyz, t, 2.1, 12, 1.0)
    assert st.truncated > 0


def test_duplicates_and_crowded_cells(ctx):
    """Coincident particles (r = 0, weight 0) and cells above the in-place sort size."""
    xyz = np.concatenate([np.tile([[5.05, 5.05, 5.05]], (150, 1)), np.tile([[1.0, 1.0, 1.0]], (40, 1)),
                          lib.generate(None, case="bulk_uniform", particles=1000, l0=1.0, seed=2)[0]])
    t = np.zeros(len(xyz), np.uint8)
    st = check_against_oracle(ctx, xyz, t, 2.1, 400, 1.0)
    assert st.max_cell_occupancy >= 150


def test_negative_and_offset_coordinates(ctx):
    xyz, t, _ = lib.generate(None, case="bulk_uniform", particles=5000, l0=0.01, jitter=0.1, seed=4)
    check_against_oracle(ctx, xyz - 0.173, t, 0.021, 96, 0.01)
    check_against_oracle(ctx, xyz + 1.0e4, t, 0.021, 96, 0.01)


def test_empty_and_single(ctx):
    ctx.upload(np.zeros((0, 3)), np.zeros(0, np.uint8))
    st = ctx.build_neighbors(0.021, 96, 0.01)
    assert st.pairs == 0
    ctx.upload(np.array([[0.5, 0.5, 0.5]]), np.array([4], np.uint8))
    st = ctx.build_neighbors(0.021, 96, 0.01)
    assert st.pairs == 0 and list(st.type_count) == [0, 0, 0, 0, 1]


def test_nonfinite_position_is_an_error(ctx):
    xyz = np.array([[0.1, 0.2, 0.3], [np.nan, 0.0, 0.0]])
    ctx.upload(xyz, np.zeros(2, np.uint8))
    with pytest.raises(lib.LsmpsError) as e:
        ctx.build_neighbors(0.021, 96, 0.01)
    assert e.value.code == lib.ERR_NONFINITE


def test_standalone_classify_matches_fused(ctx, cfg_dir):
    xyz, t, _ = lib.generate(str(cfg_dir / "rain_injection.cfg"))
    ctx.upload(xyz, t)
    st = ctx.build_neighbors(0.021, 96, 0.01, classify=True)
    fused = ctx.types()
    st2 = ctx.classify(0.01)
    assert np.array_equal(ctx.types(), fused)
    assert list(st2.type_count) == list(st.type_count)


def test_crowded_segment_global_path(ctx):
    """A segment whose 9 cell rows stage more than 1,536 candidates takes the warp-per-query
    global scan: 2,000 coincident particles plus a lattice, lists longer than 1,536."""
    xyz = np.concatenate([np.tile([[3.3, 3.3, 3.3]], (2000, 1)),
                          lib.generate(None, case="bulk_uniform", particles=1500, l0=1.0, seed=6)[0]])
    t = np.zeros(len(xyz), np.uint8)
    st = check_against_oracle(ctx, xyz, t, 2.1, 2500, 1.0)
    assert st.max_count > 1536
    st = check_against_oracle(ctx, xyz, t, 2.1, 700, 1.0)  # and truncated there
    assert st.truncated > 0


@pytest.mark.parametrize("maxn", [128, 20])
def test_single_pass_equals_two_pass(ctx, maxn):
    """The single-pass build (slot rows, then compaction) and the count + fill passes give the
    same lists, counts, truncation and classes."""
    xyz, t, _ = lib.generate(None, case="mixed", particles=300_000, l0=1.0, seed=8)
    ctx.upload(xyz, t)
    a = ctx.build_neighbors(2.1, maxn, 1.0)
    ra, ca = ctx.neighbors(a.pairs)
    ta = ctx.types()
    b = ctx.build_neighbors(2.1, maxn, 1.0, two_pass=True)
    rb, cb = ctx.neighbors(b.pairs)
    assert (a.pairs, a.truncated, list(a.type_count)) == (b.pairs, b.truncated, list(b.type_count))
    assert np.array_equal(ra, rb) and np.array_equal(ca, cb)
    assert np.array_equal(ta, ctx.types())


def test_prefetched_particles_equal_upload(ctx):
    """lsmps_prefetch_particles / lsmps_use_prefetched_particles: a prefetched set leaves the
    current one untouched until it is used, then gives the same lists and classes as a plain
    upload; the staging buffers swap back and forth across repeated prefetches."""
    sets = [lib.generate(None, case="mixed", particles=120_000, l0=1.0, seed=s)[:2] for s in (1, 2, 3)]
    want = []
    for xyz, t in sets:
        ctx.upload(xyz, t)
        st = ctx.build_neighbors(2.1, 128, 1.0)
        want.append((ctx.neighbors(st.pairs), ctx.types()))
    ctx.upload(*sets[0])
    ctx.prefetch(*sets[1])
    st = ctx.build_neighbors(2.1, 128, 1.0)  # still the uploaded set
    assert np.array_equal(ctx.neighbors(st.pairs)[1], want[0][0][1])
    for k in (1, 2, 0, 1):
        ctx.use_prefetched()
        ctx.prefetch(*sets[(k + 1) % 3])  # overlaps the build of set k
        st = ctx.build_neighbors(2.1, 128, 1.0)
        (row, col), cls = ctx.neighbors(st.pairs), ctx.types()
        assert np.array_equal(row, want[k][0][0]) and np.array_equal(col, want[k][0][1])
        assert np.array_equal(cls, want[k][1])
    ctx.use_prefetched()
    with pytest.raises(lib.LsmpsError) as e:
        ctx.use_prefetched()  # nothing prefetched
    assert e.value.code == lib.ERR_STATE
