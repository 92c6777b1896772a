"""Host-side drop-in logic without a GPU: generate_case and the new generators."""
import hashlib

import numpy as np
import pytest

import lsmps_b200 as lib
from oracle import Oracle

CASES = ["smoke", "bulk_uniform", "wall_film", "rain_injection", "narrow_gap"]


def sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("name", CASES)
def test_generate_case_bit_identical(built, golden, cfg_dir, name):
    """generate_case reproduces the reference's positions and input types (src/lsmps.cpp:68,72)."""
    xyz, t, u = lib.generate(str(cfg_dir / f"{name}.cfg"))
    assert sha(xyz, t) == golden["cases"][name]["positions_sha256"]
    if name == "rain_injection":
        splash = t == lib.SPLASH
        assert splash.sum() == len(t) - int(0.75 * len(t))
        assert np.all(u[splash] == [0, 0, -5])


def test_unknown_override_key_rejected(built, cfg_dir):
    with pytest.raises(lib.LsmpsError):
        lib.generate(str(cfg_dir / "smoke.cfg"), no_such_key=1)


def test_jitter_override(built, cfg_dir):
    a, _, _ = lib.generate(str(cfg_dir / "bulk_uniform.cfg"), particles=50653, l0=1.0, jitter=0.1)
    assert len(a) == 50653
    frac = a - np.floor(a)
    assert frac.min() >= 0.4 - 1e-12 and frac.max() <= 0.6 + 1e-12
    b, _, _ = lib.generate(str(cfg_dir / "bulk_uniform.cfg"), particles=50653, l0=1.0, jitter=0.1)
    assert np.array_equal(a, b)  # seeded


def test_rain_plate_distribution(built):
    """Rain on a 20-degree plate: 3 wall layers, a 4-layer film with 70 % of the fluid,
    30 % droplets of radius 3 l0 falling at -5 l0 / step; skewed neighbor counts."""
    n = 100_000
    xyz, t, u = lib.generate(None, case="rain_plate", particles=n, l0=1.0, seed=1)
    assert len(xyz) == n
    wall = t == lib.WALL
    fluid = ~wall
    drops = u[:, 2] < 0
    assert np.all(u[drops] == [0, 0, -5.0])
    film = fluid & ~drops
    assert film.sum() / fluid.sum() == pytest.approx(0.7, abs=0.02)
    assert wall.sum() / film.sum() == pytest.approx(3 / 4, abs=1e-9)
    row, col, _ = Oracle.neighbors(xyz, 2.1, 256)
    cnt = np.diff(row)
    p50 = np.percentile(cnt, 50)
    assert 25 <= p50 <= 40
    assert cnt.max() >= 55  # overlapping droplets make a tail above the lattice count


def test_mixed_case_sizes(built):
    n = 200_000
    xyz, t, u = lib.generate(None, case="mixed", particles=n, l0=1.0, seed=2)
    assert len(xyz) == n
    nb = int(np.ceil(np.cbrt(0.8 * n)))
    bulk, rain = xyz[: int(0.8 * n)], xyz[int(0.8 * n):]
    assert bulk[:, 0].max() < nb + 0.2
    assert rain[:, 0].min() > nb + 2.1  # no pair between the two parts


@pytest.mark.parametrize("case,n,seed,jitter", [("mixed", 60_000, 7, -1.0), ("mixed", 1_000_000, 10, -1.0),
                                                 ("rain_plate", 40_000, 3, -1.0), ("rain_plate", 25_000, 5, 0.05),
                                                 ("bulk", 30_000, 1, -1.0)])
def test_oracle_generators_match_library(built, case, n, seed, jitter):
    """The oracle's generator restatement (used by bench.py's reference arm, which must not load
    the library) yields the library's positions and types bit for bit."""
    kw = {"jitter": jitter} if jitter >= 0 else {}
    a = lib.generate(None, case="bulk_uniform" if case == "bulk" else case, particles=n, l0=1.0, seed=seed, **kw)
    b = Oracle.generate(case, n, 1.0, seed, jitter)
    assert sha(a[0], a[1]) == sha(*b)
