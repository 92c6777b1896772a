"""Test configuration: the `gpu` marker, import paths, and build-on-demand fixtures.

`-m "not gpu"` runs everything that needs no GPU: the oracle against the reference and the
golden fixtures, host-side logic (config parsing, generators, writers), the C-ABI export
table, and the multi-process (gloo) replica logic. `-m gpu` runs the parity tests, which
call the sm_100a library through its C ABI and compare against the CPU oracles.
"""
import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("oracle", "ls-mps_b200"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100a GPU (run with -m gpu)")


@pytest.fixture(scope="session")
def built():
    """Builds the oracle libraries and the product library if they are missing."""
    import oracle as orc
    import lsmps_b200 as lib

    orc.build()
    if not os.path.exists(lib.LIB_PATH) or not os.path.exists(lib.CLI_PATH):
        lib.build()
    return True


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "reference_cases.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def cfg_dir(tmp_path_factory, golden):
    """The reference's .cfg inputs, written from the fixture (no reference tree needed)."""
    d = tmp_path_factory.mktemp("cfg")
    for name, rec in golden["cases"].items():
        (d / f"{name}.cfg").write_text(rec["cfg_text"])
    return d


@pytest.fixture(scope="session")
def have_ref():
    import oracle as orc

    return os.path.exists(orc.REF_SO)
