"""The C-ABI library loads and exports every entry point the header declares (CPU only)."""
import ctypes as C
import os
import re

import lsmps_b200 as lib

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "lsmps_gpu.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(lsmps_[a-z_0-9]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("lsmps_ctx_create", "lsmps_build_neighbors", "lsmps_wls", "lsmps_ppe_assemble",
                 "lsmps_ppe_solve", "lsmps_download_pressure", "lsmps_mpnn_train"):
        assert must in names


def test_library_exports_every_declared_symbol(built):
    L = C.CDLL(lib.LIB_PATH)
    for name in declared_functions():
        assert hasattr(L, name), f"{name} declared in lsmps_gpu.h but not exported"
        assert name in lib.SIGNATURES, f"{name} has no ctypes signature in lsmps_b200.py"


def test_abi_version_and_struct_sizes(built):
    L = lib.load()
    assert L.lsmps_abi_version() == 1
    # layouts mirrored from the header (natural alignment on x86-64)
    assert C.sizeof(lib.NeighborStats) == 8 + 8 + 8 + 16 + 40 + 8 + 8
    assert C.sizeof(lib.PpeStats) == 5 * 8 + 8 + 6 * 8 + 8 + 8
    assert C.sizeof(lib.SolverOpts) == 4 + 4 + 8 + 4 + 4 + 8 + 4 + 4 + 4 + 4
    assert C.sizeof(lib.SeriesParams) == 4 * 4 + 11 * 8 + 8 * 4
    assert C.sizeof(lib.SeriesStats) == 4 * 4 + 10 * 8 + 4 * 4 + 9 * 8


def test_context_without_gpu_fails_cleanly(built):
    """On a machine without a GPU, context creation returns a status instead of crashing."""
    L = lib.load()
    h = C.c_void_p()
    rc = L.lsmps_ctx_create(0, C.byref(h))
    assert rc in (lib.OK, lib.ERR_CUDA)
    if rc == lib.OK:
        L.lsmps_ctx_destroy(h)
    assert L.lsmps_ctx_create(-1, C.byref(h)) != lib.OK
    assert L.lsmps_last_error(None) == b"null context"
