"""ORACLE — test infrastructure, not product code.

ctypes bindings for the two CPU oracles built by ``oracle/Makefile``:

* ``Ref``: the reference implementation (lilux618/LS-MPS ``src/lsmps.cpp``) compiled
  from its own sources into ``oracle/_ref/libref.so`` through ``ref_shim.cpp``;
* ``Oracle``: this repository's CPU restatement ``oracle/_build/liboracle.so``.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm
import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libref.so")
REF_BIN = os.path.join(HERE, "_ref", "lsmps-bench")
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")

# Reference quadratic test field of wls_test (src/lsmps.cpp:28) in the coefficient order
# c0 + c1 x + c2 y + c3 z + c4 x^2 + c5 y^2 + c6 z^2 + c7 xy + c8 xz + c9 yz.
REF_QUADRATIC = np.array([1, 2, -3, 0.5, 0.7, -0.2, 0.4, 0.3, -0.1, 0.25], dtype=np.float64)


def build(quiet: bool = True) -> None:
    """Build the oracle libraries (the _ref targets only where the reference exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Ref:
    """The reference's own functions on one particle set (oracle/_ref/libref.so)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(REF_SO):
                raise FileNotFoundError(f"{REF_SO} missing: build oracle/ where the reference exists")
            L = C.CDLL(REF_SO)
            L.ref_case_from_cfg.restype = C.c_void_p
            L.ref_case_from_cfg.argtypes = [C.c_char_p]
            L.ref_case_free.argtypes = [C.c_void_p]
            L.ref_cfg_get.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_double), C.c_char_p, C.c_size_t]
            L.ref_cfg_set.argtypes = [C.c_void_p, C.c_char_p, C.c_double]
            L.ref_cfg_set_case.argtypes = [C.c_void_p, C.c_char_p]
            L.ref_generate.restype = C.c_size_t
            L.ref_generate.argtypes = [C.c_void_p]
            L.ref_set_particles.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t]
            L.ref_get_particles.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
            L.ref_neighbors.restype = C.c_longlong
            L.ref_neighbors.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                        C.POINTER(C.c_ulonglong)]
            L.ref_classify.argtypes = [C.c_void_p, C.c_void_p]
            L.ref_wls_test.argtypes = [C.c_void_p, _dp]
            L.ref_wls_particle.restype = C.c_int
            L.ref_wls_particle.argtypes = [C.c_void_p, C.c_size_t, _dp]
            L.ref_assemble_ppe.argtypes = [C.c_void_p, C.POINTER(C.c_longlong * 5), C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
            L.ref_solve_ppe.argtypes = [C.c_void_p, _dp]
            L.ref_bicgstab_csr.argtypes = [C.c_size_t, _ip, _ip, _dp, _dp, _dp, C.c_int, C.c_double,
                                           C.c_void_p, _dp]
            L.ref_run_benchmark.argtypes = [C.c_void_p, _dp]
            L.ref_write_outputs.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p]
            cls._lib = L
        return cls._lib

    def __init__(self, cfg_path: str, **overrides):
        L = self.lib()
        self.h = L.ref_case_from_cfg(cfg_path.encode())
        if not self.h:
            raise RuntimeError(f"reference could not load {cfg_path}")
        for k, v in overrides.items():
            if k == "case":
                L.ref_cfg_set_case(self.h, str(v).encode())
            elif L.ref_cfg_set(self.h, k.encode(), float(v)) != 0:
                raise KeyError(k)
        self.n = 0

    def __del__(self):
        if getattr(self, "h", None):
            self.lib().ref_case_free(self.h)
            self.h = None

    def cfg(self, key: str):
        v = C.c_double()
        buf = C.create_string_buffer(256)
        if self.lib().ref_cfg_get(self.h, key.encode(), C.byref(v), buf, 256) != 0:
            raise KeyError(key)
        return buf.value.decode() if key == "case" else v.value

    def generate(self):
        self.n = self.lib().ref_generate(self.h)
        return self.particles()

    def set_particles(self, xyz: np.ndarray, types: np.ndarray):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        types = np.ascontiguousarray(types, dtype=np.uint8)
        self.n = len(types)
        self.lib().ref_set_particles(self.h, _ptr(xyz), _ptr(types), self.n)

    def particles(self):
        xyz = np.zeros((self.n, 3)); t = np.zeros(self.n, np.uint8); u = np.zeros((self.n, 3))
        self.lib().ref_get_particles(self.h, _ptr(xyz), _ptr(t), _ptr(u))
        return xyz, t, u

    def neighbors(self):
        L = self.lib()
        row = np.zeros(self.n + 1, np.int32)
        tr = C.c_ulonglong()
        pairs = L.ref_neighbors(self.h, _ptr(row), None, 0, C.byref(tr))
        col = np.zeros(max(pairs, 1), np.int32)
        L.ref_neighbors(self.h, _ptr(row), _ptr(col), pairs, C.byref(tr))
        return row, col[:pairs], int(tr.value)

    def classify(self):
        t = np.zeros(self.n, np.uint8)
        self.lib().ref_classify(self.h, _ptr(t))
        return t

    def wls_test(self):
        o = np.zeros(9)
        self.lib().ref_wls_test(self.h, o)
        keys = ["sampled", "ok", "regularized", "failed", "virtual_points", "max_gradient_error",
                "rms_gradient_error", "max_laplacian_error", "rms_laplacian_error"]
        return dict(zip(keys, o.tolist()))

    def wls_particle(self, i: int):
        x = np.zeros(9)
        st = self.lib().ref_wls_particle(self.h, i, x)
        return st, x

    def assemble_ppe(self):
        L = self.lib()
        sz = (C.c_longlong * 5)()
        L.ref_assemble_ppe(self.h, C.byref(sz), None, None, None, None, None)
        u, nnz = sz[0], sz[1]
        row = np.zeros(u + 1, np.int32); col = np.zeros(nnz, np.int32); val = np.zeros(nnz)
        b = np.zeros(u); xe = np.zeros(u)
        L.ref_assemble_ppe(self.h, C.byref(sz), _ptr(row), _ptr(col), _ptr(val), _ptr(b), _ptr(xe))
        stats = dict(unknowns=sz[0], nnz=sz[1], dirichlet=sz[2], neumann=sz[3], failed_rows=sz[4])
        return row, col, val, b, xe, stats

    def solve_ppe(self):
        o = np.zeros(10)
        self.lib().ref_solve_ppe(self.h, o)
        keys = ["iterations", "converged", "initial_residual", "final_residual", "relative_l2_error",
                "max_error", "assembly_ms", "solve_ms", "unknowns", "nnz"]
        return dict(zip(keys, o.tolist()))

    def run_benchmark(self):
        o = np.zeros(22)
        self.lib().ref_run_benchmark(self.h, o)
        keys = ["particles", "interior", "free_surface", "splash", "near_wall", "wall", "pairs",
                "truncated", "mean", "p50", "p90", "p99", "neighbor_ms", "classify_ms", "wls_ms",
                "wls_sampled", "wls_failed", "ppe_unknowns", "ppe_nnz", "ppe_iterations",
                "ppe_converged", "ppe_rel_l2"]
        return dict(zip(keys, o.tolist()))

    def write_outputs(self, json_path: str, csv_path: str):
        self.lib().ref_write_outputs(self.h, json_path.encode(), csv_path.encode())

    @classmethod
    def bicgstab_csr(cls, row, col, val, b, x_exact, max_iter, tol):
        n = len(b)
        x = np.zeros(n); o = np.zeros(6)
        cls.lib().ref_bicgstab_csr(n, row, col, val, b, x_exact, int(max_iter), float(tol), _ptr(x), o)
        keys = ["iterations", "converged", "final_residual", "relative_l2_error", "max_error", "solve_ms"]
        return x, dict(zip(keys, o.tolist()))


class Oracle:
    """This repository's CPU restatement (oracle/_build/liboracle.so)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(ORACLE_SO):
                build()
            L = C.CDLL(ORACLE_SO)
            L.orc_neighbors.restype = C.c_longlong
            L.orc_neighbors.argtypes = [_dp, C.c_size_t, C.c_double, C.c_int, C.c_void_p, C.c_void_p,
                                        C.c_size_t, C.POINTER(C.c_ulonglong)]
            L.orc_classify.argtypes = [_dp, _up, C.c_size_t, _ip, _ip, C.c_double, _up]
            L.orc_wls.argtypes = [_dp, _up, C.c_size_t, _ip, _ip, C.c_double, C.c_double, C.c_double,
                                  C.c_int, _dp, C.c_void_p, _ip, C.c_void_p, C.c_void_p]
            L.orc_wls_fields.argtypes = [_dp, _up, C.c_size_t, _ip, _ip, C.c_double, C.c_double, C.c_double,
                                         C.c_int, _dp, _dp, _ip, C.c_int]
            L.orc_ppe_assemble.restype = C.c_longlong
            L.orc_ppe_assemble.argtypes = [C.c_int, _dp, _up, C.c_size_t, _ip, _ip, C.c_double,
                                           C.c_double, C.c_longlong, C.c_double, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.POINTER(C.c_longlong * 5)]
            L.orc_spmv.argtypes = [C.c_size_t, _ip, _ip, _dp, _dp, _dp, C.c_int]
            L.orc_bicgstab.argtypes = [C.c_size_t, _ip, _ip, _dp, _dp, C.c_void_p, C.c_int, C.c_double,
                                       C.c_int, C.c_int, _dp, _dp]
            L.orc_generate.restype = C.c_size_t
            L.orc_generate.argtypes = [C.c_int, C.c_size_t, C.c_double, C.c_double, C.c_uint, _dp, _up]
            cls._lib = L
        return cls._lib

    GENERATORS = {"bulk": 0, "rain_plate": 1, "mixed": 2}

    @classmethod
    def generate(cls, case, n, l0=1.0, seed=7, jitter=-1.0):
        """Positions and types of the bench/test particle sets (bulk lattice, rain_plate,
        mixed), bit-identical to the library's generator, without loading the library."""
        xyz = np.zeros((n, 3)); t = np.zeros(n, np.uint8)
        w = cls.lib().orc_generate(cls.GENERATORS[case], n, l0, jitter, seed, xyz.reshape(-1), t)
        return xyz[:w], t[:w]

    @classmethod
    def neighbors(cls, xyz, re, maxn):
        L = cls.lib()
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        n = len(xyz)
        row = np.zeros(n + 1, np.int32)
        tr = C.c_ulonglong()
        pairs = L.orc_neighbors(xyz, n, re, maxn, _ptr(row), None, 0, C.byref(tr))
        col = np.zeros(max(pairs, 1), np.int32)
        L.orc_neighbors(xyz, n, re, maxn, _ptr(row), _ptr(col), pairs, C.byref(tr))
        return row, col[:pairs], int(tr.value)

    @classmethod
    def classify(cls, xyz, types, row, col, l0):
        out = np.zeros(len(types), np.uint8)
        cls.lib().orc_classify(np.ascontiguousarray(xyz, dtype=np.float64),
                               np.ascontiguousarray(types, dtype=np.uint8), len(types), row, col,
                               l0, out)
        return out

    @classmethod
    def wls(cls, xyz, types, row, col, re, l0, reg=1e-8, coef=None):
        coef = REF_QUADRATIC[None, :] if coef is None else np.atleast_2d(coef)
        coef = np.ascontiguousarray(coef, dtype=np.float64)
        n = len(types); nrhs = coef.shape[0]
        x = np.zeros((n, nrhs, 9)); st = np.zeros(n, np.int32); z = np.zeros((n, 9)); ws = np.zeros(n)
        cls.lib().orc_wls(np.ascontiguousarray(xyz, dtype=np.float64),
                          np.ascontiguousarray(types, dtype=np.uint8), n, row, col, re, l0, reg,
                          nrhs, coef, _ptr(x), st, _ptr(z), _ptr(ws))
        return x, st, z, ws

    @classmethod
    def wls_fields(cls, xyz, types, row, col, re, l0, fields, reg=1e-8, mirror_walls=False):
        """WLS solutions (n x nfields x 9) of per-particle fields (n x nfields), and the status.
        mirror_walls: Wall neighbors take the particle's own value (zero normal gradient)."""
        fields = np.ascontiguousarray(np.atleast_2d(np.asarray(fields, dtype=np.float64).T).T)
        n, nf = fields.shape
        x = np.zeros((n, nf, 9)); st = np.zeros(n, np.int32)
        cls.lib().orc_wls_fields(np.ascontiguousarray(xyz, dtype=np.float64),
                                 np.ascontiguousarray(types, dtype=np.uint8), n, row, col, re, l0, reg, nf, fields,
                                 x.reshape(-1), st, 1 if mirror_walls else 0)
        return x, st

    @classmethod
    def predict_velocity(cls, xyz, types, row, col, re, l0, vel, dt, nu, gravity, mirror_walls=False):
        """The viscous / gravity predictor (python/rain_plate_lsmps_cpu.py:184-196, in 3-D):
        u* = u + dt (nu lap u + g), lap u of each component = (x3 + x4 + x5) / l0 of its WLS
        solution (the basis keeps l0 f_aa in x3..x5), zero where the WLS is skipped or failed;
        wall particles keep u."""
        vel = np.asarray(vel, dtype=np.float64).reshape(-1, 3)
        x, st = cls.wls_fields(xyz, types, row, col, re, l0, vel, mirror_walls=mirror_walls)
        lap = (x[:, :, 3] + x[:, :, 4] + x[:, :, 5]) / l0
        out = vel + dt * (nu * lap + np.asarray(gravity, dtype=np.float64)[None, :])
        walls = np.asarray(types) == 4  # Wall
        out[walls] = vel[walls]
        return out

    @classmethod
    def ppe_assemble(cls, variant, xyz, types, row, col, re, l0, max_unknowns, diag_shift=0.0,
                     z=None, wsum=None, wls_status=None):
        L = cls.lib()
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        types = np.ascontiguousarray(types, dtype=np.uint8)
        n = len(types)
        sz = (C.c_longlong * 5)()
        args = (variant, xyz, types, n, row, col, re, l0, int(max_unknowns), diag_shift,
                _ptr(z), _ptr(wsum), _ptr(wls_status))
        L.orc_ppe_assemble(*args, None, None, None, None, None, None, C.byref(sz))
        u, nnz = sz[0], sz[1]
        prow = np.zeros(u + 1, np.int32); pcol = np.zeros(nnz, np.int32); val = np.zeros(nnz)
        b = np.zeros(u); xe = np.zeros(u); up = np.zeros(u, np.int32)
        L.orc_ppe_assemble(*args, _ptr(prow), _ptr(pcol), _ptr(val), _ptr(b), _ptr(xe), _ptr(up),
                           C.byref(sz))
        stats = dict(unknowns=sz[0], nnz=sz[1], dirichlet=sz[2], neumann=sz[3], failed_rows=sz[4])
        return prow, pcol, val, b, xe, up, stats

    @classmethod
    def spmv(cls, row, col, val, x, nthreads=1):
        y = np.zeros(len(row) - 1)
        cls.lib().orc_spmv(len(y), row, col, val, np.ascontiguousarray(x, dtype=np.float64), y, nthreads)
        return y

    @classmethod
    def bicgstab(cls, row, col, val, b, max_iter, tol, x0=None, precond=0, nthreads=1):
        n = len(b)
        x = np.zeros(n); o = np.zeros(4)
        x0c = None if x0 is None else np.ascontiguousarray(x0, dtype=np.float64)
        cls.lib().orc_bicgstab(n, row, col, val, b, _ptr(x0c), int(max_iter), float(tol), precond,
                               nthreads, x, o)
        return x, dict(iterations=int(o[0]), converged=bool(o[1]), final_residual=o[2], ms=o[3])
