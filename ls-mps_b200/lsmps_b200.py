"""ctypes binding of the LS-MPS sm_100a library (include/lsmps_gpu.h).

This is the Python face of the C ABI, used by the tests and bench.py; the struct layouts
below mirror the header field for field. The library is loaded from ``lib/`` next to this
file (built by ``make`` in this directory); there is no fallback of any kind: if the
shared library is missing, importing ``load()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "liblsmps_b200.so")
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "mpnn_rain200k.bin")
CLI_PATH = os.path.join(HERE, "bin", "lsmps-bench")

OK, ERR_ARG, ERR_CUDA, ERR_ALLOC, ERR_STATE, ERR_GRID, ERR_OVERFLOW, ERR_NONFINITE, ERR_TIMEOUT, ERR_IO = range(10)
INTERIOR, FREE_SURFACE, SPLASH, NEAR_WALL, WALL = range(5)
NBR_CLASSIFY = 1
NBR_TWO_PASS = 2
PPE_WALL_NEUMANN = 1
PPE_REFERENCE, PPE_SHIFTED, PPE_WLS = range(3)
SOLVER_REFERENCE, SOLVER_FP64, SOLVER_JACOBI, SOLVER_MIXED, SOLVER_LEARNED, SOLVER_MIXED_F32 = range(6)
(KB_SPMV64, KB_SPMV32, KB_NBR_COUNT, KB_NBR_FILL, KB_WLS, KB_MPNN_LAYER, KB_MG_VCYCLE, KB_NBR_SCAN, KB_NBR_COMPACT,
 KB_FP64_PEAK) = range(10)
PRECONDS = {"jacobi": 0, "multigrid": 1}
SOLVERS = {"reference": 0, "fp64": 1, "jacobi": 2, "mixed": 3, "learned": 4, "mixed_f32": 5}
VARIANTS = {"reference": 0, "shifted": 1, "wls": 2}

REF_QUADRATIC = np.array([1, 2, -3, 0.5, 0.7, -0.2, 0.4, 0.3, -0.1, 0.25], dtype=np.float64)


def build(quiet: bool = True) -> None:
    """Compile the library and CLI for sm_100a (nvcc cross-compiles without a GPU)."""
    subprocess.run(["make", "-s", "-j8", "-C", HERE], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)


class NeighborStats(C.Structure):
    _fields_ = [("pairs", C.c_uint64), ("truncated", C.c_uint64), ("mean", C.c_double),
                ("p50", C.c_int32), ("p90", C.c_int32), ("p99", C.c_int32), ("max_count", C.c_int32),
                ("type_count", C.c_uint64 * 5), ("grid_cells", C.c_int64),
                ("max_cell_occupancy", C.c_int32), ("reserved", C.c_int32)]


class WlsOpts(C.Structure):
    _fields_ = [("re", C.c_double), ("l0", C.c_double), ("regularization", C.c_double),
                ("mode", C.c_int32), ("wls_samples", C.c_int32), ("nrhs", C.c_int32),
                ("precision", C.c_int32), ("quad_coef", C.POINTER(C.c_double)),
                ("store_solutions", C.c_int32), ("reserved", C.c_int32)]


class WlsStats(C.Structure):
    _fields_ = [("sampled", C.c_uint64), ("ok", C.c_uint64), ("regularized", C.c_uint64),
                ("failed", C.c_uint64), ("virtual_points", C.c_uint64),
                ("max_gradient_error", C.c_double), ("rms_gradient_error", C.c_double),
                ("max_laplacian_error", C.c_double), ("rms_laplacian_error", C.c_double),
                ("skipped", C.c_uint64), ("fp64_fallback", C.c_uint64)]


class PpeOpts(C.Structure):
    _fields_ = [("variant", C.c_int32), ("flags", C.c_int32), ("max_unknowns", C.c_int64),
                ("re", C.c_double), ("l0", C.c_double), ("diag_shift", C.c_double)]


class ProjectionStats(C.Structure):
    _fields_ = [("unknowns", C.c_uint64), ("measured", C.c_uint64), ("div_before_rms", C.c_double),
                ("div_before_max", C.c_double), ("div_after_rms", C.c_double), ("div_after_max", C.c_double),
                ("iterations", C.c_int32), ("converged", C.c_int32), ("relative_residual", C.c_double),
                ("solve_ms", C.c_double), ("total_ms", C.c_double), ("core", C.c_uint64),
                ("div_core_before_rms", C.c_double), ("div_core_after_rms", C.c_double),
                ("wall_band1", C.c_uint64), ("wall_band2", C.c_uint64), ("div_wall1_before_rms", C.c_double),
                ("div_wall1_after_rms", C.c_double), ("div_wall2_before_rms", C.c_double),
                ("div_wall2_after_rms", C.c_double)]


class SeriesParams(C.Structure):
    _fields_ = [("steps", C.c_int32), ("injected_per_step", C.c_int32), ("cnl_rebuild_interval", C.c_int32),
                ("solver", C.c_int32), ("l0", C.c_double), ("re", C.c_double), ("skin", C.c_double),
                ("droplet_speed", C.c_double), ("film_speed", C.c_double), ("theta_deg", C.c_double),
                ("film_thickness", C.c_double), ("droplet_radius", C.c_double), ("inject_hmin", C.c_double),
                ("inject_hmax", C.c_double), ("tol", C.c_double), ("max_iter", C.c_int32),
                ("max_neighbors", C.c_int32), ("max_candidates", C.c_int32), ("wls_precision", C.c_int32),
                ("warm_start", C.c_int32), ("seed", C.c_uint32), ("precond", C.c_int32), ("reserved", C.c_int32)]


class SeriesStats(C.Structure):
    _fields_ = [("step", C.c_int32), ("rebuilt", C.c_int32), ("forced_rebuild", C.c_int32), ("converged", C.c_int32),
                ("particles", C.c_uint64), ("in_flight", C.c_uint64), ("flagged", C.c_uint64),
                ("injected_total", C.c_uint64), ("deleted_total", C.c_uint64), ("fluid_particles", C.c_uint64),
                ("mass_balance", C.c_int64), ("pairs", C.c_uint64), ("unknowns", C.c_uint64), ("nnz", C.c_uint64),
                ("iterations", C.c_int32), ("outer_iterations", C.c_int32), ("fallback", C.c_int32),
                ("reserved", C.c_int32), ("fluid_volume", C.c_double), ("max_displacement", C.c_double),
                ("relative_l2_error", C.c_double), ("relative_residual", C.c_double), ("neighbor_ms", C.c_double),
                ("wls_ms", C.c_double), ("assembly_ms", C.c_double), ("solve_ms", C.c_double),
                ("step_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


RAIN_MAX = 8


class RainValidation(C.Structure):
    _fields_ = [("nwindows", C.c_int32), ("nsections", C.c_int32), ("coverage_cells", C.c_int32),
                ("min_particles_per_cell", C.c_int32), ("wet_distance_factor", C.c_double),
                ("window_lo", C.c_double * RAIN_MAX), ("window_hi", C.c_double * RAIN_MAX),
                ("section_u", C.c_double * RAIN_MAX), ("section_max_normal", C.c_double * RAIN_MAX)]


class RainOutputs(C.Structure):
    _fields_ = [("window_particles", C.c_uint64 * RAIN_MAX), ("window_coverage", C.c_double * RAIN_MAX),
                ("film_mean", C.c_double * RAIN_MAX), ("film_p90", C.c_double * RAIN_MAX),
                ("film_max", C.c_double * RAIN_MAX), ("section_crossings", C.c_uint64 * RAIN_MAX)]


# the reference's config/rain_plate_validation.json (windows and sections in plate coordinate u)
RAIN_WINDOWS = [("impact_zone", 0.1, 0.35), ("film_zone", 0.4, 0.7), ("outlet_zone", 0.75, 0.95)]
RAIN_SECTIONS = [("mid_section", 0.55, 5.0), ("outlet_section", 0.9, 5.0)]


SERIES_DEFAULTS = dict(steps=200, injected_per_step=2000, cnl_rebuild_interval=10, solver="learned", l0=1.0, re=2.1,
                       skin=1.0, droplet_speed=0.05, film_speed=0.02, theta_deg=20.0, film_thickness=4.0,
                       droplet_radius=3.0, inject_hmin=10.0, inject_hmax=40.0, tol=3e-11, max_iter=20000,
                       max_neighbors=128, max_candidates=512, wls_precision=0, warm_start=1, seed=23,
                       precond="jacobi")


class PpeStats(C.Structure):
    _fields_ = [("unknowns", C.c_uint64), ("nnz", C.c_uint64), ("dirichlet", C.c_uint64),
                ("neumann", C.c_uint64), ("failed_rows", C.c_uint64), ("iterations", C.c_int32),
                ("converged", C.c_int32), ("initial_residual", C.c_double),
                ("final_residual", C.c_double), ("relative_l2_error", C.c_double),
                ("max_error", C.c_double), ("assembly_ms", C.c_double), ("solve_ms", C.c_double),
                ("outer_iterations", C.c_int32), ("fallback", C.c_int32),
                ("relative_residual", C.c_double)]


class SolverOpts(C.Structure):
    _fields_ = [("solver", C.c_int32), ("max_iter", C.c_int32), ("tol", C.c_double),
                ("warm_start", C.c_int32), ("use_graph", C.c_int32), ("inner_tol", C.c_double),
                ("inner_max_iter", C.c_int32), ("stall_window", C.c_int32), ("check_every", C.c_int32),
                ("precond", C.c_int32)]


class MpnnTrainOpts(C.Structure):
    _fields_ = [("steps", C.c_int32), ("batch", C.c_int32), ("lr", C.c_float),
                ("weight_decay", C.c_float), ("seed", C.c_uint32), ("loss", C.c_int32)]


# Every function the header declares, with its ctypes signature.
_vp = C.c_void_p
SIGNATURES = {
    "lsmps_ctx_create": (C.c_int, [C.c_int, C.POINTER(_vp)]),
    "lsmps_ctx_destroy": (None, [_vp]),
    "lsmps_last_error": (C.c_char_p, [_vp]),
    "lsmps_abi_version": (C.c_int, []),
    "lsmps_get_timings": (C.c_int, [_vp, C.POINTER(C.c_double * 8)]),
    "lsmps_sync": (C.c_int, [_vp]),
    "lsmps_stream": (C.c_void_p, [_vp]),
    "lsmps_launch_count": (C.c_uint64, []),
    "lsmps_kernel_bench": (C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "lsmps_upload_particles": (C.c_int, [_vp, _vp, _vp, C.c_size_t]),
    "lsmps_upload_particles_device": (C.c_int, [_vp, _vp, _vp, C.c_size_t]),
    "lsmps_build_neighbors": (C.c_int, [_vp, C.c_double, C.c_int, C.c_double, C.c_int,
                                        C.POINTER(NeighborStats)]),
    "lsmps_classify": (C.c_int, [_vp, C.c_double, C.POINTER(NeighborStats)]),
    "lsmps_build_neighbors_skin": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int, C.c_double, C.c_int,
                                             C.POINTER(NeighborStats)]),
    "lsmps_update_positions": (C.c_int, [_vp, _vp, C.c_size_t]),
    "lsmps_update_positions_device": (C.c_int, [_vp, _vp, C.c_size_t]),
    "lsmps_refresh_neighbors": (C.c_int, [_vp, C.c_int, C.POINTER(NeighborStats)]),
    "lsmps_max_displacement": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "lsmps_wls": (C.c_int, [_vp, C.POINTER(WlsOpts), C.POINTER(WlsStats)]),
    "lsmps_ppe_assemble": (C.c_int, [_vp, C.POINTER(PpeOpts), C.POINTER(PpeStats)]),
    "lsmps_ppe_solve": (C.c_int, [_vp, C.POINTER(SolverOpts), C.POINTER(PpeStats)]),
    "lsmps_download_types": (C.c_int, [_vp, _vp, C.c_size_t]),
    "lsmps_download_neighbors": (C.c_int, [_vp, _vp, _vp, C.c_size_t]),
    "lsmps_download_wls": (C.c_int, [_vp, _vp, _vp, _vp, _vp]),
    "lsmps_download_ppe": (C.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "lsmps_download_pressure": (C.c_int, [_vp, _vp, C.c_size_t]),
    "lsmps_download_pressure_async": (C.c_int, [_vp, _vp, C.c_size_t]),
    "lsmps_download_wait": (C.c_int, [_vp]),
    "lsmps_ppe_manufacture": (C.c_int, [_vp, _vp, C.c_int]),
    "lsmps_ppe_residual_static": (C.c_int, [_vp, _vp, C.c_size_t, C.c_int, _vp]),
    "lsmps_set_initial_pressure": (C.c_int, [_vp, _vp, C.c_size_t]),
    "lsmps_wls_fields": (C.c_int, [_vp, _vp, C.c_int, _vp]),
    "lsmps_ppe_load_csr": (C.c_int, [_vp, _vp, _vp, _vp, _vp, C.c_size_t, C.POINTER(PpeStats)]),
    "lsmps_mg_info": (C.c_int, [_vp, C.POINTER(C.c_int32), _vp, C.c_int32, C.POINTER(C.c_double)]),
    "lsmps_mg_apply": (C.c_int, [_vp, _vp, _vp, C.c_size_t]),
    "lsmps_projection_step": (C.c_int, [_vp, _vp, C.c_double, C.c_double, C.POINTER(SolverOpts), _vp, _vp,
                                        C.POINTER(ProjectionStats)]),
    "lsmps_series_create": (C.c_int, [_vp, C.POINTER(SeriesParams), _vp, _vp, C.c_size_t, C.POINTER(_vp)]),
    "lsmps_series_step": (C.c_int, [_vp, C.POINTER(SeriesStats)]),
    "lsmps_series_particles": (C.c_int, [_vp, _vp, _vp, _vp, C.c_size_t, C.POINTER(C.c_size_t)]),
    "lsmps_series_destroy": (None, [_vp]),
    "lsmps_series_set_validation": (C.c_int, [_vp, C.POINTER(RainValidation)]),
    "lsmps_series_rain_outputs": (C.c_int, [_vp, C.POINTER(RainOutputs)]),
    "lsmps_set_initial_pressure_device": (C.c_int, [_vp, _vp, C.c_size_t]),
    "lsmps_download_pressure_particles": (C.c_int, [_vp, _vp, C.c_size_t, C.c_double]),
    "lsmps_download_pressure_particles_device": (C.c_int, [_vp, _vp, C.c_size_t, C.c_double]),
    "lsmps_set_autotune": (C.c_int, [_vp, C.c_int]),
    "lsmps_autotune_report": (C.c_int, [_vp, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]),
    "lsmps_mpnn_param_count": (C.c_size_t, []),
    "lsmps_mpnn_init": (C.c_int, [_vp, C.c_uint32]),
    "lsmps_mpnn_get_weights": (C.c_int, [_vp, _vp, C.c_size_t]),
    "lsmps_mpnn_set_weights": (C.c_int, [_vp, _vp, C.c_size_t]),
    "lsmps_mpnn_add_sample": (C.c_int, [_vp]),
    "lsmps_mpnn_clear_samples": (C.c_int, [_vp]),
    "lsmps_mpnn_sample_count": (C.c_int, [_vp]),
    "lsmps_mpnn_grad": (C.c_int, [_vp, C.c_int, _vp, C.POINTER(C.c_float)]),
    "lsmps_mpnn_train": (C.c_int, [_vp, C.POINTER(MpnnTrainOpts), C.POINTER(C.c_float)]),
    "lsmps_mpnn_infer": (C.c_int, [_vp, _vp, _vp]),
    "lsmps_mpnn_save": (C.c_int, [_vp, C.c_char_p]),
    "lsmps_mpnn_load": (C.c_int, [_vp, C.c_char_p]),
    "lsmps_host_generate": (C.c_int, [C.c_char_p, C.c_char_p, _vp, _vp, _vp, C.POINTER(C.c_size_t)]),
    "lsmps_prefetch_particles": (C.c_int, [_vp, _vp, _vp, C.c_size_t]),
    "lsmps_predict_velocity": (C.c_int, [_vp, _vp, C.c_double, C.c_double, _vp, C.c_int, _vp]),
    "lsmps_use_prefetched_particles": (C.c_int, [_vp]),
}

_LIB = None


def load():
    """Load lib/liblsmps_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"{LIB_PATH} is missing: run make in {HERE} (or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class LsmpsError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"status {code}: {msg}")
        self.code = code


def generate(cfg_path: str | None = None, **overrides):
    """Particles of a .cfg case through the library's generate_case (host code, no GPU)."""
    L = load()
    ov = ";".join(f"{k}={v}" for k, v in overrides.items()).encode()
    n = C.c_size_t(0)
    cp = cfg_path.encode() if cfg_path else None
    rc = L.lsmps_host_generate(cp, ov, None, None, None, C.byref(n))
    if rc != OK:
        raise LsmpsError(rc, "generate failed")
    xyz = np.zeros((n.value, 3)); t = np.zeros(n.value, np.uint8); u = np.zeros((n.value, 3))
    rc = L.lsmps_host_generate(cp, ov, _p(xyz), _p(t), _p(u), C.byref(n))
    if rc != OK:
        raise LsmpsError(rc, "generate failed")
    return xyz, t, u


class Context:
    """One lsmps_ctx: device buffers and stream of one particle set on one GPU."""

    def __init__(self, device: int = 0):
        self.L = load()
        h = C.c_void_p()
        rc = self.L.lsmps_ctx_create(device, C.byref(h))
        if rc != OK:
            raise LsmpsError(rc, f"cannot create a context on device {device}")
        self.h = h
        self.n = 0

    def close(self):
        if getattr(self, "h", None):
            self.L.lsmps_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != OK:
            raise LsmpsError(rc, self.L.lsmps_last_error(self.h).decode())

    def timings(self):
        t = (C.c_double * 8)()
        self._check(self.L.lsmps_get_timings(self.h, C.byref(t)))
        return list(t)

    def sync(self):
        self._check(self.L.lsmps_sync(self.h))

    def stream(self):
        return self.L.lsmps_stream(self.h)

    def kernel_bench(self, kernel, reps=20):
        ms, nb = C.c_double(), C.c_double()
        self._check(self.L.lsmps_kernel_bench(self.h, kernel, reps, C.byref(ms), C.byref(nb)))
        return ms.value, nb.value

    def set_autotune(self, mode):
        """0 off (fixed default launch shapes), 1 on, 2 on and forget earlier choices."""
        self._check(self.L.lsmps_set_autotune(self.h, mode))

    def autotune_report(self):
        """[(key, shape, ms, is_best)] of every candidate the autotuner timed on this context."""
        need = C.c_size_t()
        self._check(self.L.lsmps_autotune_report(self.h, None, 0, C.byref(need)))
        buf = C.create_string_buffer(need.value)
        self._check(self.L.lsmps_autotune_report(self.h, buf, need.value, C.byref(need)))
        out = []
        for line in buf.value.decode().splitlines():
            f = line.split("\t")
            out.append((f[0], f[1], float(f[2]), len(f) > 3))
        return out

    def upload(self, xyz, types):
        self._xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        self._types = np.ascontiguousarray(types, dtype=np.uint8)
        self.n = len(self._types)
        self._check(self.L.lsmps_upload_particles(self.h, _p(self._xyz), _p(self._types), self.n))

    def prefetch(self, xyz, types):
        """lsmps_prefetch_particles: enqueue the copies of the next particle set (keep the arrays
        alive and unchanged until use_prefetched; pinned arrays let the copies overlap)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        types = np.ascontiguousarray(types, dtype=np.uint8)
        self._staged = (xyz, types)
        self._check(self.L.lsmps_prefetch_particles(self.h, _p(xyz), _p(types), len(types)))

    def use_prefetched(self):
        """lsmps_use_prefetched_particles: the prefetched set becomes the context's particles."""
        self._check(self.L.lsmps_use_prefetched_particles(self.h))
        self._xyz, self._types = self._staged
        self.n = len(self._types)

    def build_neighbors(self, re, max_neighbors, l0, classify=True, two_pass=False, stats=True):
        """lsmps_build_neighbors; stats=False skips the statistics (and the wait for the lists'
        last kernels) and returns None."""
        flags = (NBR_CLASSIFY if classify else 0) | (NBR_TWO_PASS if two_pass else 0)
        if not stats:
            self._check(self.L.lsmps_build_neighbors(self.h, re, max_neighbors, l0, flags, None))
            return None
        st = NeighborStats()
        self._check(self.L.lsmps_build_neighbors(self.h, re, max_neighbors, l0, flags, C.byref(st)))
        return st

    def classify(self, l0):
        st = NeighborStats()
        self._check(self.L.lsmps_classify(self.h, l0, C.byref(st)))
        return st

    def build_neighbors_skin(self, re, skin, max_neighbors, max_candidates, l0, classify=True):
        """Candidate lists of radius re + skin, then the exact lists of radius re."""
        st = NeighborStats()
        self._check(self.L.lsmps_build_neighbors_skin(self.h, re, skin, max_neighbors, max_candidates, l0,
                                                      NBR_CLASSIFY if classify else 0, C.byref(st)))
        return st

    def update_positions(self, xyz):
        """New positions of the same particles (n x 3, caller order)."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        self._check(self.L.lsmps_update_positions(self.h, _p(xyz), len(xyz)))

    def refresh_neighbors(self, classify=True):
        """Exact lists from the candidates at the current positions (LsmpsError once beyond skin / 2)."""
        st = NeighborStats()
        self._check(self.L.lsmps_refresh_neighbors(self.h, NBR_CLASSIFY if classify else 0, C.byref(st)))
        return st

    def max_displacement(self):
        d = C.c_double()
        self._check(self.L.lsmps_max_displacement(self.h, C.byref(d)))
        return d.value

    def wls(self, re, l0, mode=1, wls_samples=4096, coef=None, precision=0, store=False, reg=1e-8,
            stats=True):
        """lsmps_wls; stats=False (mode 1) skips the statistics read-back and returns None."""
        coef = REF_QUADRATIC[None, :] if coef is None else np.atleast_2d(coef)
        self._coef = np.ascontiguousarray(coef, dtype=np.float64)
        o = WlsOpts(re=re, l0=l0, regularization=reg, mode=mode, wls_samples=wls_samples,
                    nrhs=self._coef.shape[0], precision=precision,
                    quad_coef=self._coef.ctypes.data_as(C.POINTER(C.c_double)),
                    store_solutions=1 if store else 0)
        if not stats and mode == 1:
            self._check(self.L.lsmps_wls(self.h, C.byref(o), None))
            return None
        st = WlsStats()
        self._check(self.L.lsmps_wls(self.h, C.byref(o), C.byref(st)))
        return st

    def ppe_assemble(self, variant, max_unknowns, re, l0, diag_shift=1e-3, wall_neumann=False, stats=True):
        """lsmps_ppe_assemble; stats=False does not wait for the matrix's last kernel and returns
        None (its time comes with the next solve's statistics)."""
        o = PpeOpts(variant=VARIANTS.get(variant, variant), max_unknowns=int(max_unknowns), re=re,
                    l0=l0, diag_shift=diag_shift, flags=PPE_WALL_NEUMANN if wall_neumann else 0)
        if not stats:
            self._check(self.L.lsmps_ppe_assemble(self.h, C.byref(o), None))
            return None
        st = PpeStats()
        self._check(self.L.lsmps_ppe_assemble(self.h, C.byref(o), C.byref(st)))
        self._last_ppe = st
        return st

    def ppe_solve(self, solver, max_iter, tol, warm_start=False, use_graph=True, inner_tol=0.0,
                  inner_max_iter=0, stall_window=0, check_every=0, precond="jacobi"):
        """lsmps_ppe_solve. solver: a name of SOLVERS; precond: "jacobi" or "multigrid" (the MIXED
        and LEARNED solvers); use_graph: 1 device-driven graph, 2 chunk graphs, 0 eager."""
        o = SolverOpts(solver=SOLVERS.get(solver, solver), max_iter=int(max_iter), tol=tol,
                       warm_start=1 if warm_start else 0, use_graph=int(use_graph),
                       inner_tol=inner_tol, inner_max_iter=inner_max_iter, stall_window=stall_window,
                       check_every=check_every, precond=PRECONDS.get(precond, precond))
        st = PpeStats()
        self._check(self.L.lsmps_ppe_solve(self.h, C.byref(o), C.byref(st)))
        return st

    def mg_info(self):
        """Multigrid hierarchy of the assembled system: rows per level (0 = unknowns) and setup ms."""
        lv = C.c_int32(0); ms = C.c_double(0)
        rows = np.zeros(64, np.int64)
        self._check(self.L.lsmps_mg_info(self.h, C.byref(lv), _p(rows), 64, C.byref(ms)))
        return rows[: lv.value + 1].copy(), ms.value

    def mg_apply(self, z):
        """D M z: the multigrid V-cycle as the solvers apply it (reference unknown numbering)."""
        z = np.ascontiguousarray(z, dtype=np.float64)
        out = np.zeros_like(z)
        self._check(self.L.lsmps_mg_apply(self.h, _p(z), _p(out), len(z)))
        return out

    def types(self):
        t = np.zeros(self.n, np.uint8)
        self._check(self.L.lsmps_download_types(self.h, _p(t), self.n))
        return t

    def neighbors(self, pairs):
        row = np.zeros(self.n + 1, np.int32)
        col = np.zeros(max(int(pairs), 1), np.int32)
        self._check(self.L.lsmps_download_neighbors(self.h, _p(row), _p(col), int(pairs)))
        return row, col[: int(pairs)]

    def wls_result(self, nrhs=1, with_x=False):
        x = np.zeros((self.n, nrhs, 9)) if with_x else None
        st = np.zeros(self.n, np.int32); z = np.zeros((self.n, 9)); ws = np.zeros(self.n)
        self._check(self.L.lsmps_download_wls(self.h, _p(x), _p(st), _p(z), _p(ws)))
        return x, st, z, ws

    def ppe(self, unknowns, nnz):
        row = np.zeros(unknowns + 1, np.int32); col = np.zeros(max(nnz, 1), np.int32)
        val = np.zeros(max(nnz, 1)); b = np.zeros(unknowns); xe = np.zeros(unknowns)
        part = np.zeros(unknowns, np.int32)
        self._check(self.L.lsmps_download_ppe(self.h, _p(row), _p(col), _p(val), _p(b), _p(xe), _p(part)))
        return row, col[:nnz], val[:nnz], b, xe, part

    def pressure(self, unknowns):
        p = np.zeros(unknowns)
        self._check(self.L.lsmps_download_pressure(self.h, _p(p), unknowns))
        return p

    def ppe_load_csr(self, row_ptr, col, val=None, b=None):
        """Install a caller's CSR system (lsmps_ppe_load_csr); returns its PpeStats."""
        row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
        col = np.ascontiguousarray(col, dtype=np.int32)
        val = None if val is None else np.ascontiguousarray(val, dtype=np.float64)
        b = None if b is None else np.ascontiguousarray(b, dtype=np.float64)
        st = PpeStats()
        self._check(self.L.lsmps_ppe_load_csr(self.h, _p(row_ptr), _p(col), _p(val), _p(b), len(row_ptr) - 1,
                                              C.byref(st)))
        self._last_ppe = st
        return st

    def wls_fields(self, fields):
        """WLS solutions (n x k x 9) of k per-particle fields (torch CUDA tensor or array, n x k;
        caller order): gradient, l0 x second derivatives (lsmps_wls_fields)."""
        import torch

        f = torch.as_tensor(fields, dtype=torch.float64, device="cuda")
        f = f.reshape(f.shape[0], -1).contiguous()
        out = torch.zeros((f.shape[0], f.shape[1], 9), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        self._check(self.L.lsmps_wls_fields(self.h, C.c_void_p(f.data_ptr()), f.shape[1],
                                            C.c_void_p(out.data_ptr())))
        self.sync()
        return out

    def predict_velocity(self, vel, dt, nu, gravity=(0.0, 0.0, -9.81), wall_neumann=False):
        """lsmps_predict_velocity: u* = u + dt (nu lap u + gravity) (n x 3, caller order; torch tensor out)."""
        import torch

        u = torch.as_tensor(vel, dtype=torch.float64, device="cuda").reshape(-1, 3).contiguous()
        out = torch.empty_like(u)
        g = np.ascontiguousarray(gravity, dtype=np.float64)
        torch.cuda.synchronize()
        self._check(self.L.lsmps_predict_velocity(self.h, C.c_void_p(u.data_ptr()), dt, nu, _p(g),
                                                  PPE_WALL_NEUMANN if wall_neumann else 0, C.c_void_p(out.data_ptr())))
        return out

    def projection_step(self, vel, dt, rho, solver="mixed", max_iter=20000, tol=1e-10, warm_start=False):
        """One pressure projection of velocity vel (n x 3, caller order) on the assembled
        WLS-Laplacian PPE: (corrected velocity, pressure per particle, ProjectionStats)."""
        import torch

        u = torch.as_tensor(vel, dtype=torch.float64, device="cuda").reshape(-1, 3).contiguous()
        out = torch.empty_like(u)
        p = torch.zeros(u.shape[0], dtype=torch.float64, device="cuda")
        o = SolverOpts(solver=SOLVERS.get(solver, solver), max_iter=int(max_iter), tol=tol,
                       warm_start=1 if warm_start else 0, use_graph=1)
        st = ProjectionStats()
        torch.cuda.synchronize()
        self._check(self.L.lsmps_projection_step(self.h, C.c_void_p(u.data_ptr()), dt, rho, C.byref(o),
                                                 C.c_void_p(out.data_ptr()), C.c_void_p(p.data_ptr()), C.byref(st)))
        self.sync()
        return out, p, st

    def set_initial_pressure(self, p_particles):
        """Warm start of the next solve (warm_start=True) from one value per particle (caller order)."""
        p = np.ascontiguousarray(p_particles, dtype=np.float64)
        self._check(self.L.lsmps_set_initial_pressure(self.h, _p(p), len(p)))

    def pressure_particles(self, n, fill=0.0):
        """The last solution per particle (caller order); `fill` where a particle is not an unknown."""
        p = np.zeros(n)
        self._check(self.L.lsmps_download_pressure_particles(self.h, _p(p), n, fill))
        return p

    def pressure_into(self, out):
        """Download the solution into a caller buffer (e.g. pinned host memory)."""
        assert out.dtype == np.float64 and out.flags.c_contiguous
        self._check(self.L.lsmps_download_pressure(self.h, _p(out), len(out)))
        return out

    def pressure_into_async(self, out):
        """lsmps_download_pressure_async: start the download into `out` (page-locked host memory
        to overlap; keep it alive and unread until download_wait)."""
        assert out.dtype == np.float64 and out.flags.c_contiguous
        self._check(self.L.lsmps_download_pressure_async(self.h, _p(out), len(out)))
        return out

    def download_wait(self):
        """lsmps_download_wait: block until the last asynchronous download has landed."""
        self._check(self.L.lsmps_download_wait(self.h))

    def ppe_reference_numbering(self):
        """The assembled system in the reference's numbering (row, col, val, b, p*, particle)."""
        st = PpeStats()
        o = self._last_ppe
        return self.ppe(o.unknowns, o.nnz)

    def ppe_manufacture(self, c0=0.0, gz=0.0, modes=()):
        """p* = c0 + gz z + sum a sin(kx x + ky y + kz z + phi); b = A p*. modes: (a, kx, ky, kz, phi)."""
        prm = np.array([c0, gz] + [v for m in modes for v in m], dtype=np.float64)
        self._check(self.L.lsmps_ppe_manufacture(self.h, _p(prm), len(modes)))

    def mpnn_init(self, seed=0):
        self._check(self.L.lsmps_mpnn_init(self.h, seed))

    def mpnn_weights(self):
        w = np.zeros(self.L.lsmps_mpnn_param_count(), np.float32)
        self._check(self.L.lsmps_mpnn_get_weights(self.h, _p(w), len(w)))
        return w

    def mpnn_set_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        self._check(self.L.lsmps_mpnn_set_weights(self.h, _p(w), len(w)))

    def mpnn_add_sample(self):
        self._check(self.L.lsmps_mpnn_add_sample(self.h))

    def mpnn_clear_samples(self):
        self._check(self.L.lsmps_mpnn_clear_samples(self.h))

    def mpnn_sample_count(self):
        return self.L.lsmps_mpnn_sample_count(self.h)

    def mpnn_grad(self, index=0):
        g = np.zeros(self.L.lsmps_mpnn_param_count(), np.float32)
        loss = C.c_float()
        self._check(self.L.lsmps_mpnn_grad(self.h, index, _p(g), C.byref(loss)))
        return loss.value, g

    def mpnn_infer(self, r):
        r = np.ascontiguousarray(r, np.float64)
        y = np.zeros_like(r)
        self._check(self.L.lsmps_mpnn_infer(self.h, _p(r), _p(y)))
        return y

    def mpnn_train(self, steps, batch=4, lr=1e-3, weight_decay=0.0, seed=0, loss=0):
        o = MpnnTrainOpts(steps=steps, batch=batch, lr=lr, weight_decay=weight_decay, seed=seed, loss=loss)
        loss = C.c_float()
        self._check(self.L.lsmps_mpnn_train(self.h, C.byref(o), C.byref(loss)))
        return loss.value

    def mpnn_save(self, path):
        self._check(self.L.lsmps_mpnn_save(self.h, path.encode()))

    def mpnn_load(self, path):
        self._check(self.L.lsmps_mpnn_load(self.h, path.encode()))


def struct_dict(s):
    out = {}
    for name, _ in s._fields_:
        v = getattr(s, name)
        if hasattr(v, "__len__") and not isinstance(v, (bytes, str)):
            v = list(v)
        out[name] = v
    return out


class Series:
    """A rain-on-plate step series on a context (lsmps_series_*). Keyword arguments override
    SERIES_DEFAULTS; `solver` is a name of SOLVERS, `precond` one of PRECONDS. wls_precision
    defaults to FP64 for every
    solver: on B200 the FP32 factorisation with FP64 refinement measured 2x slower than the
    FP64 solve (5.5 vs 2.8 ms per step at 3M particles); None picks mixed for the mixed and
    learned solvers."""

    def __init__(self, ctx, xyz, types, **kw):
        p = dict(SERIES_DEFAULTS)
        p.update(kw)
        solver = SOLVERS.get(p["solver"], p["solver"])
        if p["wls_precision"] is None:
            p["wls_precision"] = 1 if solver in (SOLVERS["mixed"], SOLVERS["learned"], SOLVERS["mixed_f32"]) else 0
        p["solver"] = solver
        p["precond"] = PRECONDS.get(p["precond"], p["precond"])
        self.params = SeriesParams(**p)
        self.ctx = ctx
        self.h = None
        xyz = np.ascontiguousarray(xyz, dtype=np.float64)
        types = np.ascontiguousarray(types, dtype=np.uint8)
        h = _vp()
        ctx._check(ctx.L.lsmps_series_create(ctx.h, C.byref(self.params), _p(xyz), _p(types), len(types), C.byref(h)))
        self.h = h

    def step(self):
        st = SeriesStats()
        self.ctx._check(self.ctx.L.lsmps_series_step(self.h, C.byref(st)))
        return st

    def rain_outputs(self):
        """Validation outputs of the last step: {window: (particles, coverage, film mean, p90, max)},
        {section: crossings} (the default windows and sections are RAIN_WINDOWS, RAIN_SECTIONS)."""
        o = RainOutputs()
        self.ctx._check(self.ctx.L.lsmps_series_rain_outputs(self.h, C.byref(o)))
        win = {name: (o.window_particles[w], o.window_coverage[w], o.film_mean[w], o.film_p90[w], o.film_max[w])
               for w, (name, _, _) in enumerate(RAIN_WINDOWS)}
        sec = {name: o.section_crossings[c] for c, (name, _, _) in enumerate(RAIN_SECTIONS)}
        return win, sec

    def particles(self):
        """(xyz, material, pressure) of the current particle set (material: 0 wall, 1 film, 2 droplet)."""
        n = C.c_size_t()
        self.ctx._check(self.ctx.L.lsmps_series_particles(self.h, None, None, None, 0, C.byref(n)))
        xyz = np.zeros((n.value, 3))
        mat = np.zeros(n.value, np.uint8)
        pres = np.zeros(n.value)
        self.ctx._check(self.ctx.L.lsmps_series_particles(self.h, _p(xyz), _p(mat), _p(pres), n.value, C.byref(n)))
        return xyz, mat, pres

    def close(self):
        if self.h:
            self.ctx.L.lsmps_series_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
