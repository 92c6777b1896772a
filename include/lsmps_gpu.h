/* LS-MPS per-step path on an sm_100a GPU — C ABI.
 *
 * Plain C types only (pointers, sizes, PODs); no C++ exceptions cross it. One context
 * owns the device buffers and one CUDA stream (lsmps_stream), on which its work is ordered;
 * two helper streams of its own carry the prefetched uploads (ordered before the context
 * stream by lsmps_use_prefetched_particles) and, in a LEARNED solve with the multigrid from a
 * cold start, the hierarchy set-up beside the network (joined back to the context stream
 * within the solve). Calls on one context are not
 * thread-safe, separate contexts are independent. Every function returns an
 * lsmps_status; lsmps_last_error() gives the message of the last failure.
 *
 * Each entry point replaces one internal function of the reference benchmark
 * (lilux618/LS-MPS src/lsmps.cpp, which has no FFI of its own: these are the
 * functions its run_benchmark, src/lsmps.cpp:73, calls). The reference citation is
 * given beside each. Particle indices in and out are the caller's (original) order;
 * internally the library works in cell-sorted order.
 */
#ifndef LSMPS_GPU_H
#define LSMPS_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LSMPS_ABI_VERSION 1

typedef struct lsmps_ctx lsmps_ctx;

typedef enum lsmps_status {
    LSMPS_OK = 0,
    LSMPS_ERR_ARG = 1,        /* invalid argument or size */
    LSMPS_ERR_CUDA = 2,       /* CUDA runtime error (message in lsmps_last_error) */
    LSMPS_ERR_ALLOC = 3,      /* device or pinned allocation failed */
    LSMPS_ERR_STATE = 4,      /* call order: a prerequisite step has not run */
    LSMPS_ERR_GRID = 5,       /* cell grid or cell occupancy beyond the supported limits */
    LSMPS_ERR_OVERFLOW = 6,   /* a 32-bit index would overflow */
    LSMPS_ERR_NONFINITE = 7,  /* non-finite particle position or solver value */
    LSMPS_ERR_TIMEOUT = 8,    /* a bounded device-side wait expired */
    LSMPS_ERR_IO = 9          /* file read/write (weights) */
} lsmps_status;

/* Particle classes, numbered as the reference's ParticleType (include/lsmps.hpp:8). */
enum { LSMPS_INTERIOR = 0, LSMPS_FREE_SURFACE = 1, LSMPS_SPLASH = 2, LSMPS_NEAR_WALL = 3, LSMPS_WALL = 4 };

/* ---- context ---------------------------------------------------------------------- */
int lsmps_ctx_create(int device, lsmps_ctx** out);
void lsmps_ctx_destroy(lsmps_ctx* ctx);
const char* lsmps_last_error(const lsmps_ctx* ctx);
int lsmps_abi_version(void);
/* Device time (ms, CUDA events on the context stream) of the phases of the last calls:
 * [0] upload, [1] neighbor build (+classification when fused), [2] classification,
 * [3] WLS, [4] PPE assembly, [5] PPE solve, [6] last download. A WLS call without
 * statistics did not wait for its events; this call reads them (and waits for them). */
int lsmps_get_timings(lsmps_ctx* ctx, double out[8]);
/* Block until all work queued on the context stream has finished. */
int lsmps_sync(lsmps_ctx* ctx);
/* The context's CUDA stream (a cudaStream_t), for callers that time or order work on it. */
void* lsmps_stream(lsmps_ctx* ctx);
/* Kernel launches this library has issued in this process (graph replays count every
 * kernel node they run). */
uint64_t lsmps_launch_count(void);

/* Profiling hook: launches one kernel of the path `reps` times on the context stream on
 * the current data and returns its mean duration (CUDA events around the launches) and
 * its algorithmic bytes per launch (the traffic a perfect kernel would move):
 *   LSMPS_KB_SPMV64  SELL SpMV + fused dot, FP64 values (plain FP64 solver)   10 nnz + 28.25 U
 *   LSMPS_KB_SPMV32  SELL SpMV + fused dot, FP32 values, FP64 vectors (MIXED)  6 nnz + 28.25 U
 *                    (16-bit column steps and a 32-bit first column per row; with 32-bit
 *                    columns, when a row does not ascend in small steps: 12 / 8 nnz + 24.25 U)
 *   LSMPS_KB_NBR_COUNT / LSMPS_KB_NBR_FILL two-pass neighbor build   24 N + 4 N (+ 4 P + 1 N fill)
 *   LSMPS_KB_NBR_SCAN  single-pass neighbor scan into slot rows + classes   34 N + 4 P
 *   LSMPS_KB_NBR_COMPACT  slot rows packed into the CSR                     4 (N + 1) + 8 P
 *   LSMPS_KB_WLS     all-particle WLS            24 N + 4 P + 80 N (z, sum w, status)
 * No reference counterpart (the reference has no GPU path). */
enum {
    LSMPS_KB_SPMV64 = 0,
    LSMPS_KB_SPMV32 = 1,
    LSMPS_KB_NBR_COUNT = 2,
    LSMPS_KB_NBR_FILL = 3,
    LSMPS_KB_WLS = 4,
    LSMPS_KB_MPNN_LAYER = 5, /* one message-passing layer (aggregation + 64x128 tensor-core GEMM) of the
                               loaded network over the assembled PPE graph: 256 U + 8 Z */
    LSMPS_KB_MG_VCYCLE = 6,  /* one multigrid V-cycle (all its kernels) on the assembled system's
                               hierarchy: 92 U + 464 (rows of the coarse levels) */
    LSMPS_KB_NBR_SCAN = 7,
    LSMPS_KB_NBR_COMPACT = 8,
    LSMPS_KB_FP64_PEAK = 9   /* independent FP64 FMA chains on every SM: the measured FP64 peak; the
                               second output holds FLOPs per launch, not bytes. Needs no data. */
};
int lsmps_kernel_bench(lsmps_ctx* ctx, int kernel, int reps, double* ms_per_launch, double* bytes_per_launch);

/* Launch-shape autotuner. Kernels whose launch shapes (grid size, block size, loads in
 * flight) all give the same bits time each shape once on the live data at their first use
 * per problem-size class (floor(log2 n)) and keep the fastest for the context: the network's
 * message-passing layer and the all-particle WLS. mode 0: off (fixed default shapes), 1: on
 * (default), 2: on and forget earlier choices. No reference counterpart. */
int lsmps_set_autotune(lsmps_ctx* ctx, int mode);
/* The tuner's table as text, one line per candidate: "kernel n~2^k<TAB>shape<TAB>ms[<TAB>best]".
 * Writes at most cap bytes (NUL-terminated) to buf; *needed gets the full size + 1. */
int lsmps_autotune_report(lsmps_ctx* ctx, char* buf, size_t cap, size_t* needed);

/* ---- particles -------------------------------------------------------------------- */
/* xyz: n x 3 doubles (x, y, z interleaved, as the reference's Particle::r); type: n
 * class bytes (only Wall is read by classification, src/lsmps.cpp:27). Host memory. */
int lsmps_upload_particles(lsmps_ctx* ctx, const double* xyz, const uint8_t* type, size_t n);
/* Same from device pointers already on the context's device (no host copy). */
int lsmps_upload_particles_device(lsmps_ctx* ctx, const double* d_xyz, const uint8_t* d_type, size_t n);
/* Double-buffered upload for callers that stream particle sets (the next step's snapshot while
 * this one is processed): lsmps_prefetch_particles enqueues the host-to-device copies of a set
 * (from pinned memory, to overlap) on the context's copy stream and returns without waiting;
 * lsmps_use_prefetched_particles makes it the context's particle set, as lsmps_upload_particles
 * would, ordering the context stream after the copies. The host buffers must stay unchanged
 * until the copies are done (the next lsmps_use_prefetched_particles or lsmps_sync). The copy
 * into the staging buffers waits for the context stream's work enqueued so far, which may still
 * read the set they held. No reference counterpart (the reference generates its particles). */
int lsmps_prefetch_particles(lsmps_ctx* ctx, const double* xyz, const uint8_t* type, size_t n);
int lsmps_use_prefetched_particles(lsmps_ctx* ctx);

/* ---- neighbor build + classification ---------------------------------------------- */
typedef struct lsmps_neighbor_stats {
    uint64_t pairs;          /* kept directed pairs (reference NeighborData::pairs) */
    uint64_t truncated;      /* dropped pairs beyond max_neighbors (NeighborData::truncated) */
    double mean;             /* mean kept count over all particles (Metrics::neighbor_mean) */
    int32_t p50, p90, p99;   /* percentiles cnt[(size_t)(q (N-1))] of the sorted counts */
    int32_t max_count;
    uint64_t type_count[5];  /* particles per class after classification */
    int64_t grid_cells;      /* cells in the dense grid */
    int32_t max_cell_occupancy;
    int32_t reserved;
} lsmps_neighbor_stats;

#define LSMPS_NBR_CLASSIFY 1  /* fuse the 14-direction classification into the neighbor scan */
#define LSMPS_NBR_TWO_PASS 2  /* count pass + fill pass instead of the single pass (same lists; the
                                 single pass needs 4 x max_neighbors bytes per particle of scratch
                                 and falls back to two passes above 4 GB of it) */

/* Uniform-grid neighbor lists, bit-exact with the reference's neighbors()
 * (src/lsmps.cpp:16-18,26): cell = floor(r / re) per axis, 27 cells dz, dy, dx from -1
 * to 1, ascending index within a cell, |rj - ri|^2 < re^2 without FMA contraction, first
 * max_neighbors kept. With LSMPS_NBR_CLASSIFY also classify() (src/lsmps.cpp:27) with l0.
 * re must be the caller's re_ratio * l0 product, as run_benchmark (src/lsmps.cpp:73). With
 * out == NULL the statistics are neither computed nor read back, and the call returns once the
 * lists' last kernels are queued (the host waits only for the pair count, which sizes the
 * lists); its phase time is read later by lsmps_get_timings. */
int lsmps_build_neighbors(lsmps_ctx* ctx, double re, int max_neighbors, double l0, int flags,
                          lsmps_neighbor_stats* out);
/* classify() (src/lsmps.cpp:27) over the current neighbor lists, standalone. */
int lsmps_classify(lsmps_ctx* ctx, double l0, lsmps_neighbor_stats* out);

/* Neighbor lists with a skin (Verlet lists), for step series that move an unchanged particle
 * set. lsmps_build_neighbors_skin builds candidate lists of radius re + skin (at most
 * max_candidates per particle; LSMPS_ERR_ARG if any would be dropped) and from them the exact
 * lists of radius re, as lsmps_build_neighbors does. Then, per step, lsmps_update_positions
 * (same particles, same order) and lsmps_refresh_neighbors re-derive the exact lists by
 * filtering the candidates with the build's own test (src/lsmps.cpp:26): the same neighbor
 * sets as a fresh build, rows in ascending index of the candidate build's numbering.
 * refresh returns LSMPS_ERR_STATE once a particle has moved more than skin / 2 since the
 * candidate build (rebuild then); lsmps_max_displacement reports that distance. No reference
 * counterpart (the reference's cnl_rebuild_interval key is not parsed by it). */
int lsmps_build_neighbors_skin(lsmps_ctx* ctx, double re, double skin, int max_neighbors, int max_candidates,
                               double l0, int flags, lsmps_neighbor_stats* out);
int lsmps_update_positions(lsmps_ctx* ctx, const double* xyz, size_t n);
int lsmps_update_positions_device(lsmps_ctx* ctx, const double* d_xyz, size_t n);
int lsmps_refresh_neighbors(lsmps_ctx* ctx, int flags, lsmps_neighbor_stats* out);
int lsmps_max_displacement(lsmps_ctx* ctx, double* out);

/* ---- WLS -------------------------------------------------------------------------- */
typedef struct lsmps_wls_opts {
    double re, l0;
    double regularization;   /* reference Config::wls_regularization (1e-8) */
    int32_t mode;            /* 0: reference wls_test sample (src/lsmps.cpp:28), bit-exact;
                                1: every particle, nrhs quadratic fields */
    int32_t wls_samples;     /* mode 0: reference Config::wls_samples */
    int32_t nrhs;            /* mode 1: 1..3 fields */
    int32_t precision;       /* mode 1: 0 FP64; 1 FP32 Cholesky + FP64 refinement */
    const double* quad_coef; /* mode 1: nrhs x 10 coefficients of
                                c0 + c1 x + c2 y + c3 z + c4 x^2 + c5 y^2 + c6 z^2 + c7 xy + c8 xz + c9 yz */
    int32_t store_solutions; /* mode 1: keep the n x nrhs x 9 solutions for download */
    int32_t reserved;
} lsmps_wls_opts;

typedef struct lsmps_wls_stats {
    /* reference WlsStats (include/lsmps.hpp:20); mode 1 fills them over all particles
     * and all fields (errors against each field's analytic gradient / Laplacian) */
    uint64_t sampled, ok, regularized, failed, virtual_points;
    double max_gradient_error, rms_gradient_error, max_laplacian_error, rms_laplacian_error;
    uint64_t skipped;        /* Wall / Splash particles */
    uint64_t fp64_fallback;  /* precision 1: systems refactored in FP64 */
} lsmps_wls_stats;

/* wls_test (mode 0) or the all-particle batched WLS (mode 1). Mode 1 also keeps each
 * particle's Laplacian vector z = M^-1 (e3+e4+e5) and sum of weights for the WLS PPE; with
 * out == NULL it returns without reading its statistics back, so the host does not wait for
 * the device (the next call is ordered after it on the context stream). */
int lsmps_wls(lsmps_ctx* ctx, const lsmps_wls_opts* opts, lsmps_wls_stats* out);

/* ---- PPE assembly ----------------------------------------------------------------- */
enum { LSMPS_PPE_REFERENCE = 0, LSMPS_PPE_SHIFTED = 1, LSMPS_PPE_WLS = 2, LSMPS_PPE_LOADED = 3 /* lsmps_ppe_load_csr */ };
/* WLS rows with Neumann walls: wall neighbors take the row particle's own pressure (zero normal
 * gradient), so they add neither an entry nor a diagonal term; without it walls are Dirichlet
 * neighbors like the free surface. No reference counterpart in 3-D (the reference's 2-D step
 * mirrors the wall value: python/rain_plate_lsmps_cpu.py:90-100,179). */
#define LSMPS_PPE_WALL_NEUMANN 1

typedef struct lsmps_ppe_opts {
    int32_t variant;         /* LSMPS_PPE_* */
    int32_t flags;           /* LSMPS_PPE_WALL_NEUMANN (variant WLS only) */
    int64_t max_unknowns;    /* reference Config::ppe_max_unknowns */
    double re, l0;
    double diag_shift;       /* SHIFTED / WLS: diagonal times (1 + diag_shift) */
} lsmps_ppe_opts;

typedef struct lsmps_ppe_stats {
    /* reference PpeStats (include/lsmps.hpp:21) */
    uint64_t unknowns, nnz, dirichlet, neumann, failed_rows;
    int32_t iterations, converged;
    double initial_residual, final_residual, relative_l2_error, max_error, assembly_ms, solve_ms;
    /* final_residual is |b - A x| in FP64; for a converged MIXED or LEARNED solve it is the
     * convergence test's own FP64 residual of the final iterate, |b - (A D^-1)(D x)|, the same
     * quantity up to rounding (no further SpMV) */
    /* extensions */
    int32_t outer_iterations;   /* FP64 refinement sweeps (mixed / learned) */
    int32_t fallback;           /* 1 when the solve continued as Jacobi MIXED: LEARNED after a stall or a
                                   discarded guess, MULTIGRID after a stall or a breakdown */
    double relative_residual;   /* |b - Ax| / |b| at exit (FP64) */
} lsmps_ppe_stats;

/* assemble_ppe (src/lsmps.cpp:30-64) and its variants; keeps A, b = A p*, p* on the device.
 * With out == NULL the call returns once the matrix's last kernel is queued (the host waits
 * only for the unknown and nonzero counts); its phase time is read by lsmps_get_timings or
 * reported by the next lsmps_ppe_solve. */
int lsmps_ppe_assemble(lsmps_ctx* ctx, const lsmps_ppe_opts* opts, lsmps_ppe_stats* out);

/* A caller's sparse system in place of an assembled PPE, for the solvers and kernel benches
 * (e.g. the synthetic CSR that the reference's python/workload_calibration.py:253-301 writes):
 * host CSR with n rows, row_ptr (n + 1, 64-bit), col (row_ptr[n] entries, any order,
 * duplicates allowed; entries on the diagonal are summed into it), val (NULL: -1 for every
 * off-diagonal entry and a diagonal of (off-diagonal count) (1 + 1e-3), at least 1), b (NULL:
 * b = A 1, and the error statistics measure against p* = 1). Rows are the unknowns in the given
 * numbering. The learned solver and the per-particle calls refuse a loaded system. */
int lsmps_ppe_load_csr(lsmps_ctx* ctx, const int64_t* row_ptr, const int32_t* col, const double* val,
                       const double* b, size_t n, lsmps_ppe_stats* out);

/* ---- PPE solve -------------------------------------------------------------------- */
enum {
    LSMPS_SOLVER_REFERENCE = 0, /* bit-identical to the reference's FP64 BiCGStab (src/lsmps.cpp:67):
                                   sequential-order dot products; for small systems */
    LSMPS_SOLVER_FP64 = 1,      /* the reference iteration in FP64, GPU reductions */
    LSMPS_SOLVER_JACOBI = 2,    /* FP64, Jacobi right preconditioning */
    LSMPS_SOLVER_MIXED = 3,     /* Jacobi BiCGStab, FP64 vectors, FP32 matrix in the iteration's SpMVs,
                                   FP64 true-residual replacement every `inner_tol` drop */
    LSMPS_SOLVER_LEARNED = 4,   /* MIXED started from the message-passing network's guess; plain
                                   Jacobi continuation when the residual stalls */
    LSMPS_SOLVER_MIXED_F32 = 5  /* FP32 vectors and matrix, FP64 solution and residual refinement */
};

/* Right preconditioner of MIXED and LEARNED (lsmps_solver_opts.precond; the other solvers take
 * only JACOBI). MULTIGRID: a cell-aggregation multigrid V-cycle in FP32. Level 1 has one
 * aggregate per neighbor-grid cell; each coarser level groups 2x2x2 blocks of the level below.
 * Coarse operators are the Galerkin products, stored as 27-slot stencils. One Jacobi sweep
 * smooths each level; the coarsest level (at most 256 rows, or 640 from level 3 on) gets 10
 * sweeps. It is rebuilt after each assembly (its setup time is in solve_ms). No reference
 * counterpart: the reference's BiCGStab (src/lsmps.cpp:67) is unpreconditioned. Not for loaded
 * CSR systems, which have no cells. Opt-in: cell aggregates ignore connection strength, so
 * systems with weakly coupled particles or strong row contrasts can need more iterations than
 * JACOBI. A multigrid run that stalls (stall_window) or breaks down continues as Jacobi MIXED
 * from its iterate (from zero if that is no longer finite) and reports fallback = 1. With
 * LEARNED and no warm start the hierarchy is built on the context's side stream while the
 * network runs on the context stream (the set-up reads level sizes back to the host; the
 * network fills the GPU meanwhile); the result is the same bits. */
enum {
    LSMPS_PRECOND_JACOBI = 0,
    LSMPS_PRECOND_MULTIGRID = 1
};

typedef struct lsmps_solver_opts {
    int32_t solver;          /* LSMPS_SOLVER_* */
    int32_t max_iter;        /* total BiCGStab iterations (inner ones for MIXED / LEARNED) */
    double tol;              /* converged when |r| <= tol * max(1, |b|) (src/lsmps.cpp:67) */
    int32_t warm_start;      /* start from the last solution held by the context */
    int32_t use_graph;       /* FP64 / JACOBI / MIXED / LEARNED: 1 (default) the whole iteration loop as one
                                CUDA graph whose WHILE node repeats check_every iterations and the
                                replacement / restart / stop decisions on the device (no host round
                                trip per solve); 2 graphs of check_every iterations launched from a
                                host loop that makes the decisions; 0 eager launches, same host loop.
                                All three run the same kernels in the same order (same bits). */
    double inner_tol;        /* MIXED / LEARNED: residual drop between FP64 residual replacements
                                (default 0.01); MIXED_F32: the same (default 0.1) */
    int32_t inner_max_iter;  /* reserved */
    int32_t stall_window;    /* LEARNED / MULTIGRID: iterations without 1 % progress of |r| before the
                                fallback to Jacobi MIXED (default 20) */
    int32_t check_every;     /* iterations between host convergence checks (default 8) */
    int32_t precond;         /* LSMPS_PRECOND_* (MIXED / LEARNED; default JACOBI) */
} lsmps_solver_opts;

int lsmps_ppe_solve(lsmps_ctx* ctx, const lsmps_solver_opts* opts, lsmps_ppe_stats* out);

/* The multigrid hierarchy of the assembled system, built by the last multigrid solve (or by
 * lsmps_mg_apply): the number of coarse levels, the rows of levels 0 (the unknowns) .. levels
 * (up to `cap` entries) and its setup time. lsmps_mg_apply: out = D M z for one host vector
 * of U values in the reference's unknown numbering (D the diagonal of A, M the V-cycle), the
 * operator the solvers apply in their iteration on y = D x. No reference counterpart. */
int lsmps_mg_info(lsmps_ctx* ctx, int32_t* levels, int64_t* rows, int32_t cap, double* setup_ms);
int lsmps_mg_apply(lsmps_ctx* ctx, const double* z, double* out, size_t u);

/* ---- downloads (host buffers, caller's particle / unknown order) ------------------- */
int lsmps_download_types(lsmps_ctx* ctx, uint8_t* type, size_t n);
/* row_ptr: n + 1; col: pairs entries (original particle indices, reference order). */
int lsmps_download_neighbors(lsmps_ctx* ctx, int32_t* row_ptr, int32_t* col, size_t col_cap);
/* mode-1 WLS: x (n x nrhs x 9, if stored), status (n: 0 ok, 1 regularised, 2 skipped,
 * 3 sum w <= 0, 4 Cholesky failed), z (n x 9), wsum (n). Any pointer may be NULL. */
int lsmps_download_wls(lsmps_ctx* ctx, double* x, int32_t* status, double* z, double* wsum);
/* PPE in the reference's numbering (unknown rank in particle order): row (U+1), col, val
 * (nnz), b, p* (U), unknown_particle (U). Any pointer may be NULL. */
int lsmps_download_ppe(lsmps_ctx* ctx, int32_t* row, int32_t* col, double* val, double* b,
                       double* x_exact, int32_t* unknown_particle);
/* Solution of the last solve (U, reference numbering). */
int lsmps_download_pressure(lsmps_ctx* ctx, double* p, size_t u);
/* The same download without waiting for it: the values are reordered on the context stream
 * and copied to `p` on the context's copy stream, so a time loop can start its next step while
 * the result travels. `p` must be page-locked host memory to overlap, and must stay valid and
 * unread until lsmps_download_wait returns (or the next asynchronous download, which orders
 * itself after the previous copy, has been waited for). lsmps_download_wait blocks until the
 * last asynchronous download has landed (at once when none is pending). No reference
 * counterpart (the reference's solution lives in host memory, src/lsmps.cpp:67). */
int lsmps_download_pressure_async(lsmps_ctx* ctx, double* p, size_t u);
int lsmps_download_wait(lsmps_ctx* ctx);

/* Per-particle pressure (n values, caller order) for step series whose unknowns change from
 * step to step. set_initial_pressure: the next lsmps_ppe_solve with warm_start = 1 starts from
 * these values at the unknowns (call after lsmps_ppe_assemble). download_pressure_particles:
 * the last solution at the unknowns' particles, `fill` at the others (NaN: the others keep the
 * values the buffer holds). No reference counterpart (the reference solves one snapshot from
 * zero, src/lsmps.cpp:67). */
int lsmps_set_initial_pressure(lsmps_ctx* ctx, const double* p, size_t n);
int lsmps_set_initial_pressure_device(lsmps_ctx* ctx, const double* d_p, size_t n);
int lsmps_download_pressure_particles(lsmps_ctx* ctx, double* p, size_t n, double fill);
int lsmps_download_pressure_particles_device(lsmps_ctx* ctx, double* d_p, size_t n, double fill);

/* ---- manufactured right-hand sides ------------------------------------------------ */
/* p* = c0 + sum_m a_m sin(kx_m x + ky_m y + kz_m z + phi_m) + gz z over the unknowns'
 * particle positions, b = A p* (the reference's discrete manufactured solution,
 * src/lsmps.cpp:59-61, with a caller-chosen smooth field). params: c0, gz, then nmodes x
 * (a, kx, ky, kz, phi). No reference counterpart beyond the fixed p* of the variants. */
int lsmps_ppe_manufacture(lsmps_ctx* ctx, const double* params, int nmodes);

/* ---- residual check that allocates nothing ------------------------------------------ */
/* No counterpart in the reference. out[v] = |b - A p_v|_2 for the nvec (1..8) device
 * vectors p_v = d_p + v * ld (U doubles each, the reference's unknown numbering), and
 * out[nvec] = |b|_2, written to the device buffer d_out (nvec + 1 doubles), over the
 * assembled system. Enqueued on the context stream (lsmps_stream) and returns without
 * waiting: order the producer of d_p before it and read d_out after lsmps_sync.
 * It allocates nothing: no cudaMalloc / cudaFree and no context buffer growth. It is for
 * callers that keep the pressure in their own device memory and check it inside a time
 * loop that overlaps work on other streams, where an allocation would synchronise the
 * device, or whose device memory is already in their own pool. The reduction scratch is
 * one static device array of 42,880 bytes per device (partial sums of at most 592 blocks
 * for at most 8 vectors); nvec outside 1..8 fails with LSMPS_ERR_ARG. Its ticket word must
 * start at zero: each call clears it on the stream before the launch. Every call resolves
 * the array's address on the context's device (cudaGetSymbolAddress, checked; nothing is
 * cached, so a device reset between calls is harmless). The first call on a device may load
 * the module, so make that first call before any stream capture begins. The scratch is shared
 * by every context on the device: calls whose executions overlap in time (two contexts, two
 * streams, two threads) race on it and must be serialised by the caller. */
int lsmps_ppe_residual_static(lsmps_ctx* ctx, const double* d_p, size_t ld, int nvec, double* d_out);

/* ---- WLS of caller fields, pressure projection ------------------------------------ */
/* The all-particle WLS (mode 1 moments, FP64) of nfields (1..3) per-particle fields given in
 * device memory (n x nfields, caller order): out (n x nfields x 9, caller order) holds per
 * particle and field the WLS solution (df/dx, df/dy, df/dz, l0 d2f/dx2, l0 d2f/dy2,
 * l0 d2f/dz2, l0 d2f/dxdy, l0 d2f/dxdz, l0 d2f/dydz), as the reference's wls_test solves for
 * its quadratic (src/lsmps.cpp:28), with f_j - f_i from the array; zeros where the WLS is
 * skipped (wall, splash) or failed. Needs neighbor lists and classes. */
int lsmps_wls_fields(lsmps_ctx* ctx, const double* d_fields, int nfields, double* d_out);

typedef struct lsmps_projection_stats {
    uint64_t unknowns;       /* PPE unknowns */
    uint64_t measured;       /* particles the divergence statistics cover (the unknowns) */
    double div_before_rms, div_before_max;  /* div u* */
    double div_after_rms, div_after_max;    /* div u after the correction */
    int32_t iterations, converged;
    double relative_residual, solve_ms, total_ms;
    uint64_t core;           /* Interior unknowns at least 3 neighbor hops from any other particle */
    double div_core_before_rms, div_core_after_rms;  /* over the core */
    /* the wall bands: unknowns 1 (band 1) or 2 (band 2) neighbor hops from a wall particle and
       at least 3 hops from any free-surface or splash particle */
    uint64_t wall_band1, wall_band2;
    double div_wall1_before_rms, div_wall1_after_rms, div_wall2_before_rms, div_wall2_after_rms;
} lsmps_projection_stats;

/* One pressure projection (the reference's 2-D python/rain_plate_lsmps_cpu.py:202-260 in
 * 3-D): div u* from lsmps_wls_fields of the velocity, the assembled WLS-Laplacian PPE (variant
 * LSMPS_PPE_WLS; free-surface / splash Dirichlet p = 0) solved with opts for
 * lap p = rho / dt div u* (b = -rho / dt div u*, as A ~ -lap), and u = u* - dt / rho grad p
 * (walls keep u*). With a PPE assembled with LSMPS_PPE_WALL_NEUMANN the walls are Neumann
 * boundaries: in the divergence, the pressure gradient and the PPE rows, wall neighbors take
 * the particle's own value (zero normal gradient), the mirrored wall value of the reference's
 * virtual points (python/rain_plate_lsmps_cpu.py:90-100,179); the wall particles themselves
 * serve as the mirrored points in the moment matrices. d_vel / d_vel_out: n x 3 device arrays,
 * caller order; d_pressure: n values, 0 off the unknowns. Overwrites the assembled b (and p*
 * with 0). */
int lsmps_projection_step(lsmps_ctx* ctx, const double* d_vel, double dt, double rho, const lsmps_solver_opts* opts,
                          double* d_vel_out, double* d_pressure, lsmps_projection_stats* out);
/* The viscous and gravity predictor of the fractional-step scheme (the reference's 2-D
 * provisional_velocity, python/rain_plate_lsmps_cpu.py:184-196, in 3-D): u* = u + dt (nu lap u
 * + gravity) with lap u of each component from the all-particle WLS of the velocity,
 * (x3 + x4 + x5) / l0; walls keep u; splash particles (no WLS) fall freely (u + dt gravity).
 * d_vel / d_vel_out: n x 3 device arrays, caller order; gravity: 3 host doubles; flags:
 * LSMPS_PPE_WALL_NEUMANN gives wall neighbors the particle's own velocity in the WLS (the
 * mirrored wall value). Needs neighbor lists and classes. */
int lsmps_predict_velocity(lsmps_ctx* ctx, const double* d_vel, double dt, double nu, const double* gravity, int flags,
                           double* d_vel_out);

/* ---- step series (rain-on-plate proxy) ------------------------------------------------ */
/* A 3-D step series on one context: wall fixed, droplets fall droplet_speed l0 per step and
 * join the film at film_thickness l0 above the plate, the film slides film_speed l0 per step
 * down the plate (angle theta_deg, plate frame of the rain_plate generator), particles past
 * the plate's lower edge (the outflow plane) leave, injected_per_step particles arrive per
 * step as droplets of droplet_radius l0 at heights inject_hmin..inject_hmax l0 above the
 * plate. Every step runs neighbor lists (lsmps_build_neighbors_skin every
 * cnl_rebuild_interval steps or when the skin no longer covers the motion, the refresh in
 * between), classification, all-particle WLS, the WLS-Laplacian PPE and the solve, warm-started
 * from the previous step's pressure per particle. Injected droplets join and flagged
 * outflow particles leave at rebuild steps. The fluid count is taken on the device each step
 * and compared with initial + injected - deleted (mass_balance, 0 when conserved). The
 * reference's series is the 2-D python/rain_plate_cpu.py baseline (inject:67-87,
 * remove_outflow:146-154); its C++ benchmark ignores these keys of config/rain_injection.cfg. */
typedef struct lsmps_series lsmps_series;
typedef struct lsmps_series_params {
    int32_t steps;                /* informational: steps the caller will run */
    int32_t injected_per_step;    /* config key injected_per_step */
    int32_t cnl_rebuild_interval; /* config key cnl_rebuild_interval */
    int32_t solver;               /* LSMPS_SOLVER_FP64 .. LSMPS_SOLVER_MIXED_F32 */
    double l0, re;                /* spacing; support radius in l0 (re_ratio) */
    double skin;                  /* candidate skin in l0 */
    double droplet_speed;         /* l0 per step */
    double film_speed;            /* l0 per step */
    double theta_deg;             /* plate angle */
    double film_thickness;        /* l0 */
    double droplet_radius;        /* l0 */
    double inject_hmin, inject_hmax; /* l0 above the plate */
    double tol;                   /* PPE tolerance as lsmps_solver_opts.tol */
    int32_t max_iter;
    int32_t max_neighbors;
    int32_t max_candidates;
    int32_t wls_precision;        /* 0 FP64, 1 FP32 + FP64 refinement */
    int32_t warm_start;           /* 1: start each solve from the previous pressure */
    uint32_t seed;                /* injection positions */
    int32_t precond;              /* LSMPS_PRECOND_* for the MIXED and LEARNED solvers */
    int32_t reserved;
} lsmps_series_params;

typedef struct lsmps_series_stats {
    int32_t step, rebuilt, forced_rebuild, converged;
    uint64_t particles;           /* the set the PPE sees */
    uint64_t in_flight;           /* injected, joining at the next rebuild */
    uint64_t flagged;             /* past the outflow plane, leaving at the next rebuild */
    uint64_t injected_total, deleted_total;
    uint64_t fluid_particles;     /* counted on the device: set + in flight, not wall */
    int64_t mass_balance;         /* fluid_particles - (initial fluid + injected - deleted) */
    uint64_t pairs, unknowns, nnz;
    int32_t iterations, outer_iterations, fallback, reserved;
    double fluid_volume;          /* fluid_particles x l0^3 */
    double max_displacement;      /* since the last candidate build */
    double relative_l2_error;     /* |x - p*| / |p*| of this step's PPE */
    double relative_residual;
    double neighbor_ms, wls_ms, assembly_ms, solve_ms, step_ms;
} lsmps_series_stats;

/* Rain validation outputs of each step, the reference's schema (python/rain_plate_cpu.py
 * compute_window_metrics:182-213, compute_section_crossings:216-239, validated by
 * python/validate_outputs.py): plate coordinate u = 1 - s / L (0 at the upper edge, 1 at the
 * outflow edge, s along the plate, L its length), normal distance d above the plate surface.
 * Window w: fluid particles with lo <= u < hi and 0 <= d <= wet_distance_factor l0, binned in
 * coverage_cells cells along u; coverage = share of cells holding at least
 * min_particles_per_cell; film thickness per occupied cell = max d + l0, and its mean, 90th
 * percentile (linear interpolation) and maximum. Section: particles whose u went from below to
 * at least section_u this step with 0 <= d <= max normal distance l0. Defaults: the reference's
 * config/rain_plate_validation.json. */
#define LSMPS_RAIN_MAX_WINDOWS 8
#define LSMPS_RAIN_MAX_SECTIONS 8
#define LSMPS_RAIN_MAX_CELLS 64
typedef struct lsmps_rain_validation {
    int32_t nwindows, nsections, coverage_cells, min_particles_per_cell;
    double wet_distance_factor;
    double window_lo[LSMPS_RAIN_MAX_WINDOWS], window_hi[LSMPS_RAIN_MAX_WINDOWS];
    double section_u[LSMPS_RAIN_MAX_SECTIONS], section_max_normal[LSMPS_RAIN_MAX_SECTIONS];
} lsmps_rain_validation;

typedef struct lsmps_rain_outputs {
    uint64_t window_particles[LSMPS_RAIN_MAX_WINDOWS];
    double window_coverage[LSMPS_RAIN_MAX_WINDOWS];
    double film_mean[LSMPS_RAIN_MAX_WINDOWS], film_p90[LSMPS_RAIN_MAX_WINDOWS], film_max[LSMPS_RAIN_MAX_WINDOWS];
    uint64_t section_crossings[LSMPS_RAIN_MAX_SECTIONS];
} lsmps_rain_outputs;

/* xyz / type: the initial particles (host, as lsmps_upload_particles; Wall marks the plate).
 * The series borrows ctx (and its network for LSMPS_SOLVER_LEARNED) until destroyed. */
int lsmps_series_create(lsmps_ctx* ctx, const lsmps_series_params* params, const double* xyz, const uint8_t* type,
                        size_t n, lsmps_series** out);
int lsmps_series_step(lsmps_series* series, lsmps_series_stats* out);
/* The current particle set (host): positions n x 3, material (0 wall, 1 film, 2 droplet),
 * pressure; any pointer may be NULL; *n gets the count. */
int lsmps_series_particles(lsmps_series* series, double* xyz, uint8_t* material, double* pressure, size_t cap,
                           size_t* n);
void lsmps_series_destroy(lsmps_series* series);
/* Replace the validation windows and sections (takes effect at the next step). */
int lsmps_series_set_validation(lsmps_series* series, const lsmps_rain_validation* cfg);
/* The validation outputs of the last step. */
int lsmps_series_rain_outputs(lsmps_series* series, lsmps_rain_outputs* out);

/* ---- learned preconditioner (message-passing network over the PPE graph) ----------- */
/* No reference counterpart (this library's learned preconditioner). Nodes are the PPE unknowns, edges the
 * off-diagonal entries with weight -a_ij / a_ii. Input features per node: residual
 * (unit-norm residual times sqrt(U)), diagonal a_ii / mean(a) - 1, NearWall flag,
 * row length / 32 - 1. Encoder 4 -> 64 (ReLU); three residual message-passing layers
 * h += ReLU(W_l [h | sum_j w_ij h_j] + b_l), W_l 64 x 128; decoder 64 -> 1; output y / sqrt(U)
 * is the guess for the Jacobi-scaled solution y = D A^-1 r of the unit residual r.
 * Activations and weights BF16, accumulation FP32 (tensor-core mma). FP32 master weights
 * in this order: W_enc[64][4], b_enc[64], 3 x (W_l[64][128], b_l[64]), w_dec[64], b_dec. */
#define LSMPS_MPNN_HIDDEN 64
#define LSMPS_MPNN_LAYERS 3
#define LSMPS_MPNN_FEATURES 4
size_t lsmps_mpnn_param_count(void);

typedef struct lsmps_mpnn_train_opts {
    int32_t steps;           /* optimiser steps */
    int32_t batch;           /* samples accumulated per step */
    float lr;                /* Adam learning rate */
    float weight_decay;      /* decoupled weight decay */
    uint32_t seed;           /* sample order */
    int32_t loss;            /* 0: error |y - t|^2 / |t|^2; 1: residual |r - A D^-1 y|^2 / |r|^2; 2: both */
} lsmps_mpnn_train_opts;

/* Initialise the weights from a seed (He-scaled normals; residual branches scaled down). */
int lsmps_mpnn_init(lsmps_ctx* ctx, uint32_t seed);
int lsmps_mpnn_get_weights(lsmps_ctx* ctx, float* w, size_t n);
int lsmps_mpnn_set_weights(lsmps_ctx* ctx, const float* w, size_t n);
/* Store a training pair from the current state: input b / |b| of the assembled system,
 * target D x / |b| with x the last solution. The graph is stored once per assembly. */
int lsmps_mpnn_add_sample(lsmps_ctx* ctx);
int lsmps_mpnn_clear_samples(lsmps_ctx* ctx);
int lsmps_mpnn_sample_count(lsmps_ctx* ctx);
/* Loss of stored sample `index` (the kind last used by lsmps_mpnn_train; error loss
 * before any training) and its gradient (FP32, parameter order above; grad may be NULL). */
int lsmps_mpnn_grad(lsmps_ctx* ctx, int index, float* grad, float* loss);
/* Adam on the stored samples; loss_out: mean loss of the last `batch` samples. */
int lsmps_mpnn_train(lsmps_ctx* ctx, const lsmps_mpnn_train_opts* opts, float* loss_out);
/* y = net(r) on the current assembled system (reference numbering, U entries each). */
int lsmps_mpnn_infer(lsmps_ctx* ctx, const double* r, double* y);
int lsmps_mpnn_save(lsmps_ctx* ctx, const char* path);
int lsmps_mpnn_load(lsmps_ctx* ctx, const char* path);

/* ---- host helpers (no GPU) --------------------------------------------------------- */
/* Parse a .cfg file and generate its particle set with the library's generate_case
 * (bit-identical to the reference's for the reference's cases). Two calls: first with
 * xyz == NULL for *n, then with buffers of n. Extra key=value overrides ("k=v;k=v"). */
int lsmps_host_generate(const char* cfg_path, const char* overrides, double* xyz, uint8_t* type,
                        double* uvw, size_t* n);

#ifdef __cplusplus
}
#endif
#endif /* LSMPS_GPU_H */
