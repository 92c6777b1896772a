// Internal entry points of the library's phases (called by the C ABI in capi.cu).
#pragma once
#include <functional>

#include "ctx.cuh"

namespace lsmps_gpu {

// neighbors.cu
void particles_upload(lsmps_ctx* ctx, const double* xyz, const uint8_t* type, size_t n, bool device);
void series_create(lsmps_ctx* ctx, const lsmps_series_params* p, const double* xyz, const uint8_t* type, size_t n,
                   lsmps_series** out);
void series_step(lsmps_series* s, lsmps_series_stats* out);
void series_particles(lsmps_series* s, double* xyz, uint8_t* material, double* pressure, size_t cap, size_t* n);
void series_destroy(lsmps_series* s);
void series_set_validation(lsmps_series* s, const lsmps_rain_validation* v);
void series_rain_outputs(lsmps_series* s, lsmps_rain_outputs* out);
lsmps_ctx* series_context(lsmps_series* s);
void nb_build(lsmps_ctx* ctx, double re, int maxn, double l0, int flags, lsmps_neighbor_stats* out);
void nb_classify(lsmps_ctx* ctx, double l0, lsmps_neighbor_stats* out);
// Neighbor statistics (one read-back; with `where`, the device error flags in the same one).
void nb_stats(lsmps_ctx* ctx, lsmps_neighbor_stats* out, const char* where = nullptr);
void nb_download(lsmps_ctx* ctx, int32_t* row_ptr, int32_t* col, size_t col_cap);
void nb_download_types(lsmps_ctx* ctx, uint8_t* type, size_t n);
void nb_build_skin(lsmps_ctx* ctx, double re, double skin, int maxn, int maxc, double l0, int flags,
                   lsmps_neighbor_stats* out);
void nb_refresh(lsmps_ctx* ctx, int flags, lsmps_neighbor_stats* out);
// the exact lists from the candidate lists in one pass (slot rows, compaction), with the
// classes when `classify`; false (nothing done) when the slot rows exceed their budget
bool nb_filter_single(lsmps_ctx* ctx, int classify);
double nb_max_displacement(lsmps_ctx* ctx);
void nb_update_positions(lsmps_ctx* ctx, const double* xyz, size_t n, bool device);

// wls.cu
void wls_run(lsmps_ctx* ctx, const lsmps_wls_opts* opts, lsmps_wls_stats* out);
void wls_download(lsmps_ctx* ctx, double* x, int32_t* status, double* z, double* wsum);
void wls_fields(lsmps_ctx* ctx, const double* d_fields, int nrhs, double* d_out, bool mirror_walls = false);
void projection_step(lsmps_ctx* ctx, const double* d_vel, double dt, double rho, const lsmps_solver_opts* so,
                     double* d_vel_out, double* d_pressure, lsmps_projection_stats* out);
void predict_velocity(lsmps_ctx* ctx, const double* d_vel, double dt, double nu, const double* g, int flags,
                      double* d_vel_out);

// ppe.cu
void ppe_assemble(lsmps_ctx* ctx, const lsmps_ppe_opts* opts, lsmps_ppe_stats* out);
void ppe_load_csr(lsmps_ctx* ctx, const int64_t* row_ptr, const int32_t* col, const double* val, const double* b,
                  size_t n, lsmps_ppe_stats* out);
void ppe_download(lsmps_ctx* ctx, int32_t* row, int32_t* col, double* val, double* b, double* xe,
                  int32_t* unknown_particle);

// solver.cu
void ppe_solve(lsmps_ctx* ctx, const lsmps_solver_opts* opts, lsmps_ppe_stats* out);
void ppe_download_pressure(lsmps_ctx* ctx, double* p, size_t u);
void ppe_download_pressure_async(lsmps_ctx* ctx, double* p, size_t u);
void ppe_download_wait(lsmps_ctx* ctx);
void ppe_set_initial_particles(lsmps_ctx* ctx, const double* pp, size_t n, bool device);
void ppe_pressure_particles(lsmps_ctx* ctx, double* pp, size_t n, double fill, bool device);

// mpnn.cu
bool mpnn_ready(lsmps_ctx* ctx);
void mpnn_destroy(lsmps_ctx* ctx);
size_t mpnn_param_count();
void mpnn_init(lsmps_ctx* ctx, uint32_t seed);
void mpnn_get_weights(lsmps_ctx* ctx, float* w, size_t n);
void mpnn_set_weights(lsmps_ctx* ctx, const float* w, size_t n);
void mpnn_add_sample(lsmps_ctx* ctx);
void mpnn_clear_samples(lsmps_ctx* ctx);
int mpnn_sample_count(lsmps_ctx* ctx);
void mpnn_grad(lsmps_ctx* ctx, int index, float* grad, float* loss);
void mpnn_train(lsmps_ctx* ctx, const lsmps_mpnn_train_opts* opts, float* loss);
void mpnn_infer(lsmps_ctx* ctx, const double* r, double* y);
void mpnn_warm_start(lsmps_ctx* ctx, const float* rhs, float* y);
void mpnn_save(lsmps_ctx* ctx, const char* path);
void mpnn_load(lsmps_ctx* ctx, const char* path);
void ppe_manufacture(lsmps_ctx* ctx, const double* params, int nmodes);
void ppe_residual_static(lsmps_ctx* ctx, const double* d_p, size_t ld, int nvec, double* d_out);

// multigrid.cu: the cell-aggregation V-cycle preconditioner (out = D M z, gated by the
// solver scalars; need_s also skips once the |s| test has passed; restricted: the caller
// has already written the level-1 right-hand side P^T z)
struct BcgScalars;
void mg_setup(lsmps_ctx* ctx);
void mg_apply(lsmps_ctx* ctx, const double* z, double* out, const BcgScalars* S, int need_s,
              bool restricted = false);
int mg_launches_per_apply(lsmps_ctx* ctx, bool restricted = false);
void mg_destroy(lsmps_ctx* ctx);
void mg_info(lsmps_ctx* ctx, int* levels, int64_t* rows, int cap, double* setup_ms);
void mg_apply_host(lsmps_ctx* ctx, const double* z, double* out, size_t n);

// Profiling hooks behind lsmps_kernel_bench (mean ms per launch, algorithmic bytes).
void nb_kernel_bench(lsmps_ctx* ctx, int kernel, int reps, double* ms, double* bytes);
void wls_kernel_bench(lsmps_ctx* ctx, int reps, double* ms, double* bytes);
void fp64_peak_bench(lsmps_ctx* ctx, int reps, double* ms, double* flops);
void solver_kernel_bench(lsmps_ctx* ctx, int kernel, int reps, double* ms, double* bytes);
void mpnn_kernel_bench(lsmps_ctx* ctx, int reps, double* ms, double* bytes);
void mg_kernel_bench(lsmps_ctx* ctx, int reps, double* ms, double* bytes);

// Timing helpers: record event `slot` on the context stream.
// Launch-shape autotuner. For a kernel whose candidate launch shapes all compute the same
// bits and whose launches are idempotent: at the first call for (kernel, size class of n =
// floor(log2 n)) each candidate is launched once to warm and `reps` times between CUDA events
// on the context stream, and the fastest is kept in the context. Returns the candidate to
// launch. With tuning off or while the stream is captured it returns the stored choice if
// any, else `fallback`. launch(c) enqueues candidate c on the context stream.
int autotune(lsmps_ctx* ctx, const char* kernel, long long n, const std::vector<std::string>& names, int fallback,
             const std::function<void(int)>& launch, int reps = 2);
std::string autotune_report(lsmps_ctx* ctx);

void ev_record(lsmps_ctx* ctx, int slot);
double ev_elapsed(lsmps_ctx* ctx, int a, int b);
// Reads the phase times of calls that did not wait (statistics not requested).
void resolve_timings(lsmps_ctx* ctx);

}  // namespace lsmps_gpu
