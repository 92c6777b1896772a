// The C ABI of lsmps_gpu.h: argument checks, exception-to-status translation, context
// lifetime, uploads and phase timing. The phases live in neighbors.cu, wls.cu, ppe.cu,
// solver.cu and mpnn.cu.
#include <atomic>
#include <cstring>
#include <new>

#include "ops.cuh"

namespace lsmps_gpu {

static std::atomic<uint64_t> g_launches{0};
void note_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void* pinned_ensure(lsmps_ctx* ctx, size_t bytes) {
    if (bytes > ctx->pinned_bytes) {
        if (ctx->pinned) cudaFreeHost(ctx->pinned);
        ctx->pinned = nullptr;
        ctx->pinned_bytes = 0;
        if (cudaMallocHost(&ctx->pinned, bytes) != cudaSuccess) {
            cudaGetLastError();
            throw Error{LSMPS_ERR_ALLOC, "pinned host allocation failed"};
        }
        ctx->pinned_bytes = bytes;
    }
    return ctx->pinned;
}

// Clears the device error flags and throws the error that set flag f names.
static void raise_device_flags(lsmps_ctx* ctx, int f, const char* where) {
    LSMPS_CUDA(cudaMemsetAsync(ctx->dflags.get<int>(), 0, sizeof(int), ctx->stream));
    std::string w(where);
    if (f & DFLAG_NONFINITE) throw Error{LSMPS_ERR_NONFINITE, w + ": non-finite particle position"};
    if (f & DFLAG_CELL_OVERFLOW) throw Error{LSMPS_ERR_GRID, w + ": a cell holds more than 8192 particles"};
    if (f & DFLAG_INDEX) throw Error{LSMPS_ERR_OVERFLOW, w + ": a count exceeds the int32 range"};
    if (f & DFLAG_TIMEOUT) throw Error{LSMPS_ERR_TIMEOUT, w + ": a bounded device wait expired"};
    if (f & DFLAG_STENCIL) throw Error{LSMPS_ERR_GRID, w + ": a coupling spans more than one neighbor cell"};
    throw Error{LSMPS_ERR_CUDA, w + ": device error flag " + std::to_string(f)};
}

void check_device_flags(lsmps_ctx* ctx, const char* where) { read_back(ctx, {}, where); }

void read_back(lsmps_ctx* ctx, std::initializer_list<ReadBack> items, const char* where) {
    auto span = [](size_t b) { return (b + 15) & ~(size_t)15; };
    size_t total = 16;
    for (const ReadBack& r : items) total += span(r.bytes);
    char* pin = static_cast<char*>(pinned_ensure(ctx, total));
    cudaStream_t s = ctx->stream;
    if (where) LSMPS_CUDA(cudaMemcpyAsync(pin, ctx->dflags.get<int>(), sizeof(int), cudaMemcpyDeviceToHost, s));
    size_t off = 16;
    for (const ReadBack& r : items) {
        if (r.bytes) LSMPS_CUDA(cudaMemcpyAsync(pin + off, r.src, r.bytes, cudaMemcpyDeviceToHost, s));
        off += span(r.bytes);
    }
    LSMPS_CUDA(cudaStreamSynchronize(s));
    off = 16;
    for (const ReadBack& r : items) {
        if (r.bytes) std::memcpy(r.dst, pin + off, r.bytes);
        off += span(r.bytes);
    }
    if (!where) return;
    int f = 0;
    std::memcpy(&f, pin, sizeof(int));
    if (f) raise_device_flags(ctx, f, where);
}

void ev_record(lsmps_ctx* ctx, int slot) { LSMPS_CUDA(cudaEventRecord(ctx->ev[slot], ctx->stream)); }

void resolve_timings(lsmps_ctx* ctx) {
    if (ctx->timing_pending & 2u) ctx->timings[1] = ev_elapsed(ctx, 2, 3);
    if (ctx->timing_pending & 8u) ctx->timings[3] = ev_elapsed(ctx, 6, 7);
    if (ctx->timing_pending & 16u) {
        ctx->timings[4] = ctx->ppe_assembly.assembly_ms = ev_elapsed(ctx, 8, 9);
    }
    ctx->timing_pending = 0;
}

double ev_elapsed(lsmps_ctx* ctx, int a, int b) {
    LSMPS_CUDA(cudaEventSynchronize(ctx->ev[b]));
    float ms = 0;
    LSMPS_CUDA(cudaEventElapsedTime(&ms, ctx->ev[a], ctx->ev[b]));
    return ms;
}

namespace {
__global__ void k_pack_particles(const double* __restrict__ xyz, size_t n, double* __restrict__ pos) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i < 3 * n) pos[i] = xyz[i];
}
}  // namespace

void particles_upload(lsmps_ctx* ctx, const double* xyz, const uint8_t* type, size_t n, bool device) {
    LSMPS_REQUIRE(n == 0 || (xyz && type), LSMPS_ERR_ARG, "null particle buffers");
    LSMPS_REQUIRE(n < (size_t)(1u << 31) - 1, LSMPS_ERR_OVERFLOW, "particle count beyond int32");
    ev_record(ctx, 0);
    double* pos = ctx->pos.ensure<double>(3 * n + 1);
    uint8_t* t = ctx->type_in.ensure<uint8_t>(n + 1);
    if (n) {
        if (device) {
            k_pack_particles<<<blocks_for(3 * n, 256), 256, 0, ctx->stream>>>(xyz, n, pos);
            LSMPS_CHECK_LAUNCH();
            LSMPS_CUDA(cudaMemcpyAsync(t, type, n, cudaMemcpyDeviceToDevice, ctx->stream));
        } else {
            LSMPS_CUDA(cudaMemcpyAsync(pos, xyz, 3 * n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
            LSMPS_CUDA(cudaMemcpyAsync(t, type, n, cudaMemcpyHostToDevice, ctx->stream));
        }
    }
    ev_record(ctx, 1);
    ctx->n = n;
    ctx->have_neighbors = ctx->have_classes = ctx->have_wls = ctx->have_ppe = ctx->have_solution = false;
    ctx->have_candidates = false;
    ctx->timings[0] = ev_elapsed(ctx, 0, 1);
}

void particles_prefetch(lsmps_ctx* ctx, const double* xyz, const uint8_t* type, size_t n) {
    LSMPS_REQUIRE(n == 0 || (xyz && type), LSMPS_ERR_ARG, "null particle buffers");
    LSMPS_REQUIRE(n < (size_t)(1u << 31) - 1, LSMPS_ERR_OVERFLOW, "particle count beyond int32");
    if (!ctx->copy_stream)  // also created by an asynchronous download
        LSMPS_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    if (!ctx->stage_done) {
        LSMPS_CUDA(cudaEventCreateWithFlags(&ctx->stage_done, cudaEventDisableTiming));
        LSMPS_CUDA(cudaEventCreateWithFlags(&ctx->stage_free, cudaEventDisableTiming));
    }
    // the staging buffers held the set before the last swap: work already enqueued on the
    // context stream may still read them
    LSMPS_CUDA(cudaEventRecord(ctx->stage_free, ctx->stream));
    LSMPS_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->stage_free, 0));
    double* pos = ctx->stage_pos.ensure<double>(3 * n + 1);
    uint8_t* t = ctx->stage_type.ensure<uint8_t>(n + 1);
    if (n) {
        LSMPS_CUDA(cudaMemcpyAsync(pos, xyz, 3 * n * sizeof(double), cudaMemcpyHostToDevice, ctx->copy_stream));
        LSMPS_CUDA(cudaMemcpyAsync(t, type, n, cudaMemcpyHostToDevice, ctx->copy_stream));
    }
    LSMPS_CUDA(cudaEventRecord(ctx->stage_done, ctx->copy_stream));
    ctx->stage_n = n;
    ctx->have_stage = true;
}

void particles_use_prefetched(lsmps_ctx* ctx) {
    LSMPS_REQUIRE(ctx->have_stage, LSMPS_ERR_STATE, "no prefetched particle set (lsmps_prefetch_particles first)");
    LSMPS_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->stage_done, 0));
    std::swap(ctx->pos, ctx->stage_pos);
    std::swap(ctx->type_in, ctx->stage_type);
    ctx->n = ctx->stage_n;
    ctx->have_stage = false;
    ctx->have_neighbors = ctx->have_classes = ctx->have_wls = ctx->have_ppe = ctx->have_solution = false;
    ctx->have_candidates = false;
    ctx->timings[0] = 0.0;  // the copies overlapped other work
}

}  // namespace lsmps_gpu

using namespace lsmps_gpu;

namespace {
template <class F>
int guarded(lsmps_ctx* ctx, F&& f) {
    if (!ctx) return LSMPS_ERR_ARG;
    try {
        LSMPS_CUDA(cudaSetDevice(ctx->device));
        f();
        ctx->last_error.clear();
        return LSMPS_OK;
    } catch (const Error& e) {
        ctx->last_error = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        ctx->last_error = "host allocation failed";
        return LSMPS_ERR_ALLOC;
    } catch (const std::exception& e) {
        ctx->last_error = e.what();
        return LSMPS_ERR_ARG;
    }
}
}  // namespace

extern "C" {

int lsmps_abi_version(void) { return LSMPS_ABI_VERSION; }

int lsmps_ctx_create(int device, lsmps_ctx** out) {
    if (!out) return LSMPS_ERR_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return LSMPS_ERR_CUDA;
    }
    lsmps_ctx* ctx = new (std::nothrow) lsmps_ctx();
    if (!ctx) return LSMPS_ERR_ALLOC;
    ctx->device = device;
    int rc = guarded(ctx, [&] {
        LSMPS_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
        for (auto& e : ctx->ev) LSMPS_CUDA(cudaEventCreate(&e));
        int* f = ctx->dflags.ensure<int>(16);
        LSMPS_CUDA(cudaMemsetAsync(f, 0, 16 * sizeof(int), ctx->stream));
        ctx->scratch.ensure<int>(4096);  // small device scalars (see the offsets at their uses)
        LSMPS_CUDA(cudaStreamSynchronize(ctx->stream));
    });
    if (rc != LSMPS_OK) {
        lsmps_ctx_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return LSMPS_OK;
}

void lsmps_ctx_destroy(lsmps_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    if (ctx->side_stream) cudaStreamSynchronize(ctx->side_stream);
    lsmps_gpu::DevBuf* bufs[] = {&ctx->dflags, &ctx->scratch, &ctx->scan_tmp, &ctx->host_dummy, &ctx->pos,
                                 &ctx->type_in, &ctx->cell_of, &ctx->slot, &ctx->cell_count, &ctx->cell_start,
                                 &ctx->perm, &ctx->iperm, &ctx->sx, &ctx->sy, &ctx->sz, &ctx->stype,
                                 &ctx->scell, &ctx->cls, &ctx->nbr_cnt, &ctx->nbr_row, &ctx->nbr_col, &ctx->seg_list,
                                 &ctx->cand_row, &ctx->cand_col, &ctx->ref_sx, &ctx->ref_sy, &ctx->ref_sz,
                                 &ctx->nbr_stats, &ctx->wls_status, &ctx->wls_z, &ctx->wls_wsum, &ctx->wls_x,
                                 &ctx->wf_in, &ctx->wf_x, &ctx->wf_status, &ctx->wf_z, &ctx->wf_wsum, &ctx->wf_stats,
                                 &ctx->pj_grad, &ctx->pj_gradp, &ctx->pj_div, &ctx->pj_mask, &ctx->pj_stats,
                                 &ctx->pj_hop, &ctx->ld_ident, &ctx->S_dcol, &ctx->S_rbase,
                                 &ctx->wls_stats, &ctx->wls_sample, &ctx->ref_rank, &ctx->u_of_sorted,
                                 &ctx->sorted_of_u, &ctx->ref_of_u, &ctx->u_of_ref, &ctx->A_row, &ctx->A_col,
                                 &ctx->A_val, &ctx->A_valf, &ctx->A_b, &ctx->A_xexact, &ctx->A_dinv,
                                 &ctx->A_dinvf, &ctx->A_cnt, &ctx->vx, &ctx->vr, &ctx->vr0, &ctx->vp, &ctx->vv,
                                 &ctx->vs, &ctx->vt, &ctx->vph, &ctx->vsh, &ctx->vtmp, &ctx->fx, &ctx->fr,
                                 &ctx->fr0, &ctx->fp, &ctx->fv, &ctx->fs, &ctx->ft, &ctx->fph, &ctx->fsh,
                                 &ctx->red, &ctx->S_ptr, &ctx->S_len,
                                 &ctx->S_col, &ctx->S_val, &ctx->S_vals, &ctx->S_valf, &ctx->nbr_slots,
                                 &ctx->A_slot_col, &ctx->A_slot_val, &ctx->A_xep, &ctx->stage_pos,
                                 &ctx->stage_type, &ctx->dl_stage};
    for (auto* b : bufs) b->release();
    mpnn_destroy(ctx);
    mg_destroy(ctx);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    if (ctx->stage_done) cudaEventDestroy(ctx->stage_done);
    if (ctx->stage_free) cudaEventDestroy(ctx->stage_free);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->dl_ready) cudaEventDestroy(ctx->dl_ready);
    if (ctx->dl_done) cudaEventDestroy(ctx->dl_done);
    if (ctx->side_fork) cudaEventDestroy(ctx->side_fork);
    if (ctx->side_join) cudaEventDestroy(ctx->side_join);
    if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* lsmps_last_error(const lsmps_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int lsmps_get_timings(lsmps_ctx* ctx, double out[8]) {
    if (!ctx || !out) return LSMPS_ERR_ARG;
    if (ctx->timing_pending) {  // calls that did not wait: their events are read now
        const int rc = guarded(ctx, [&] { resolve_timings(ctx); });
        if (rc != LSMPS_OK) return rc;
    }
    std::memcpy(out, ctx->timings, sizeof(ctx->timings));
    return LSMPS_OK;
}

int lsmps_sync(lsmps_ctx* ctx) {
    return guarded(ctx, [&] { LSMPS_CUDA(cudaStreamSynchronize(ctx->stream)); });
}

void* lsmps_stream(lsmps_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

uint64_t lsmps_launch_count(void) { return g_launches.load(); }

int lsmps_kernel_bench(lsmps_ctx* ctx, int kernel, int reps, double* ms_per_launch, double* bytes_per_launch) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(ms_per_launch && bytes_per_launch && reps > 0, LSMPS_ERR_ARG, "kernel bench arguments");
        if (kernel == LSMPS_KB_SPMV64 || kernel == LSMPS_KB_SPMV32)
            solver_kernel_bench(ctx, kernel, reps, ms_per_launch, bytes_per_launch);
        else if (kernel == LSMPS_KB_NBR_COUNT || kernel == LSMPS_KB_NBR_FILL || kernel == LSMPS_KB_NBR_SCAN ||
                 kernel == LSMPS_KB_NBR_COMPACT)
            nb_kernel_bench(ctx, kernel, reps, ms_per_launch, bytes_per_launch);
        else if (kernel == LSMPS_KB_WLS)
            wls_kernel_bench(ctx, reps, ms_per_launch, bytes_per_launch);
        else if (kernel == LSMPS_KB_MPNN_LAYER)
            mpnn_kernel_bench(ctx, reps, ms_per_launch, bytes_per_launch);
        else if (kernel == LSMPS_KB_MG_VCYCLE)
            mg_kernel_bench(ctx, reps, ms_per_launch, bytes_per_launch);
        else if (kernel == LSMPS_KB_FP64_PEAK)
            fp64_peak_bench(ctx, reps, ms_per_launch, bytes_per_launch);
        else
            throw Error{LSMPS_ERR_ARG, "unknown kernel id"};
    });
}

int lsmps_set_autotune(lsmps_ctx* ctx, int mode) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(mode >= 0 && mode <= 2, LSMPS_ERR_ARG, "autotune mode must be 0, 1 or 2");
        ctx->tuner.enabled = mode != 0;
        if (mode == 2) ctx->tuner.table.clear();
    });
}

int lsmps_autotune_report(lsmps_ctx* ctx, char* buf, size_t cap, size_t* needed) {
    return guarded(ctx, [&] {
        const std::string r = autotune_report(ctx);
        if (needed) *needed = r.size() + 1;
        if (buf && cap) {
            const size_t k = std::min(cap - 1, r.size());
            std::memcpy(buf, r.data(), k);
            buf[k] = 0;
        }
    });
}

int lsmps_upload_particles(lsmps_ctx* ctx, const double* xyz, const uint8_t* type, size_t n) {
    return guarded(ctx, [&] { particles_upload(ctx, xyz, type, n, false); });
}

int lsmps_upload_particles_device(lsmps_ctx* ctx, const double* d_xyz, const uint8_t* d_type, size_t n) {
    return guarded(ctx, [&] { particles_upload(ctx, d_xyz, d_type, n, true); });
}

int lsmps_prefetch_particles(lsmps_ctx* ctx, const double* xyz, const uint8_t* type, size_t n) {
    return guarded(ctx, [&] { particles_prefetch(ctx, xyz, type, n); });
}

int lsmps_use_prefetched_particles(lsmps_ctx* ctx) {
    return guarded(ctx, [&] { particles_use_prefetched(ctx); });
}

int lsmps_build_neighbors(lsmps_ctx* ctx, double re, int max_neighbors, double l0, int flags,
                          lsmps_neighbor_stats* out) {
    return guarded(ctx, [&] {
        ev_record(ctx, 2);
        nb_build(ctx, re, max_neighbors, l0, flags, out);
        ev_record(ctx, 3);
        // without statistics the call does not wait for its last kernels; its time is read later
        if (out) {
            ctx->timing_pending &= ~2u;
            ctx->timings[1] = ev_elapsed(ctx, 2, 3);
        } else {
            ctx->timing_pending |= 2u;
        }
    });
}

int lsmps_build_neighbors_skin(lsmps_ctx* ctx, double re, double skin, int max_neighbors, int max_candidates,
                               double l0, int flags, lsmps_neighbor_stats* out) {
    return guarded(ctx, [&] {
        ev_record(ctx, 2);
        nb_build_skin(ctx, re, skin, max_neighbors, max_candidates, l0, flags, out);
        ev_record(ctx, 3);
        ctx->timings[1] = ev_elapsed(ctx, 2, 3);
        ctx->timing_pending &= ~2u;
    });
}

int lsmps_update_positions(lsmps_ctx* ctx, const double* xyz, size_t n) {
    return guarded(ctx, [&] { nb_update_positions(ctx, xyz, n, false); });
}

int lsmps_update_positions_device(lsmps_ctx* ctx, const double* d_xyz, size_t n) {
    return guarded(ctx, [&] { nb_update_positions(ctx, d_xyz, n, true); });
}

int lsmps_refresh_neighbors(lsmps_ctx* ctx, int flags, lsmps_neighbor_stats* out) {
    return guarded(ctx, [&] {
        ev_record(ctx, 2);
        nb_refresh(ctx, flags, out);
        ev_record(ctx, 3);
        ctx->timings[1] = ev_elapsed(ctx, 2, 3);
        ctx->timing_pending &= ~2u;
    });
}

int lsmps_max_displacement(lsmps_ctx* ctx, double* out) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(out, LSMPS_ERR_ARG, "null output");
        *out = nb_max_displacement(ctx);
    });
}

int lsmps_classify(lsmps_ctx* ctx, double l0, lsmps_neighbor_stats* out) {
    return guarded(ctx, [&] {
        ev_record(ctx, 4);
        nb_classify(ctx, l0, out);
        ev_record(ctx, 5);
        ctx->timings[2] = ev_elapsed(ctx, 4, 5);
    });
}

int lsmps_wls(lsmps_ctx* ctx, const lsmps_wls_opts* opts, lsmps_wls_stats* out) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(opts, LSMPS_ERR_ARG, "null WLS options");
        ev_record(ctx, 6);
        wls_run(ctx, opts, out);
        ev_record(ctx, 7);
        // without statistics the call does not wait; its time is read by lsmps_get_timings
        if (out) {
            ctx->timing_pending &= ~8u;
            ctx->timings[3] = ev_elapsed(ctx, 6, 7);
        } else {
            ctx->timing_pending |= 8u;
        }
    });
}

int lsmps_ppe_assemble(lsmps_ctx* ctx, const lsmps_ppe_opts* opts, lsmps_ppe_stats* out) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(opts, LSMPS_ERR_ARG, "null PPE options");
        ppe_assemble(ctx, opts, out);
        // without statistics the call does not wait for its last kernels; its time is read later
        if (out) {
            ctx->timing_pending &= ~16u;
            ctx->timings[4] = ctx->ppe_assembly.assembly_ms;
        } else {
            ctx->timing_pending |= 16u;
        }
    });
}

int lsmps_ppe_solve(lsmps_ctx* ctx, const lsmps_solver_opts* opts, lsmps_ppe_stats* out) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(opts, LSMPS_ERR_ARG, "null solver options");
        ppe_solve(ctx, opts, out);
        // an assembly that did not wait: its events are complete once the solve has returned
        if (ctx->timing_pending & 16u) {
            resolve_timings(ctx);
            if (out) out->assembly_ms = ctx->ppe_assembly.assembly_ms;
        }
    });
}

int lsmps_mg_info(lsmps_ctx* ctx, int32_t* levels, int64_t* rows, int32_t cap, double* setup_ms) {
    return guarded(ctx, [&] {
        int lv = 0;
        mg_info(ctx, &lv, rows, cap, setup_ms);
        if (levels) *levels = lv;
    });
}

int lsmps_mg_apply(lsmps_ctx* ctx, const double* z, double* out, size_t u) {
    return guarded(ctx, [&] { mg_apply_host(ctx, z, out, u); });
}

int lsmps_download_types(lsmps_ctx* ctx, uint8_t* type, size_t n) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(type || n == 0, LSMPS_ERR_ARG, "null type buffer");
        nb_download_types(ctx, type, n);
    });
}

int lsmps_download_neighbors(lsmps_ctx* ctx, int32_t* row_ptr, int32_t* col, size_t col_cap) {
    return guarded(ctx, [&] { nb_download(ctx, row_ptr, col, col_cap); });
}

int lsmps_download_wls(lsmps_ctx* ctx, double* x, int32_t* status, double* z, double* wsum) {
    return guarded(ctx, [&] { wls_download(ctx, x, status, z, wsum); });
}

int lsmps_download_ppe(lsmps_ctx* ctx, int32_t* row, int32_t* col, double* val, double* b, double* x_exact,
                       int32_t* unknown_particle) {
    return guarded(ctx, [&] { ppe_download(ctx, row, col, val, b, x_exact, unknown_particle); });
}

int lsmps_download_pressure(lsmps_ctx* ctx, double* p, size_t u) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(p || u == 0, LSMPS_ERR_ARG, "null pressure buffer");
        ev_record(ctx, 12);
        ppe_download_pressure(ctx, p, u);
        ev_record(ctx, 13);
        ctx->timings[6] = ev_elapsed(ctx, 12, 13);
    });
}

int lsmps_download_pressure_async(lsmps_ctx* ctx, double* p, size_t u) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(p || u == 0, LSMPS_ERR_ARG, "null pressure buffer");
        ppe_download_pressure_async(ctx, p, u);
    });
}

int lsmps_download_wait(lsmps_ctx* ctx) {
    return guarded(ctx, [&] { ppe_download_wait(ctx); });
}

int lsmps_set_initial_pressure(lsmps_ctx* ctx, const double* p, size_t n) {
    return guarded(ctx, [&] { ppe_set_initial_particles(ctx, p, n, false); });
}
int lsmps_set_initial_pressure_device(lsmps_ctx* ctx, const double* d_p, size_t n) {
    return guarded(ctx, [&] { ppe_set_initial_particles(ctx, d_p, n, true); });
}
int lsmps_download_pressure_particles(lsmps_ctx* ctx, double* p, size_t n, double fill) {
    return guarded(ctx, [&] { ppe_pressure_particles(ctx, p, n, fill, false); });
}
int lsmps_download_pressure_particles_device(lsmps_ctx* ctx, double* d_p, size_t n, double fill) {
    return guarded(ctx, [&] { ppe_pressure_particles(ctx, d_p, n, fill, true); });
}

static_assert(sizeof(lsmps_series_params) == 136, "lsmps_series_params layout");
static_assert(sizeof(lsmps_series_stats) == 184, "lsmps_series_stats layout");

int lsmps_series_create(lsmps_ctx* ctx, const lsmps_series_params* params, const double* xyz, const uint8_t* type,
                        size_t n, lsmps_series** out) {
    return guarded(ctx, [&] { series_create(ctx, params, xyz, type, n, out); });
}

int lsmps_series_step(lsmps_series* series, lsmps_series_stats* out) {
    return guarded(series_context(series), [&] { series_step(series, out); });
}

int lsmps_series_particles(lsmps_series* series, double* xyz, uint8_t* material, double* pressure, size_t cap,
                           size_t* n) {
    return guarded(series_context(series), [&] { series_particles(series, xyz, material, pressure, cap, n); });
}

int lsmps_series_set_validation(lsmps_series* series, const lsmps_rain_validation* cfg) {
    return guarded(series_context(series), [&] { series_set_validation(series, cfg); });
}

int lsmps_series_rain_outputs(lsmps_series* series, lsmps_rain_outputs* out) {
    return guarded(series_context(series), [&] { series_rain_outputs(series, out); });
}

void lsmps_series_destroy(lsmps_series* series) {
    if (!series) return;
    cudaSetDevice(series_context(series)->device);
    series_destroy(series);
}

int lsmps_ppe_load_csr(lsmps_ctx* ctx, const int64_t* row_ptr, const int32_t* col, const double* val,
                       const double* b, size_t n, lsmps_ppe_stats* out) {
    return guarded(ctx, [&] { ppe_load_csr(ctx, row_ptr, col, val, b, n, out); });
}

int lsmps_wls_fields(lsmps_ctx* ctx, const double* d_fields, int nfields, double* d_out) {
    return guarded(ctx, [&] { wls_fields(ctx, d_fields, nfields, d_out); });
}

int lsmps_projection_step(lsmps_ctx* ctx, const double* d_vel, double dt, double rho, const lsmps_solver_opts* opts,
                          double* d_vel_out, double* d_pressure, lsmps_projection_stats* out) {
    return guarded(ctx, [&] { projection_step(ctx, d_vel, dt, rho, opts, d_vel_out, d_pressure, out); });
}

int lsmps_predict_velocity(lsmps_ctx* ctx, const double* d_vel, double dt, double nu, const double* gravity, int flags,
                           double* d_vel_out) {
    return guarded(ctx, [&] { predict_velocity(ctx, d_vel, dt, nu, gravity, flags, d_vel_out); });
}

int lsmps_ppe_manufacture(lsmps_ctx* ctx, const double* params, int nmodes) {
    return guarded(ctx, [&] { ppe_manufacture(ctx, params, nmodes); });
}

int lsmps_ppe_residual_static(lsmps_ctx* ctx, const double* d_p, size_t ld, int nvec, double* d_out) {
    return guarded(ctx, [&] { ppe_residual_static(ctx, d_p, ld, nvec, d_out); });
}

size_t lsmps_mpnn_param_count(void) { return mpnn_param_count(); }

int lsmps_mpnn_init(lsmps_ctx* ctx, uint32_t seed) {
    return guarded(ctx, [&] { mpnn_init(ctx, seed); });
}
int lsmps_mpnn_get_weights(lsmps_ctx* ctx, float* w, size_t n) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(w, LSMPS_ERR_ARG, "null weight buffer");
        mpnn_get_weights(ctx, w, n);
    });
}
int lsmps_mpnn_set_weights(lsmps_ctx* ctx, const float* w, size_t n) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(w, LSMPS_ERR_ARG, "null weight buffer");
        mpnn_set_weights(ctx, w, n);
    });
}
int lsmps_mpnn_add_sample(lsmps_ctx* ctx) {
    return guarded(ctx, [&] { mpnn_add_sample(ctx); });
}
int lsmps_mpnn_clear_samples(lsmps_ctx* ctx) {
    return guarded(ctx, [&] { mpnn_clear_samples(ctx); });
}
int lsmps_mpnn_sample_count(lsmps_ctx* ctx) { return ctx ? mpnn_sample_count(ctx) : 0; }
int lsmps_mpnn_grad(lsmps_ctx* ctx, int index, float* grad, float* loss) {
    return guarded(ctx, [&] { mpnn_grad(ctx, index, grad, loss); });
}
int lsmps_mpnn_train(lsmps_ctx* ctx, const lsmps_mpnn_train_opts* opts, float* loss_out) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(opts, LSMPS_ERR_ARG, "null training options");
        mpnn_train(ctx, opts, loss_out);
    });
}
int lsmps_mpnn_infer(lsmps_ctx* ctx, const double* r, double* y) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(r && y, LSMPS_ERR_ARG, "null vectors");
        mpnn_infer(ctx, r, y);
    });
}
int lsmps_mpnn_save(lsmps_ctx* ctx, const char* path) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(path, LSMPS_ERR_ARG, "null path");
        mpnn_save(ctx, path);
    });
}
int lsmps_mpnn_load(lsmps_ctx* ctx, const char* path) {
    return guarded(ctx, [&] {
        LSMPS_REQUIRE(path, LSMPS_ERR_ARG, "null path");
        mpnn_load(ctx, path);
    });
}

}  // extern "C"
