// The opaque lsmps_ctx: device buffers and state of one particle set on one GPU.
//
// HBM layout (n particles, P kept pairs, U unknowns, Z nonzeros):
//   particles (caller order)   pos: n x double3 AoS (24 B), type_in: n x u8
//   cell-sorted copies         perm/iperm: n x i32, sx/sy/sz: 3 x n x f64 (SoA), stype, cls:
//                              n x u8, scell: n x i32
//   dense cell grid            cell_start: cells + 1 x i32
//   neighbor CSR (sorted)      nbr_row: n + 1 x i32, nbr_col: P x i32 (sorted indices; the
//                              reference's row order is ascending sorted index)
//   WLS                        wls_status: n x i32, wls_z: n x 9 f64, wls_wsum: n x f64
//   PPE (unknowns in sorted    A_row: U + 1 x i32, A_col: Z x i32, A_val: Z x f64, b, x*,
//   order)                     diag_inv: U x f64, u_of_sorted: n x i32, sorted_of_u /
//                              ref_of_u / u_of_ref: U x i32
//   SELL-32 solver copies      S_ptr / S_len: U/32 x i32, S_col: E x i32, S_val (A) and
//                              S_vals (A D^-1): E x f64, S_valf (A D^-1): E x f32, with
//                              E = Z + padding (each slice padded to its longest row)
#pragma once
#include <initializer_list>
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace lsmps_gpu {
struct MpnnState;
struct MgState;

// Autotuner table of one context: per "kernel n~2^k" key, the candidate launch shapes,
// their measured ms per launch and the chosen one.
struct TuneResult {
    std::vector<std::string> names;
    std::vector<float> ms;
    int best = 0;
};
struct Tuner {
    bool enabled = true;
    std::map<std::string, TuneResult> table;
};
}  // namespace lsmps_gpu

struct lsmps_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string last_error;
    cudaEvent_t ev[18] = {};
    // double-buffered particle upload (lsmps_prefetch_particles): staging buffers, copy stream,
    // copy-done and buffer-free events, created at first use
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t stage_done = nullptr, stage_free = nullptr;
    // the learned solver with the multigrid builds the hierarchy on side_stream (highest priority)
    // while the network runs on `stream`; fork / join events, all created at first use
    cudaStream_t side_stream = nullptr;
    cudaEvent_t side_fork = nullptr, side_join = nullptr;
    // asynchronous result download (lsmps_download_pressure_async): staging buffer on the
    // device, reordered-result-ready and copy-done events, a copy in flight
    lsmps_gpu::DevBuf dl_stage;
    cudaEvent_t dl_ready = nullptr, dl_done = nullptr;
    bool dl_pending = false;
    size_t stage_n = 0;
    bool have_stage = false;
    double timings[8] = {};
    // phase times of calls made without statistics, which do not wait: their events are read
    // later (bit 1: neighbors, events 2-3; bit 3: WLS, 6-7; bit 4: assembly, 8-9)
    unsigned timing_pending = 0;

    lsmps_gpu::DevBuf dflags;      // int device error flags
    lsmps_gpu::DevBuf scratch;     // general reduction scratch
    lsmps_gpu::DevBuf scan_tmp;    // block sums of scans
    lsmps_gpu::DevBuf host_dummy;

    // ---- particles ----
    size_t n = 0;
    lsmps_gpu::DevBuf pos, type_in;
    lsmps_gpu::DevBuf stage_pos, stage_type;  // the prefetched set (swapped in by use_prefetched)

    // ---- grid + neighbors ----
    double re = 0, re2 = 0, l0 = 0;
    int maxn = 0;
    int gmin[3] = {0, 0, 0};
    int gdim[3] = {0, 0, 0};
    long long ncells = 0;
    bool have_neighbors = false, have_classes = false;
    uint64_t pairs = 0, truncated = 0;
    int max_cell_occupancy = 0;
    int nsegs = 0;  // non-empty 12-cell segments of the grid (neighbor passes)
    lsmps_gpu::DevBuf cell_of, slot, cell_count, cell_start, perm, iperm;
    lsmps_gpu::DevBuf sx, sy, sz, stype, scell, cls;
    lsmps_gpu::DevBuf nbr_cnt, nbr_row, nbr_col, nbr_stats, seg_list;
    lsmps_gpu::DevBuf nbr_slots;  // single-pass build: maxn slots per particle before compaction
    bool nbr_single = false;      // the last build used the single pass
    // candidate lists of radius re + skin (sorted numbering) and the sorted positions they
    // were built at, for refreshes of an unchanged particle set
    bool have_candidates = false;
    double skin = 0, cand_re = 0;
    uint64_t cand_pairs = 0;
    lsmps_gpu::DevBuf cand_row, cand_col, ref_sx, ref_sy, ref_sz;

    // ---- WLS ----
    bool have_wls = false;
    int wls_nrhs = 0;
    bool wls_stored = false;
    lsmps_gpu::DevBuf wls_status, wls_z, wls_wsum, wls_x, wls_stats, wls_sample;
    // WLS of caller fields (gradients for the projection step): inputs, solutions, scratch
    lsmps_gpu::DevBuf wf_in, wf_x, wf_status, wf_z, wf_wsum, wf_stats;
    // projection step: WLS solutions of u and p, divergence, unknown mask, statistics
    lsmps_gpu::DevBuf pj_grad, pj_gradp, pj_div, pj_mask, pj_stats, pj_hop;

    // ---- PPE ----
    bool have_ppe = false;
    int ppe_variant = 0;
    long long U = 0, nnz = 0;
    lsmps_gpu::DevBuf ref_rank, u_of_sorted, sorted_of_u, ref_of_u, u_of_ref;
    lsmps_gpu::DevBuf A_row, A_col, A_val, A_valf, A_b, A_xexact, A_dinv, A_dinvf, A_cnt;
    lsmps_gpu::DevBuf A_slot_col, A_slot_val, A_xep;  // A_xep: p* per sorted particle
    bool ppe_wall_neumann = false;  // the assembled WLS rows treat walls as Neumann boundaries  // assembly: rows at their neighbor-row slots before packing
    lsmps_ppe_stats ppe_assembly{};
    bool ppe_loaded = false;        // the system came from lsmps_ppe_load_csr (no particles behind it)
    lsmps_gpu::DevBuf ld_ident;     // identity map standing in for the particle permutation
    // SELL-32 copies of A for the fast solvers (built on first use after an assembly)
    bool have_sell = false, have_sell_s = false, have_sell_f = false;
    bool have_sell_raw = false;  // the unscaled FP64 values and 32-bit columns of the SELL copy
    long long sell_nslices = 0, sell_entries = 0;
    lsmps_gpu::DevBuf S_ptr, S_len, S_col, S_val, S_vals, S_valf;
    // 16-bit column steps of the SELL copies (used when every row ascends in steps < 65536)
    bool have_steps = false, sell_steps_enabled = true;
    lsmps_gpu::DevBuf S_dcol, S_rbase;

    // ---- solver state ----
    bool have_solution = false;
    lsmps_gpu::DevBuf vx, vr, vr0, vp, vv, vs, vt, vph, vsh, vtmp;   // FP64 vectors
    lsmps_gpu::DevBuf fx, fr, fr0, fp, fv, fs, ft, fph, fsh;         // FP32 vectors
    lsmps_gpu::DevBuf red;                                           // reduction partials + scalars

    // ---- learned preconditioner (weights, training store, workspace) ----
    lsmps_gpu::MpnnState* mpnn = nullptr;
    // cell-aggregation multigrid hierarchy of the assembled system (multigrid.cu)
    lsmps_gpu::MgState* mg = nullptr;
    long long assembly_gen = 0;  // bumped by every PPE assembly

    lsmps_gpu::Tuner tuner;  // launch shapes chosen by the autotuner

    void* pinned = nullptr;
    size_t pinned_bytes = 0;
};

namespace lsmps_gpu {
// Pinned host staging buffer of the context (grow-only).
void* pinned_ensure(lsmps_ctx* ctx, size_t bytes);
// Read device int flags, clear them, and throw on any set flag.
void check_device_flags(lsmps_ctx* ctx, const char* where);
// A device value to read back to the host: bytes from src (device) to dst (host).
struct ReadBack {
    const void* src;
    void* dst;
    size_t bytes;
};
// Reads the values, and the device error flags unless where is null, in one synchronisation of
// the context stream (copies into the context's pinned staging buffer), then throws on a set
// flag as check_device_flags does.
void read_back(lsmps_ctx* ctx, std::initializer_list<ReadBack> items, const char* where);
}  // namespace lsmps_gpu
