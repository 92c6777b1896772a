// Neighbor lists with a skin (Verlet lists) for step series: a full cell-list build at radius
// re + skin keeps every pair closer than re + skin as a candidate; while no particle has moved
// more than skin / 2 since that build, the exact lists for radius re are the candidates that
// pass the build's own test |r_j - r_i|^2 < re^2 (src/lsmps.cpp:26), which a filter over the
// candidate CSR finds without touching the cell grid. Rows keep candidate order, which is
// ascending sorted index, the order a build gives (numbering of the candidate build).
#include <cmath>
#include <cstring>
#include <utility>

#include "ops.cuh"
#include "scan.cuh"

namespace lsmps_gpu {
namespace {

// Sorted copies of new positions of the same particles (caller order AoS -> sorted SoA).
__global__ void k_regather(const int* __restrict__ perm, size_t n, const double* __restrict__ pos,
                           double* __restrict__ sx, double* __restrict__ sy, double* __restrict__ sz, int* dflag) {
    size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    const size_t i = (size_t)perm[k];
    const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    if (!isfinite(x) || !isfinite(y) || !isfinite(z)) atomicOr(dflag, DFLAG_NONFINITE);
    sx[k] = x;
    sy[k] = y;
    sz[k] = z;
}

// Largest |r - r_build|^2 (non-negative doubles order as their bit patterns).
__global__ void k_max_disp2(size_t n, const double* __restrict__ sx, const double* __restrict__ sy,
                            const double* __restrict__ sz, const double* __restrict__ rx,
                            const double* __restrict__ ry, const double* __restrict__ rz,
                            unsigned long long* out) {
    double m = 0.0;
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const double dx = sx[k] - rx[k], dy = sy[k] - ry[k], dz = sz[k] - rz[k];
        m = fmax(m, dx * dx + dy * dy + dz * dz);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// Warp per row: candidates j != i with |r_j - r_i|^2 < re^2 (exact FP64, the build's test), in
// candidate order, the first maxn kept. Count pass: kept count and dropped pairs; fill pass:
// ordered compaction by ballot.
template <bool FILL>
__global__ void __launch_bounds__(256) k_filter(int n, const int* __restrict__ crow, const int* __restrict__ ccol,
                                                const double* __restrict__ sx, const double* __restrict__ sy,
                                                const double* __restrict__ sz, double re2, int maxn,
                                                int* __restrict__ cnt, unsigned long long* trunc,
                                                const int* __restrict__ row, int* __restrict__ col) {
    const int lane = threadIdx.x & 31;
    const int nw = (int)((gridDim.x * (size_t)blockDim.x) >> 5);
    for (int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5); i < n; i += nw) {
        const double xi = sx[i], yi = sy[i], zi = sz[i];
        const int c0 = crow[i], c1 = crow[i + 1];
        const int out0 = FILL ? row[i] : 0;
        int kept = 0;
        for (int b = c0; b < c1; b += 32) {
            const int e = b + lane;
            bool ok = false;
            int j = 0;
            if (e < c1) {
                j = ccol[e];
                ok = j != i && xnorm2(xsub(sx[j], xi), xsub(sy[j], yi), xsub(sz[j], zi)) < re2;
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (FILL && ok) {
                const int p = kept + __popc(m & ((1u << lane) - 1u));
                if (p < maxn) col[out0 + p] = j;
            }
            kept += __popc(m);
        }
        if (!FILL && lane == 0) {
            cnt[i] = min(kept, maxn);
            if (kept > maxn) atomicAdd(trunc, (unsigned long long)(kept - maxn));
        }
    }
}

}  // namespace

void nb_build_skin(lsmps_ctx* ctx, double re, double skin, int maxn, int maxc, double l0, int flags,
                   lsmps_neighbor_stats* out) {
    LSMPS_REQUIRE(skin >= 0 && std::isfinite(skin), LSMPS_ERR_ARG, "skin must be non-negative and finite");
    LSMPS_REQUIRE(maxc >= maxn, LSMPS_ERR_ARG, "max_candidates must be at least max_neighbors");
    nb_build(ctx, re + skin, maxc, l0, 0, nullptr);
    LSMPS_REQUIRE(ctx->truncated == 0, LSMPS_ERR_ARG,
                  "candidate lists truncated (" + std::to_string(ctx->truncated) +
                      " pairs beyond max_candidates): raise max_candidates");
    std::swap(ctx->nbr_row, ctx->cand_row);
    std::swap(ctx->nbr_col, ctx->cand_col);
    ctx->cand_pairs = ctx->pairs;
    const size_t n = ctx->n;
    cudaStream_t s = ctx->stream;
    double* rx = ctx->ref_sx.ensure<double>(n + 1);
    double* ry = ctx->ref_sy.ensure<double>(n + 1);
    double* rz = ctx->ref_sz.ensure<double>(n + 1);
    if (n) {
        LSMPS_CUDA(cudaMemcpyAsync(rx, ctx->sx.get<double>(), n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        LSMPS_CUDA(cudaMemcpyAsync(ry, ctx->sy.get<double>(), n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        LSMPS_CUDA(cudaMemcpyAsync(rz, ctx->sz.get<double>(), n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    ctx->have_candidates = true;
    ctx->skin = skin;
    ctx->cand_re = re + skin;
    ctx->re = re;
    ctx->re2 = re * re;
    ctx->maxn = maxn;
    ctx->l0 = l0;
    nb_refresh(ctx, flags, out);
}

double nb_max_displacement(lsmps_ctx* ctx) {
    LSMPS_REQUIRE(ctx->have_candidates, LSMPS_ERR_STATE, "no candidate lists: lsmps_build_neighbors_skin first");
    const size_t n = ctx->n;
    if (!n) return 0.0;
    cudaStream_t s = ctx->stream;
    auto* d2 = reinterpret_cast<unsigned long long*>(ctx->scratch.get<int>() + 44);  // ints 44-45
    LSMPS_CUDA(cudaMemsetAsync(d2, 0, sizeof(unsigned long long), s));
    k_max_disp2<<<std::min<unsigned>(blocks_for(n, 256), 148 * 8), 256, 0, s>>>(
        n, ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(), ctx->ref_sx.get<double>(),
        ctx->ref_sy.get<double>(), ctx->ref_sz.get<double>(), d2);
    LSMPS_CHECK_LAUNCH();
    unsigned long long h = 0;
    LSMPS_CUDA(cudaMemcpyAsync(&h, d2, sizeof(h), cudaMemcpyDeviceToHost, s));
    LSMPS_CUDA(cudaStreamSynchronize(s));
    double m2;
    std::memcpy(&m2, &h, sizeof(m2));
    return std::sqrt(m2);
}

void nb_refresh(lsmps_ctx* ctx, int flags, lsmps_neighbor_stats* out) {
    LSMPS_REQUIRE(ctx->have_candidates, LSMPS_ERR_STATE, "no candidate lists: lsmps_build_neighbors_skin first");
    const double disp = nb_max_displacement(ctx);
    // |r_j - r_i| < re now and both moved at most skin / 2  =>  they were closer than re + skin
    LSMPS_REQUIRE(disp <= 0.5 * ctx->skin * (1.0 - 1e-9), LSMPS_ERR_STATE,
                  "a particle moved " + std::to_string(disp) + " since the candidate build, more than half the skin " +
                      std::to_string(ctx->skin) + ": rebuild with lsmps_build_neighbors_skin");
    const int classify = (flags & LSMPS_NBR_CLASSIFY) ? 1 : 0;
    if (nb_filter_single(ctx, classify)) {  // one pass, classes fused
        ctx->have_neighbors = true;
        ctx->have_classes = classify != 0;
        ctx->have_wls = ctx->have_ppe = ctx->have_solution = false;
        nb_stats(ctx, out, "neighbor filter");
        return;
    }
    cudaStream_t s = ctx->stream;
    const int n = (int)ctx->n;
    const int maxn = ctx->maxn;
    int* dflag = ctx->dflags.get<int>();
    int* cnt = ctx->nbr_cnt.ensure<int>(n + 1);
    int* row = ctx->nbr_row.ensure<int>(n + 1);
    auto* trunc_d = reinterpret_cast<unsigned long long*>(ctx->scratch.get<int>() + 16);
    LSMPS_CUDA(cudaMemsetAsync(trunc_d, 0, sizeof(unsigned long long), s));
    const unsigned grid = std::max(1u, std::min<unsigned>(blocks_for((size_t)n * 32, 256), 148 * 8));
    if (n) {
        k_filter<false><<<grid, 256, 0, s>>>(n, ctx->cand_row.get<int>(), ctx->cand_col.get<int>(),
                                            ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(),
                                            ctx->re2, maxn, cnt, trunc_d, nullptr, nullptr);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<int>(cnt, row, (long long)n, s, ctx->scan_tmp, dflag);
    int hpairs = 0;
    unsigned long long htr = 0;
    read_back(ctx, {{row + n, &hpairs, sizeof(int)}, {trunc_d, &htr, sizeof(htr)}}, "neighbor filter count");
    ctx->pairs = (uint64_t)hpairs;
    ctx->truncated = htr;
    int* col = ctx->nbr_col.ensure<int>((size_t)hpairs + 1);
    if (n) {
        k_filter<true><<<grid, 256, 0, s>>>(n, ctx->cand_row.get<int>(), ctx->cand_col.get<int>(),
                                           ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(),
                                           ctx->re2, maxn, nullptr, nullptr, row, col);
        LSMPS_CHECK_LAUNCH();
    }
    ctx->have_neighbors = true;
    ctx->have_classes = false;
    ctx->have_wls = ctx->have_ppe = ctx->have_solution = false;
    if (flags & LSMPS_NBR_CLASSIFY) {
        nb_classify(ctx, ctx->l0, out);
    } else {
        ctx->cls.ensure<uint8_t>(ctx->n + 1);
        nb_stats(ctx, out, "neighbor filter");
        return;
    }
    check_device_flags(ctx, "neighbor filter");
}

void nb_update_positions(lsmps_ctx* ctx, const double* xyz, size_t n, bool device) {
    LSMPS_REQUIRE(ctx->have_candidates, LSMPS_ERR_STATE,
                  "position updates keep the particle set of lsmps_build_neighbors_skin: build it first");
    LSMPS_REQUIRE(n == ctx->n, LSMPS_ERR_ARG, "position update must keep the particle count");
    LSMPS_REQUIRE(n == 0 || xyz, LSMPS_ERR_ARG, "null position buffer");
    cudaStream_t s = ctx->stream;
    ev_record(ctx, 0);
    double* pos = ctx->pos.get<double>();
    if (n) {
        LSMPS_CUDA(cudaMemcpyAsync(pos, xyz, 3 * n * sizeof(double),
                                   device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
        k_regather<<<blocks_for(n, 256), 256, 0, s>>>(ctx->perm.get<int>(), n, pos, ctx->sx.get<double>(),
                                                     ctx->sy.get<double>(), ctx->sz.get<double>(),
                                                     ctx->dflags.get<int>());
        LSMPS_CHECK_LAUNCH();
    }
    ev_record(ctx, 1);
    ctx->have_neighbors = ctx->have_classes = ctx->have_wls = ctx->have_ppe = ctx->have_solution = false;
    ctx->timings[0] = ev_elapsed(ctx, 0, 1);
    check_device_flags(ctx, "position update");
}

}  // namespace lsmps_gpu
