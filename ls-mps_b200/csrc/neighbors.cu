// Uniform-grid neighbor build and 14-direction classification on sm_100a.
//
// Semantics follow the reference's neighbors() and classify() (src/lsmps.cpp:16-18,26-27)
// bit for bit; the data flow is the GPU's own:
//   1. cell coordinates floor(r / re) (IEEE division) and their bounding box;
//   2. a counting sort of particles into a dense cell grid (atomic slots, scan), then
//      each cell's members sorted by particle index, so that every 3-cell x-row of the grid
//      is one contiguous, index-ascending range of the sorted arrays;
//   3. a count pass and a fill pass, one warp per particle: the warp tests the 9 contiguous
//      row ranges 32 candidates at a time, and a ballot gives each accepted candidate its
//      position. Scanning the 9 rows in (dz, dy) order with candidates in sorted order is
//      exactly the reference's order (27 cells dz, dy, dx; ascending index in a cell), so
//      the sorted column indices of a row ascend and the first max_neighbors are the ones
//      the reference keeps. The fill pass fuses the classification over the kept list.
// Distances use __dadd_rn/__dmul_rn: the reference evaluates (dx*dx + dy*dy) + dz*dz
// without fused multiply-adds, and the acceptance test d^2 < re^2 must match at the ulp.
#include <algorithm>
#include <cmath>
#include <climits>
#include <vector>

#include "ops.cuh"
#include "scan.cuh"

namespace lsmps_gpu {
namespace {

constexpr long long MAX_CELLS = 1ll << 29;   // 2 GiB of int32 cell starts
constexpr int SMALL_CELL = 64;                // in-place insertion sort up to this occupancy
constexpr int BIG_CELL_MAX = 8192;            // shared-memory bitonic sort up to this occupancy
constexpr int NB_WARPS = 8;                   // warps (= particles) per block in the passes

// ---- 1. cell coordinates --------------------------------------------------------------
__global__ void k_cell_coords(const double* __restrict__ pos, size_t n, double re,
                              int3* __restrict__ cell, int* bounds, int* dflag) {
    int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
    bool bad = false;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double c[3];
        int ci[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double v = pos[3 * i + a];
            c[a] = floor(xdiv(v, re));
            if (!isfinite(c[a]) || fabs(c[a]) > (double)(1 << 30)) { bad = true; c[a] = 0; }
            ci[a] = (int)c[a];
            mn[a] = min(mn[a], ci[a]);
            mx[a] = max(mx[a], ci[a]);
        }
        cell[i] = make_int3(ci[0], ci[1], ci[2]);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = min(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = max(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (mn[a] != INT_MAX) atomicMin(&bounds[a], mn[a]);
            if (mx[a] != INT_MIN) atomicMax(&bounds[3 + a], mx[a]);
        }
    }
    if (bad) atomicOr(dflag, DFLAG_NONFINITE);
}

// ---- 2. counting sort -------------------------------------------------------------------
__global__ void k_cell_count(const int3* __restrict__ cell, size_t n, int3 g0, int3 gd,
                             int* __restrict__ lin_out, int* __restrict__ slot, int* __restrict__ count) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int3 c = cell[i];
    int lin = ((c.z - g0.z) * gd.y + (c.y - g0.y)) * gd.x + (c.x - g0.x);
    lin_out[i] = lin;
    slot[i] = atomicAdd(&count[lin], 1);
}

__global__ void k_scatter(const int* __restrict__ lin, const int* __restrict__ slot, size_t n,
                          const int* __restrict__ cell_start, int* __restrict__ perm) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    perm[cell_start[lin[i]] + slot[i]] = (int)i;
}

// Atomic slots leave a cell's members in arbitrary order; restore ascending index.
__global__ void k_sort_small_cells(const int* __restrict__ cell_start, long long ncells,
                                   int* __restrict__ perm, int* big_list, int* big_count,
                                   int* max_occ) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    int occ = 0;
    if (c < ncells) {
        int b = cell_start[c], e = cell_start[c + 1];
        occ = e - b;
        if (occ > SMALL_CELL) {
            int slot = atomicAdd(big_count, 1);
            big_list[slot] = (int)c;
        } else if (occ > 1) {
            for (int a = b + 1; a < e; ++a) {
                int v = perm[a];
                int t = a - 1;
                while (t >= b && perm[t] > v) {
                    perm[t + 1] = perm[t];
                    --t;
                }
                perm[t + 1] = v;
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) occ = max(occ, __shfl_xor_sync(0xffffffffu, occ, o));
    if ((threadIdx.x & 31) == 0 && occ > 0) atomicMax(max_occ, occ);
}

// One block per crowded cell: bitonic sort in shared memory (padding with INT_MAX).
__global__ void __launch_bounds__(1024) k_sort_big_cells(const int* __restrict__ cell_start,
                                                         int* __restrict__ perm,
                                                         const int* __restrict__ big_list,
                                                         const int* big_count, int* dflag) {
    __shared__ int s[BIG_CELL_MAX];
    int nbig = *big_count;
    for (int bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
        int c = big_list[bi];
        int b = cell_start[c], e = cell_start[c + 1], occ = e - b;
        if (occ > BIG_CELL_MAX) {
            if (threadIdx.x == 0) atomicOr(dflag, DFLAG_CELL_OVERFLOW);
            continue;
        }
        int len = 1;
        while (len < occ) len <<= 1;
        for (int t = threadIdx.x; t < len; t += blockDim.x) s[t] = t < occ ? perm[b + t] : INT_MAX;
        __syncthreads();
        for (int k = 2; k <= len; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int t = threadIdx.x; t < len; t += blockDim.x) {
                    int p = t ^ j;
                    if (p > t) {
                        bool up = (t & k) == 0;
                        int a = s[t], d = s[p];
                        if ((a > d) == up) { s[t] = d; s[p] = a; }
                    }
                }
                __syncthreads();
            }
        }
        for (int t = threadIdx.x; t < occ; t += blockDim.x) perm[b + t] = s[t];
        __syncthreads();
    }
}

__global__ void k_gather_sorted(const int* __restrict__ perm, size_t n, const double* __restrict__ pos,
                                const uint8_t* __restrict__ type_in, const int* __restrict__ lin,
                                double* __restrict__ sx, double* __restrict__ sy, double* __restrict__ sz,
                                uint8_t* __restrict__ stype, int* __restrict__ scell, int* __restrict__ iperm) {
    size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    int i = perm[k];
    sx[k] = pos[3 * (size_t)i];
    sy[k] = pos[3 * (size_t)i + 1];
    sz[k] = pos[3 * (size_t)i + 2];
    stype[k] = type_in[i];
    scell[k] = lin[i];
    iperm[i] = (int)k;
}

// ---- 3. count / fill passes ---------------------------------------------------------------
struct GridView {
    const int* cell_start;
    int nx, ny, nz;
};

// Candidate range of row (dz, dy) around cell (cx, cy, cz): cells x-1..x+1 of that row.
__device__ __forceinline__ bool row_range(const GridView& g, int cx, int cy, int cz, int dy, int dz,
                                          int& beg, int& end) {
    int y = cy + dy, z = cz + dz;
    if (y < 0 || y >= g.ny || z < 0 || z >= g.nz) return false;
    int xlo = max(cx - 1, 0), xhi = min(cx + 1, g.nx - 1);
    int base = (z * g.ny + y) * g.nx;
    beg = g.cell_start[base + xlo];
    end = g.cell_start[base + xhi + 1];
    return beg < end;
}

__device__ __forceinline__ unsigned sector_bits(double dx, double dy, double dz) {
    double ax = fabs(dx), ay = fabs(dy), az = fabs(dz);
    int s = (ax >= ay && ax >= az) ? (dx >= 0 ? 0 : 1)
                                   : ((ay >= ax && ay >= az) ? (dy >= 0 ? 2 : 3) : (dz >= 0 ? 4 : 5));
    int o = 6 + (dx >= 0) + 2 * (dy >= 0) + 4 * (dz >= 0);
    return (1u << s) | (1u << o);
}

// The reference's decision (src/lsmps.cpp:27) from the kept count and sector mask.
__device__ __forceinline__ uint8_t classify_rule(uint8_t tin, int kept, unsigned sectors_mask, double z,
                                                 double l0) {
    if (tin == LSMPS_WALL) return LSMPS_WALL;
    if (kept < 10) return LSMPS_SPLASH;
    int sectors = __popc(sectors_mask);
    if (z < xmul(1.5, l0)) return LSMPS_NEAR_WALL;
    if (sectors < 11) return LSMPS_FREE_SURFACE;
    return LSMPS_INTERIOR;
}

__global__ void __launch_bounds__(NB_WARPS * 32) k_count(GridView g, const double* __restrict__ sx,
                                                       const double* __restrict__ sy,
                                                       const double* __restrict__ sz,
                                                       const int* __restrict__ scell, int n, double re2,
                                                       int maxn, int* __restrict__ cnt,
                                                       unsigned long long* trunc_total) {
    int k = blockIdx.x * NB_WARPS + (threadIdx.x >> 5);
    int lane = threadIdx.x & 31;
    unsigned long long tr = 0;
    if (k < n) {
        int lin = scell[k];
        int cx = lin % g.nx, t = lin / g.nx, cy = t % g.ny, cz = t / g.ny;
        double xi = sx[k], yi = sy[k], zi = sz[k];
        int count = 0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy) {
                int beg, end;
                if (!row_range(g, cx, cy, cz, dy, dz, beg, end)) continue;
                for (int mb = beg; mb < end; mb += 32) {
                    int m = mb + lane;
                    bool ok = false;
                    if (m < end && m != k)
                        ok = xnorm2(xsub(sx[m], xi), xsub(sy[m], yi), xsub(sz[m], zi)) < re2;
                    count += __popc(__ballot_sync(0xffffffffu, ok));
                }
            }
        if (lane == 0) {
            cnt[k] = min(count, maxn);
            tr = count > maxn ? (unsigned long long)(count - maxn) : 0ull;
        }
    }
    if (lane == 0 && tr) atomicAdd(trunc_total, tr);
}

__global__ void __launch_bounds__(NB_WARPS * 32) k_fill(GridView g, const double* __restrict__ sx,
                                                      const double* __restrict__ sy,
                                                      const double* __restrict__ sz,
                                                      const int* __restrict__ scell,
                                                      const uint8_t* __restrict__ stype, int n,
                                                      double re2, int maxn, double l0, int classify,
                                                      const int* __restrict__ row,
                                                      int* __restrict__ col, uint8_t* __restrict__ cls) {
    int k = blockIdx.x * NB_WARPS + (threadIdx.x >> 5);
    if (k >= n) return;
    int lane = threadIdx.x & 31;
    unsigned lt = (1u << lane) - 1u;
    int lin = scell[k];
    int cx = lin % g.nx, t = lin / g.nx, cy = t % g.ny, cz = t / g.ny;
    double xi = sx[k], yi = sy[k], zi = sz[k];
    int out0 = row[k];
    const int room = row[k + 1] - out0;  // = min(count, maxn) from the count pass
    int written = 0;
    unsigned sec = 0;
    for (int dz = -1; dz <= 1 && written < maxn; ++dz)
        for (int dy = -1; dy <= 1 && written < maxn; ++dy) {
            int beg, end;
            if (!row_range(g, cx, cy, cz, dy, dz, beg, end)) continue;
            for (int mb = beg; mb < end && written < maxn; mb += 32) {
                int m = mb + lane;
                bool ok = false;
                double dx = 0, dyv = 0, dzv = 0;
                if (m < end && m != k) {
                    dx = xsub(sx[m], xi);
                    dyv = xsub(sy[m], yi);
                    dzv = xsub(sz[m], zi);
                    ok = xnorm2(dx, dyv, dzv) < re2;
                }
                unsigned bal = __ballot_sync(0xffffffffu, ok);
                if (ok) {
                    int p = written + __popc(bal & lt);
                    if (p < maxn && p < room) {
                        col[out0 + p] = m;
                        if (classify) sec |= sector_bits(dx, dyv, dzv);
                    }
                }
                written += __popc(bal);
            }
        }
    if (classify) {
        sec = __reduce_or_sync(0xffffffffu, sec);
        if (lane == 0) cls[k] = classify_rule(stype[k], min(written, maxn), sec, zi, l0);
    }
}

// Standalone classification over an existing CSR (warp per particle).
__global__ void __launch_bounds__(NB_WARPS * 32) k_classify(const double* __restrict__ sx,
                                                          const double* __restrict__ sy,
                                                          const double* __restrict__ sz,
                                                          const uint8_t* __restrict__ stype, int n,
                                                          double l0, const int* __restrict__ row,
                                                          const int* __restrict__ col,
                                                          uint8_t* __restrict__ cls) {
    int k = blockIdx.x * NB_WARPS + (threadIdx.x >> 5);
    if (k >= n) return;
    int lane = threadIdx.x & 31;
    double xi = sx[k], yi = sy[k], zi = sz[k];
    int b = row[k], e = row[k + 1];
    unsigned sec = 0;
    for (int p = b + lane; p < e; p += 32) {
        int m = col[p];
        sec |= sector_bits(xsub(sx[m], xi), xsub(sy[m], yi), xsub(sz[m], zi));
    }
    sec = __reduce_or_sync(0xffffffffu, sec);
    if (lane == 0) cls[k] = classify_rule(stype[k], e - b, sec, zi, l0);
}

// Histogram of kept counts and class counts (block-private in shared memory).
// stats layout (u64): [0..4] class counts, [5] truncated pairs, [6] max count,
// [8 .. 8+maxn] count histogram.
__global__ void k_nbr_stats(const int* __restrict__ cnt, const uint8_t* __restrict__ cls, int n, int maxn,
                            int have_cls, unsigned long long* stats) {
    extern __shared__ unsigned int sh[];
    unsigned int* hist = sh;              // maxn + 1
    unsigned int* tc = sh + maxn + 1;     // 5
    unsigned int* mxc = tc + 5;           // 1
    for (int t = threadIdx.x; t < maxn + 7; t += blockDim.x) sh[t] = 0;
    __syncthreads();
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        int c = cnt[k];
        atomicAdd(&hist[c], 1u);
        atomicMax(mxc, (unsigned)c);
        if (have_cls) atomicAdd(&tc[cls[k] < 5 ? cls[k] : 0], 1u);
    }
    __syncthreads();
    for (int t = threadIdx.x; t <= maxn; t += blockDim.x)
        if (hist[t]) atomicAdd(&stats[8 + t], (unsigned long long)hist[t]);
    if (threadIdx.x < 5 && tc[threadIdx.x]) atomicAdd(&stats[threadIdx.x], (unsigned long long)tc[threadIdx.x]);
    if (threadIdx.x == 0) atomicMax(&stats[6], (unsigned long long)*mxc);
}

// ---- downloads in caller order ------------------------------------------------------------
__global__ void k_orig_counts(const int* __restrict__ iperm, const int* __restrict__ row, size_t n,
                              int* __restrict__ ocnt) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int k = iperm[i];
    ocnt[i] = row[k + 1] - row[k];
}

__global__ void k_orig_fill(const int* __restrict__ iperm, const int* __restrict__ perm,
                            const int* __restrict__ row, const int* __restrict__ col, int n,
                            const int* __restrict__ orow, int* __restrict__ ocol) {
    int i = blockIdx.x * NB_WARPS + (threadIdx.x >> 5);
    if (i >= n) return;
    int lane = threadIdx.x & 31;
    int k = iperm[i];
    int b = row[k], e = row[k + 1], o = orow[i];
    for (int p = b + lane; p < e; p += 32) ocol[o + (p - b)] = perm[col[p]];
}

__global__ void k_orig_types(const int* __restrict__ iperm, const uint8_t* __restrict__ cls, size_t n,
                             uint8_t* __restrict__ out) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = cls[iperm[i]];
}

}  // namespace

// Percentiles as the reference computes them (src/lsmps.cpp:73): sort the counts and take
// cnt[(size_t)(q * (N - 1))], here from the count histogram.
static void fill_stats(lsmps_ctx* ctx, const std::vector<unsigned long long>& st, lsmps_neighbor_stats* out) {
    size_t n = ctx->n;
    lsmps_neighbor_stats s{};
    for (int t = 0; t < 5; ++t) s.type_count[t] = st[t];
    s.truncated = st[5];
    s.max_count = (int32_t)st[6];
    s.pairs = ctx->pairs;
    s.mean = n ? (double)ctx->pairs / (double)n : 0.0;
    auto pct = [&](double q) -> int {
        if (!n) return 0;
        size_t idx = (size_t)(q * (double)(n - 1));
        unsigned long long cum = 0;
        for (int c = 0; c <= ctx->maxn; ++c) {
            cum += st[8 + c];
            if (cum > idx) return c;
        }
        return ctx->maxn;
    };
    s.p50 = pct(.5);
    s.p90 = pct(.9);
    s.p99 = pct(.99);
    s.grid_cells = ctx->ncells;
    s.max_cell_occupancy = (int32_t)st[7];
    if (out) *out = s;
}

void nb_stats(lsmps_ctx* ctx, lsmps_neighbor_stats* out) {
    int n = (int)ctx->n;
    int maxn = ctx->maxn;
    auto* st = ctx->nbr_stats.ensure<unsigned long long>(8 + maxn + 1);
    LSMPS_CUDA(cudaMemsetAsync(st, 0, (8 + maxn + 1) * sizeof(unsigned long long), ctx->stream));
    if (n > 0) {
        size_t shm = (maxn + 7) * sizeof(unsigned int);
        k_nbr_stats<<<std::min(148 * 4, (int)blocks_for(n, 256)), 256, shm, ctx->stream>>>(
            ctx->nbr_cnt.get<int>(), ctx->cls.get<uint8_t>(), n, maxn, ctx->have_classes ? 1 : 0, st);
        LSMPS_CHECK_LAUNCH();
    }
    std::vector<unsigned long long> h(8 + maxn + 1);
    LSMPS_CUDA(cudaMemcpyAsync(h.data(), st, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                               ctx->stream));
    LSMPS_CUDA(cudaStreamSynchronize(ctx->stream));
    h[5] = ctx->truncated;
    h[7] = (unsigned long long)ctx->max_cell_occupancy;
    fill_stats(ctx, h, out);
}

void nb_build(lsmps_ctx* ctx, double re, int maxn, double l0, int flags, lsmps_neighbor_stats* out) {
    LSMPS_REQUIRE(re > 0 && std::isfinite(re), LSMPS_ERR_ARG, "re must be positive and finite");
    LSMPS_REQUIRE(maxn >= 0 && maxn <= 8192, LSMPS_ERR_ARG, "max_neighbors must be in [0, 8192]");
    LSMPS_REQUIRE(ctx->n < (size_t)INT_MAX, LSMPS_ERR_OVERFLOW, "particle count beyond int32");
    cudaStream_t s = ctx->stream;
    const size_t n = ctx->n;
    ctx->re = re;
    ctx->re2 = re * re;
    ctx->l0 = l0;
    ctx->maxn = maxn;
    ctx->have_neighbors = ctx->have_classes = false;
    ctx->have_wls = ctx->have_ppe = ctx->have_solution = false;
    int* dflag = ctx->dflags.get<int>();

    // 1. cell coordinates + bounds
    int3* cell = ctx->cell_of.ensure<int3>(n);
    int* bounds = ctx->scratch.ensure<int>(64);
    int init[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
    LSMPS_CUDA(cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, s));
    if (n) {
        k_cell_coords<<<std::min<unsigned>(blocks_for(n, 256), 148 * 8), 256, 0, s>>>(
            ctx->pos.get<double>(), n, re, cell, bounds, dflag);
        LSMPS_CHECK_LAUNCH();
    }
    int hb[6];
    LSMPS_CUDA(cudaMemcpyAsync(hb, bounds, sizeof(hb), cudaMemcpyDeviceToHost, s));
    LSMPS_CUDA(cudaStreamSynchronize(s));
    check_device_flags(ctx, "cell coordinates");
    if (n == 0) { hb[0] = hb[1] = hb[2] = 0; hb[3] = hb[4] = hb[5] = 0; }
    for (int a = 0; a < 3; ++a) {
        ctx->gmin[a] = hb[a];
        ctx->gdim[a] = hb[3 + a] - hb[a] + 1;
    }
    long long ncells = (long long)ctx->gdim[0] * ctx->gdim[1] * ctx->gdim[2];
    LSMPS_REQUIRE(ncells > 0 && ncells <= MAX_CELLS, LSMPS_ERR_GRID,
                  "dense cell grid of " + std::to_string(ncells) + " cells exceeds the limit of " +
                      std::to_string(MAX_CELLS));
    ctx->ncells = ncells;

    // 2. counting sort
    int* lin = ctx->slot.ensure<int>(2 * n + 1);  // lin[0..n) and slot[n..2n)
    int* slot = lin + n;
    int* count = ctx->cell_count.ensure<int>(ncells + 1);
    int* cstart = ctx->cell_start.ensure<int>(ncells + 1);
    int* perm = ctx->perm.ensure<int>(n);
    LSMPS_CUDA(cudaMemsetAsync(count, 0, (ncells + 1) * sizeof(int), s));
    int3 g0 = make_int3(ctx->gmin[0], ctx->gmin[1], ctx->gmin[2]);
    int3 gd = make_int3(ctx->gdim[0], ctx->gdim[1], ctx->gdim[2]);
    if (n) {
        k_cell_count<<<blocks_for(n, 256), 256, 0, s>>>(cell, n, g0, gd, lin, slot, count);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<int>(count, cstart, ncells, s, ctx->scan_tmp, dflag);
    if (n) {
        k_scatter<<<blocks_for(n, 256), 256, 0, s>>>(lin, slot, n, cstart, perm);
        LSMPS_CHECK_LAUNCH();
    }
    int* big = ctx->scratch.get<int>() + 8;  // [8] big count, [9] max occupancy
    LSMPS_CUDA(cudaMemsetAsync(big, 0, 2 * sizeof(int), s));
    int* big_list = count;  // counts are no longer needed: reuse as the crowded-cell list
    k_sort_small_cells<<<(unsigned)((ncells + 255) / 256), 256, 0, s>>>(cstart, ncells, perm, big_list, big,
                                                                       big + 1);
    LSMPS_CHECK_LAUNCH();
    k_sort_big_cells<<<148, 1024, 0, s>>>(cstart, perm, big_list, big, dflag);
    LSMPS_CHECK_LAUNCH();

    double* sx = ctx->sx.ensure<double>(n);
    double* sy = ctx->sy.ensure<double>(n);
    double* sz = ctx->sz.ensure<double>(n);
    uint8_t* stype = ctx->stype.ensure<uint8_t>(n);
    int* scell = ctx->scell.ensure<int>(n);
    int* iperm = ctx->iperm.ensure<int>(n);
    if (n) {
        k_gather_sorted<<<blocks_for(n, 256), 256, 0, s>>>(perm, n, ctx->pos.get<double>(),
                                                           ctx->type_in.get<uint8_t>(), lin, sx, sy, sz,
                                                           stype, scell, iperm);
        LSMPS_CHECK_LAUNCH();
    }

    // 3. count pass, row pointers, fill pass (+ classification)
    int* cnt = ctx->nbr_cnt.ensure<int>(n + 1);
    int* row = ctx->nbr_row.ensure<int>(n + 1);
    unsigned long long* trunc_d = reinterpret_cast<unsigned long long*>(ctx->scratch.get<int>() + 16);
    LSMPS_CUDA(cudaMemsetAsync(trunc_d, 0, sizeof(unsigned long long), s));
    GridView gv{cstart, gd.x, gd.y, gd.z};
    unsigned nb_blocks = (unsigned)((n + NB_WARPS - 1) / NB_WARPS);
    if (n) {
        k_count<<<nb_blocks, NB_WARPS * 32, 0, s>>>(gv, sx, sy, sz, scell, (int)n, ctx->re2, maxn, cnt, trunc_d);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<int>(cnt, row, (long long)n, s, ctx->scan_tmp, dflag);
    int hpairs = 0;
    LSMPS_CUDA(cudaMemcpyAsync(&hpairs, row + n, sizeof(int), cudaMemcpyDeviceToHost, s));
    int hocc = 0;
    unsigned long long htr = 0;
    LSMPS_CUDA(cudaMemcpyAsync(&hocc, big + 1, sizeof(int), cudaMemcpyDeviceToHost, s));
    LSMPS_CUDA(cudaMemcpyAsync(&htr, trunc_d, sizeof(htr), cudaMemcpyDeviceToHost, s));
    LSMPS_CUDA(cudaStreamSynchronize(s));
    check_device_flags(ctx, "neighbor count");
    ctx->pairs = (uint64_t)hpairs;
    ctx->truncated = htr;
    ctx->max_cell_occupancy = hocc;
    int* col = ctx->nbr_col.ensure<int>((size_t)hpairs + 1);
    uint8_t* cls = ctx->cls.ensure<uint8_t>(n);
    const int do_cls = (flags & LSMPS_NBR_CLASSIFY) ? 1 : 0;
    if (n) {
        k_fill<<<nb_blocks, NB_WARPS * 32, 0, s>>>(gv, sx, sy, sz, scell, stype, (int)n, ctx->re2, maxn, l0,
                                                 do_cls, row, col, cls);
        LSMPS_CHECK_LAUNCH();
    }
    ctx->have_neighbors = true;
    ctx->have_classes = do_cls != 0;
    nb_stats(ctx, out);
    LSMPS_CUDA(cudaStreamSynchronize(s));
    check_device_flags(ctx, "neighbor fill");
}

void nb_kernel_bench(lsmps_ctx* ctx, int kernel, int reps, double* ms, double* bytes) {
    LSMPS_REQUIRE(ctx->have_neighbors, LSMPS_ERR_STATE, "kernel bench needs neighbor lists");
    cudaStream_t s = ctx->stream;
    int n = (int)ctx->n;
    GridView gv{ctx->cell_start.get<int>(), ctx->gdim[0], ctx->gdim[1], ctx->gdim[2]};
    unsigned nb_blocks = (unsigned)((n + NB_WARPS - 1) / NB_WARPS);
    auto* trunc_d = reinterpret_cast<unsigned long long*>(ctx->scratch.get<int>() + 16);
    auto launch = [&] {
        if (kernel == LSMPS_KB_NBR_COUNT)
            k_count<<<nb_blocks, NB_WARPS * 32, 0, s>>>(gv, ctx->sx.get<double>(), ctx->sy.get<double>(),
                                                        ctx->sz.get<double>(), ctx->scell.get<int>(), n, ctx->re2,
                                                        ctx->maxn, ctx->nbr_cnt.get<int>(), trunc_d);
        else
            k_fill<<<nb_blocks, NB_WARPS * 32, 0, s>>>(gv, ctx->sx.get<double>(), ctx->sy.get<double>(),
                                                       ctx->sz.get<double>(), ctx->scell.get<int>(),
                                                       ctx->stype.get<uint8_t>(), n, ctx->re2, ctx->maxn, ctx->l0,
                                                       ctx->have_classes ? 1 : 0, ctx->nbr_row.get<int>(),
                                                       ctx->nbr_col.get<int>(), ctx->cls.get<uint8_t>());
        LSMPS_CHECK_LAUNCH();
    };
    if (n == 0) { *ms = 0; *bytes = 0; return; }
    launch();  // warm
    ev_record(ctx, 14);
    for (int r = 0; r < reps; ++r) launch();
    ev_record(ctx, 15);
    *ms = ev_elapsed(ctx, 14, 15) / reps;
    double N = (double)n, P = (double)ctx->pairs, cells = (double)ctx->ncells;
    *bytes = kernel == LSMPS_KB_NBR_COUNT ? 32.0 * N + 4.0 * cells : 34.0 * N + 4.0 * P + 4.0 * cells;
}

void nb_classify(lsmps_ctx* ctx, double l0, lsmps_neighbor_stats* out) {
    LSMPS_REQUIRE(ctx->have_neighbors, LSMPS_ERR_STATE, "classify needs lsmps_build_neighbors first");
    int n = (int)ctx->n;
    ctx->l0 = l0;
    uint8_t* cls = ctx->cls.ensure<uint8_t>(ctx->n);
    if (n) {
        k_classify<<<(unsigned)((n + NB_WARPS - 1) / NB_WARPS), NB_WARPS * 32, 0, ctx->stream>>>(
            ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(), ctx->stype.get<uint8_t>(), n,
            l0, ctx->nbr_row.get<int>(), ctx->nbr_col.get<int>(), cls);
        LSMPS_CHECK_LAUNCH();
    }
    ctx->have_classes = true;
    ctx->have_wls = ctx->have_ppe = ctx->have_solution = false;
    nb_stats(ctx, out);
}

void nb_download(lsmps_ctx* ctx, int32_t* row_ptr, int32_t* col, size_t col_cap) {
    LSMPS_REQUIRE(ctx->have_neighbors, LSMPS_ERR_STATE, "no neighbor lists built");
    cudaStream_t s = ctx->stream;
    size_t n = ctx->n;
    int* ocnt = ctx->vtmp.ensure<int>(2 * n + 2);
    int* orow = ocnt + n + 1;
    if (n) {
        k_orig_counts<<<blocks_for(n, 256), 256, 0, s>>>(ctx->iperm.get<int>(), ctx->nbr_row.get<int>(), n, ocnt);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<int>(ocnt, orow, (long long)n, s, ctx->scan_tmp, ctx->dflags.get<int>());
    if (row_ptr) LSMPS_CUDA(cudaMemcpyAsync(row_ptr, orow, (n + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (col) {
        LSMPS_REQUIRE(col_cap >= ctx->pairs, LSMPS_ERR_ARG, "col buffer smaller than the pair count");
        int* ocol = ctx->vs.ensure<int>(ctx->pairs + 1);
        if (n) {
            k_orig_fill<<<(unsigned)((n + NB_WARPS - 1) / NB_WARPS), NB_WARPS * 32, 0, s>>>(
                ctx->iperm.get<int>(), ctx->perm.get<int>(), ctx->nbr_row.get<int>(), ctx->nbr_col.get<int>(),
                (int)n, orow, ocol);
            LSMPS_CHECK_LAUNCH();
        }
        LSMPS_CUDA(cudaMemcpyAsync(col, ocol, ctx->pairs * sizeof(int), cudaMemcpyDeviceToHost, s));
    }
    LSMPS_CUDA(cudaStreamSynchronize(s));
}

void nb_download_types(lsmps_ctx* ctx, uint8_t* type, size_t n) {
    LSMPS_REQUIRE(ctx->have_classes, LSMPS_ERR_STATE, "no classification computed");
    LSMPS_REQUIRE(n == ctx->n, LSMPS_ERR_ARG, "type buffer size differs from the particle count");
    uint8_t* tmp = ctx->vtmp.ensure<uint8_t>(n + 1);
    if (n) {
        k_orig_types<<<blocks_for(n, 256), 256, 0, ctx->stream>>>(ctx->iperm.get<int>(), ctx->cls.get<uint8_t>(),
                                                                  n, tmp);
        LSMPS_CHECK_LAUNCH();
        LSMPS_CUDA(cudaMemcpyAsync(type, tmp, n, cudaMemcpyDeviceToHost, ctx->stream));
    }
    LSMPS_CUDA(cudaStreamSynchronize(ctx->stream));
}

}  // namespace lsmps_gpu
