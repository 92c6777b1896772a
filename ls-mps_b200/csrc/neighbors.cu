// Uniform-grid neighbor build and 14-direction classification on sm_100a.
//
// Semantics follow the reference's neighbors() and classify() (src/lsmps.cpp:16-18,26-27)
// bit for bit; the data flow is the GPU's own:
//   1. cell coordinates floor(r / re) (IEEE division) and their bounding box;
//   2. a counting sort of particles into a dense cell grid (atomic slots, scan), then
//      each cell's members sorted by particle index, so that every 3-cell x-row of the grid
//      is one contiguous, index-ascending range of the sorted arrays;
//   3. a count pass and a fill pass, one block per segment of 4 cells along x, one warp per
//      particle: the block stages its 9 cell rows' candidates in shared memory, a warp tests
//      a particle's 9 contiguous row ranges 32 candidates at a time (FP32 guard band, exact
//      FP64 near the cutoff), and a ballot gives each accepted candidate its position. Scanning the 9 rows in (dz, dy) order with candidates in sorted order is
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
constexpr double SLOT_BUDGET_BYTES = 4e9;     // slot rows of the single-pass build (n x maxn x 4 B)

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
    // the block's bounds, then six atomics per block (per-warp atomics on the same six words
    // serialise in L2: ~9.5k per word at 1M particles)
    __shared__ int sb[6][32];
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            sb[a][warp] = mn[a];
            sb[3 + a][warp] = mx[a];
        }
    }
    __syncthreads();
    if (threadIdx.x < 6) {
        const int a = threadIdx.x;
        int v = sb[a][0];
        for (int w = 1; w < nwarps; ++w) v = a < 3 ? min(v, sb[a][w]) : max(v, sb[a][w]);
        if (a < 3 ? v != INT_MAX : v != INT_MIN) {
            if (a < 3) atomicMin(&bounds[a], v);
            else atomicMax(&bounds[a], v);
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

// Atomic slots leave a cell's members in arbitrary order; restore ascending index (cells of up
// to 32 members sorted in registers, up to SMALL_CELL in place).
// Ascending bitonic sort of N (a power of two) values held in registers (the loops unroll to
// fixed indices).
template <int N>
__device__ __forceinline__ void bitonic_sort_regs(int (&v)[N]) {
#pragma unroll
    for (int k = 2; k <= N; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int l = i ^ j;
                if (l > i) {
                    const int a = v[i], c = v[l];
                    const bool asc = (i & k) == 0;
                    v[i] = asc ? min(a, c) : max(a, c);
                    v[l] = asc ? max(a, c) : min(a, c);
                }
            }
}

// A cell's members (occ <= N, distinct indices) sorted ascending in registers: all loads in
// flight at once, padding INT_MAX sorts last.
template <int N>
__device__ __forceinline__ void sort_cell_regs(int* __restrict__ perm, int b, int occ) {
    int v[N];
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = i < occ ? perm[b + i] : INT_MAX;
    bitonic_sort_regs<N>(v);
#pragma unroll
    for (int i = 0; i < N; ++i)
        if (i < occ) perm[b + i] = v[i];
}

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
        } else if (occ > 1 && occ <= 16) {
            sort_cell_regs<16>(perm, b, occ);
        } else if (occ > 1 && occ <= 32) {
            sort_cell_regs<32>(perm, b, occ);
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
    // one atomic per block (per-warp atomics on one word serialise in L2)
    __shared__ int socc[32];
    if ((threadIdx.x & 31) == 0) socc[threadIdx.x >> 5] = occ;
    __syncthreads();
    if (threadIdx.x == 0) {
        int m = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = max(m, socc[w]);
        if (m > 0) atomicMax(max_occ, m);
    }
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

// Global-memory form of one query (one warp): count / fill the accepted candidates of
// sorted particle k; used by the staged kernels when a segment's neighborhood does not fit
// in shared memory.
__device__ __forceinline__ int count_query_global(const GridView& g, const double* __restrict__ sx,
                                                  const double* __restrict__ sy, const double* __restrict__ sz,
                                                  const int* __restrict__ scell, int k, double re2, int lane) {
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
                if (m < end && m != k) ok = xnorm2(xsub(sx[m], xi), xsub(sy[m], yi), xsub(sz[m], zi)) < re2;
                count += __popc(__ballot_sync(0xffffffffu, ok));
            }
        }
    return count;
}

__device__ __forceinline__ void fill_query_global(const GridView& g, const double* __restrict__ sx,
                                                  const double* __restrict__ sy, const double* __restrict__ sz,
                                                  const int* __restrict__ scell, const uint8_t* __restrict__ stype,
                                                  int k, double re2, int maxn, double l0, int classify,
                                                  const int* __restrict__ row, int* __restrict__ col,
                                                  uint8_t* __restrict__ cls, int lane) {
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

// ---- staged passes: one block per segment of SEG cells along x, one thread per particle -----
// The block copies the candidates of its 9 cell rows (cells cx0-1 .. cx1+1 of rows (cy+dy,
// cz+dz)) into shared memory once, as FP32 positions relative to the segment's corner, plus
// the row pointers of its own particles (a contiguous range of the sorted arrays). Each
// thread then walks one particle's 9 row ranges (cells cx-1 .. cx+1 of each row, contiguous
// in the sorted order) candidate by candidate, so its kept list comes out in the reference's
// order without any cross-lane bookkeeping. Cells whose box is farther than re (plus a 1e-4
// relative margin) are skipped. A candidate is accepted when its FP32 distance^2 is below
// re^2 (1 - 2e-5) and rejected above re^2 (1 + 2e-5); in between the exact FP64 test on the
// global positions decides. Coordinates lie within (SEG + 2) re of the corner, so the FP32
// distance^2 is within 1e-5 re^2 of the exact one and the kept lists are the reference's bit
// for bit. The sector bits of the classification use the FP32 differences when every sign
// and |d| comparison they need is separated by more than 4e-6 re, else the exact FP64 ones.
constexpr int SEG = 12;
constexpr int SEG_THREADS = 128;
constexpr int SEG_MAXC = 1536;  // staged candidates (24 KB)
constexpr int SEG_MAXQ = 512;   // queries per segment

struct SegGrid {
    GridView g;
    int3 g0;   // grid origin cell
    double re;
    int nsegx;
};

__device__ __forceinline__ bool sector_bits_f32(float dx, float dy, float dz, float margin, unsigned& bits) {
    const float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
    if (fminf(fminf(ax, ay), az) <= margin || fabsf(ax - ay) <= margin || fabsf(ax - az) <= margin ||
        fabsf(ay - az) <= margin)
        return false;
    const int s = (ax >= ay && ax >= az) ? (dx >= 0 ? 0 : 1) : ((ay >= ax && ay >= az) ? (dy >= 0 ? 2 : 3) : (dz >= 0 ? 4 : 5));
    const int o = 6 + (dx >= 0) + 2 * (dy >= 0) + 4 * (dz >= 0);
    bits = (1u << s) | (1u << o);
    return true;
}

// Non-empty segments of the grid, listed in any order (each segment's outputs are addressed
// by its own particles, so the order does not affect the result).
__global__ void k_list_segments(SegGrid G, long long nseg, int* __restrict__ list, int* __restrict__ count) {
    const long long seg = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    bool nonempty = false;
    if (seg < nseg) {
        const int sxi = (int)(seg % G.nsegx);
        const long long tt = seg / G.nsegx;
        const int cy = (int)(tt % G.g.ny), cz = (int)(tt / G.g.ny);
        const int cx0 = sxi * SEG, cx1 = min(cx0 + SEG, G.g.nx) - 1;
        const int rowlin = (cz * G.g.ny + cy) * G.g.nx;
        nonempty = G.g.cell_start[rowlin + cx0] != G.g.cell_start[rowlin + cx1 + 1];
    }
    const unsigned bal = __ballot_sync(0xffffffffu, nonempty);
    int base = 0;
    if ((threadIdx.x & 31) == 0 && bal) base = atomicAdd(count, __popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (nonempty) list[base + __popc(bal & ((1u << (threadIdx.x & 31)) - 1u))] = (int)seg;
}

// One accepted-or-band candidate of the thread's query (the rare path of the scan).
template <bool FILL>
__device__ __forceinline__ void seg_accept(float d2, float lo_th, float dx, float dy, float dz, int m, int k,
                                           const double* __restrict__ sx, const double* __restrict__ sy,
                                           const double* __restrict__ sz, double re2, int maxn, int room, int out0,
                                           int classify, float margin, int* __restrict__ col, int& written,
                                           unsigned& sec) {
    if (m == k) return;
    if (d2 >= lo_th && !(xnorm2(xsub(sx[m], sx[k]), xsub(sy[m], sy[k]), xsub(sz[m], sz[k])) < re2)) return;
    if (FILL && written < maxn && written < room) {
        col[out0 + written] = m;
        if (classify) {
            unsigned bb;
            if (!sector_bits_f32(dx, dy, dz, margin, bb))
                bb = sector_bits(xsub(sx[m], sx[k]), xsub(sy[m], sy[k]), xsub(sz[m], sz[k]));
            sec |= bb;
        }
    }
    ++written;
}

template <bool FILL>
__global__ void __launch_bounds__(SEG_THREADS, 8) k_seg_pass(SegGrid G, const int* __restrict__ seg_list,
                                                            const double* __restrict__ sx,
                                                            const double* __restrict__ sy,
                                                            const double* __restrict__ sz,
                                                            const int* __restrict__ scell,
                                                            const uint8_t* __restrict__ stype, double re2,
                                                            int maxn, double l0, int classify,
                                                            int* __restrict__ cnt,
                                                            unsigned long long* trunc_total,
                                                            const int* __restrict__ row, int* __restrict__ col,
                                                            uint8_t* __restrict__ cls) {
    __shared__ float4 cf[SEG_MAXC];
    __shared__ int qrow[SEG_MAXQ + 1];
    __shared__ int rbase[10], rfirst[9], rcs[9][SEG + 3];
    const float re_f = (float)G.re;
    const float re2f = (float)re2;
    const float lo_th = re2f * (1.f - 2e-5f), hi_th = re2f * (1.f + 2e-5f);
    const float cull = re2f * (1.f + 1e-4f);
    const float margin = 4e-6f * re_f;
    const int seg = seg_list[blockIdx.x];
    const int sxi = seg % G.nsegx, tt = seg / G.nsegx, cy = tt % G.g.ny, cz = tt / G.g.ny;
    const int cx0 = sxi * SEG, cx1 = min(cx0 + SEG, G.g.nx) - 1;
    const int lo = max(cx0 - 1, 0), hi = min(cx1 + 1, G.g.nx - 1);
    const int rowlin = (cz * G.g.ny + cy) * G.g.nx;
    const int q0 = G.g.cell_start[rowlin + cx0], q1 = G.g.cell_start[rowlin + cx1 + 1];
    for (int t = threadIdx.x; t < 9 * (SEG + 3); t += blockDim.x) {
        const int r = t / (SEG + 3), c = lo + t % (SEG + 3);
        const int y = cy + (r % 3 - 1), z = cz + (r / 3 - 1);
        int v = 0;
        if (y >= 0 && y < G.g.ny && z >= 0 && z < G.g.nz && c <= hi + 1) v = G.g.cell_start[(z * G.g.ny + y) * G.g.nx + c];
        rcs[r][c - lo] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        rbase[0] = 0;
        for (int r = 0; r < 9; ++r) {
            rfirst[r] = rcs[r][0];
            rbase[r + 1] = rbase[r] + (rcs[r][hi + 1 - lo] - rcs[r][0]);
        }
    }
    __syncthreads();
    const int total = rbase[9];
    if (total > SEG_MAXC || q1 - q0 > SEG_MAXQ) {
        // crowded neighborhood: the global-memory form, one query per warp
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int k = q0 + warp; k < q1; k += SEG_THREADS / 32) {
            if (FILL) {
                fill_query_global(G.g, sx, sy, sz, scell, stype, k, re2, maxn, l0, classify, row, col, cls, lane);
            } else {
                int c = count_query_global(G.g, sx, sy, sz, scell, k, re2, lane);
                if (lane == 0) {
                    cnt[k] = min(c, maxn);
                    if (c > maxn) atomicAdd(trunc_total, (unsigned long long)(c - maxn));
                }
            }
        }
        return;
    }
    const double ox = (G.g0.x + cx0) * G.re, oy = (G.g0.y + cy) * G.re, oz = (G.g0.z + cz) * G.re;
    for (int r = 0; r < 9; ++r) {  // row by row: consecutive threads load consecutive particles
        const int n_r = rbase[r + 1] - rbase[r], f = rfirst[r], b = rbase[r];
        for (int i = threadIdx.x; i < n_r; i += blockDim.x)
            cf[b + i] = make_float4((float)(sx[f + i] - ox), (float)(sy[f + i] - oy), (float)(sz[f + i] - oz), 0.f);
    }
    if (FILL)
        for (int i = threadIdx.x; i <= q1 - q0; i += blockDim.x) qrow[i] = row[q0 + i];
    __syncthreads();
    for (int k = q0 + threadIdx.x; k < q1; k += blockDim.x) {
        int ck = cx0;
        while (ck < cx1 && k >= rcs[4][ck + 1 - lo]) ++ck;
        const float4 qf = cf[rbase[4] + (k - rfirst[4])];  // the query is staged in the centre row
        const float qx = qf.x - (ck - cx0) * re_f;          // position inside its own cell (x)
        int written = 0, out0 = 0, room = 0;
        unsigned sec = 0;
        if (FILL) {
            out0 = qrow[k - q0];
            room = qrow[k - q0 + 1] - out0;
        }
        for (int r = 0; r < 9; ++r) {
            const int dy = r % 3 - 1, dz = r / 3 - 1;
            const float gy = dy < 0 ? qf.y : (dy > 0 ? re_f - qf.y : 0.f);
            const float gz = dz < 0 ? qf.z : (dz > 0 ? re_f - qf.z : 0.f);
            const float gyz = gy * gy + gz * gz;
            if (gyz > cull) continue;
            // cells ck-1 .. ck+1 of this row, each kept when its box is within re
            int clo = max(ck - 1, lo), chi = min(ck + 1, hi);
            if (clo < ck && gyz + qx * qx > cull) clo = ck;
            if (chi > ck && gyz + (re_f - qx) * (re_f - qx) > cull) chi = ck;
            const int gb = rcs[r][clo - lo], ge = rcs[r][chi + 1 - lo];
            const int sb = rbase[r] + (gb - rfirst[r]);
            const int se = sb + (ge - gb);
            const int mshift = rfirst[r] - rbase[r];  // global index = staged index + mshift
            int si = sb;
            for (; si + 4 <= se; si += 4) {
                float d2[4], ddx[4], ddy[4], ddz[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const float4 cj = cf[si + u];
                    ddx[u] = cj.x - qf.x;
                    ddy[u] = cj.y - qf.y;
                    ddz[u] = cj.z - qf.z;
                    d2[u] = ddx[u] * ddx[u] + ddy[u] * ddy[u] + ddz[u] * ddz[u];
                }
#pragma unroll
                for (int u = 0; u < 4; ++u)
                    if (d2[u] <= hi_th)
                        seg_accept<FILL>(d2[u], lo_th, ddx[u], ddy[u], ddz[u], si + u + mshift, k, sx, sy, sz, re2,
                                         maxn, room, out0, classify, margin, col, written, sec);
            }
            for (; si < se; ++si) {
                const float4 cj = cf[si];
                const float dx = cj.x - qf.x, dyf = cj.y - qf.y, dzf = cj.z - qf.z;
                const float d2 = dx * dx + dyf * dyf + dzf * dzf;
                if (d2 <= hi_th)
                    seg_accept<FILL>(d2, lo_th, dx, dyf, dzf, si + mshift, k, sx, sy, sz, re2, maxn, room, out0,
                                     classify, margin, col, written, sec);
            }
        }
        if (FILL) {
            if (classify) cls[k] = classify_rule(stype[k], min(written, maxn), sec, sz[k], l0);
        } else {
            cnt[k] = min(written, maxn);
            if (written > maxn) atomicAdd(trunc_total, (unsigned long long)(written - maxn));
        }
    }
}

// ---- single pass: each query's kept list straight into its slot row ------------------------
// The staging, the cell culling and the FP32 guard band of k_seg_pass, in one pass instead of
// a count and a fill pass that repeat every distance test. A thread tests its row window 32
// staged candidates at a time into a hit mask (no branch per candidate), then walks the set
// bits in order: the rare guard-band hits are decided exactly in FP64, and each kept candidate
// p < maxn goes to slots[k * maxn + p] with its sector bits. Counting continues past maxn for
// the truncation statistic. k_slots_compact then packs the slot rows into the CSR once the
// kept counts are scanned. The kept order is the staged order of the 9 row windows, which is
// the reference's order, as in k_seg_pass.
__device__ __forceinline__ void scan_query_global(const GridView& g, const double* __restrict__ sx,
                                                  const double* __restrict__ sy, const double* __restrict__ sz,
                                                  const int* __restrict__ scell, const uint8_t* __restrict__ stype,
                                                  int k, double re2, int maxn, double l0, int classify,
                                                  int* __restrict__ slots, int* __restrict__ cnt,
                                                  unsigned long long* trunc_total, uint8_t* __restrict__ cls,
                                                  int lane) {
    const unsigned lt = (1u << lane) - 1u;
    const int lin = scell[k];
    const int cx = lin % g.nx, t = lin / g.nx, cy = t % g.ny, cz = t / g.ny;
    const double xi = sx[k], yi = sy[k], zi = sz[k];
    int* out = slots + (size_t)k * maxn;
    int written = 0;
    unsigned sec = 0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy) {
            int beg, end;
            if (!row_range(g, cx, cy, cz, dy, dz, beg, end)) continue;
            for (int mb = beg; mb < end; mb += 32) {
                const int m = mb + lane;
                bool ok = false;
                double dx = 0, dyv = 0, dzv = 0;
                if (m < end && m != k) {
                    dx = xsub(sx[m], xi);
                    dyv = xsub(sy[m], yi);
                    dzv = xsub(sz[m], zi);
                    ok = xnorm2(dx, dyv, dzv) < re2;
                }
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                if (ok) {
                    const int p = written + __popc(bal & lt);
                    if (p < maxn) {
                        out[p] = m;
                        if (classify) sec |= sector_bits(dx, dyv, dzv);
                    }
                }
                written += __popc(bal);
            }
        }
    if (lane == 0) {
        cnt[k] = min(written, maxn);
        if (written > maxn) atomicAdd(trunc_total, (unsigned long long)(written - maxn));
    }
    if (classify) {
        sec = __reduce_or_sync(0xffffffffu, sec);
        if (lane == 0) cls[k] = classify_rule(stype[k], min(written, maxn), sec, zi, l0);
    }
}

__global__ void __launch_bounds__(SEG_THREADS, 8) k_seg_scan(SegGrid G, const int* __restrict__ seg_list,
                                                            const double* __restrict__ sx,
                                                            const double* __restrict__ sy,
                                                            const double* __restrict__ sz,
                                                            const int* __restrict__ scell,
                                                            const uint8_t* __restrict__ stype, double re2,
                                                            int maxn, double l0, int classify,
                                                            int* __restrict__ cnt,
                                                            unsigned long long* trunc_total,
                                                            int* __restrict__ slots, uint8_t* __restrict__ cls) {
    // staged candidates in pairs, for the packed FP32x2 arithmetic: pair p holds the x and y
    // of candidates 2p and 2p + 1 in cxy[p] and their z in cz[p]
    __shared__ float4 cxy[SEG_MAXC / 2 + 1];
    __shared__ float2 cz[SEG_MAXC / 2 + 1];
    __shared__ int rbase[10], rfirst[9], rcs[9][SEG + 3];
    const float re_f = (float)G.re;
    const float re2f = (float)re2;
    const float lo_th = re2f * (1.f - 2e-5f), hi_th = re2f * (1.f + 2e-5f);
    const float cull = re2f * (1.f + 1e-4f);
    const float margin = 4e-6f * re_f;
    const int seg = seg_list[blockIdx.x];
    const int sxi = seg % G.nsegx, tt = seg / G.nsegx, cy = tt % G.g.ny, cz0 = tt / G.g.ny;
    const int cx0 = sxi * SEG, cx1 = min(cx0 + SEG, G.g.nx) - 1;
    const int lo = max(cx0 - 1, 0), hi = min(cx1 + 1, G.g.nx - 1);
    const int rowlin = (cz0 * G.g.ny + cy) * G.g.nx;
    const int q0 = G.g.cell_start[rowlin + cx0], q1 = G.g.cell_start[rowlin + cx1 + 1];
    for (int t = threadIdx.x; t < 9 * (SEG + 3); t += blockDim.x) {
        const int r = t / (SEG + 3), c = lo + t % (SEG + 3);
        const int y = cy + (r % 3 - 1), z = cz0 + (r / 3 - 1);
        int v = 0;
        if (y >= 0 && y < G.g.ny && z >= 0 && z < G.g.nz && c <= hi + 1) v = G.g.cell_start[(z * G.g.ny + y) * G.g.nx + c];
        rcs[r][c - lo] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        rbase[0] = 0;
        for (int r = 0; r < 9; ++r) {
            rfirst[r] = rcs[r][0];
            rbase[r + 1] = rbase[r] + (rcs[r][hi + 1 - lo] - rcs[r][0]);
        }
    }
    __syncthreads();
    const int total = rbase[9];
    if (total > SEG_MAXC) {
        // crowded neighborhood: the global-memory form, one query per warp
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int k = q0 + warp; k < q1; k += SEG_THREADS / 32)
            scan_query_global(G.g, sx, sy, sz, scell, stype, k, re2, maxn, l0, classify, slots, cnt, trunc_total, cls,
                              lane);
        return;
    }
    const double ox = (G.g0.x + cx0) * G.re, oy = (G.g0.y + cy) * G.re, oz = (G.g0.z + cz0) * G.re;
    float* fxy = reinterpret_cast<float*>(cxy);
    float* fz = reinterpret_cast<float*>(cz);
    for (int r = 0; r < 9; ++r) {  // row by row: consecutive threads load consecutive particles
        const int n_r = rbase[r + 1] - rbase[r], f = rfirst[r], b = rbase[r];
        for (int i = threadIdx.x; i < n_r; i += blockDim.x) {
            const int si = b + i, p = si >> 1, h = si & 1;
            fxy[4 * p + h] = (float)(sx[f + i] - ox);
            fxy[4 * p + 2 + h] = (float)(sy[f + i] - oy);
            fz[2 * p + h] = (float)(sz[f + i] - oz);
        }
    }
    __syncthreads();
    for (int k = q0 + threadIdx.x; k < q1; k += blockDim.x) {
        const int ck = scell[k] - rowlin;                   // the query's cell along x
        const int kst = rbase[4] + (k - rfirst[4]);         // the query staged in the centre row
        const float qxs = fxy[4 * (kst >> 1) + (kst & 1)], qys = fxy[4 * (kst >> 1) + 2 + (kst & 1)];
        const float qzs = fz[2 * (kst >> 1) + (kst & 1)];
        const float2 nqx = make_float2(-qxs, -qxs), nqy = make_float2(-qys, -qys), nqz = make_float2(-qzs, -qzs);
        const float qx = qxs - (ck - cx0) * re_f;          // position inside its own cell (x)
        int* out = slots + (size_t)k * maxn;
        int written = 0;
        unsigned sec = 0;
        for (int r = 0; r < 9; ++r) {
            const int dy = r % 3 - 1, dz = r / 3 - 1;
            const float gy = dy < 0 ? qys : (dy > 0 ? re_f - qys : 0.f);
            const float gz = dz < 0 ? qzs : (dz > 0 ? re_f - qzs : 0.f);
            const float gyz = gy * gy + gz * gz;
            if (gyz > cull) continue;
            // cells ck-1 .. ck+1 of this row, each kept when its box is within re
            int clo = max(ck - 1, lo), chi = min(ck + 1, hi);
            if (clo < ck && gyz + qx * qx > cull) clo = ck;
            if (chi > ck && gyz + (re_f - qx) * (re_f - qx) > cull) chi = ck;
            const int gb = rcs[r][clo - lo], ge = rcs[r][chi + 1 - lo];
            const int sb = rbase[r] + (gb - rfirst[r]);
            const int se = sb + (ge - gb);
            const int mshift = rfirst[r] - rbase[r];  // global index = staged index + mshift
            const int pend = (se + 1) >> 1;
            for (int pb = sb >> 1; pb < pend; pb += 16) {
                const int c0 = pb << 1;  // first staged candidate of this chunk of 32
                const int np = min(16, pend - pb);
                unsigned hit = 0;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    if (j < np) {
                        const float4 a = cxy[pb + j];
                        const float2 dxv = __fadd2_rn(make_float2(a.x, a.y), nqx);
                        const float2 dyv = __fadd2_rn(make_float2(a.z, a.w), nqy);
                        const float2 dzv = __fadd2_rn(cz[pb + j], nqz);
                        float2 d2 = __fmul2_rn(dxv, dxv);
                        d2 = __ffma2_rn(dyv, dyv, d2);
                        d2 = __ffma2_rn(dzv, dzv, d2);
                        if (d2.x <= hi_th) hit |= 1u << (2 * j);
                        if (d2.y <= hi_th) hit |= 2u << (2 * j);
                    }
                }
                // keep the window [sb, se) and drop the query itself
                const int wlo = sb - c0, whi = se - c0;
                if (whi < 32) hit &= (1u << whi) - 1u;
                if (wlo > 0) hit &= ~((1u << wlo) - 1u);
                if (r == 4 && kst >= c0 && kst < c0 + 32) hit &= ~(1u << (kst - c0));
                while (hit) {
                    const int i = __ffs(hit) - 1;
                    hit &= hit - 1;
                    const int si = c0 + i, p = si >> 1, h = si & 1;
                    const float dx = fxy[4 * p + h] - qxs, dyf = fxy[4 * p + 2 + h] - qys, dzf = fz[2 * p + h] - qzs;
                    const float d2 = dx * dx + dyf * dyf + dzf * dzf;
                    const int m = si + mshift;
                    if (d2 >= lo_th && !(xnorm2(xsub(sx[m], sx[k]), xsub(sy[m], sy[k]), xsub(sz[m], sz[k])) < re2))
                        continue;
                    if (written < maxn) {
                        out[written] = m;
                        if (classify) {
                            unsigned bb;
                            if (!sector_bits_f32(dx, dyf, dzf, margin, bb))
                                bb = sector_bits(xsub(sx[m], sx[k]), xsub(sy[m], sy[k]), xsub(sz[m], sz[k]));
                            sec |= bb;
                        }
                    }
                    ++written;
                }
            }
        }
        cnt[k] = min(written, maxn);
        if (written > maxn) atomicAdd(trunc_total, (unsigned long long)(written - maxn));
        if (classify) cls[k] = classify_rule(stype[k], min(written, maxn), sec, sz[k], l0);
    }
}

// Packs the slot rows into the CSR: eight lanes per row, row k's kept list from
// slots[k * maxn] to col[row[k]].
__global__ void __launch_bounds__(256) k_slots_compact(int n, int maxn, const int* __restrict__ slots,
                                                       const int* __restrict__ row, int* __restrict__ col) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int k = (int)(g >> 3), sub = (int)(g & 7);
    if (k >= n) return;
    const int b = row[k], c = row[k + 1] - b;
    const int* src = slots + (size_t)k * maxn;
    for (int p = sub; p < c; p += 8) col[b + p] = __ldcs(src + p);
}

// Refresh of skin lists in one pass (warp per particle): the candidates j != i of the candidate
// CSR (radius re + skin, ascending sorted index) that pass the build's exact FP64 test
// |r_j - r_i|^2 < re^2, in candidate order, go to the particle's slot row (the first maxn),
// with the sector bits of the kept ones for the classification; counting continues past maxn.
__global__ void __launch_bounds__(256) k_filter_slots(int n, const int* __restrict__ crow,
                                                      const int* __restrict__ ccol, const double* __restrict__ sx,
                                                      const double* __restrict__ sy, const double* __restrict__ sz,
                                                      const uint8_t* __restrict__ stype, double re2, int maxn,
                                                      double l0, int classify, int* __restrict__ slots,
                                                      int* __restrict__ cnt, unsigned long long* trunc,
                                                      uint8_t* __restrict__ cls) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int nw = (int)((gridDim.x * (size_t)blockDim.x) >> 5);
    for (int i = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5); i < n; i += nw) {
        const double xi = sx[i], yi = sy[i], zi = sz[i];
        const int c0 = crow[i], c1 = crow[i + 1];
        int* out = slots + (size_t)i * maxn;
        int kept = 0;
        unsigned sec = 0;
        for (int b = c0; b < c1; b += 32) {
            const int e = b + lane;
            bool ok = false;
            int j = 0;
            double dx = 0, dy = 0, dz = 0;
            if (e < c1) {
                j = ccol[e];
                dx = xsub(sx[j], xi);
                dy = xsub(sy[j], yi);
                dz = xsub(sz[j], zi);
                ok = j != i && xnorm2(dx, dy, dz) < re2;
            }
            const unsigned m = __ballot_sync(0xffffffffu, ok);
            if (ok) {
                const int p = kept + __popc(m & lt);
                if (p < maxn) {
                    out[p] = j;
                    if (classify) sec |= sector_bits(dx, dy, dz);
                }
            }
            kept += __popc(m);
        }
        if (lane == 0) {
            cnt[i] = min(kept, maxn);
            if (kept > maxn) atomicAdd(trunc, (unsigned long long)(kept - maxn));
        }
        if (classify) {
            sec = __reduce_or_sync(0xffffffffu, sec);
            if (lane == 0) cls[i] = classify_rule(stype[i], min(kept, maxn), sec, zi, l0);
        }
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

void nb_stats(lsmps_ctx* ctx, lsmps_neighbor_stats* out, const char* where) {
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
    read_back(ctx, {{st, h.data(), h.size() * sizeof(unsigned long long)}}, where);
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
    ctx->have_candidates = false;  // the sorted numbering changes
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
    read_back(ctx, {{bounds, hb, sizeof(hb)}}, "cell coordinates");
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
    SegGrid sg{gv, g0, re, (gd.x + SEG - 1) / SEG};
    const long long nseg = (long long)sg.nsegx * gd.y * gd.z;
    LSMPS_REQUIRE(nseg < (1ll << 31), LSMPS_ERR_GRID, "too many cell segments");
    int* seg_list = ctx->seg_list.ensure<int>(nseg + 1);
    int* seg_count = ctx->scratch.get<int>() + 40;
    LSMPS_CUDA(cudaMemsetAsync(seg_count, 0, sizeof(int), s));
    k_list_segments<<<(unsigned)((nseg + 255) / 256), 256, 0, s>>>(sg, nseg, seg_list, seg_count);
    LSMPS_CHECK_LAUNCH();
    int hsegs = 0;
    read_back(ctx, {{seg_count, &hsegs, sizeof(int)}}, nullptr);
    ctx->nsegs = hsegs;
    const unsigned seg_grid = (unsigned)std::max(hsegs, 1);
    const int do_cls = (flags & LSMPS_NBR_CLASSIFY) ? 1 : 0;
    uint8_t* cls = ctx->cls.ensure<uint8_t>(n);
    // one pass into maxn slots per particle while they fit (the usual case: 0.5 GB at 1M
    // particles and maxn 128), else the count and fill passes
    const bool single = !(flags & LSMPS_NBR_TWO_PASS) && (double)n * (double)maxn * 4.0 <= SLOT_BUDGET_BYTES;
    ctx->nbr_single = single;
    int* slots = single ? ctx->nbr_slots.ensure<int>((size_t)n * maxn + 1) : nullptr;
    if (n && hsegs) {
        if (single)
            k_seg_scan<<<seg_grid, SEG_THREADS, 0, s>>>(sg, seg_list, sx, sy, sz, scell, stype, ctx->re2, maxn, l0,
                                                       do_cls, cnt, trunc_d, slots, cls);
        else
            k_seg_pass<false><<<seg_grid, SEG_THREADS, 0, s>>>(sg, seg_list, sx, sy, sz, scell, stype,
                                                                 ctx->re2, maxn, l0, 0, cnt, trunc_d, nullptr, nullptr,
                                                                 nullptr);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<int>(cnt, row, (long long)n, s, ctx->scan_tmp, dflag);
    int hpairs = 0, hocc = 0;
    unsigned long long htr = 0;
    read_back(ctx, {{row + n, &hpairs, sizeof(int)}, {big + 1, &hocc, sizeof(int)}, {trunc_d, &htr, sizeof(htr)}},
              "neighbor count");
    ctx->pairs = (uint64_t)hpairs;
    ctx->truncated = htr;
    ctx->max_cell_occupancy = hocc;
    int* col = ctx->nbr_col.ensure<int>((size_t)hpairs + 1);
    if (n && hsegs) {
        if (single)
            k_slots_compact<<<(unsigned)((8ull * n + 255) / 256), 256, 0, s>>>((int)n, maxn, slots, row, col);
        else
            k_seg_pass<true><<<seg_grid, SEG_THREADS, 0, s>>>(sg, seg_list, sx, sy, sz, scell, stype,
                                                                ctx->re2, maxn, l0, do_cls, nullptr, nullptr, row, col,
                                                                cls);
        LSMPS_CHECK_LAUNCH();
    }
    ctx->have_neighbors = true;
    ctx->have_classes = do_cls != 0;
    // without statistics nothing is read back here (no device flag is set after the count's
    // read-back), so the host does not wait for the compaction
    if (out) nb_stats(ctx, out, "neighbor fill");
}

bool nb_filter_single(lsmps_ctx* ctx, int classify) {
    const size_t n = ctx->n;
    const int maxn = ctx->maxn;
    if ((double)n * (double)maxn * 4.0 > SLOT_BUDGET_BYTES) return false;
    cudaStream_t s = ctx->stream;
    int* dflag = ctx->dflags.get<int>();
    int* cnt = ctx->nbr_cnt.ensure<int>(n + 1);
    int* row = ctx->nbr_row.ensure<int>(n + 1);
    int* slots = ctx->nbr_slots.ensure<int>(n * maxn + 1);
    uint8_t* cls = ctx->cls.ensure<uint8_t>(n + 1);
    auto* trunc_d = reinterpret_cast<unsigned long long*>(ctx->scratch.get<int>() + 16);
    LSMPS_CUDA(cudaMemsetAsync(trunc_d, 0, sizeof(unsigned long long), s));
    if (n) {
        const unsigned grid = std::max(1u, std::min<unsigned>(blocks_for(n * 32, 256), 148 * 16));
        k_filter_slots<<<grid, 256, 0, s>>>((int)n, ctx->cand_row.get<int>(), ctx->cand_col.get<int>(),
                                            ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(),
                                            ctx->stype.get<uint8_t>(), ctx->re2, maxn, ctx->l0, classify, slots, cnt,
                                            trunc_d, cls);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<int>(cnt, row, (long long)n, s, ctx->scan_tmp, dflag);
    int hpairs = 0;
    unsigned long long htr = 0;
    read_back(ctx, {{row + n, &hpairs, sizeof(int)}, {trunc_d, &htr, sizeof(htr)}}, "neighbor filter");
    ctx->pairs = (uint64_t)hpairs;
    ctx->truncated = htr;
    int* col = ctx->nbr_col.ensure<int>((size_t)hpairs + 1);
    if (n) {
        k_slots_compact<<<(unsigned)((8ull * n + 255) / 256), 256, 0, s>>>((int)n, maxn, slots, row, col);
        LSMPS_CHECK_LAUNCH();
    }
    return true;
}

void nb_kernel_bench(lsmps_ctx* ctx, int kernel, int reps, double* ms, double* bytes) {
    LSMPS_REQUIRE(ctx->have_neighbors, LSMPS_ERR_STATE, "kernel bench needs neighbor lists");
    cudaStream_t s = ctx->stream;
    int n = (int)ctx->n;
    GridView gv{ctx->cell_start.get<int>(), ctx->gdim[0], ctx->gdim[1], ctx->gdim[2]};
    SegGrid sg{gv, make_int3(ctx->gmin[0], ctx->gmin[1], ctx->gmin[2]), ctx->re, (ctx->gdim[0] + SEG - 1) / SEG};
    auto* trunc_d = reinterpret_cast<unsigned long long*>(ctx->scratch.get<int>() + 16);
    const int* seg_list = ctx->seg_list.get<int>();
    const unsigned seg_grid = (unsigned)std::max(ctx->nsegs, 1);
    int* slots = nullptr;
    if (kernel == LSMPS_KB_NBR_SCAN || kernel == LSMPS_KB_NBR_COMPACT) {
        LSMPS_REQUIRE((double)n * (double)ctx->maxn * 4.0 <= SLOT_BUDGET_BYTES, LSMPS_ERR_STATE,
                      "single-pass neighbor bench: slot rows exceed the budget");
        LSMPS_REQUIRE(kernel == LSMPS_KB_NBR_SCAN || ctx->nbr_single, LSMPS_ERR_STATE,
                      "compaction bench needs a single-pass build");
        slots = ctx->nbr_slots.ensure<int>((size_t)n * ctx->maxn + 1);
    }
    auto launch = [&] {
        if (kernel == LSMPS_KB_NBR_SCAN)
            k_seg_scan<<<seg_grid, SEG_THREADS, 0, s>>>(
                sg, seg_list, ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(), ctx->scell.get<int>(),
                ctx->stype.get<uint8_t>(), ctx->re2, ctx->maxn, ctx->l0, ctx->have_classes ? 1 : 0,
                ctx->nbr_cnt.get<int>(), trunc_d, slots, ctx->cls.get<uint8_t>());
        else if (kernel == LSMPS_KB_NBR_COMPACT)
            k_slots_compact<<<(unsigned)((8ull * n + 255) / 256), 256, 0, s>>>(n, ctx->maxn, slots,
                                                                               ctx->nbr_row.get<int>(),
                                                                               ctx->nbr_col.get<int>());
        else if (kernel == LSMPS_KB_NBR_COUNT)
            k_seg_pass<false><<<seg_grid, SEG_THREADS, 0, s>>>(
                sg, seg_list, ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(), ctx->scell.get<int>(),
                ctx->stype.get<uint8_t>(), ctx->re2, ctx->maxn, ctx->l0, 0, ctx->nbr_cnt.get<int>(), trunc_d, nullptr,
                nullptr, nullptr);
        else
            k_seg_pass<true><<<seg_grid, SEG_THREADS, 0, s>>>(
                sg, seg_list, ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(), ctx->scell.get<int>(),
                ctx->stype.get<uint8_t>(), ctx->re2, ctx->maxn, ctx->l0, ctx->have_classes ? 1 : 0, nullptr, nullptr,
                ctx->nbr_row.get<int>(), ctx->nbr_col.get<int>(), ctx->cls.get<uint8_t>());
        LSMPS_CHECK_LAUNCH();
    };
    if (n == 0 || ctx->nsegs == 0) { *ms = 0; *bytes = 0; return; }
    launch();  // warm
    ev_record(ctx, 14);
    for (int r = 0; r < reps; ++r) launch();
    ev_record(ctx, 15);
    *ms = ev_elapsed(ctx, 14, 15) / reps;
    // algorithmic bytes: positions (24 B) and cell (4 B) of every particle once, cell starts;
    // the count pass writes 4 B per particle, the fill pass reads types and row pointers and
    // writes the columns and classes
    double N = (double)n, P = (double)ctx->pairs, cells = (double)ctx->ncells;
    if (kernel == LSMPS_KB_NBR_SCAN)  // + scell, types, counts, kept slots, classes
        *bytes = 24.0 * N + 4.0 * N + 1.0 * N + 4.0 * N + 4.0 * P + 1.0 * N + 4.0 * cells;
    else if (kernel == LSMPS_KB_NBR_COMPACT)  // row pointers, the kept slots read and the CSR written
        *bytes = 4.0 * (N + 1) + 8.0 * P;
    else
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
