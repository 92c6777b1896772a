// Cell-aggregation multigrid V-cycle: the right preconditioner of the MIXED and LEARNED
// solvers when lsmps_solver_opts.precond = LSMPS_PRECOND_MULTIGRID. No reference counterpart
// (the reference's BiCGStab, src/lsmps.cpp:67, is unpreconditioned); the system it
// preconditions is the assembled PPE A p = b (src/lsmps.cpp:29-64 and its variants).
//
// Hierarchy, rebuilt after every assembly from the particles' cells:
//   level 1   one aggregate per cell of the neighbor grid (cell size re) holding unknowns.
//             Unknowns are numbered in cell-sorted order, so an aggregate is a contiguous
//             range of rows [ustart[I], ustart[I+1]).
//   level l+1 one aggregate per 2x2x2 block of level-l aggregates.
//   coarsest  the first level of at most MG_COARSE_SMALL rows, or of at most MG_COARSE_MAX rows
//             from level MG_COARSE_DEEP on (is_coarsest).
// Coarse operators are Galerkin products with piecewise-constant prolongation,
// A_{l+1} = P^T A_l P. An unknown's neighbors lie within re, so every coupling of an
// aggregate reaches only the 27 aggregates around it. Every coarse operator is therefore a
// 27-slot stencil on its block grid: slot t = 9 (dz + 1) + 3 (dy + 1) + (dx + 1) holds the
// coupling to the aggregate at offset (dx, dy, dz) (nbr = -1 where there is none). The fine
// level keeps its SELL matrix for the solver. The V-cycle uses AP = A P instead: for each
// fine row, the 27 sums of its entries per neighbor aggregate, scaled by the row's inverse
// diagonal and stored in FP16. The one fine-level smoothing sweep after the coarse
// correction (a piecewise-constant vector) then streams 56 bytes per row instead of the
// row's entries.
//
// V-cycle M z (FP32 inside, FP64 in and out), with omega = MG_OMEGA, alpha = MG_ALPHA:
//   fine:   r1 = P^T z (no pre-smoothing), e1 = cycle(1, r1),
//           x = alpha P e1 + omega D^-1 (z - A alpha P e1)
//   level l < coarsest: x_l = omega D_l^-1 r_l (one Jacobi sweep from 0),
//           r_{l+1} = P^T (r_l - A_l x_l), e_{l+1} = cycle(l + 1, r_{l+1}),
//           x' = x_l + alpha P e_{l+1}, e_l = x' + omega D_l^-1 (r_l - A_l x')
//   coarsest: MG_SWEEPS Jacobi sweeps from 0.
// The solvers iterate on y = D x with A D^-1, so they apply D M (the fine kernel multiplies
// by the diagonal). Each level's down and up step is one grid-wide kernel (level 1's down step
// two), the coarsest one block. Every sum has a fixed order, so a V-cycle is
// deterministic and a fixed linear operator, as BiCGStab requires. The V-cycle kernels take
// the solver's device scalars and return at once when the iteration has stopped (the gated
// kernels of the device-driven loop), and start under programmatic dependent launch.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "ops.cuh"
#include "scan.cuh"
#include "solver.cuh"

namespace lsmps_gpu {

constexpr int MG_MAX_LEVELS = 40;
constexpr int MG_COARSE_MAX = 640;       // rows of the coarsest level (one block)
constexpr int MG_COARSE_SMALL = 256;     // ... of a hierarchy of fewer than MG_COARSE_DEEP levels
constexpr int MG_COARSE_DEEP = 3;
// The coarsest level's 10 Jacobi sweeps: enough for a level of up to 640 rows at the bottom of
// a deep hierarchy (at 1M particles, level 4 of 537 rows), not for level 1 or 2 of a small
// system, which keep the 256-row limit (4,000 particles: 18 iterations against 27 with 640).
__host__ __device__ constexpr bool is_coarsest(long long n, int level) {
    return n <= MG_COARSE_SMALL || (n <= MG_COARSE_MAX && level >= MG_COARSE_DEEP);
}
constexpr int MG_SWEEPS = 10;            // Jacobi sweeps on the coarsest level
constexpr float MG_OMEGA = 1.0f;         // smoother damping
constexpr float MG_ALPHA = 1.5f;         // coarse-correction scaling
constexpr int MG_SLOTS = 27;
constexpr int MG_CENTER = 13;

struct MgLevel {
    long long n = 0;
    int dims[3] = {0, 0, 0};  // block grid of this level
    DevBuf coord;             // n x int3 block coordinates
    DevBuf val;               // 27-slot stencil, slice-major: [(I / 32) * 27 + t] * 32 + I % 32 (float)
    DevBuf nbr;               // same layout, int row index or -1 (whose stencil value is 0)
    DevBuf dinv;              // n float inverse diagonals (0 where the diagonal is not positive)
    DevBuf parent;            // n int rows of level + 1
    DevBuf pn;                // slice-major like nbr: parent of the slot's row, or -1
    DevBuf child;             // n x 8 int rows of level - 1 (levels >= 2), -1 where absent
    DevBuf r, x, e;           // float vectors
};

struct MgState {
    long long gen = -1;  // assembly the hierarchy belongs to
    int levels = 0;      // coarse levels 1 .. levels
    double setup_ms = 0;
    MgLevel L[MG_MAX_LEVELS + 1];
    DevBuf agg0, ustart, ucell, upack, head, hscan, ap, aph, map, flags, pos;
    DevBuf nsz;  // int: size of level l at [l] (levels >= 2, written on the device)
};

namespace {

__host__ __device__ __forceinline__ long long slot_index(long long i, int t) {
    return (((i >> 5) * MG_SLOTS + t) << 5) + (i & 31);
}
__host__ __device__ __forceinline__ long long padded(long long n) { return ((n + 31) >> 5) << 5; }

__device__ __forceinline__ bool gated(const BcgScalars* S, int need_s) {
    return S && (S->done || (need_s && S->s_conv));
}

// ---- setup ------------------------------------------------------------------------------
// Cell coordinates packed into 32 bits (x | y << bx | z << (bx + by)): the grid has at most
// 2^29 cells, so the three widths ceil(log2(dim)) sum to at most 31.
struct Pack {
    int bx, by;
    unsigned mx, my, mz;
};
__device__ __forceinline__ int3 unpack(unsigned p, const Pack& k) {
    return make_int3((int)(p & k.mx), (int)((p >> k.bx) & k.my), (int)((p >> (k.bx + k.by)) & k.mz));
}
__device__ __forceinline__ int slot_of(int3 a, int3 b) {  // offset of b from a, clamped to one block
    int dx = max(-1, min(1, b.x - a.x)), dy = max(-1, min(1, b.y - a.y)), dz = max(-1, min(1, b.z - a.z));
    return 9 * (dz + 1) + 3 * (dy + 1) + (dx + 1);
}

__global__ void k_mg_heads(long long U, const int* __restrict__ sorted_of_u, const int* __restrict__ scell, int gx,
                           int gy, Pack pk, int* __restrict__ ucell, unsigned* __restrict__ upack,
                           int* __restrict__ head) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= U) return;
    int c = scell[sorted_of_u[i]];
    ucell[i] = c;
    unsigned x = (unsigned)(c % gx), y = (unsigned)((c / gx) % gy), z = (unsigned)(c / (gx * gy));
    upack[i] = x | (y << pk.bx) | (z << (pk.bx + pk.by));
    head[i] = (i == 0 || scell[sorted_of_u[i - 1]] != c) ? 1 : 0;
}

__global__ void k_mg_aggregates(long long U, const int* __restrict__ ucell, const int* __restrict__ head,
                                const int* __restrict__ hscan, int gx, int gy, int* __restrict__ agg0,
                                int* __restrict__ ustart, int3* __restrict__ coord, int* __restrict__ map,
                                long long n1) {
    long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= U) return;
    int I = hscan[i] + head[i] - 1;
    agg0[i] = I;
    if (head[i]) {
        int c = ucell[i];
        ustart[I] = (int)i;
        coord[I] = make_int3(c % gx, (c / gx) % gy, c / (gx * gy));
        map[c] = I;
    }
    if (i == U - 1) ustart[n1] = (int)U;
}

// nbr[I][t]: the row at offset t of row I's block, through the dense map of its grid
// Set-up kernels of a coarse level run before the host knows its size: they take an upper
// bound n for the grid and, when nd is set, the level's size from the device (*nd <= n).
__device__ __forceinline__ long long dev_size(long long n, const int* nd) { return nd ? (long long)*nd : n; }

__global__ void k_mg_nbr(long long n, const int* nd, const int3* __restrict__ coord, int gx, int gy, int gz,
                         const int* __restrict__ map, int* __restrict__ nbr) {
    long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (I >= dev_size(n, nd)) return;
    int3 c = coord[I];
#pragma unroll
    for (int t = 0; t < MG_SLOTS; ++t) {
        int x = c.x + t % 3 - 1, y = c.y + (t / 3) % 3 - 1, z = c.z + t / 9 - 1;
        int J = -1;
        if (x >= 0 && y >= 0 && z >= 0 && x < gx && y < gy && z < gz)
            J = map[((long long)z * gy + y) * gx + x];
        nbr[slot_index(I, t)] = J;
    }
}

// AP[i][t]: row i's entries summed per neighbor aggregate, in FP32 slice-major (for level 1)
// and as AP / a_ii in FP16 row-major, MG_APH_STRIDE halves per row (for the V-cycle). One warp
// per SELL slice, one lane per row, four entries per load (coalesced), read from the solver's
// FP32 copy of A D^-1 (a_ij = (a_ij / a_jj) a_jj, the column's diagonal from D^-1; the copy's
// 16-bit column steps or 32-bit columns), so the set-up needs no unscaled FP64 copy. Each lane
// adds its entries, in entry order, into its own column of a shared-memory table of 27 slots;
// the table is then written out with coalesced stores. AP is deterministic.
constexpr int MG_APH_STRIDE = 28;  // 27 slots + 1 zero pad: 56 B rows, read as seven 8-byte loads
constexpr int AP_WARPS = 4;
__global__ void __launch_bounds__(AP_WARPS * 32) k_mg_fine_ap(Sell<float> A, const unsigned* __restrict__ upack,
                                                              Pack pk, const double* __restrict__ dinv,
                                                              float* __restrict__ ap, __half* __restrict__ aph,
                                                              int* __restrict__ dflag) {
    __shared__ float acc[AP_WARPS][MG_APH_STRIDE][33];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long sl = blockIdx.x * (long long)AP_WARPS + w;
    if (sl >= A.nslices) return;  // whole warp
    const long long i = (sl << 5) + lane;
    const bool live = i < A.n;
#pragma unroll
    for (int t = 0; t < MG_APH_STRIDE; ++t) acc[w][t][lane] = 0.0f;
    const int3 ci = unpack(live ? upack[i] : 0u, pk);
    const long long base = (long long)A.sptr[sl] + 4 * lane;
    const int chunks = A.slen[sl] >> 2;
    int cur = A.dcol ? A.rbase[i] : 0;  // the row's first column (16-bit steps)
    for (int c = 0; c < chunks; ++c) {
        const float4 v4 = __ldcs(reinterpret_cast<const float4*>(A.val + base + 128 * c));
        int col[4];
        if (A.dcol) {
            const uint2 q = __ldcs(reinterpret_cast<const uint2*>(A.dcol + base + 128 * c));
            cur += (int)(q.x & 0xffffu);
            col[0] = cur;
            cur += (int)(q.x >> 16);
            col[1] = cur;
            cur += (int)(q.y & 0xffffu);
            col[2] = cur;
            cur += (int)(q.y >> 16);
            col[3] = cur;
        } else {
            const int4 cc = __ldcs(reinterpret_cast<const int4*>(A.col + base + 128 * c));
            col[0] = cc.x, col[1] = cc.y, col[2] = cc.z, col[3] = cc.w;
        }
        const float v[4] = {v4.x, v4.y, v4.z, v4.w};
        unsigned pj[4];
        double dj[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            pj[k] = live ? upack[col[k]] : 0u;
            dj[k] = live ? dinv[col[k]] : 1.0;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int3 cj = unpack(pj[k], pk);
            // a coupling beyond the adjacent cells has no slot: flag it (clamped slot, no write
            // out of bounds; the setup then fails with LSMPS_ERR_GRID)
            if (abs(cj.x - ci.x) > 1 || abs(cj.y - ci.y) > 1 || abs(cj.z - ci.z) > 1) atomicOr(dflag, DFLAG_STENCIL);
            acc[w][slot_of(ci, cj)][lane] += v[k] / (float)dj[k];  // padding: v = 0
        }
    }
    __syncwarp();
    if (!live) return;
#pragma unroll
    for (int t = 0; t < MG_SLOTS; ++t) ap[slot_index(i, t)] = acc[w][t][lane];
    const double di = dinv[i];
    uint2* hr = reinterpret_cast<uint2*>(aph + i * MG_APH_STRIDE);
#pragma unroll
    for (int k = 0; k < MG_APH_STRIDE / 4; ++k) {
        __half2 h0 = __floats2half2_rn((float)(acc[w][4 * k][lane] * di), (float)(acc[w][4 * k + 1][lane] * di));
        __half2 h1 = __floats2half2_rn((float)(acc[w][4 * k + 2][lane] * di),
                                       4 * k + 3 < MG_SLOTS ? (float)(acc[w][4 * k + 3][lane] * di) : 0.0f);
        uint2 q;
        q.x = *reinterpret_cast<unsigned*>(&h0);
        q.y = *reinterpret_cast<unsigned*>(&h1);
        hr[k] = q;
    }
}

__device__ __forceinline__ float safe_inv(double d) {
    return (d > 0 && isfinite(d)) ? (float)(1.0 / d) : 0.0f;
}

// level 1 = P^T (A P): one warp per aggregate, lane t sums slot t over the aggregate's rows
// (FP64, row order)
__global__ void k_mg_level1(long long n1, const int* __restrict__ ustart, const float* __restrict__ ap,
                            float* __restrict__ val1, float* __restrict__ dinv1) {
    const long long I = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const int t = threadIdx.x & 31;
    if (I >= n1 || t >= MG_SLOTS) return;
    double a = 0;
    const int b = ustart[I], e = ustart[I + 1];
    int i = b;
    for (; i + 4 <= e; i += 4) {
        const float v0 = ap[slot_index(i, t)], v1 = ap[slot_index(i + 1, t)], v2 = ap[slot_index(i + 2, t)],
                    v3 = ap[slot_index(i + 3, t)];
        a += (double)v0;
        a += (double)v1;
        a += (double)v2;
        a += (double)v3;
    }
    for (; i < e; ++i) a += (double)ap[slot_index(i, t)];
    val1[slot_index(I, t)] = (float)a;
    if (t == MG_CENTER) dinv1[I] = safe_inv(a);
}

__global__ void k_mg_mark(long long n, const int* nd, const int3* __restrict__ coord, int gx, int gy,
                          int* __restrict__ flags) {
    long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (I >= dev_size(n, nd)) return;
    int3 c = coord[I];
    flags[((long long)(c.z >> 1) * gy + (c.y >> 1)) * gx + (c.x >> 1)] = 1;
}

__global__ void k_mg_assign(long long nb, const int* __restrict__ flags, const int* __restrict__ pos, int gx,
                            int gy, int3* __restrict__ coord, int* __restrict__ map) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= nb) return;
    if (flags[q]) {
        int B = pos[q];
        coord[B] = make_int3((int)(q % gx), (int)((q / gx) % gy), (int)(q / ((long long)gx * gy)));
        map[q] = B;
    } else {
        map[q] = -1;
    }
}

__global__ void k_mg_parent(long long n, const int* nd, const int3* __restrict__ coord, int gx, int gy,
                            const int* __restrict__ map, int* __restrict__ parent, int* __restrict__ child) {
    long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (I >= dev_size(n, nd)) return;
    int3 c = coord[I];
    int B = map[((long long)(c.z >> 1) * gy + (c.y >> 1)) * gx + (c.x >> 1)];
    parent[I] = B;
    child[8ll * B + ((c.x & 1) | ((c.y & 1) << 1) | ((c.z & 1) << 2))] = (int)I;
}

// pn[I][t] = parent of row I's neighbor in slot t (or -1)
__global__ void k_mg_pn(long long ncap, const int* nd, const int* __restrict__ nbr, const int* __restrict__ parent,
                        int* __restrict__ pn) {
    long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long n = dev_size(ncap, nd);
    if (q >= padded(n) * MG_SLOTS) return;
    const long long I = ((q >> 5) / MG_SLOTS) * 32 + (q & 31);  // padding rows hold no neighbors
    const int J = I < n ? nbr[q] : -1;
    pn[q] = J >= 0 ? parent[J] : -1;
}

// A_{l+1}[B][t'], one thread per (B, t'): the child in octant o = (ox, oy, oz) of B couples
// through its slot offset d to the block at offset (o + d) >> 1 (per axis) of B, so slot t'
// = e collects, per axis, the offsets d in [2e - o, 2e - o + 1] within [-1, 1] of every
// child (children in octant order, offsets in slot order).
__global__ void k_mg_coarsen(long long ncap, const int* nd, const int* __restrict__ child,
                             const float* __restrict__ val, float* __restrict__ valc, float* __restrict__ dinvc) {
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (q >= dev_size(ncap, nd) * MG_SLOTS) return;
    const long long B = q / MG_SLOTS;
    const int tp = (int)(q - B * MG_SLOTS);
    const int ex = tp % 3 - 1, ey = (tp / 3) % 3 - 1, ez = tp / 9 - 1;
    double a = 0;
    for (int o = 0; o < 8; ++o) {
        const int I = child[8 * B + o];
        if (I < 0) continue;
        const int ox = o & 1, oy = (o >> 1) & 1, oz = o >> 2;
        for (int dz = max(-1, 2 * ez - oz); dz <= min(1, 2 * ez - oz + 1); ++dz)
            for (int dy = max(-1, 2 * ey - oy); dy <= min(1, 2 * ey - oy + 1); ++dy)
                for (int dx = max(-1, 2 * ex - ox); dx <= min(1, 2 * ex - ox + 1); ++dx)
                    a += (double)val[slot_index(I, 9 * (dz + 1) + 3 * (dy + 1) + (dx + 1))];
    }
    valc[slot_index(B, tp)] = (float)a;
    if (tp == MG_CENTER) dinvc[B] = safe_inv(a);
}

// ---- V-cycle ------------------------------------------------------------------------------
// r1[I] = sum of z over the aggregate's rows
__global__ void k_mg_restrict0(long long n1, const int* __restrict__ ustart, const double* __restrict__ z,
                               float* __restrict__ r1, const BcgScalars* S, int need_s) {
    pdl_begin();
    if (gated(S, need_s)) return;
    long long I = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (I >= n1) return;
    double a = 0;
    for (int i = ustart[I], e = ustart[I + 1]; i < e; ++i) a += z[i];
    r1[I] = (float)a;
}

// Partial sum over the slots t = g, g + 4, ... of row I of A_l times the vector f, where
// f(J) = omega r[J] dinv[J] (down: the pre-smoothed iterate) or x[J] + alpha ec[pn] (up).
// Empty slots (nbr = -1) hold 0, so their index is clamped to 0 instead of branching, and all
// of the row's loads are issued before the gathers that depend on them.
__device__ __forceinline__ float row_part_down(long long I, int g, const float* __restrict__ val,
                                               const int* __restrict__ nbr, const float* __restrict__ r,
                                               const float* __restrict__ dinv) {
    int J[7];
    float v[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        const int t = g + 4 * k;
        const long long si = slot_index(I, min(t, MG_SLOTS - 1));
        J[k] = max(nbr[si], 0);
        v[k] = t < MG_SLOTS ? val[si] : 0.0f;
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 7; ++k) s += v[k] * (MG_OMEGA * r[J[k]] * dinv[J[k]]);
    return s;
}
__device__ __forceinline__ float row_part_up(long long I, int g, const float* __restrict__ val,
                                             const int* __restrict__ nbr, const int* __restrict__ pn,
                                             const float* __restrict__ x, const float* __restrict__ ec) {
    int J[7], P[7];
    float v[7];
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        const int t = g + 4 * k;
        const long long si = slot_index(I, min(t, MG_SLOTS - 1));
        J[k] = max(nbr[si], 0);
        P[k] = max(pn[si], 0);
        v[k] = t < MG_SLOTS ? val[si] : 0.0f;
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < 7; ++k) s += v[k] * (x[J[k]] + MG_ALPHA * ec[P[k]]);
    return s;
}

// Level l, four lanes per row (slots t = g mod 4): x_l[I] = omega r_l[I] / d_I and the
// residual r_l[I] - (A_l x_l)[I] into res (the four partial sums added in a fixed tree).
__global__ void k_mg_res(long long n, const float* __restrict__ val, const int* __restrict__ nbr,
                         const float* __restrict__ dinv, const float* __restrict__ r, float* __restrict__ x,
                         float* __restrict__ res, const BcgScalars* S, int need_s) {
    pdl_begin();
    if (gated(S, need_s)) return;
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long I = q >> 2;
    const int g = (int)(q & 3);
    float s = I < n ? row_part_down(I, g, val, nbr, r, dinv) : 0.0f;
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (I < n && g == 0) {
        const float rI = r[I];
        x[I] = MG_OMEGA * rI * dinv[I];
        res[I] = rI - s;
    }
}

// r_{l+1}[B] = sum of the children's residuals (octant order)
__global__ void k_mg_restrict(long long nc, const int* __restrict__ child, const float* __restrict__ res,
                              float* __restrict__ rc, const BcgScalars* S, int need_s) {
    pdl_begin();
    if (gated(S, need_s)) return;
    const long long B = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (B >= nc) return;
    float a = 0.0f;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const int I = child[8 * B + o];
        if (I >= 0) a += res[I];
    }
    rc[B] = a;
}

// One warp per coarse row B; four lanes per child I (octant o = lane / 4): x_l[I] and the
// child's residual as in k_mg_res, then the eight residuals added in a fixed tree.
__global__ void k_mg_down(long long nc, const int* __restrict__ child, const float* __restrict__ val,
                          const int* __restrict__ nbr, const float* __restrict__ dinv, const float* __restrict__ r,
                          float* __restrict__ x, float* __restrict__ rc, const BcgScalars* S, int need_s) {
    pdl_begin();
    if (gated(S, need_s)) return;
    const long long B = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    if (B >= nc) return;  // whole warp
    const int lane = threadIdx.x & 31, g = lane & 3;
    const int I = child[8 * B + (lane >> 2)];
    float s = I >= 0 ? row_part_down(I, g, val, nbr, r, dinv) : 0.0f;
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    float res = 0.0f;
    if (I >= 0) {
        const float rI = r[I];
        res = rI - s;
        if (g == 0) x[I] = MG_OMEGA * rI * dinv[I];
    }
    res += __shfl_xor_sync(0xffffffffu, res, 4);
    res += __shfl_xor_sync(0xffffffffu, res, 8);
    res += __shfl_xor_sync(0xffffffffu, res, 16);
    if (lane == 0) rc[B] = res;
}

// Coarsest level (n <= MG_COARSE_MAX rows): Jacobi sweeps from 0 in one block of nb >= n
// threads (a multiple of 32), one thread per row with its 27 stencil values and neighbor rows
// in registers, the iterate in shared memory (no large shared-memory carve-out, which would
// make the SM reconfigure between the V-cycle's kernels). A single block pays each dependent
// L2 round trip in series, so only this level runs in one (the levels above it get grid-wide
// kernels). At 1M particles a coarsest level of up to 640 rows ends the hierarchy one level
// earlier (537 rows instead of a further level of 82): the restatement's iterations stay the
// same (26-28 against 28), and each V-cycle saves a down and an up step.
__global__ void __launch_bounds__(MG_COARSE_MAX) k_mg_coarsest(int n, const float* __restrict__ val,
                                                               const int* __restrict__ nbr,
                                                               const float* __restrict__ dinv,
                                                               const float* __restrict__ r, float* __restrict__ e,
                                                               const BcgScalars* S, int need_s) {
    pdl_begin();
    if (gated(S, need_s)) return;
    __shared__ float cur[2][MG_COARSE_MAX];
    const int I = threadIdx.x;
    const bool own = I < n;
    float cv[MG_SLOTS];
    int cn[MG_SLOTS];
#pragma unroll
    for (int t = 0; t < MG_SLOTS; ++t) {
        cv[t] = own ? val[slot_index(I, t)] : 0.0f;
        cn[t] = own ? max(nbr[slot_index(I, t)], 0) : 0;  // empty slots hold 0
    }
    const float ri = own ? r[I] : 0.0f, di = own ? dinv[I] : 0.0f;
    float x = MG_OMEGA * ri * di;  // first sweep from 0
    cur[0][I] = x;
    __syncthreads();
    int b = 0;
    for (int it = 1; it < MG_SWEEPS; ++it) {
        float s = 0.0f;
#pragma unroll
        for (int t = 0; t < MG_SLOTS; ++t) s += cv[t] * cur[b][cn[t]];
        x = x + MG_OMEGA * di * (ri - s);
        cur[b ^ 1][I] = x;
        __syncthreads();
        b ^= 1;
    }
    if (own) e[I] = x;
}

// e_l = x' + omega D^-1 (r_l - A_l x'), x' = x_l + alpha P e_{l+1}; four lanes per row.
__global__ void k_mg_up(long long n, const float* __restrict__ val, const int* __restrict__ nbr,
                        const int* __restrict__ pn, const float* __restrict__ dinv, const int* __restrict__ parent,
                        const float* __restrict__ r, const float* __restrict__ x, const float* __restrict__ ec,
                        float* __restrict__ e, const BcgScalars* S, int need_s) {
    pdl_begin();
    if (gated(S, need_s)) return;
    const long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long I = q >> 2;
    const int g = (int)(q & 3);
    float s = I < n ? row_part_up(I, g, val, nbr, pn, x, ec) : 0.0f;
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (I < n && g == 0) {
        const float xi = x[I] + MG_ALPHA * ec[parent[I]];
        e[I] = xi + MG_OMEGA * dinv[I] * (r[I] - s);
    }
}

// out_i = d_i x_i with x = alpha P e1 + omega D^-1 (z - A alpha P e1):
// out_i = omega z_i + alpha d_i (e1[I] - omega sum_t (AP[i][t] / d_i) e1[J_t]).
// A block's rows span a contiguous range of aggregates; the block first gathers e1 at the 27
// neighbors of each of them into shared memory, so each row reads its 27 values from there.
constexpr int UP0_THREADS = 256;
__global__ void __launch_bounds__(UP0_THREADS) k_mg_up0(long long U, const int* __restrict__ agg0,
                                                        const __half* __restrict__ aph,
                                                        const int* __restrict__ nbr1, const float* __restrict__ e1,
                                                        const double* __restrict__ z, const double* __restrict__ dinv,
                                                        double* __restrict__ out, const BcgScalars* S, int need_s) {
    pdl_begin();
    if (gated(S, need_s)) return;
    __shared__ float E[UP0_THREADS * MG_SLOTS];
    const long long i0 = blockIdx.x * (long long)UP0_THREADS;
    const long long i = i0 + threadIdx.x;
    const bool live = i < U;
    // the row's own data first, so its loads overlap the neighbor gathers below
    uint2 h[MG_APH_STRIDE / 4];
    const uint2* hr = reinterpret_cast<const uint2*>(aph + (live ? i : i0) * MG_APH_STRIDE);
#pragma unroll
    for (int k = 0; k < MG_APH_STRIDE / 4; ++k) h[k] = __ldcs(hr + k);
    const double zi = live ? z[i] : 0.0, di = live ? dinv[i] : 1.0;
    const int I = agg0[live ? i : i0];
    const int I0 = agg0[i0];
    const int na = agg0[min(i0 + UP0_THREADS - 1, U - 1)] - I0 + 1;  // <= UP0_THREADS
    const int nq = na * MG_SLOTS;
    if (nq <= 4 * UP0_THREADS) {
        // the usual block (up to 37 aggregates): all neighbor-slot indices first, then all
        // gathers, so that each step's loads are in flight together
        int idx[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int q = threadIdx.x + r * UP0_THREADS;
            const int a = q / MG_SLOTS;
            idx[r] = q < nq ? nbr1[slot_index(I0 + a, q - a * MG_SLOTS)] : 0;
        }
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int q = threadIdx.x + r * UP0_THREADS;
            if (q < nq) E[q] = e1[max(idx[r], 0)];  // empty slots: AP is 0 there
        }
    } else {
        for (int q = threadIdx.x; q < nq; q += UP0_THREADS) {
            const int a = q / MG_SLOTS;
            E[q] = e1[max(nbr1[slot_index(I0 + a, q - a * MG_SLOTS)], 0)];
        }
    }
    const float eI = e1[I];
    __syncthreads();
    if (!live) return;
    const float* Er = E + (I - I0) * MG_SLOTS;
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < MG_APH_STRIDE / 4; ++k) {
        const float2 f0 = __half22float2(*reinterpret_cast<const __half2*>(&h[k].x));
        const float2 f1 = __half22float2(*reinterpret_cast<const __half2*>(&h[k].y));
        s += f0.x * Er[4 * k] + f0.y * Er[4 * k + 1] + f1.x * Er[4 * k + 2];
        if (4 * k + 3 < MG_SLOTS) s += f1.y * Er[4 * k + 3];
    }
    out[i] = (double)MG_OMEGA * zi + (double)MG_ALPHA * ((double)eI - (double)MG_OMEGA * (double)s) / di;
}

inline unsigned grid_for(long long n, int threads) {
    return (unsigned)std::max<long long>(1, (n + threads - 1) / threads);
}

}  // namespace

void mg_destroy(lsmps_ctx* ctx) {
    MgState* m = ctx->mg;
    if (!m) return;
    for (auto& l : m->L)
        for (DevBuf* d : {&l.coord, &l.val, &l.nbr, &l.dinv, &l.parent, &l.pn, &l.child, &l.r, &l.x, &l.e})
            d->release();
    for (DevBuf* d : {&m->agg0, &m->ustart, &m->ucell, &m->upack, &m->head, &m->hscan, &m->ap, &m->aph, &m->map,
                      &m->flags, &m->pos, &m->nsz})
        d->release();
    delete m;
    ctx->mg = nullptr;
}

// Builds (or keeps) the hierarchy of the context's assembled system.
void mg_setup(lsmps_ctx* ctx) {
    LSMPS_REQUIRE(ctx->have_ppe, LSMPS_ERR_STATE, "multigrid needs an assembled PPE");
    LSMPS_REQUIRE(!ctx->ppe_loaded, LSMPS_ERR_STATE,
                  "the multigrid preconditioner aggregates particle cells: a loaded CSR system has none");
    if (!ctx->mg) ctx->mg = new MgState();
    MgState& M = *ctx->mg;
    if (M.gen == ctx->assembly_gen) return;
    cudaStream_t s = ctx->stream;
    int* dflag = ctx->dflags.get<int>();
    const long long U = ctx->U;
    LSMPS_REQUIRE(U > 0, LSMPS_ERR_STATE, "multigrid needs at least one unknown");
    ev_record(ctx, 16);
    const int gx = ctx->gdim[0], gy = ctx->gdim[1], gz = ctx->gdim[2];
    const long long ncells = ctx->ncells;
    // level 1: cells
    auto bits = [](int g) {
        int b = 1;
        while ((1ll << b) < g) ++b;
        return b;
    };
    LSMPS_REQUIRE(bits(gx) + bits(gy) + bits(gz) <= 32, LSMPS_ERR_GRID, "cell grid too large for packed coordinates");
    Pack pk{bits(gx), bits(gy), (1u << bits(gx)) - 1, (1u << bits(gy)) - 1, (unsigned)((1ull << bits(gz)) - 1)};
    int* ucell = M.ucell.ensure<int>(U + 1);
    unsigned* upack = M.upack.ensure<unsigned>(U + 1);
    int* head = M.head.ensure<int>(U + 1);
    int* hscan = M.hscan.ensure<int>(U + 1);
    k_mg_heads<<<grid_for(U, 256), 256, 0, s>>>(U, ctx->sorted_of_u.get<int>(), ctx->scell.get<int>(), gx, gy, pk,
                                                ucell, upack, head);
    LSMPS_CHECK_LAUNCH();
    scan_exclusive<int>(head, hscan, U, s, ctx->scan_tmp, dflag);
    int hn = 0;
    read_back(ctx, {{hscan + U, &hn, sizeof(int)}}, "multigrid aggregates");
    long long n1 = hn;
    MgLevel& L1 = M.L[1];
    L1.n = n1;
    L1.dims[0] = gx;
    L1.dims[1] = gy;
    L1.dims[2] = gz;
    int* agg0 = M.agg0.ensure<int>(U + 1);
    int* ustart = M.ustart.ensure<int>(n1 + 1);
    int3* coord1 = L1.coord.ensure<int3>(n1);
    int* map = M.map.ensure<int>(ncells + 1);
    LSMPS_CUDA(cudaMemsetAsync(map, 0xff, (ncells + 1) * sizeof(int), s));
    k_mg_aggregates<<<grid_for(U, 256), 256, 0, s>>>(U, ucell, head, hscan, gx, gy, agg0, ustart, coord1, map, n1);
    LSMPS_CHECK_LAUNCH();
    int* nbr1 = L1.nbr.ensure<int>(padded(n1) * MG_SLOTS);
    k_mg_nbr<<<grid_for(n1, 256), 256, 0, s>>>(n1, nullptr, coord1, gx, gy, gz, map, nbr1);
    LSMPS_CHECK_LAUNCH();
    float* ap = M.ap.ensure<float>(padded(U) * MG_SLOTS);
    const Sell<float> Af = sell_scaled32_view(ctx);
    k_mg_fine_ap<<<grid_for(Af.nslices, AP_WARPS), AP_WARPS * 32, 0, s>>>(
        Af, upack, pk, ctx->A_dinv.get<double>(), ap, M.aph.ensure<__half>(U * MG_APH_STRIDE + 8), dflag);
    LSMPS_CHECK_LAUNCH();
    k_mg_level1<<<grid_for(32 * n1, 256), 256, 0, s>>>(n1, ustart, ap, L1.val.ensure<float>(padded(n1) * MG_SLOTS),
                                                       L1.dinv.ensure<float>(n1));
    LSMPS_CHECK_LAUNCH();
    // levels 2..: 2x2x2 blocks of the level below, until the coarsest is small enough. The
    // coarse levels are built before the host knows their sizes: arrays and grids take upper
    // bounds (a level has at most as many rows as the level below and as its block grid has
    // blocks), and the kernels read the sizes from the device. Once a level's bound is within
    // 8x of MG_COARSE_MAX the sizes so far are read back (with the device flags) in one
    // synchronisation, so the loop stops at the first level is_coarsest accepts.
    int* nsz = M.nsz.ensure<int>(MG_MAX_LEVELS + 2);
    int lv = 1;
    long long ub = n1;  // upper bound of level lv's size (its size, for level 1)
    int hsz[MG_MAX_LEVELS + 2] = {};
    while (!is_coarsest(ub, lv)) {
        LSMPS_REQUIRE(lv < MG_MAX_LEVELS, LSMPS_ERR_STATE, "multigrid coarsening did not converge");
        MgLevel& F = M.L[lv];
        MgLevel& C = M.L[lv + 1];
        const int* fn = lv == 1 ? nullptr : nsz + lv;  // F's size on the device (level 1: n1)
        for (int a = 0; a < 3; ++a) C.dims[a] = (F.dims[a] + 1) >> 1;
        const long long nb = (long long)C.dims[0] * C.dims[1] * C.dims[2];
        const long long cub = std::min(nb, ub);
        int* flags = M.flags.ensure<int>(nb + 1);
        int* pos = M.pos.ensure<int>(nb + 1);
        LSMPS_CUDA(cudaMemsetAsync(flags, 0, (nb + 1) * sizeof(int), s));
        k_mg_mark<<<grid_for(ub, 256), 256, 0, s>>>(ub, fn, F.coord.get<int3>(), C.dims[0], C.dims[1], flags);
        LSMPS_CHECK_LAUNCH();
        scan_exclusive<int>(flags, pos, nb, s, ctx->scan_tmp, dflag);
        LSMPS_CUDA(cudaMemcpyAsync(nsz + lv + 1, pos + nb, sizeof(int), cudaMemcpyDeviceToDevice, s));
        const int* cn = nsz + lv + 1;
        C.n = cub;  // the bound until the read-back
        int3* cc = C.coord.ensure<int3>(cub);
        k_mg_assign<<<grid_for(nb, 256), 256, 0, s>>>(nb, flags, pos, C.dims[0], C.dims[1], cc, map);
        LSMPS_CHECK_LAUNCH();
        int* child = C.child.ensure<int>(8 * cub);
        LSMPS_CUDA(cudaMemsetAsync(child, 0xff, 8 * cub * sizeof(int), s));
        k_mg_parent<<<grid_for(ub, 256), 256, 0, s>>>(ub, fn, F.coord.get<int3>(), C.dims[0], C.dims[1], map,
                                                     F.parent.ensure<int>(ub), child);
        LSMPS_CHECK_LAUNCH();
        k_mg_pn<<<grid_for(padded(ub) * MG_SLOTS, 256), 256, 0, s>>>(ub, fn, F.nbr.get<int>(), F.parent.get<int>(),
                                                                      F.pn.ensure<int>(padded(ub) * MG_SLOTS));
        LSMPS_CHECK_LAUNCH();
        k_mg_nbr<<<grid_for(cub, 256), 256, 0, s>>>(cub, cn, cc, C.dims[0], C.dims[1], C.dims[2], map,
                                                    C.nbr.ensure<int>(padded(cub) * MG_SLOTS));
        LSMPS_CHECK_LAUNCH();
        k_mg_coarsen<<<grid_for(MG_SLOTS * cub, 256), 256, 0, s>>>(cub, cn, child, F.val.get<float>(),
                                                                   C.val.ensure<float>(padded(cub) * MG_SLOTS),
                                                                   C.dinv.ensure<float>(cub));
        LSMPS_CHECK_LAUNCH();
        ub = cub;
        ++lv;
        if (ub <= 8 * MG_COARSE_MAX) {
            read_back(ctx, {{nsz + 2, hsz + 2, (size_t)(lv - 1) * sizeof(int)}}, "multigrid setup");
            for (int l = 2; l <= lv; ++l) M.L[l].n = hsz[l];
            ub = M.L[lv].n;
        }
    }
    ev_record(ctx, 17);
    // the loop ends on a size read back (is_coarsest needs at most MG_COARSE_MAX, within 8x), which
    // checked the device flags; a single-level hierarchy checks them here
    if (lv == 1) check_device_flags(ctx, "multigrid setup");
    int levels = 1;
    while (levels < lv && !is_coarsest(M.L[levels].n, levels)) ++levels;
    M.levels = levels;
    for (int l = 1; l <= levels; ++l) {
        MgLevel& Ll = M.L[l];
        Ll.r.ensure<float>(Ll.n + 1);
        Ll.x.ensure<float>(Ll.n + 1);
        Ll.e.ensure<float>(Ll.n + 1);
    }
    M.setup_ms = ev_elapsed(ctx, 16, 17);
    M.gen = ctx->assembly_gen;
}

// restrict0 (unless the caller restricted), the down steps (two kernels for level 1), the
// coarsest, the up steps and the fine kernel
int mg_launches_per_apply(lsmps_ctx* ctx, bool restricted) {
    if (!ctx->mg) return 0;
    const int Lc = ctx->mg->levels;
    return (restricted ? 0 : 1) + (Lc > 1 ? 2 + (Lc - 2) : 0) + 1 + (Lc - 1) + 1;
}

MgFine mg_fine(lsmps_ctx* ctx) {
    MgState& M = *ctx->mg;
    return MgFine{M.L[1].n, M.ustart.get<int>(), M.agg0.get<int>(), M.L[1].r.get<float>()};
}

// out = D M z on the context stream (z, out: U doubles); gated by the solver scalars S
// (need_s: also skip once the |s| test has passed).
void mg_apply(lsmps_ctx* ctx, const double* z, double* out, const BcgScalars* S, int need_s, bool restricted) {
    MgState& M = *ctx->mg;
    cudaStream_t s = ctx->stream;
    const long long U = ctx->U;
    const int Lc = M.levels;
    MgLevel* L = M.L;
    if (!restricted)
        launch_pdl(k_mg_restrict0, grid_for(L[1].n, 256), 256, 0, s, L[1].n, M.ustart.get<int>(), z,
                   L[1].r.get<float>(), S, need_s);
    for (int l = 1; l < Lc; ++l) {
        if (l == 1) {
            launch_pdl(k_mg_res, grid_for(4 * L[1].n, 256), 256, 0, s, L[1].n, L[1].val.get<float>(),
                       L[1].nbr.get<int>(), L[1].dinv.get<float>(), L[1].r.get<float>(), L[1].x.get<float>(),
                       L[1].e.get<float>(), S, need_s);
            launch_pdl(k_mg_restrict, grid_for(L[2].n, 256), 256, 0, s, L[2].n, L[2].child.get<int>(),
                       L[1].e.get<float>(), L[2].r.get<float>(), S, need_s);
        } else {
            launch_pdl(k_mg_down, grid_for(32 * L[l + 1].n, 256), 256, 0, s, L[l + 1].n, L[l + 1].child.get<int>(),
                       L[l].val.get<float>(), L[l].nbr.get<int>(), L[l].dinv.get<float>(), L[l].r.get<float>(),
                       L[l].x.get<float>(), L[l + 1].r.get<float>(), S, need_s);
        }
    }
    const int nbc = (int)std::max<long long>(32, (L[Lc].n + 31) / 32 * 32);
    launch_pdl(k_mg_coarsest, 1, nbc, 0, s, (int)L[Lc].n, L[Lc].val.get<float>(), L[Lc].nbr.get<int>(),
               L[Lc].dinv.get<float>(), L[Lc].r.get<float>(), L[Lc].e.get<float>(), S, need_s);
    for (int l = Lc - 1; l >= 1; --l)
        launch_pdl(k_mg_up, grid_for(4 * L[l].n, 256), 256, 0, s, L[l].n, L[l].val.get<float>(), L[l].nbr.get<int>(),
                   L[l].pn.get<int>(), L[l].dinv.get<float>(), L[l].parent.get<int>(), L[l].r.get<float>(),
                   L[l].x.get<float>(), L[l + 1].e.get<float>(), L[l].e.get<float>(), S, need_s);
    launch_pdl(k_mg_up0, grid_for(U, UP0_THREADS), UP0_THREADS, 0, s, U, M.agg0.get<int>(), M.aph.get<__half>(), L[1].nbr.get<int>(),
               L[1].e.get<float>(), z, ctx->A_dinv.get<double>(), out, S, need_s);
    note_launches((uint64_t)mg_launches_per_apply(ctx, restricted));
}

// One V-cycle (ungated) `reps` times between events; algorithmic bytes: the fine level reads
// z twice, the FP16 AP rows (56 B), agg0 and the diagonal and writes out (92 U); each coarse
// row is read as stencil values and neighbor rows twice (down and up, 432 B) plus its vectors.
void mg_kernel_bench(lsmps_ctx* ctx, int reps, double* ms, double* bytes) {
    mg_setup(ctx);
    const long long U = ctx->U;
    double* z = ctx->vtmp.ensure<double>(2 * U + 2);
    double* out = z + U + 1;
    LSMPS_CUDA(cudaMemcpyAsync(z, ctx->A_b.get<double>(), U * sizeof(double), cudaMemcpyDeviceToDevice,
                               ctx->stream));
    mg_apply(ctx, z, out, nullptr, 0);
    ev_record(ctx, 16);
    for (int k = 0; k < reps; ++k) mg_apply(ctx, z, out, nullptr, 0);
    ev_record(ctx, 17);
    *ms = ev_elapsed(ctx, 16, 17) / reps;
    double rows = 0;
    for (int l = 1; l <= ctx->mg->levels; ++l) rows += (double)ctx->mg->L[l].n;
    *bytes = 92.0 * (double)U + 464.0 * rows;
}

void mg_info(lsmps_ctx* ctx, int* levels, int64_t* rows, int cap, double* setup_ms) {
    LSMPS_REQUIRE(ctx->mg && ctx->mg->gen == ctx->assembly_gen, LSMPS_ERR_STATE,
                  "no multigrid hierarchy for the assembled system (solve with the multigrid preconditioner first)");
    const MgState& M = *ctx->mg;
    if (levels) *levels = M.levels;
    if (rows) {
        if (cap > 0) rows[0] = ctx->U;
        for (int l = 1; l <= M.levels && l < cap; ++l) rows[l] = M.L[l].n;
    }
    if (setup_ms) *setup_ms = M.setup_ms;
}

// Host-facing application of the preconditioner (tests): out = D M z in the reference's
// unknown numbering.
__global__ void k_mg_perm(long long U, const int* __restrict__ idx, const double* __restrict__ in,
                          double* __restrict__ out, int gather) {
    long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (u >= U) return;
    if (gather) out[u] = in[idx[u]];
    else out[idx[u]] = in[u];
}

void mg_apply_host(lsmps_ctx* ctx, const double* z, double* out, size_t n) {
    mg_setup(ctx);
    const long long U = ctx->U;
    LSMPS_REQUIRE((long long)n == U && z && out, LSMPS_ERR_ARG, "multigrid apply needs U values in and out");
    cudaStream_t s = ctx->stream;
    double* buf = ctx->vtmp.ensure<double>(3 * U + 3);
    double* zr = buf;
    double* zs = buf + U + 1;
    double* os = buf + 2 * (U + 1);
    LSMPS_CUDA(cudaMemcpyAsync(zr, z, U * sizeof(double), cudaMemcpyHostToDevice, s));
    // reference numbering -> solver numbering: z_s[u] = z_ref[ref_of_u[u]]
    const int* ref_of_u = ctx->ref_of_u.get<int>();
    k_mg_perm<<<grid_for(U, 256), 256, 0, s>>>(U, ref_of_u, zr, zs, 1);
    LSMPS_CHECK_LAUNCH();
    mg_apply(ctx, zs, os, nullptr, 0);
    k_mg_perm<<<grid_for(U, 256), 256, 0, s>>>(U, ref_of_u, os, zr, 0);
    LSMPS_CHECK_LAUNCH();
    LSMPS_CUDA(cudaMemcpyAsync(out, zr, U * sizeof(double), cudaMemcpyDeviceToHost, s));
    LSMPS_CUDA(cudaStreamSynchronize(s));
}

}  // namespace lsmps_gpu
