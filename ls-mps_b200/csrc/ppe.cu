#include <algorithm>
#include <vector>
#include <climits>
// Pressure-Poisson (PPE) CSR assembly on sm_100a.
//
// Unknowns are the Interior / NearWall particles ranked in caller order and capped at
// max_unknowns, as the reference's assemble_ppe (src/lsmps.cpp:33-36). Internally they
// are numbered in cell-sorted order (unknown u = rank among unknowns in the sorted
// arrays), so a row's column indices ascend and its x-gathers fall in a few contiguous
// ranges; lsmps_download_ppe maps rows and columns back to the reference's numbering.
// Each row holds its neighbors that are unknowns in neighbor-list order and the
// diagonal last, like the reference (src/lsmps.cpp:40-57).
//
// One pass over the rows (a group of lanes per row) computes every coefficient once and
// writes the kept entries, p*, b = A p* in entry order and D^-1; a pack kernel moves the
// rows into the CSR after the row lengths are scanned. The reference variant uses exactly
// rounded FP64 operations in the reference's order, so its CSR values and b are
// bit-identical to the reference.
#include <cmath>

#include "ops.cuh"
#include "scan.cuh"

namespace lsmps_gpu {
namespace {

struct PpeParams {
    int variant;
    double re, l0, shift;
    int pinned_ref;  // reference variant: the unknown of rank 0 is an identity row
    int neumann;     // WLS rows: wall neighbors take the row's own value (no entry, no diagonal term)
};

__global__ void k_elig_orig(const int* __restrict__ iperm, const uint8_t* __restrict__ cls, size_t n,
                            uint8_t* __restrict__ elig) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint8_t t = cls[iperm[i]];
    elig[i] = (t == LSMPS_INTERIOR || t == LSMPS_NEAR_WALL) ? 1 : 0;
}

__global__ void k_is_unknown(const int* __restrict__ perm, const uint8_t* __restrict__ elig_orig,
                             const int* __restrict__ rank_orig, long long cap, size_t n,
                             uint8_t* __restrict__ isu) {
    size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    int i = perm[k];
    isu[k] = (elig_orig[i] && rank_orig[i] < cap) ? 1 : 0;
}

__global__ void k_number_unknowns(const int* __restrict__ perm, const uint8_t* __restrict__ isu,
                                  const int* __restrict__ rank_orig, size_t n, int* __restrict__ uidx,
                                  int* __restrict__ sorted_of_u, int* __restrict__ ref_of_u,
                                  int* __restrict__ u_of_ref) {
    size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (k >= n) return;
    int u = uidx[k];  // exclusive scan of isu
    if (isu[k]) {
        int rr = rank_orig[perm[k]];
        sorted_of_u[u] = (int)k;
        ref_of_u[u] = rr;
        u_of_ref[rr] = u;
    } else {
        uidx[k] = -1;
    }
}

// Off-diagonal coefficient a_ij (> 0 means the row gets -a_ij at column j) of row k for
// neighbor m; returns false when the pair contributes nothing. For the WLS rows, zk holds the
// row's Laplacian vector z prescaled (z0..z2, z3..z5 times 1 / (2 l0), z6..z8 times 1 / l0)
// and ws holds 1 / (sum_w l0).
__device__ __forceinline__ bool row_coeff(const PpeParams& P, double xi, double yi, double zi, double xm,
                                          double ym, double zm, const double* zk, double ws, double& a) {
    double dx = xsub(xm, xi), dy = xsub(ym, yi), dz = xsub(zm, zi);
    if (P.variant == LSMPS_PPE_WLS) {
        // c = w (q . z) / (r sum_w l0) with w = (re / r - 1)^2 and q . z = P / r, where P is the
        // polynomial below: c = (re - r)^2 P / (r^4 sum_w l0), from one reciprocal square root
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (!(d2 > 1e-24) || d2 >= P.re * P.re) return false;  // r <= 1e-12 or r >= re: weight 0
        const double ir = rsqrt(d2), ir2 = ir * ir;
        const double t = P.re - d2 * ir;
        const double poly = dx * zk[0] + dy * zk[1] + dz * zk[2] + dx * dx * zk[3] + dy * dy * zk[4] +
                            dz * dz * zk[5] + dx * dy * zk[6] + dx * dz * zk[7] + dy * dz * zk[8];
        a = t * t * poly * ws * (ir2 * ir2);
        return a > 0;  // clipped: only c > 0 contributes
    }
    double r = __dsqrt_rn(xnorm2(dx, dy, dz));
    double w = xweight(r, P.re);
    if (w <= 0) return false;
    if (P.variant == LSMPS_PPE_REFERENCE) {
        a = xdiv(w, xmul(r, r));  // src/lsmps.cpp:48
        return true;
    }
    a = w;  // shifted graph Laplacian
    return true;
}

__device__ __forceinline__ bool wls_row_valid(int st) { return st == 0 || st == 1; }

// p*(x) of the variant at one particle (reference: x^2 + y^2, src/lsmps.cpp:29; otherwise
// the smooth manufactured field), the same expression for a row's own value and its
// neighbors' so that b = A p* is computed from the entries as they are written.
__device__ __forceinline__ double exact_p(int variant, double x, double y, double z) {
    return variant == LSMPS_PPE_REFERENCE ? xadd(xmul(x, x), xmul(y, y)) : sin(0.3 * x) * cos(0.2 * y) + 0.1 * z;
}

// p* at every sorted particle, once (the rows read it for their own and their neighbors' values)
__global__ void k_ppe_exact(size_t n, int variant, const double* __restrict__ sx, const double* __restrict__ sy,
                            const double* __restrict__ sz, double* __restrict__ xep) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        xep[k] = exact_p(variant, sx[k], sy[k], sz[k]);
}

// One pass over the rows, PPE_G lanes per row: the lanes of a row's group take its neighbors
// PPE_G at a time and compute their coefficients; every lane then replays the group's
// coefficients in neighbor order, so the diagonal and b = A p* are the sequential sums of
// the reference's order (exact FP64 operations), identical in all lanes. Kept off-diagonal
// entries go, in order, to the row's slot range at nbr_row[k] + k (room for every neighbor
// plus the diagonal); k_ppe_pack moves them into the CSR once the row lengths are scanned.
// Writes cnt[u] (entries with the diagonal), p*[u], b[u], D^-1[u].
// stats (u64): [0] neumann, [1] failed rows. Capped at 64 registers (8 blocks of 128 threads
// per SM; 72 uncapped): 0.80 against 0.82 ms for the assembly at 1M particles.
constexpr int PPE_G = 8;
__global__ void __launch_bounds__(128, 8) k_ppe_rows(PpeParams P, long long U, const int* __restrict__ sorted_of_u,
                                                  const int* __restrict__ ref_of_u, const int* __restrict__ uidx,
                                                  const double* __restrict__ sx, const double* __restrict__ sy,
                                                  const double* __restrict__ sz, const uint8_t* __restrict__ cls,
                                                  const int* __restrict__ row, const int* __restrict__ col,
                                                  const int* __restrict__ wst, const double* __restrict__ wz,
                                                  const double* __restrict__ wws, int* __restrict__ cnt,
                                                  int* __restrict__ scol, double* __restrict__ sval,
                                                  const double* __restrict__ xep, double* __restrict__ xexact,
                                                  double* __restrict__ b,
                                                  double* __restrict__ dinv, unsigned long long* stats) {
    const int lane = threadIdx.x & 31, sub = lane & (PPE_G - 1), gbase = lane & ~(PPE_G - 1);
    const long long u = (blockIdx.x * (long long)blockDim.x + threadIdx.x) / PPE_G;
    const bool live = u < U;
    int k = 0, e0 = 0, e1 = 0;
    bool pinned = false, identity = false;
    double xi = 0, yi = 0, zi = 0, ws = 0;
    if (live) {
        k = sorted_of_u[u];
        xi = sx[k], yi = sy[k], zi = sz[k];
        pinned = P.variant == LSMPS_PPE_REFERENCE && ref_of_u[u] == P.pinned_ref;
        identity = P.variant == LSMPS_PPE_WLS && !wls_row_valid(wst[k]);
        if (!pinned && !identity) e0 = row[k], e1 = row[k + 1];
    }
    double zk[K];
#pragma unroll
    for (int a = 0; a < K; ++a) zk[a] = 0.0;
    if (live && P.variant == LSMPS_PPE_WLS && !pinned && !identity) {
        const double h = 0.5 / P.l0, g = 1.0 / P.l0;
#pragma unroll
        for (int a = 0; a < K; ++a) zk[a] = wz[(size_t)k * K + a] * (a < 3 ? 1.0 : a < 6 ? h : g);
        ws = 1.0 / (wws[k] * P.l0);
    }
    const long long sbase = live ? (long long)row[k] + k : 0;  // the row's slot range
    // the warp walks the longest of its groups' rows; shorter rows idle (flags stay 0)
    const int chunks = __reduce_max_sync(0xffffffffu, (e1 - e0 + PPE_G - 1) / PPE_G);
    double diag = 0.0, bsum = 0.0;
    int written = 0;
    // the neighbor index of the next chunk is loaded one chunk ahead, so each chunk waits for
    // one round trip (its gathers) instead of two
    int mnext = e0 + sub < e1 ? col[e0 + sub] : 0;
    for (int c = 0; c < chunks; ++c) {
        const int e = e0 + c * PPE_G + sub;
        const int m_cur = mnext;
        mnext = e + PPE_G < e1 ? col[e + PPE_G] : 0;
        bool contrib = false, keep = false;
        double a = 0.0, xem = 0.0;
        int cj = -1;
        if (e < e1) {
            // every load of the pair at once
            const int m = m_cur;
            cj = uidx[m];
            const double xm = sx[m], ym = sy[m], zm = sz[m];
            const double xpm = xep[m];
            const bool wall = P.neumann && cls[m] == LSMPS_WALL;
            if ((P.variant == LSMPS_PPE_WLS || cj >= 0) && !wall) {
                contrib = row_coeff(P, xi, yi, zi, xm, ym, zm, zk, ws, a);
                keep = contrib && cj >= 0;
                if (keep) xem = xpm;
            }
        }
        const unsigned kb = (__ballot_sync(0xffffffffu, keep) >> gbase) & ((1u << PPE_G) - 1u);
        if (keep) {
            const long long p = sbase + written + __popc(kb & ((1u << sub) - 1u));
            scol[p] = cj;
            sval[p] = -a;
        }
        written += __popc(kb);
        // the group's coefficients in neighbor order: diagonal and b as sequential sums
#pragma unroll
        for (int j = 0; j < PPE_G; ++j) {
            const double aj = __shfl_sync(0xffffffffu, a, gbase + j);
            const double xj = __shfl_sync(0xffffffffu, xem, gbase + j);
            const int fj = __shfl_sync(0xffffffffu, (contrib ? 1 : 0) | (keep ? 2 : 0), gbase + j);
            if (fj & 1) diag = xadd(diag, aj);
            if (fj & 2) bsum = xadd(bsum, xmul(-aj, xj));
        }
    }
    int neumann = 0, failed = 0;
    if (live) {
        const double xe = xep[k];
        int c = written;
        if (pinned) {
            c = 0;
            diag = 1.0;
            bsum = 0.0;
        } else {
            // WLS rows without a positive, finite diagonal become identity rows
            if (P.variant == LSMPS_PPE_WLS && !identity && !(diag > 0 && isfinite(diag))) identity = true;
            if (identity) {
                c = 0;
                bsum = 0.0;
                failed = 1;
                diag = 1.0;
            } else {
                if (P.variant != LSMPS_PPE_REFERENCE) diag = diag * (1.0 + P.shift);
                if (diag <= 0 || !isfinite(diag)) {  // src/lsmps.cpp:52
                    failed = 1;
                    diag = 1.0;
                }
            }
            if (cls[k] == LSMPS_NEAR_WALL) neumann = 1;
        }
        if (sub == 0) {
            scol[sbase + c] = (int)u;
            sval[sbase + c] = diag;
            cnt[u] = c + 1;
            xexact[u] = xe;
            b[u] = xadd(bsum, xmul(diag, xe));
            dinv[u] = 1.0 / diag;
        }
    }
    if (sub != 0) neumann = failed = 0;
    neumann = __reduce_add_sync(0xffffffffu, neumann);
    failed = __reduce_add_sync(0xffffffffu, failed);
    if (lane == 0) {
        if (neumann) atomicAdd(&stats[0], (unsigned long long)neumann);
        if (failed) atomicAdd(&stats[1], (unsigned long long)failed);
    }
}

// Moves each row's slot range into the CSR. A block takes PACK_ROWS consecutive rows, whose
// entries are one contiguous range of the CSR: each warp loads the first 32 entries of four
// rows at once (the rest of a longer row after them) into shared memory at their CSR offsets,
// then the block writes the range with consecutive stores. A block whose range exceeds
// PACK_CAP entries copies its rows directly.
constexpr int PACK_ROWS = 32, PACK_CAP = 2048, PACK_THREADS = 256;
__global__ void __launch_bounds__(PACK_THREADS) k_ppe_pack(long long U, const int* __restrict__ sorted_of_u,
                                                           const int* __restrict__ nrow, const int* __restrict__ arow,
                                                           const int* __restrict__ scol,
                                                           const double* __restrict__ sval, int* __restrict__ acol,
                                                           double* __restrict__ aval) {
    __shared__ double bval[PACK_CAP];
    __shared__ int bcol[PACK_CAP];
    __shared__ int roff[PACK_ROWS + 1];
    __shared__ long long rsrc[PACK_ROWS];
    const long long u0 = blockIdx.x * (long long)PACK_ROWS;
    const int nr = (int)min((long long)PACK_ROWS, U - u0);
    if (threadIdx.x <= nr) roff[threadIdx.x] = arow[u0 + threadIdx.x];
    if (threadIdx.x < nr) {
        const int k = sorted_of_u[u0 + threadIdx.x];
        rsrc[threadIdx.x] = (long long)nrow[k] + k;
    }
    __syncthreads();
    const int base = roff[0], total = roff[nr] - base;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int RPW = PACK_ROWS / (PACK_THREADS / 32);  // rows per warp
    if (total <= PACK_CAP) {
        int cc[RPW];
        double vv[RPW];
#pragma unroll
        for (int j = 0; j < RPW; ++j) {
            const int r = warp + j * (PACK_THREADS / 32);
            const bool on = r < nr && lane < roff[r + 1] - roff[r];
            cc[j] = on ? __ldcs(scol + rsrc[r] + lane) : 0;
            vv[j] = on ? __ldcs(sval + rsrc[r] + lane) : 0.0;
        }
#pragma unroll
        for (int j = 0; j < RPW; ++j) {
            const int r = warp + j * (PACK_THREADS / 32);
            if (r < nr && lane < roff[r + 1] - roff[r]) {
                bcol[roff[r] - base + lane] = cc[j];
                bval[roff[r] - base + lane] = vv[j];
            }
        }
        for (int j = 0; j < RPW; ++j) {  // rows longer than 32 entries
            const int r = warp + j * (PACK_THREADS / 32);
            if (r >= nr) break;
            const int o = roff[r] - base, c = roff[r + 1] - roff[r];
            for (int p = 32 + lane; p < c; p += 32) {
                bcol[o + p] = __ldcs(scol + rsrc[r] + p);
                bval[o + p] = __ldcs(sval + rsrc[r] + p);
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < total; i += PACK_THREADS) {
            acol[base + i] = bcol[i];
            aval[base + i] = bval[i];
        }
    } else {
        for (int r = warp; r < nr; r += PACK_THREADS / 32) {
            const int o = roff[r], c = roff[r + 1] - o;
            for (int p = lane; p < c; p += 32) {
                acol[o + p] = __ldcs(scol + rsrc[r] + p);
                aval[o + p] = __ldcs(sval + rsrc[r] + p);
            }
        }
    }
}

// ---- download in the reference numbering ----
__global__ void k_ref_counts(const int* __restrict__ u_of_ref, const int* __restrict__ arow, long long U,
                             int* __restrict__ cnt) {
    long long rr = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (rr >= U) return;
    int u = u_of_ref[rr];
    cnt[rr] = arow[u + 1] - arow[u];
}

__global__ void k_ref_fill(const int* __restrict__ u_of_ref, const int* __restrict__ ref_of_u,
                           const int* __restrict__ arow, const int* __restrict__ acol,
                           const double* __restrict__ aval, const double* __restrict__ b,
                           const double* __restrict__ xe, const int* __restrict__ sorted_of_u,
                           const int* __restrict__ perm, long long U, const int* __restrict__ orow,
                           int* __restrict__ ocol, double* __restrict__ oval, double* __restrict__ ob,
                           double* __restrict__ oxe, int* __restrict__ opart) {
    long long rr = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (rr >= U) return;
    int u = u_of_ref[rr];
    int o = orow[rr];
    for (int e = arow[u]; e < arow[u + 1]; ++e, ++o) {
        ocol[o] = ref_of_u[acol[e]];
        oval[o] = aval[e];
    }
    ob[rr] = b[u];
    oxe[rr] = xe[u];
    opart[rr] = perm[sorted_of_u[u]];
}

}  // namespace

void ppe_assemble(lsmps_ctx* ctx, const lsmps_ppe_opts* o, lsmps_ppe_stats* out) {
    LSMPS_REQUIRE(ctx->have_neighbors && ctx->have_classes, LSMPS_ERR_STATE,
                  "PPE assembly needs neighbor lists and classification first");
    LSMPS_REQUIRE(o && o->variant >= 0 && o->variant <= 2, LSMPS_ERR_ARG, "unknown PPE variant");
    LSMPS_REQUIRE(o->variant != LSMPS_PPE_WLS || ctx->have_wls, LSMPS_ERR_STATE,
                  "WLS-Laplacian PPE needs the all-particle WLS (lsmps_wls mode 1) first");
    LSMPS_REQUIRE(o->re > 0 && o->l0 > 0, LSMPS_ERR_ARG, "PPE options need re > 0 and l0 > 0");
    cudaStream_t s = ctx->stream;
    size_t n = ctx->n;
    int* dflag = ctx->dflags.get<int>();
    ev_record(ctx, 8);
    long long cap = std::min<long long>((long long)n, std::max<long long>(0, o->max_unknowns));

    uint8_t* elig = ctx->A_cnt.ensure<uint8_t>(2 * n + 16);
    uint8_t* isu = elig + n + 8;
    int* rank = ctx->ref_rank.ensure<int>(n + 1);
    int* uidx = ctx->u_of_sorted.ensure<int>(n + 1);
    if (n) {
        k_elig_orig<<<blocks_for(n, 256), 256, 0, s>>>(ctx->iperm.get<int>(), ctx->cls.get<uint8_t>(), n, elig);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<uint8_t>(elig, rank, (long long)n, s, ctx->scan_tmp, dflag);
    if (n) {
        k_is_unknown<<<blocks_for(n, 256), 256, 0, s>>>(ctx->perm.get<int>(), elig, rank, cap, n, isu);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<uint8_t>(isu, uidx, (long long)n, s, ctx->scan_tmp, dflag);
    int hU = 0;
    read_back(ctx, {{uidx + n, &hU, sizeof(int)}}, nullptr);
    const long long U = hU;
    int* sorted_of_u = ctx->sorted_of_u.ensure<int>(U + 1);
    int* ref_of_u = ctx->ref_of_u.ensure<int>(U + 1);
    int* u_of_ref = ctx->u_of_ref.ensure<int>(U + 1);
    if (n) {
        k_number_unknowns<<<blocks_for(n, 256), 256, 0, s>>>(ctx->perm.get<int>(), isu, rank, n, uidx, sorted_of_u,
                                                             ref_of_u, u_of_ref);
        LSMPS_CHECK_LAUNCH();
    }
    LSMPS_REQUIRE((o->flags & ~LSMPS_PPE_WALL_NEUMANN) == 0 &&
                      (!(o->flags & LSMPS_PPE_WALL_NEUMANN) || o->variant == LSMPS_PPE_WLS),
                  LSMPS_ERR_ARG, "PPE flags: LSMPS_PPE_WALL_NEUMANN is for the WLS variant");
    const int neumann = (o->flags & LSMPS_PPE_WALL_NEUMANN) ? 1 : 0;
    PpeParams P{o->variant, o->re, o->l0, o->diag_shift, 0, neumann};
    int* cnt = ctx->vtmp.ensure<int>(U + 1);
    int* arow = ctx->A_row.ensure<int>(U + 1);
    const int* wst = ctx->have_wls ? ctx->wls_status.get<int>() : nullptr;
    const double* wz = ctx->have_wls ? ctx->wls_z.get<double>() : nullptr;
    const double* wws = ctx->have_wls ? ctx->wls_wsum.get<double>() : nullptr;
    // slot ranges: a row of sorted particle k at nbr_row[k] + k, room for its neighbors and the diagonal
    const size_t slots = (size_t)ctx->pairs + n + 1;
    int* scol = ctx->A_slot_col.ensure<int>(slots);
    double* sval = ctx->A_slot_val.ensure<double>(slots);
    double* xe = ctx->A_xexact.ensure<double>(U + 1);
    double* b = ctx->A_b.ensure<double>(U + 1);
    double* dinv = ctx->A_dinv.ensure<double>(U + 1);
    auto* st = reinterpret_cast<unsigned long long*>(ctx->scratch.get<int>() + 32);
    LSMPS_CUDA(cudaMemsetAsync(st, 0, 2 * sizeof(unsigned long long), s));
    if (U) {
        double* xep = ctx->A_xep.ensure<double>(n + 1);
        k_ppe_exact<<<std::min<unsigned>(blocks_for(n, 256), 148 * 8), 256, 0, s>>>(
            n, o->variant, ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(), xep);
        k_ppe_rows<<<blocks_for((size_t)U * PPE_G, 128), 128, 0, s>>>(
            P, U, sorted_of_u, ref_of_u, uidx, ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(),
            ctx->cls.get<uint8_t>(), ctx->nbr_row.get<int>(), ctx->nbr_col.get<int>(), wst, wz, wws, cnt, scol, sval,
            xep, xe, b, dinv, st);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<int>(cnt, arow, U, s, ctx->scan_tmp, dflag);
    int hnnz = 0;
    unsigned long long hs[2];  // the rows' statistics are final here
    read_back(ctx, {{arow + U, &hnnz, sizeof(int)}, {st, hs, sizeof(hs)}}, "PPE rows");
    const long long nnz = hnnz;
    int* acol = ctx->A_col.ensure<int>(nnz + 1);
    double* aval = ctx->A_val.ensure<double>(nnz + 1);
    if (U) {
        k_ppe_pack<<<blocks_for((size_t)U, PACK_ROWS), PACK_THREADS, 0, s>>>(U, sorted_of_u, ctx->nbr_row.get<int>(),
                                                                             arow, scol, sval, acol, aval);
        LSMPS_CHECK_LAUNCH();
    }
    ev_record(ctx, 9);
    lsmps_ppe_stats ps{};
    ps.unknowns = (uint64_t)U;
    ps.nnz = (uint64_t)nnz;
    ps.dirichlet = (uint64_t)(n - U);
    // the reference counts NearWall rows except the pinned row 0 (src/lsmps.cpp:45,56)
    ps.neumann = hs[0];
    ps.failed_rows = hs[1];
    ps.assembly_ms = out ? ev_elapsed(ctx, 8, 9) : 0.0;  // without statistics: read later
    ctx->U = U;
    ctx->nnz = nnz;
    ctx->ppe_variant = o->variant;
    ctx->ppe_wall_neumann = neumann != 0;
    ctx->ppe_loaded = false;
    ctx->have_ppe = true;
    ctx->have_solution = false;
    ctx->assembly_gen += 1;
    ctx->have_sell = ctx->have_sell_s = ctx->have_sell_f = ctx->have_sell_raw = false;
    ctx->ppe_assembly = ps;
    if (out) *out = ps;
}

// A caller's system in place of an assembled one (rows = unknowns, identity numbering). The
// diagonal goes last in every row, as the assembly stores it; entries j == i are summed into it.
// Without values: -1 for every off-diagonal entry and a diagonal of (off-diagonal count)
// (1 + 1e-3) (at least 1), a diagonally dominant operator; without b: b = A 1 and p* = 1.
void ppe_load_csr(lsmps_ctx* ctx, const int64_t* row_ptr, const int32_t* col, const double* val, const double* b,
                  size_t n, lsmps_ppe_stats* out) {
    LSMPS_REQUIRE(row_ptr && (n == 0 || col || row_ptr[n] == 0), LSMPS_ERR_ARG, "null CSR arrays");
    LSMPS_REQUIRE(n < (size_t)INT_MAX && row_ptr[0] == 0, LSMPS_ERR_ARG, "row_ptr[0] must be 0 and n < 2^31");
    const int64_t nnz_in = row_ptr[n];
    std::vector<int> arow(n + 1), acol;
    std::vector<double> aval, adinv(n), ab(n), axe(n);
    acol.reserve((size_t)nnz_in + n);
    aval.reserve((size_t)nnz_in + n);
    arow[0] = 0;
    for (size_t i = 0; i < n; ++i) {
        const int64_t e0 = row_ptr[i], e1 = row_ptr[i + 1];
        LSMPS_REQUIRE(e1 >= e0 && e1 <= nnz_in, LSMPS_ERR_ARG, "row_ptr must be non-decreasing up to row_ptr[n]");
        double diag = 0;
        int off = 0;
        for (int64_t e = e0; e < e1; ++e) {
            const int32_t j = col[e];
            LSMPS_REQUIRE(j >= 0 && (size_t)j < n, LSMPS_ERR_ARG, "column index out of range");
            if ((size_t)j == i) {
                if (val) diag += val[e];
                continue;
            }
            acol.push_back(j);
            aval.push_back(val ? val[e] : -1.0);
            ++off;
        }
        if (!val) diag = std::max(1.0, off * (1.0 + 1e-3));
        LSMPS_REQUIRE(std::isfinite(diag) && diag != 0.0, LSMPS_ERR_ARG,
                      "row " + std::to_string(i) + " has a zero or non-finite diagonal");
        acol.push_back((int)i);
        aval.push_back(diag);
        adinv[i] = 1.0 / diag;
        LSMPS_REQUIRE(acol.size() < (size_t)INT_MAX, LSMPS_ERR_OVERFLOW, "more than 2^31 entries");
        arow[i + 1] = (int)acol.size();
    }
    for (size_t i = 0; i < n; ++i) {
        if (b) {
            ab[i] = b[i];
            axe[i] = 0.0;
        } else {
            double s = 0;
            for (int e = arow[i]; e < arow[i + 1]; ++e) s += aval[e];
            ab[i] = s;
            axe[i] = 1.0;
        }
    }
    std::vector<int> ident(n);
    for (size_t i = 0; i < n; ++i) ident[i] = (int)i;
    cudaStream_t s = ctx->stream;
    const size_t nnz = acol.size();
    auto up = [&](DevBuf& d, const void* h, size_t bytes) {
        void* p = d.ensure<char>(bytes + 16);
        if (bytes) LSMPS_CUDA(cudaMemcpyAsync(p, h, bytes, cudaMemcpyHostToDevice, s));
    };
    up(ctx->A_row, arow.data(), (n + 1) * sizeof(int));
    up(ctx->A_col, acol.data(), nnz * sizeof(int));
    up(ctx->A_val, aval.data(), nnz * sizeof(double));
    up(ctx->A_b, ab.data(), n * sizeof(double));
    up(ctx->A_xexact, axe.data(), n * sizeof(double));
    up(ctx->A_dinv, adinv.data(), n * sizeof(double));
    for (DevBuf* d : {&ctx->ref_of_u, &ctx->u_of_ref, &ctx->sorted_of_u, &ctx->ld_ident})
        up(*d, ident.data(), n * sizeof(int));
    LSMPS_CUDA(cudaStreamSynchronize(s));
    lsmps_ppe_stats ps{};
    ps.unknowns = n;
    ps.nnz = nnz;
    ctx->U = (long long)n;
    ctx->nnz = (long long)nnz;
    ctx->ppe_variant = LSMPS_PPE_LOADED;
    ctx->ppe_loaded = true;
    ctx->have_ppe = true;
    ctx->have_solution = false;
    ctx->assembly_gen += 1;
    ctx->have_sell = ctx->have_sell_s = ctx->have_sell_f = ctx->have_sell_raw = false;
    ctx->ppe_assembly = ps;
    ctx->timing_pending &= ~16u;  // a loaded system has no pending assembly time
    if (out) *out = ps;
}

void ppe_download(lsmps_ctx* ctx, int32_t* row, int32_t* col, double* val, double* b, double* xe,
                  int32_t* unknown_particle) {
    LSMPS_REQUIRE(ctx->have_ppe, LSMPS_ERR_STATE, "no PPE assembled");
    cudaStream_t s = ctx->stream;
    long long U = ctx->U, nnz = ctx->nnz;
    size_t bytes = (U + 1) * 4 * 2 + nnz * 12 + U * 16 + U * 4 + 256;
    char* base = ctx->vtmp.ensure<char>(bytes);
    int* cnt = reinterpret_cast<int*>(base);
    int* orow = cnt + (U + 1);
    double* oval = reinterpret_cast<double*>(base + (((U + 1) * 8 + 15) / 16) * 16);
    double* ob = oval + nnz;
    double* oxe = ob + U;
    int* ocol = reinterpret_cast<int*>(oxe + U);
    int* opart = ocol + nnz;
    if (U) {
        k_ref_counts<<<blocks_for(U, 256), 256, 0, s>>>(ctx->u_of_ref.get<int>(), ctx->A_row.get<int>(), U, cnt);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<int>(cnt, orow, U, s, ctx->scan_tmp, ctx->dflags.get<int>());
    if (U) {
        k_ref_fill<<<blocks_for(U, 128), 128, 0, s>>>(ctx->u_of_ref.get<int>(), ctx->ref_of_u.get<int>(),
                                                      ctx->A_row.get<int>(), ctx->A_col.get<int>(),
                                                      ctx->A_val.get<double>(), ctx->A_b.get<double>(),
                                                      ctx->A_xexact.get<double>(), ctx->sorted_of_u.get<int>(),
                                                      ctx->ppe_loaded ? ctx->ld_ident.get<int>() : ctx->perm.get<int>(),
                                                      U, orow, ocol, oval, ob, oxe, opart);
        LSMPS_CHECK_LAUNCH();
    }
    if (row) LSMPS_CUDA(cudaMemcpyAsync(row, orow, (U + 1) * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (U) {
        if (col) LSMPS_CUDA(cudaMemcpyAsync(col, ocol, nnz * sizeof(int), cudaMemcpyDeviceToHost, s));
        if (val) LSMPS_CUDA(cudaMemcpyAsync(val, oval, nnz * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (b) LSMPS_CUDA(cudaMemcpyAsync(b, ob, U * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (xe) LSMPS_CUDA(cudaMemcpyAsync(xe, oxe, U * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (unknown_particle)
            LSMPS_CUDA(cudaMemcpyAsync(unknown_particle, opart, U * sizeof(int), cudaMemcpyDeviceToHost, s));
    }
    LSMPS_CUDA(cudaStreamSynchronize(s));
}

}  // namespace lsmps_gpu
