// One pressure projection of the LS-MPS fractional-step scheme on the current particle set,
// in 3-D with the all-particle WLS (the reference's 2-D step: python/rain_plate_lsmps_cpu.py
// divergence:202-206, solve_pressure:209-252, pressure_correct:255-260):
//   div u*    sum over c of the c-th gradient component of u*_c, from the WLS of the three
//             velocity components (wls_fields);
//   PPE       the assembled WLS-Laplacian system (variant WLS: free-surface and splash
//             particles are Dirichlet p = 0, walls are not unknowns), A ~ -lap, so the
//             right-hand side of lap p = rho / dt div u* is b = -rho / dt div u*;
//   u         u* - dt / rho grad p from the WLS gradient of p (p = 0 off the unknowns); wall
//             particles keep u*.
// The divergence before and after is measured over the unknowns (where the PPE holds) and over
// the core: Interior unknowns at least three neighbor hops from any other particle (free
// surface, splash, wall, near-wall). In the first two layers inside a Dirichlet surface the clipped
// WLS-Laplacian rows and the one-sided WLS gradients disagree and leave a divergence of the
// order of the pressure jump times dt / rho; in the core the projection works as intended.
#include <cmath>

#include "ops.cuh"

namespace lsmps_gpu {
namespace {

constexpr int KB = 9;  // WLS unknowns per field

// mask[i] = 1 for the particles that are unknowns
__global__ void k_unknown_mask(long long U, const int* __restrict__ sorted_of_u, const int* __restrict__ perm,
                               uint8_t* __restrict__ mask) {
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < U; u += (long long)gridDim.x * blockDim.x)
        mask[perm[sorted_of_u[u]]] = 1;
}

// Neighbor-hop distances (sorted order) from a seed set, exact up to 3: seed particles 0,
// the others HOP_FAR, then three passes of hop = min(hop, 1 + min over neighbors). Seeds:
//   SEED_BOUNDARY  every particle but the Interior unknowns (free surface, splash, wall, near-wall)
//   SEED_SURFACE   free-surface and splash particles
//   SEED_WALL      wall particles
constexpr uint8_t HOP_FAR = 255;
enum { SEED_BOUNDARY = 0, SEED_SURFACE = 1, SEED_WALL = 2 };
__global__ void k_hop_seed(size_t n, int mode, const uint8_t* __restrict__ cls, const uint8_t* __restrict__ isu,
                           uint8_t* __restrict__ hop) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const uint8_t c = cls[k];
        bool seed;
        if (mode == SEED_BOUNDARY) seed = !(isu[k] && c == LSMPS_INTERIOR);
        else if (mode == SEED_SURFACE) seed = c == LSMPS_FREE_SURFACE || c == LSMPS_SPLASH;
        else seed = c == LSMPS_WALL;
        hop[k] = seed ? 0 : HOP_FAR;
    }
}
// isu[k] = 1 for the sorted particles that are unknowns
__global__ void k_unknown_sorted(long long U, const int* __restrict__ sorted_of_u, uint8_t* __restrict__ isu) {
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < U; u += (long long)gridDim.x * blockDim.x)
        isu[sorted_of_u[u]] = 1;
}
__global__ void k_hop_pass(size_t n, const int* __restrict__ row, const int* __restrict__ col,
                           const uint8_t* __restrict__ in, uint8_t* __restrict__ out) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        int h = in[k];
        for (int e = row[k]; e < row[k + 1] && h > 0; ++e) h = min(h, in[col[e]] + 1);
        out[k] = (uint8_t)h;
    }
}
// mask[i] (caller order): bit 0 unknown, bit 1 core (at least three hops from any boundary
// particle), bit 2 wall band 1 and bit 3 wall band 2 (unknowns one / two hops from a wall and
// at least three from the free surface)
__global__ void k_region_mask(size_t n, const int* __restrict__ iperm, const uint8_t* __restrict__ hb,
                              const uint8_t* __restrict__ hs, const uint8_t* __restrict__ hw,
                              uint8_t* __restrict__ mask) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (!mask[i]) continue;
        const int k = iperm[i];
        uint8_t m = mask[i];
        if (hb[k] >= 3) m |= 2;
        if (hs[k] >= 3 && hw[k] == 1) m |= 4;
        if (hs[k] >= 3 && hw[k] == 2) m |= 8;
        mask[i] = m;
    }
}

// div[i] = d u_x / dx + d u_y / dy + d u_z / dz from the WLS solutions of the three fields;
// stats: [0] sum div^2, [1] max |div| (bits), [2] count over the unknowns, then sum div^2 and
// count over the core [3, 4], wall band 1 [5, 6] and wall band 2 [7, 8]
__global__ void k_divergence(size_t n, const double* __restrict__ G, const uint8_t* __restrict__ mask,
                             double* __restrict__ div, double* stats) {
    double s2 = 0, mx = 0, cnt = 0;
    double rs[3] = {0, 0, 0}, rc[3] = {0, 0, 0};  // core, wall band 1, wall band 2
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double* g = G + i * 3 * KB;
        const double d = g[0] + g[KB + 1] + g[2 * KB + 2];
        if (div) div[i] = d;
        if (mask[i] & 1) {
            s2 += d * d;
            mx = fmax(mx, fabs(d));
            cnt += 1;
        }
#pragma unroll
        for (int r = 0; r < 3; ++r)
            if (mask[i] & (2 << r)) {
                rs[r] += d * d;
                rc[r] += 1;
            }
    }
    s2 = warp_sum(s2);
    cnt = warp_sum(cnt);
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        rs[r] = warp_sum(rs[r]);
        rc[r] = warp_sum(rc[r]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&stats[0], s2);
        atomicAdd(&stats[2], cnt);
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            atomicAdd(&stats[3 + 2 * r], rs[r]);
            atomicAdd(&stats[4 + 2 * r], rc[r]);
        }
        atomicMax(reinterpret_cast<unsigned long long*>(&stats[1]), (unsigned long long)__double_as_longlong(mx));
    }
}

// b[u] = scale div(particle of u); p* = 0 (no manufactured solution)
__global__ void k_rhs_from_div(long long U, const int* __restrict__ sorted_of_u, const int* __restrict__ perm,
                               const double* __restrict__ div, double scale, double* __restrict__ b,
                               double* __restrict__ xe) {
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < U; u += (long long)gridDim.x * blockDim.x) {
        b[u] = scale * div[perm[sorted_of_u[u]]];
        xe[u] = 0.0;
    }
}

// u = u* - c grad p (walls keep u*); grad p = the first three WLS unknowns of the field p
__global__ void k_correct(size_t n, const uint8_t* __restrict__ type, const double* __restrict__ ustar,
                          const double* __restrict__ Gp, double c, double* __restrict__ u) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const bool wall = type[i] == LSMPS_WALL;
#pragma unroll
        for (int a = 0; a < 3; ++a) u[3 * i + a] = wall ? ustar[3 * i + a] : ustar[3 * i + a] - c * Gp[i * KB + a];
    }
}

// u* = u + dt (nu lap u + g); lap u of each component from its WLS solution, (x3 + x4 + x5) / l0
// (zero where the WLS is skipped or failed: splash particles fall freely); walls keep u
__global__ void k_predict(size_t n, const uint8_t* __restrict__ type, const double* __restrict__ u,
                          const double* __restrict__ G, double l0inv, double dt, double nu, double3 g,
                          double* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const bool wall = type[i] == LSMPS_WALL;
        const double ga[3] = {g.x, g.y, g.z};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double* x = G + (i * 3 + a) * KB;
            const double lap = (x[3] + x[4] + x[5]) * l0inv;
            out[3 * i + a] = wall ? u[3 * i + a] : u[3 * i + a] + dt * (nu * lap + ga[a]);
        }
    }
}

unsigned grid_n(size_t n) { return std::max(1u, std::min<unsigned>(blocks_for(n, 256), 148 * 8)); }

}  // namespace

void predict_velocity(lsmps_ctx* ctx, const double* d_vel, double dt, double nu, const double* g, int flags,
                      double* d_vel_out) {
    LSMPS_REQUIRE(ctx->have_neighbors && ctx->have_classes, LSMPS_ERR_STATE,
                  "the predictor needs neighbor lists and classification first");
    LSMPS_REQUIRE(dt > 0 && std::isfinite(dt) && nu >= 0 && std::isfinite(nu) && g, LSMPS_ERR_ARG,
                  "predictor: dt > 0, nu >= 0 and a gravity vector");
    LSMPS_REQUIRE((flags & ~LSMPS_PPE_WALL_NEUMANN) == 0, LSMPS_ERR_ARG, "predictor flags");
    const size_t n = ctx->n;
    LSMPS_REQUIRE(n == 0 || (d_vel && d_vel_out), LSMPS_ERR_ARG, "null velocity buffer");
    double* G = ctx->pj_grad.ensure<double>(n * 3 * KB + 1);
    wls_fields(ctx, d_vel, 3, G, (flags & LSMPS_PPE_WALL_NEUMANN) != 0);
    if (n) {
        k_predict<<<grid_n(n), 256, 0, ctx->stream>>>(n, ctx->type_in.get<uint8_t>(), d_vel, G, 1.0 / ctx->l0, dt, nu,
                                                      make_double3(g[0], g[1], g[2]), d_vel_out);
        LSMPS_CHECK_LAUNCH();
    }
    LSMPS_CUDA(cudaStreamSynchronize(ctx->stream));
}

void projection_step(lsmps_ctx* ctx, const double* d_vel, double dt, double rho, const lsmps_solver_opts* so,
                     double* d_vel_out, double* d_pressure, lsmps_projection_stats* out) {
    LSMPS_REQUIRE(ctx->have_ppe && ctx->ppe_variant == LSMPS_PPE_WLS, LSMPS_ERR_STATE,
                  "the projection needs the WLS-Laplacian PPE assembled (lsmps_ppe_assemble, variant WLS)");
    LSMPS_REQUIRE(dt > 0 && rho > 0 && std::isfinite(dt) && std::isfinite(rho), LSMPS_ERR_ARG,
                  "dt and rho must be positive and finite");
    LSMPS_REQUIRE(so, LSMPS_ERR_ARG, "null solver options");
    const size_t n = ctx->n;
    LSMPS_REQUIRE(n == 0 || (d_vel && d_vel_out && d_pressure), LSMPS_ERR_ARG, "null velocity or pressure buffer");
    cudaStream_t s = ctx->stream;
    lsmps_projection_stats st{};
    ev_record(ctx, 12);
    double* G = ctx->pj_grad.ensure<double>(n * 3 * KB + 1);
    double* div = ctx->pj_div.ensure<double>(n + 1);
    uint8_t* mask = ctx->pj_mask.ensure<uint8_t>(n + 1);
    double* stats = ctx->pj_stats.ensure<double>(32);
    const long long U = ctx->U;
    const bool neumann = ctx->ppe_wall_neumann;
    LSMPS_CUDA(cudaMemsetAsync(mask, 0, n + 1, s));
    LSMPS_CUDA(cudaMemsetAsync(stats, 0, 32 * sizeof(double), s));
    if (U) {
        k_unknown_mask<<<1184, 256, 0, s>>>(U, ctx->sorted_of_u.get<int>(), ctx->perm.get<int>(), mask);
        uint8_t* hop = ctx->pj_hop.ensure<uint8_t>(5 * (n + 1));
        uint8_t* isu = hop + 3 * (n + 1);
        uint8_t* tmp = isu + (n + 1);
        LSMPS_CUDA(cudaMemsetAsync(isu, 0, n + 1, s));
        k_unknown_sorted<<<1184, 256, 0, s>>>(U, ctx->sorted_of_u.get<int>(), isu);
        for (int mode = 0; mode < 3; ++mode) {  // three passes ping-pong between tmp and the result
            uint8_t* h = hop + mode * (n + 1);
            k_hop_seed<<<grid_n(n), 256, 0, s>>>(n, mode, ctx->cls.get<uint8_t>(), isu, h);
            for (int pass = 0; pass < 3; ++pass)
                k_hop_pass<<<grid_n(n), 256, 0, s>>>(n, ctx->nbr_row.get<int>(), ctx->nbr_col.get<int>(),
                                                     pass % 2 ? tmp : h, pass % 2 ? h : tmp);
            LSMPS_CUDA(cudaMemcpyAsync(h, tmp, n, cudaMemcpyDeviceToDevice, s));  // after an odd pass count
        }
        k_region_mask<<<grid_n(n), 256, 0, s>>>(n, ctx->iperm.get<int>(), hop, hop + (n + 1), hop + 2 * (n + 1), mask);
        note_launches(15);
        LSMPS_CHECK_LAUNCH();
    }
    // 1. div u*
    wls_fields(ctx, d_vel, 3, G, neumann);
    if (n) {
        k_divergence<<<grid_n(n), 256, 0, s>>>(n, G, mask, div, stats);
        LSMPS_CHECK_LAUNCH();
    }
    // 2. PPE right-hand side and solve
    if (U) {
        k_rhs_from_div<<<1184, 256, 0, s>>>(U, ctx->sorted_of_u.get<int>(), ctx->perm.get<int>(), div, -rho / dt,
                                            ctx->A_b.get<double>(), ctx->A_xexact.get<double>());
        LSMPS_CHECK_LAUNCH();
    }
    lsmps_ppe_stats ps{};
    ppe_solve(ctx, so, &ps);
    if (U) {
        ppe_pressure_particles(ctx, d_pressure, n, 0.0, true);
    } else if (n) {
        LSMPS_CUDA(cudaMemsetAsync(d_pressure, 0, n * sizeof(double), s));
    }
    // 3. u = u* - dt / rho grad p
    double* Gp = ctx->pj_gradp.ensure<double>(n * KB + 1);
    wls_fields(ctx, d_pressure, 1, Gp, neumann);
    if (n) {
        k_correct<<<grid_n(n), 256, 0, s>>>(n, ctx->type_in.get<uint8_t>(), d_vel, Gp, dt / rho, d_vel_out);
        LSMPS_CHECK_LAUNCH();
    }
    // 4. div u
    wls_fields(ctx, d_vel_out, 3, G, neumann);
    if (n) {
        k_divergence<<<grid_n(n), 256, 0, s>>>(n, G, mask, nullptr, stats + 16);
        LSMPS_CHECK_LAUNCH();
    }
    ev_record(ctx, 13);
    double h[32];
    LSMPS_CUDA(cudaMemcpyAsync(h, stats, sizeof(h), cudaMemcpyDeviceToHost, s));
    LSMPS_CUDA(cudaStreamSynchronize(s));
    const double cnt = std::max(h[2], 1.0), ccnt = std::max(h[4], 1.0);
    const double w1 = std::max(h[6], 1.0), w2 = std::max(h[8], 1.0);
    st.unknowns = (uint64_t)U;
    st.measured = (uint64_t)h[2];
    st.div_before_rms = std::sqrt(h[0] / cnt);
    st.div_before_max = h[1];
    st.div_after_rms = std::sqrt(h[16] / cnt);
    st.div_after_max = h[17];
    st.core = (uint64_t)h[4];
    st.div_core_before_rms = std::sqrt(h[3] / ccnt);
    st.div_core_after_rms = std::sqrt(h[19] / ccnt);
    st.wall_band1 = (uint64_t)h[6];
    st.wall_band2 = (uint64_t)h[8];
    st.div_wall1_before_rms = std::sqrt(h[5] / w1);
    st.div_wall1_after_rms = std::sqrt(h[21] / w1);
    st.div_wall2_before_rms = std::sqrt(h[7] / w2);
    st.div_wall2_after_rms = std::sqrt(h[23] / w2);
    st.iterations = ps.iterations;
    st.converged = ps.converged;
    st.relative_residual = ps.relative_residual;
    st.solve_ms = ps.solve_ms;
    st.total_ms = ev_elapsed(ctx, 12, 13);
    if (out) *out = st;
}

}  // namespace lsmps_gpu
