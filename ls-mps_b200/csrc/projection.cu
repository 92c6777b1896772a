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

// hop[k] (sorted order) = HOP_FAR for Interior unknowns, 0 for every other particle (boundary:
// free surface, splash, wall, near-wall); then three passes of hop = min(hop, 1 + min over
// neighbors) (hop counts up to 3 are exact)
constexpr uint8_t HOP_FAR = 255;
__global__ void k_hop_init(long long U, const int* __restrict__ sorted_of_u, size_t n, uint8_t* __restrict__ hop) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
        hop[k] = 0;
}
__global__ void k_hop_mark(long long U, const int* __restrict__ sorted_of_u, const uint8_t* __restrict__ cls,
                           uint8_t* __restrict__ hop) {
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < U; u += (long long)gridDim.x * blockDim.x) {
        const int k = sorted_of_u[u];
        if (cls[k] == LSMPS_INTERIOR) hop[k] = HOP_FAR;
    }
}
__global__ void k_hop_pass(size_t n, const int* __restrict__ row, const int* __restrict__ col,
                           const uint8_t* __restrict__ in, uint8_t* __restrict__ out) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        int h = in[k];
        for (int e = row[k]; e < row[k + 1] && h > 0; ++e) h = min(h, in[col[e]] + 1);
        out[k] = (uint8_t)h;
    }
}
// mask[i] (caller order): bit 0 unknown, bit 1 core (at least three hops from a non-unknown)
__global__ void k_core_mask(size_t n, const int* __restrict__ iperm, const uint8_t* __restrict__ hop,
                            uint8_t* __restrict__ mask) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (mask[i] && hop[iperm[i]] >= 3) mask[i] |= 2;
}

// div[i] = d u_x / dx + d u_y / dy + d u_z / dz from the WLS solutions of the three fields;
// stats: [0] sum div^2, [1] max |div| (bits), [2] count over the unknowns, [3] sum div^2 over
// the core, [4] count over the core
__global__ void k_divergence(size_t n, const double* __restrict__ G, const uint8_t* __restrict__ mask,
                             double* __restrict__ div, double* stats) {
    double s2 = 0, mx = 0, cnt = 0, c2 = 0, ccnt = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double* g = G + i * 3 * KB;
        const double d = g[0] + g[KB + 1] + g[2 * KB + 2];
        if (div) div[i] = d;
        if (mask[i] & 1) {
            s2 += d * d;
            mx = fmax(mx, fabs(d));
            cnt += 1;
        }
        if (mask[i] & 2) {
            c2 += d * d;
            ccnt += 1;
        }
    }
    s2 = warp_sum(s2);
    cnt = warp_sum(cnt);
    c2 = warp_sum(c2);
    ccnt = warp_sum(ccnt);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&stats[0], s2);
        atomicAdd(&stats[2], cnt);
        atomicAdd(&stats[3], c2);
        atomicAdd(&stats[4], ccnt);
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

unsigned grid_n(size_t n) { return std::max(1u, std::min<unsigned>(blocks_for(n, 256), 148 * 8)); }

}  // namespace

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
    double* stats = ctx->pj_stats.ensure<double>(16);
    const long long U = ctx->U;
    LSMPS_CUDA(cudaMemsetAsync(mask, 0, n + 1, s));
    LSMPS_CUDA(cudaMemsetAsync(stats, 0, 16 * sizeof(double), s));
    if (U) {
        k_unknown_mask<<<1184, 256, 0, s>>>(U, ctx->sorted_of_u.get<int>(), ctx->perm.get<int>(), mask);
        uint8_t* hop = ctx->pj_hop.ensure<uint8_t>(2 * n + 2);
        uint8_t* hop2 = hop + n + 1;
        k_hop_init<<<grid_n(n), 256, 0, s>>>(U, ctx->sorted_of_u.get<int>(), n, hop);
        k_hop_mark<<<1184, 256, 0, s>>>(U, ctx->sorted_of_u.get<int>(), ctx->cls.get<uint8_t>(), hop);
        for (int pass = 0; pass < 3; ++pass) {
            k_hop_pass<<<grid_n(n), 256, 0, s>>>(n, ctx->nbr_row.get<int>(), ctx->nbr_col.get<int>(),
                                                 pass % 2 ? hop2 : hop, pass % 2 ? hop : hop2);
        }
        k_core_mask<<<grid_n(n), 256, 0, s>>>(n, ctx->iperm.get<int>(), hop2, mask);
        note_launches(6);
        LSMPS_CHECK_LAUNCH();
    }
    // 1. div u*
    wls_fields(ctx, d_vel, 3, G);
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
    wls_fields(ctx, d_pressure, 1, Gp);
    if (n) {
        k_correct<<<grid_n(n), 256, 0, s>>>(n, ctx->type_in.get<uint8_t>(), d_vel, Gp, dt / rho, d_vel_out);
        LSMPS_CHECK_LAUNCH();
    }
    // 4. div u
    wls_fields(ctx, d_vel_out, 3, G);
    if (n) {
        k_divergence<<<grid_n(n), 256, 0, s>>>(n, G, mask, nullptr, stats + 8);
        LSMPS_CHECK_LAUNCH();
    }
    ev_record(ctx, 13);
    double h[16];
    LSMPS_CUDA(cudaMemcpyAsync(h, stats, sizeof(h), cudaMemcpyDeviceToHost, s));
    LSMPS_CUDA(cudaStreamSynchronize(s));
    const double cnt = std::max(h[2], 1.0), ccnt = std::max(h[4], 1.0);
    st.unknowns = (uint64_t)U;
    st.measured = (uint64_t)h[2];
    st.div_before_rms = std::sqrt(h[0] / cnt);
    st.div_before_max = h[1];
    st.div_after_rms = std::sqrt(h[8] / cnt);
    st.div_after_max = h[9];
    st.core = (uint64_t)h[4];
    st.div_core_before_rms = std::sqrt(h[3] / ccnt);
    st.div_core_after_rms = std::sqrt(h[11] / ccnt);
    st.iterations = ps.iterations;
    st.converged = ps.converged;
    st.relative_residual = ps.relative_residual;
    st.solve_ms = ps.solve_ms;
    st.total_ms = ev_elapsed(ctx, 12, 13);
    if (out) *out = st;
}

}  // namespace lsmps_gpu
