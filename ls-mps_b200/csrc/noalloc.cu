// PPE residual check that allocates nothing: ||b - A p_v|| for up to eight caller-owned
// device vectors p_v (reference numbering) over the assembled system, with the reduction's
// partial sums and ticket in a fixed static device array instead of context buffers.
//
// Callers this is for: a simulation that keeps the pressure in its own device buffer and
// checks it inside its time loop while it overlaps other work on other streams. There the
// library must not grow a buffer (cudaMalloc / cudaFree synchronise the device and would
// stall that overlap) and the device memory may already be handed to the caller's own pool.
// The residual the solver reports goes through a U-sized temporary and the lazily built
// SELL copy of A; this variant reads the CSR the assembly left and keeps nothing but
// partial sums.
#include <algorithm>
#include <climits>

#include "ops.cuh"

namespace lsmps_gpu {
namespace {

constexpr int NA_THREADS = 256;
constexpr int NA_GRID = 148 * 4;  // at most this many blocks: one partial sum per block
constexpr int NA_MAX_VEC = 8;     // vectors per call
constexpr int NA_SLOTS = NA_MAX_VEC + 1;  // |r_v|^2 for each vector, then |b|^2
constexpr int NA_TICKET = NA_SLOTS * NA_GRID;  // double offset of the ticket word
constexpr int NA_DOUBLES = NA_TICKET + 32;     // 42,880 bytes

// Slot s of block k at [s * NA_GRID + k]; the ticket (an unsigned int) at [NA_TICKET]. The
// ticket must be zero when a launch starts: the host clears it before every launch and the
// last block clears it again. The partial sums need no initial value.
static __device__ __align__(256) double g_residual_scratch[NA_DOUBLES];

// Device address of the scratch on the current device (`device`), resolved on every call:
// the lookup allocates nothing, and a cached address would go stale after a device reset or
// a re-created primary context. The first lookup on a device may load this module onto it.
double* scratch_address(int device) {
    LSMPS_REQUIRE(device >= 0, LSMPS_ERR_ARG, "negative device ordinal");
    void* p = nullptr;
    LSMPS_CUDA(cudaGetSymbolAddress(&p, g_residual_scratch));
    return static_cast<double*>(p);
}

// One warp per row (grid-stride); lane 0 accumulates (b_i - (A p_v)_i)^2 and b_i^2, the
// block's sums go to the scratch and the last block to arrive adds them in block order.
__global__ void __launch_bounds__(NA_THREADS) k_residual_static(long long U, const int* __restrict__ row,
                                                                const int* __restrict__ col,
                                                                const double* __restrict__ val,
                                                                const double* __restrict__ b,
                                                                const int* __restrict__ ref_of_u,
                                                                const double* __restrict__ p, long long ld,
                                                                int nvec, double* scratch, double* out) {
    __shared__ double red[NA_THREADS / 32][NA_SLOTS];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double acc[NA_SLOTS];
#pragma unroll
    for (int v = 0; v < NA_SLOTS; ++v) acc[v] = 0.0;
    const long long nw = (long long)gridDim.x * (NA_THREADS / 32);
    for (long long i = (long long)blockIdx.x * (NA_THREADS / 32) + warp; i < U; i += nw) {
        double ax[NA_MAX_VEC];
#pragma unroll
        for (int v = 0; v < NA_MAX_VEC; ++v) ax[v] = 0.0;
        for (int e = row[i] + lane; e < row[i + 1]; e += 32) {
            const double a = val[e];
            const long long c = ref_of_u[col[e]];
#pragma unroll
            for (int v = 0; v < NA_MAX_VEC; ++v)
                if (v < nvec) ax[v] += a * p[v * ld + c];
        }
        const double bi = b[i];
#pragma unroll
        for (int v = 0; v < NA_MAX_VEC; ++v)
            if (v < nvec) {
                const double ri = bi - warp_sum(ax[v]);
                acc[v] += ri * ri;
            }
        acc[NA_MAX_VEC] += bi * bi;
    }
    if (lane == 0)
#pragma unroll
        for (int v = 0; v < NA_SLOTS; ++v) red[warp][v] = acc[v];
    __syncthreads();
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch + NA_TICKET);
    if (threadIdx.x < NA_SLOTS) {
        double t = 0.0;
        for (int w = 0; w < NA_THREADS / 32; ++w) t += red[w][threadIdx.x];
        scratch[threadIdx.x * NA_GRID + blockIdx.x] = t;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // fixed-order sum: thread t adds blocks t, t + 256, ...; then warps; then thread 0
    __shared__ double wsum[NA_THREADS / 32];
    for (int s = 0; s < NA_SLOTS; ++s) {
        if (s >= nvec && s < NA_MAX_VEC) continue;
        double t = 0.0;
        for (int k = threadIdx.x; k < (int)gridDim.x; k += NA_THREADS) t += __ldcg(scratch + s * NA_GRID + k);
        t = warp_sum(t);
        if (lane == 0) wsum[warp] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int w = 0; w < NA_THREADS / 32; ++w) tot += wsum[w];
            out[s < NA_MAX_VEC ? s : nvec] = sqrt(tot);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

}  // namespace

void ppe_residual_static(lsmps_ctx* ctx, const double* d_p, size_t ld, int nvec, double* d_out) {
    LSMPS_REQUIRE(nvec >= 1 && nvec <= NA_MAX_VEC, LSMPS_ERR_ARG,
                  "nvec must be in [1, 8]: the static scratch (42,880 bytes per device) holds partial sums "
                  "for at most 8 vectors");
    LSMPS_REQUIRE(ctx->have_ppe, LSMPS_ERR_STATE, "residual check needs lsmps_ppe_assemble first");
    LSMPS_REQUIRE(d_p && d_out, LSMPS_ERR_ARG, "null vector or output pointer");
    const long long U = ctx->U;
    LSMPS_REQUIRE(nvec == 1 || ld >= (size_t)U, LSMPS_ERR_ARG, "ld must be at least the number of unknowns");
    LSMPS_REQUIRE(ld <= (size_t)LLONG_MAX / NA_MAX_VEC, LSMPS_ERR_ARG, "ld too large");
    cudaStream_t s = ctx->stream;
    double* scratch = scratch_address(ctx->device);
    LSMPS_CUDA(cudaMemsetAsync(scratch + NA_TICKET, 0, sizeof(unsigned), s));
    if (U == 0) {
        LSMPS_CUDA(cudaMemsetAsync(d_out, 0, (nvec + 1) * sizeof(double), s));
        return;
    }
    const unsigned grid = (unsigned)std::min<long long>(NA_GRID, (U + NA_THREADS / 32 - 1) / (NA_THREADS / 32));
    k_residual_static<<<grid, NA_THREADS, 0, s>>>(U, ctx->A_row.get<int>(), ctx->A_col.get<int>(),
                                                  ctx->A_val.get<double>(), ctx->A_b.get<double>(),
                                                  ctx->ref_of_u.get<int>(), d_p, (long long)ld, nvec, scratch,
                                                  d_out);
    LSMPS_CHECK_LAUNCH();
}

}  // namespace lsmps_gpu
