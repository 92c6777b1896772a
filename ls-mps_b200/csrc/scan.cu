// Exclusive scans: tiles of 4096 items per 1024-thread block (4 per thread).
#include <climits>

#include "scan.cuh"

namespace lsmps_gpu {
namespace {

constexpr int SCAN_THREADS = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;

// Block-wide inclusive scan of one long long per thread; returns the inclusive value and
// the block total in *total.
__device__ long long block_inclusive_scan(long long v, long long* total) {
    __shared__ long long warp_tot[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        long long t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) warp_tot[warp] = v;
    __syncthreads();
    if (warp == 0) {
        int nw = blockDim.x >> 5;
        long long w = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            long long t = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += t;
        }
        if (lane < nw) warp_tot[lane] = w;
    }
    __syncthreads();
    if (warp > 0) v += warp_tot[warp - 1];
    *total = warp_tot[(blockDim.x >> 5) - 1];
    __syncthreads();
    return v;
}

template <class InT>
__global__ void __launch_bounds__(SCAN_THREADS) k_tile_sums(const InT* __restrict__ in, long long n,
                                                            long long* __restrict__ tile_sum) {
    long long base = (long long)blockIdx.x * SCAN_TILE;
    long long s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        long long i = base + (long long)k * SCAN_THREADS + threadIdx.x;
        if (i < n) s += (long long)in[i];
    }
    s = warp_sum(s);
    __shared__ long long ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        long long v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0;
        v = warp_sum(v);
        if (threadIdx.x == 0) tile_sum[blockIdx.x] = v;
    }
}

// One block: exclusive scan of the tile sums in place; tile_sum[ntiles] = total.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(long long* tile_sum, long long ntiles) {
    long long per = (ntiles + SCAN_THREADS - 1) / SCAN_THREADS;
    long long lo = (long long)threadIdx.x * per, hi = min(lo + per, ntiles);
    long long s = 0;
    for (long long i = lo; i < hi; ++i) s += tile_sum[i];
    long long tot;
    long long inc = block_inclusive_scan(s, &tot);
    long long run = inc - s;
    for (long long i = lo; i < hi; ++i) {
        long long v = tile_sum[i];
        tile_sum[i] = run;
        run += v;
    }
    if (threadIdx.x == 0) tile_sum[ntiles] = tot;
}

template <class InT>
__global__ void __launch_bounds__(SCAN_THREADS) k_downsweep(const InT* in, int* out, long long n,
                                                            const long long* __restrict__ tile_sum,
                                                            long long ntiles, int* dflag) {
    long long base = (long long)blockIdx.x * SCAN_TILE + (long long)threadIdx.x * SCAN_ITEMS;
    long long v[SCAN_ITEMS];
    long long s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        long long i = base + k;
        v[k] = i < n ? (long long)in[i] : 0;
        s += v[k];
    }
    long long tot;
    long long inc = block_inclusive_scan(s, &tot);
    long long run = tile_sum[blockIdx.x] + inc - s;
    bool over = false;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        long long i = base + k;
        if (i < n) {
            over |= run > INT_MAX;
            out[i] = (int)run;
        }
        run += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        long long total = tile_sum[ntiles];
        if (total > INT_MAX) over = true;
        out[n] = (int)total;
    }
    if (over) atomicOr(dflag, DFLAG_INDEX);
}

}  // namespace

template <class InT>
void scan_exclusive(const InT* in, int* out, long long n, cudaStream_t s, DevBuf& tmp, int* dflag) {
    long long ntiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (ntiles == 0) ntiles = 1;
    long long* ts = tmp.ensure<long long>(ntiles + 1);
    k_tile_sums<InT><<<(unsigned)ntiles, SCAN_THREADS, 0, s>>>(in, n, ts);
    LSMPS_CHECK_LAUNCH();
    k_scan_tiles<<<1, SCAN_THREADS, 0, s>>>(ts, ntiles);
    LSMPS_CHECK_LAUNCH();
    k_downsweep<InT><<<(unsigned)ntiles, SCAN_THREADS, 0, s>>>(in, out, n, ts, ntiles, dflag);
    LSMPS_CHECK_LAUNCH();
}

template void scan_exclusive<int>(const int*, int*, long long, cudaStream_t, DevBuf&, int*);
template void scan_exclusive<uint8_t>(const uint8_t*, int*, long long, cudaStream_t, DevBuf&, int*);

namespace {
__global__ void k_reduce_i32(const int* __restrict__ in, long long n, long long* out) {
    long long s = 0;
    for (long long i = threadIdx.x; i < n; i += blockDim.x) s += in[i];
    s = warp_sum(s);
    __shared__ long long ws[32];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        long long v = threadIdx.x < (blockDim.x >> 5) ? ws[threadIdx.x] : 0;
        v = warp_sum(v);
        if (threadIdx.x == 0) *out = v;
    }
}
}  // namespace

void reduce_sum_i32(const int* in, long long n, long long* out, cudaStream_t s) {
    k_reduce_i32<<<1, 1024, 0, s>>>(in, n, out);
    LSMPS_CHECK_LAUNCH();
}

}  // namespace lsmps_gpu
