// FP64 CUDA-core peak of this GPU, measured: the roofline denominator of the FP64-bound
// kernels (the all-particle WLS moments and Cholesky solves), which have no tensor-core form.
// Each thread runs FP64_CHAINS independent FMA chains (enough to cover the pipe latency) for
// `iters` steps; the result is written only if it is the (never reached) sentinel, so the
// compiler keeps every FMA.
#include "ops.cuh"

namespace lsmps_gpu {
namespace {

constexpr int FP64_CHAINS = 8;
constexpr int FP64_THREADS = 256;

__global__ void __launch_bounds__(FP64_THREADS) k_fp64_fma(int iters, double a, double b, double* sink) {
    double x[FP64_CHAINS];
#pragma unroll
    for (int c = 0; c < FP64_CHAINS; ++c) x[c] = (double)(threadIdx.x + c);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < FP64_CHAINS; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0;
#pragma unroll
    for (int c = 0; c < FP64_CHAINS; ++c) s += x[c];
    if (s == -12345.6789) sink[blockIdx.x] = s;
}

}  // namespace

// FLOPs per launch in *flops (2 per FMA).
void fp64_peak_bench(lsmps_ctx* ctx, int reps, double* ms, double* flops) {
    int sms = 0;
    LSMPS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const int blocks = sms * 8, iters = 4096;
    double* sink = ctx->scratch.ensure<double>(blocks + 1);
    // a = 1 - 2^-30, b = 2^-30: the chains stay finite and bounded
    const double a = 1.0 - 9.313225746154785e-10, b = 9.313225746154785e-10;
    k_fp64_fma<<<blocks, FP64_THREADS, 0, ctx->stream>>>(iters, a, b, sink);
    LSMPS_CHECK_LAUNCH();
    ev_record(ctx, 14);
    for (int r = 0; r < reps; ++r) k_fp64_fma<<<blocks, FP64_THREADS, 0, ctx->stream>>>(iters, a, b, sink);
    LSMPS_CHECK_LAUNCH();
    ev_record(ctx, 15);
    *ms = ev_elapsed(ctx, 14, 15) / reps;
    *flops = 2.0 * FP64_CHAINS * (double)iters * (double)blocks * FP64_THREADS;
}

}  // namespace lsmps_gpu
