// Launch-shape autotuner: picks, per context, kernel and problem-size class, the fastest of
// a kernel's launch shapes (grid size, block size, loads in flight) that all compute the same
// bits, by timing each candidate once on the live data.
#include <cmath>
#include <sstream>

#include "ops.cuh"

namespace lsmps_gpu {

int autotune(lsmps_ctx* ctx, const char* kernel, long long n, const std::vector<std::string>& names, int fallback,
             const std::function<void(int)>& launch, int reps) {
    Tuner& T = ctx->tuner;
    const int size_class = n > 0 ? 63 - __builtin_clzll((unsigned long long)n) : 0;
    const std::string key = std::string(kernel) + " n~2^" + std::to_string(size_class);
    auto it = T.table.find(key);
    if (it != T.table.end()) return it->second.best;
    if (!T.enabled || names.size() < 2 || n <= 0) return fallback;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    LSMPS_CUDA(cudaStreamIsCapturing(ctx->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return fallback;  // no timing inside a capture
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    LSMPS_CUDA(cudaEventCreate(&e0));
    cudaError_t err = cudaEventCreate(&e1);
    if (err != cudaSuccess) {
        cudaEventDestroy(e0);
        LSMPS_CUDA(err);
    }
    TuneResult R;
    R.names = names;
    R.ms.assign(names.size(), 0.f);
    try {
        for (size_t c = 0; c < names.size(); ++c) {
            launch((int)c);  // warm: instruction cache, L2 state of the inputs
            LSMPS_CUDA(cudaEventRecord(e0, ctx->stream));
            for (int r = 0; r < reps; ++r) launch((int)c);
            LSMPS_CUDA(cudaEventRecord(e1, ctx->stream));
            LSMPS_CUDA(cudaEventSynchronize(e1));
            float ms = 0;
            LSMPS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            R.ms[c] = ms / reps;
        }
    } catch (...) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    R.best = 0;
    for (size_t c = 1; c < names.size(); ++c)
        if (R.ms[c] < R.ms[R.best]) R.best = (int)c;
    T.table[key] = R;
    return R.best;
}

std::string autotune_report(lsmps_ctx* ctx) {
    std::ostringstream os;
    for (const auto& kv : ctx->tuner.table) {
        const TuneResult& R = kv.second;
        for (size_t c = 0; c < R.names.size(); ++c)
            os << kv.first << '\t' << R.names[c] << '\t' << R.ms[c] << ((int)c == R.best ? "\tbest" : "") << '\n';
    }
    return os.str();
}

}  // namespace lsmps_gpu
