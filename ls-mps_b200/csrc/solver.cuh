// BiCGStab engine shared by the FP64, Jacobi, mixed-precision and learned solvers.
#pragma once
#include "ctx.cuh"

namespace lsmps_gpu {

// Scalars of one BiCGStab run, resident in device memory and updated by the last block of
// each reduction kernel, so the iteration runs without host round trips.
struct BcgScalars {
    double rho, rho0, alpha, omega, beta;
    double thresh;        // converged when |s| or |r| <= thresh
    double sn, rn;        // last |s| and |r|
    double tt;
    double best_rn;       // smallest |r| seen (stall detection)
    double bnorm;         // |b| of the run (set by the init kernel)
    int done;             // 0 running, 1 converged, 2 breakdown, 3 iteration cap, 4 stalled
    int s_conv;           // |s| test passed this iteration
    int iters;            // completed iterations (reference bookkeeping)
    int it;               // iteration counter
    int max_iter;
    int stall_window, since_best;
    int nonfinite;
    unsigned int counter[8];  // last-block tickets of the reduction kernels
};

// A SELL-32x4 matrix view in the solver's numbering: rows in slices of 32, slice s holding
// slen[s] (a multiple of 4) entries per row from sptr[s], in chunks of four consecutive
// entries per row (entry k of row 32 s + l at sptr[s] + 128 (k / 4) + 4 l + k % 4),
// zero-padded to its longest row. Every row's columns ascend (the diagonal in place). With
// dcol set, the columns are stored as 16-bit steps: column k = rbase[row] + dcol[0] + ... +
// dcol[k] (dcol of the first entry and of padding entries is 0), and col is not read.
template <class T>
struct Sell {
    long long n;
    long long nslices;
    const int* sptr;
    const int* slen;
    const int* col;
    const T* val;
    const unsigned short* dcol = nullptr;
    const int* rbase = nullptr;
};

// The assembled system's SELL copy with FP64 values of A (built on first use).
Sell<double> sell_a64_view(lsmps_ctx* ctx);
// The SELL copy of A D^-1 with FP32 values (built with the structure).
Sell<float> sell_scaled32_view(lsmps_ctx* ctx);

// The multigrid's level-1 aggregates (contiguous row ranges ustart[I] .. ustart[I+1], and each
// row's aggregate agg0[i]) and its level-1 right-hand side, for solver kernels that restrict a
// vector while producing it.
struct MgFine {
    long long n1;
    const int* ustart;
    const int* agg0;
    float* r1;
};
MgFine mg_fine(lsmps_ctx* ctx);

}  // namespace lsmps_gpu
