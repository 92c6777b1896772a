// PPE solvers on sm_100a.
//
// * REFERENCE: the reference's unpreconditioned FP64 BiCGStab (src/lsmps.cpp:65-67)
//   reproduced bit for bit: exactly rounded FP64 vector updates in the reference's
//   expression order, row-sequential SpMV in stored entry order, and dot products summed
//   sequentially in the reference's unknown order by one thread (products formed in
//   parallel). Slow by design; it exists so small cases match the reference exactly.
// * FP64 / JACOBI: the same iteration with GPU reductions. Jacobi right preconditioning
//   is applied as a column scaling of the matrix (A D^-1, solve for y, x = D^-1 y), which
//   costs nothing per iteration.
// * MIXED / LEARNED: FP64 iterative refinement, r = b - A x with the FP64 matrix, around
//   FP32 Jacobi-BiCGStab inner solves of A D^-1 y = r / |r| on an FP32 copy of the matrix.
//   LEARNED starts each inner solve from the message-passing network's guess.
//
// The fast engine runs five kernels per iteration. Each reduction is fused into the
// kernel that produces its operands; the last block of the grid to finish (atomic ticket)
// sums the per-block partials in a fixed order, so results are deterministic, and updates
// the scalars in device memory. Every kernel returns at once when the run is done, so a
// CUDA graph of several iterations can be replayed without host round trips; the host
// reads the status once per graph launch.
#include <algorithm>
#include <cmath>
#include <climits>
#include <cstring>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "ops.cuh"
#include "scan.cuh"
#include "solver.cuh"

namespace lsmps_gpu {


namespace {

constexpr int RB = 256;            // threads per block
constexpr int RGRID = 148 * 6;     // persistent grid of the vector / SpMV kernels

// ---------------------------------------------------------------------------------------
// REFERENCE (bit-exact) solver
// ---------------------------------------------------------------------------------------
struct ExactState {
    double rho, rho0, alpha, omega, beta, bnorm, thresh, den, tt;
    int done;    // 1 converged, 2 break
    int s_conv;
    int iters;
    int it;
    int converged;
};

__global__ void k_x_prod(const double* __restrict__ a, const double* __restrict__ b,
                         const int* __restrict__ u_of_ref, long long U, double* __restrict__ prod,
                         const ExactState* st) {
    if (st->done) return;
    for (long long rr = blockIdx.x * (long long)blockDim.x + threadIdx.x; rr < U;
         rr += (long long)gridDim.x * blockDim.x) {
        int u = u_of_ref[rr];
        prod[rr] = xmul(a[u], b[u]);
    }
}

enum ExactOp { OP_BNORM, OP_RHO, OP_DEN, OP_SN, OP_TT, OP_TS, OP_RN };

// One thread: sequential sum (the reference's dot, src/lsmps.cpp:66) and the scalar step.
__global__ void k_x_tail(const double* __restrict__ prod, long long U, ExactState* st, int op, double tol,
                         int max_iter) {
    if (threadIdx.x || blockIdx.x) return;
    if (st->done) return;
    double s = 0;
    for (long long rr = 0; rr < U; ++rr) s = xadd(s, prod[rr]);
    switch (op) {
        case OP_BNORM:
            st->bnorm = __dsqrt_rn(s);
            st->thresh = xmul(tol, fmax(1.0, st->bnorm));
            st->rho0 = st->alpha = st->omega = 1.0;
            st->it = 0;
            st->iters = 0;
            if (max_iter <= 0) st->done = 2;
            break;
        case OP_RHO:
            st->rho = s;
            if (fabs(s) < 1e-30) { st->done = 2; break; }
            st->beta = xmul(xdiv(st->rho, st->rho0), xdiv(st->alpha, st->omega));
            break;
        case OP_DEN:
            if (fabs(s) < 1e-30) { st->done = 2; break; }
            st->alpha = xdiv(st->rho, s);
            break;
        case OP_SN:
            if (__dsqrt_rn(s) <= st->thresh) { st->s_conv = 1; st->iters = st->it + 1; st->converged = 1; }
            break;
        case OP_TT:
            st->tt = s;
            if (s < 1e-30) st->done = 2;
            break;
        case OP_TS:
            st->omega = xdiv(s, st->tt);
            break;
        case OP_RN:
            st->iters = st->it + 1;
            if (__dsqrt_rn(s) <= st->thresh) { st->converged = 1; st->done = 1; break; }
            if (fabs(st->omega) < 1e-30) { st->done = 2; break; }
            st->rho0 = st->rho;
            st->it += 1;
            if (st->it >= max_iter) st->done = 2;
            break;
    }
}

__global__ void k_x_spmv(long long U, const int* __restrict__ row, const int* __restrict__ col,
                         const double* __restrict__ val, const double* __restrict__ x, double* __restrict__ y,
                         const ExactState* st, int check) {
    if (check && st->done) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < U;
         i += (long long)gridDim.x * blockDim.x) {
        double s = 0;
        for (int e = row[i]; e < row[i + 1]; ++e) s = xadd(s, xmul(val[e], x[col[e]]));
        y[i] = s;
    }
}

// kind 0: p = r + beta (p - omega v); 1: s = r - alpha v; 2: x += alpha p (and finish when
// the |s| test passed); 3: x += alpha p + omega s, r = s - omega t.
__global__ void k_x_vec(long long U, int kind, double* __restrict__ x, double* __restrict__ r,
                        double* __restrict__ p, const double* __restrict__ v, double* __restrict__ s,
                        const double* __restrict__ t, ExactState* st) {
    if (st->done) return;
    if (kind == 2 && !st->s_conv) return;
    if (kind == 3 && st->s_conv) return;
    const double alpha = st->alpha, beta = st->beta, omega = st->omega;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < U;
         i += (long long)gridDim.x * blockDim.x) {
        if (kind == 0) p[i] = xadd(r[i], xmul(beta, xsub(p[i], xmul(omega, v[i]))));
        else if (kind == 1) s[i] = xsub(r[i], xmul(alpha, v[i]));
        else if (kind == 2) { x[i] = xadd(x[i], xmul(alpha, p[i])); r[i] = s[i]; }
        else {
            x[i] = xadd(x[i], xadd(xmul(alpha, p[i]), xmul(omega, s[i])));
            r[i] = xsub(s[i], xmul(omega, t[i]));
        }
    }
}

__global__ void k_x_finish_sconv(ExactState* st) {
    if (st->s_conv && !st->done) st->done = 1;
}

// Final statistics (src/lsmps.cpp:67 tail): sequential sums in reference order.
__global__ void k_x_final(const double* __restrict__ Ax, const double* __restrict__ b,
                          const double* __restrict__ x, const double* __restrict__ xe,
                          const int* __restrict__ u_of_ref, long long U, double* out) {
    if (threadIdx.x || blockIdx.x) return;
    double res = 0, se = 0, mx = 0, exn = 0;
    for (long long rr = 0; rr < U; ++rr) {
        int u = u_of_ref[rr];
        double d = xsub(Ax[u], b[u]);
        res = xadd(res, xmul(d, d));
        double e = xsub(x[u], xe[u]);
        se = xadd(se, xmul(e, e));
        exn = xadd(exn, xmul(xe[u], xe[u]));
        mx = fmax(mx, fabs(e));
    }
    out[0] = __dsqrt_rn(res);
    out[1] = __dsqrt_rn(xdiv(se, fmax(exn, 1e-30)));
    out[2] = mx;
}

// ---------------------------------------------------------------------------------------
// Fast engine
// ---------------------------------------------------------------------------------------
struct Partials {
    double* a;   // RGRID entries
    double* b;   // RGRID entries
};

// Block sum of two doubles into partials[blockIdx]; returns true in the last block to
// arrive, after which the caller may read all partials (fixed-order final sum).
__device__ __forceinline__ bool block_partials(double va, double vb, Partials P, unsigned int* counter) {
    __shared__ double sa[RB / 32], sb[RB / 32];
    __shared__ bool last;
    va = warp_sum(va);
    vb = warp_sum(vb);
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { sa[w] = va; sb[w] = vb; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0, tb = 0;
        for (int k = 0; k < RB / 32; ++k) { ta += sa[k]; tb += sb[k]; }
        P.a[blockIdx.x] = ta;
        P.b[blockIdx.x] = tb;
        __threadfence();
        unsigned int ticket = atomicAdd(counter, 1u);
        last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    return last;
}

// In the last block: fixed-order sum of the partials (thread t sums entries t, t+RB, ...
// then a fixed tree), result in *ra / *rb for thread 0.
__device__ __forceinline__ void final_sum(Partials P, double* ra, double* rb) {
    __shared__ double sa[RB / 32], sb[RB / 32];
    double va = 0, vb = 0;
    for (int k = threadIdx.x; k < (int)gridDim.x; k += RB) {
        va += __ldcg(P.a + k);
        vb += __ldcg(P.b + k);
    }
    va = warp_sum(va);
    vb = warp_sum(vb);
    if ((threadIdx.x & 31) == 0) { sa[threadIdx.x >> 5] = va; sb[threadIdx.x >> 5] = vb; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0, tb = 0;
        for (int k = 0; k < RB / 32; ++k) { ta += sa[k]; tb += sb[k]; }
        *ra = ta;
        *rb = tb;
    }
}

// Row i of a SELL-32x4 matrix: slice s = i / 32 stores its 32 rows in chunks of four
// consecutive entries per row (entries 4c..4c+3 of lane l at sptr[s] + 128 c + 4 l), zero-
// padded to the slice's longest row rounded up to a multiple of four. One thread per row,
// one warp per slice: each thread reads its next four values and four columns with two
// 16-byte loads (a warp covers 512 contiguous bytes per load), and two chunks are issued
// before their eight x gathers, so each thread keeps 64-96 bytes of matrix loads and eight
// gathers in flight. Matrix loads stream past L1/L2 (__ldcs) so the vectors, re-read every
// iteration, stay in the 126 MB L2.
__device__ __forceinline__ void ld4(const float* p, float v[4]) {
    float4 q = __ldcs(reinterpret_cast<const float4*>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
__device__ __forceinline__ void ld4(const double* p, double v[4]) {
    double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void ld4(const int* p, int v[4]) {
    int4 q = __ldcs(reinterpret_cast<const int4*>(p));
    v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
}
// four 16-bit column steps (8 bytes) -> four columns continuing from c
__device__ __forceinline__ void ld4_steps(const unsigned short* p, int& c, int out[4]) {
    uint2 q = __ldcs(reinterpret_cast<const uint2*>(p));
    c += (int)(q.x & 0xffffu);
    out[0] = c;
    c += (int)(q.x >> 16);
    out[1] = c;
    c += (int)(q.y & 0xffffu);
    out[2] = c;
    c += (int)(q.y >> 16);
    out[3] = c;
}

// The row product with 16-bit column steps (2 bytes per entry instead of 4).
template <class TM, class T>
__device__ __forceinline__ double sell_row16(const Sell<TM>& A, long long s, int lane, const T* __restrict__ x) {
    const long long base = (long long)A.sptr[s] + 4 * lane;
    const TM* __restrict__ val = A.val + base;
    const unsigned short* __restrict__ dc = A.dcol + base;
    int cur = A.rbase[(s << 5) + lane];
    const int chunks = A.slen[s] >> 2;
    double a0 = 0, a1 = 0;
    int c = 0;
    for (; c + 2 <= chunks; c += 2) {
        TM v0[4], v1[4];
        int c0[4], c1[4];
        ld4(val + 128 * c, v0);
        ld4(val + 128 * (c + 1), v1);
        ld4_steps(dc + 128 * c, cur, c0);
        ld4_steps(dc + 128 * (c + 1), cur, c1);
        T x0[4], x1[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            x0[j] = x[c0[j]];
            x1[j] = x[c1[j]];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            a0 += (double)v0[j] * (double)x0[j];
            a1 += (double)v1[j] * (double)x1[j];
        }
    }
    if (c < chunks) {
        TM v0[4];
        int c0[4];
        ld4(val + 128 * c, v0);
        ld4_steps(dc + 128 * c, cur, c0);
#pragma unroll
        for (int j = 0; j < 4; ++j) a0 += (double)v0[j] * (double)x[c0[j]];
    }
    return a0 + a1;
}

// The same row product, software-pipelined: the next pair of chunks' values and column steps
// are loaded while the current pair's gathers are in flight, so a pair of chunks waits for one
// round trip instead of two. The sums are added in the same order as sell_row16 (same bits);
// it needs ~64 registers, so its kernels run 4 blocks of RB threads per SM instead of 6.
__device__ __forceinline__ void steps_to_cols(uint2 q, int& c, int out[4]) {
    c += (int)(q.x & 0xffffu);
    out[0] = c;
    c += (int)(q.x >> 16);
    out[1] = c;
    c += (int)(q.y & 0xffffu);
    out[2] = c;
    c += (int)(q.y >> 16);
    out[3] = c;
}
template <class TM, class T>
__device__ __forceinline__ double sell_row16_pipe(const Sell<TM>& A, long long s, int lane,
                                                  const T* __restrict__ x) {
    const long long base = (long long)A.sptr[s] + 4 * lane;
    const TM* __restrict__ val = A.val + base;
    const unsigned short* __restrict__ dc = A.dcol + base;
    int cur = A.rbase[(s << 5) + lane];
    const int chunks = A.slen[s] >> 2;
    double a0 = 0, a1 = 0;
    int c = 0;
    TM v0[4], v1[4];
    uint2 s0 = make_uint2(0, 0), s1 = make_uint2(0, 0);
    if (chunks >= 2) {
        ld4(val, v0);
        ld4(val + 128, v1);
        s0 = __ldcs(reinterpret_cast<const uint2*>(dc));
        s1 = __ldcs(reinterpret_cast<const uint2*>(dc + 128));
    }
    for (; c + 2 <= chunks; c += 2) {
        int c0[4], c1[4];
        steps_to_cols(s0, cur, c0);
        steps_to_cols(s1, cur, c1);
        T x0[4], x1[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            x0[j] = x[c0[j]];
            x1[j] = x[c1[j]];
        }
        if (c + 4 <= chunks) {  // the next pair, in flight with the gathers above
            TM w0[4], w1[4];
            ld4(val + 128 * (c + 2), w0);
            ld4(val + 128 * (c + 3), w1);
            const uint2 t0 = __ldcs(reinterpret_cast<const uint2*>(dc + 128 * (c + 2)));
            const uint2 t1 = __ldcs(reinterpret_cast<const uint2*>(dc + 128 * (c + 3)));
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                a0 += (double)v0[j] * (double)x0[j];
                a1 += (double)v1[j] * (double)x1[j];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                v0[j] = w0[j];
                v1[j] = w1[j];
            }
            s0 = t0;
            s1 = t1;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                a0 += (double)v0[j] * (double)x0[j];
                a1 += (double)v1[j] * (double)x1[j];
            }
        }
    }
    if (c < chunks) {
        TM u0[4];
        int c0[4];
        ld4(val + 128 * c, u0);
        ld4_steps(dc + 128 * c, cur, c0);
#pragma unroll
        for (int j = 0; j < 4; ++j) a0 += (double)u0[j] * (double)x[c0[j]];
    }
    return a0 + a1;
}

// The solver SpMVs with FP32 values and 16-bit steps use the pipelined product.
template <class TM, bool C16>
constexpr bool sell_pipe() {
    return C16 && sizeof(TM) == 4;
}
template <class TM, bool C16>
constexpr int spmv_blocks_per_sm() {
    return sell_pipe<TM, C16>() ? 4 : 6;
}
template <class TM, bool C16>
constexpr unsigned spmv_grid() {
    return 148u * spmv_blocks_per_sm<TM, C16>();
}

// C16: the view's columns are 16-bit steps (a compile-time choice: one code path per kernel)
template <bool C16, class TM, class T>
__device__ __forceinline__ double sell_row(const Sell<TM>& A, long long s, int lane, const T* __restrict__ x) {
    if constexpr (C16) return sell_row16(A, s, lane, x);
    const long long base = (long long)A.sptr[s] + 4 * lane;
    const TM* __restrict__ val = A.val + base;
    const int* __restrict__ col = A.col + base;
    const int chunks = A.slen[s] >> 2;
    double a0 = 0, a1 = 0;
    int c = 0;
    for (; c + 2 <= chunks; c += 2) {
        TM v0[4], v1[4];
        int c0[4], c1[4];
        ld4(val + 128 * c, v0);
        ld4(col + 128 * c, c0);
        ld4(val + 128 * (c + 1), v1);
        ld4(col + 128 * (c + 1), c1);
        T x0[4], x1[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            x0[j] = x[c0[j]];
            x1[j] = x[c1[j]];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            a0 += (double)v0[j] * (double)x0[j];
            a1 += (double)v1[j] * (double)x1[j];
        }
    }
    if (c < chunks) {
        TM v0[4];
        int c0[4];
        ld4(val + 128 * c, v0);
        ld4(col + 128 * c, c0);
#pragma unroll
        for (int j = 0; j < 4; ++j) a0 += (double)v0[j] * (double)x[c0[j]];
    }
    return a0 + a1;
}

#define SELL_LOOP(A)                                                              \
    const int lane = threadIdx.x & 31;                                            \
    const long long w0 = (blockIdx.x * (long long)RB + threadIdx.x) >> 5;         \
    const long long nw = ((long long)gridDim.x * RB) >> 5;                        \
    for (long long s = w0; s < (A).nslices; s += nw)

// Four consecutive vector elements per thread and access (float4, or two double2), so
// the elementwise kernels keep 16-32 bytes per array in flight per thread.
template <class T>
struct V4 {
    T a[4];
};
__device__ __forceinline__ V4<float> ld_v4(const float* p) {
    float4 q = *reinterpret_cast<const float4*>(p);
    return {{q.x, q.y, q.z, q.w}};
}
__device__ __forceinline__ V4<double> ld_v4(const double* p) {
    double2 u = reinterpret_cast<const double2*>(p)[0], w = reinterpret_cast<const double2*>(p)[1];
    return {{u.x, u.y, w.x, w.y}};
}
__device__ __forceinline__ void st_v4(float* p, const V4<float>& v) {
    *reinterpret_cast<float4*>(p) = make_float4(v.a[0], v.a[1], v.a[2], v.a[3]);
}
__device__ __forceinline__ void st_v4(double* p, const V4<double>& v) {
    reinterpret_cast<double2*>(p)[0] = make_double2(v.a[0], v.a[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(v.a[2], v.a[3]);
}

// Calls f4(i) for i = 0, 4, 8, ... (groups of four elements), then f1(i) for the tail.
template <class F4, class F1>
__device__ __forceinline__ void vec_loop(long long n, F4&& f4, F1&& f1) {
    const long long n4 = n >> 2;
    for (long long q = blockIdx.x * (long long)RB + threadIdx.x; q < n4; q += (long long)gridDim.x * RB) f4(q << 2);
    for (long long i = (n4 << 2) + blockIdx.x * (long long)RB + threadIdx.x; i < n; i += (long long)gridDim.x * RB)
        f1(i);
}

// p = r + beta (p - omega v)
template <class T>
__global__ void __launch_bounds__(RB) k_bcg_p(long long n, const T* __restrict__ r, T* __restrict__ p,
                                              const T* __restrict__ v, const BcgScalars* S) {
    pdl_begin();
    if (S->done) return;
    const T beta = (T)S->beta, omega = (T)S->omega;
    vec_loop(n, [&](long long i) {
        V4<T> rr = ld_v4(r + i), pp = ld_v4(p + i), vv = ld_v4(v + i);
#pragma unroll
        for (int j = 0; j < 4; ++j) pp.a[j] = rr.a[j] + beta * (pp.a[j] - omega * vv.a[j]);
        st_v4(p + i, pp);
    }, [&](long long i) { p[i] = r[i] + beta * (p[i] - omega * v[i]); });
}

// v = A p; den = (r0, v); alpha = rho / den
template <class T, class TM = T, bool C16 = false>
__global__ void __launch_bounds__(RB, spmv_blocks_per_sm<TM, C16>()) k_bcg_v(Sell<TM> A, const T* __restrict__ p, T* __restrict__ v,
                                              const T* __restrict__ r0, BcgScalars* S, Partials P) {
    pdl_begin();
    if (S->done) return;
    double acc = 0;
    SELL_LOOP(A) {
        double y = sell_pipe<TM, C16>() ? sell_row16_pipe(A, s, lane, p) : sell_row<C16>(A, s, lane, p);
        long long i = (s << 5) + lane;
        if (i < A.n) {
            T yi = (T)y;
            v[i] = yi;
            acc += (double)r0[i] * (double)yi;
        }
    }
    if (block_partials(acc, 0.0, P, &S->counter[0])) {
        double den, unused;
        final_sum(P, &den, &unused);
        if (threadIdx.x == 0) {
            S->counter[0] = 0;
            if (!isfinite(den)) { S->nonfinite = 1; S->done = 2; }
            else if (fabs(den) < 1e-30) S->done = 2;
            else S->alpha = S->rho / den;
        }
    }
}

// s = r - alpha v; |s|
template <class T>
__global__ void __launch_bounds__(RB) k_bcg_s(long long n, const T* __restrict__ r, const T* __restrict__ v,
                                              T* __restrict__ s, BcgScalars* S, Partials P) {
    pdl_begin();
    if (S->done) return;
    const T alpha = (T)S->alpha;
    double acc = 0;
    vec_loop(n, [&](long long i) {
        V4<T> rr = ld_v4(r + i), vv = ld_v4(v + i), ss;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            ss.a[j] = rr.a[j] - alpha * vv.a[j];
            acc += (double)ss.a[j] * (double)ss.a[j];
        }
        st_v4(s + i, ss);
    }, [&](long long i) {
        T si = r[i] - alpha * v[i];
        s[i] = si;
        acc += (double)si * (double)si;
    });
    if (block_partials(acc, 0.0, P, &S->counter[1])) {
        double ss, unused;
        final_sum(P, &ss, &unused);
        if (threadIdx.x == 0) {
            S->counter[1] = 0;
            S->sn = sqrt(ss);
            if (S->sn <= S->thresh) { S->s_conv = 1; S->iters = S->it + 1; }
        }
    }
}

// With the multigrid, the p and s updates also restrict the new vector to level 1
// (r1 = P^T p, a sum over each aggregate's contiguous rows). A warp takes AGG_W consecutive
// aggregates, i.e. the rows ustart[Ia] .. ustart[Ia + AGG_W], and walks them 32 consecutive rows
// per step, so every load and store is coalesced. A segmented shuffle scan sums each step's
// rows per aggregate and the segment's last lane adds that sum into the aggregate's shared-
// memory slot; steps run in order, so the summation order is fixed.
constexpr int AGG_W = 16;  // aggregates per warp task

inline unsigned agg_blocks(long long n1) {
    return (unsigned)(((n1 + AGG_W - 1) / AGG_W + RB / 32 - 1) / (RB / 32));
}

// Calls f(i) (which returns the new value of row i) for every row of aggregates [Ia, Ib) and
// returns, in lane l < Ib - Ia, the sum over aggregate Ia + l. `sh` is the warp's AGG_W slots.
template <class F>
__device__ __forceinline__ double warp_agg_sums(const MgFine& G, long long Ia, long long Ib, double* sh, F&& f) {
    const int lane = threadIdx.x & 31;
    if (lane < AGG_W) sh[lane] = 0.0;
    __syncwarp();
    const int rb = G.ustart[Ia], re = G.ustart[Ib];
    // segment sums of one step: inclusive scan within runs of equal a, the run's last lane adds
    auto deliver = [&](double x, int a, bool live) {
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, x, o);
            const int ay = __shfl_up_sync(0xffffffffu, a, o);
            if (lane >= o && ay == a) x += y;
        }
        const int an = __shfl_down_sync(0xffffffffu, a, 1);
        if (live && (lane == 31 || an != a)) sh[a] += x;
        __syncwarp();
    };
    // two steps per pass: both steps' loads are in flight before either scan
    for (int base = rb; base < re; base += 64) {
        const int i0 = base + lane, i1 = base + 32 + lane;
        const bool l0 = i0 < re, l1 = i1 < re;
        int a0 = AGG_W + lane, a1 = AGG_W + lane;  // past the last row: a key of its own, in no run
        if (l0) a0 = G.agg0[i0] - (int)Ia;
        if (l1) a1 = G.agg0[i1] - (int)Ia;
        const double x0 = l0 ? f(i0) : 0.0;
        const double x1 = l1 ? f(i1) : 0.0;
        deliver(x0, a0, l0);
        deliver(x1, a1, l1);
    }
    const double sum = lane < AGG_W ? sh[lane] : 0.0;
    __syncwarp();  // before the next task clears the slots
    return sum;
}

__global__ void __launch_bounds__(RB) k_bcg_p_agg(MgFine G, const double* __restrict__ r, double* __restrict__ p,
                                                  const double* __restrict__ v, const BcgScalars* S) {
    pdl_begin();
    if (S->done) return;
    __shared__ double sh[RB / 32][AGG_W];
    const double beta = S->beta, omega = S->omega;
    const int lane = threadIdx.x & 31;
    const long long nt = (G.n1 + AGG_W - 1) / AGG_W;
    for (long long task = (blockIdx.x * (long long)RB + threadIdx.x) >> 5; task < nt;
         task += ((long long)gridDim.x * RB) >> 5) {
        const long long Ia = task * AGG_W, Ib = min(Ia + AGG_W, G.n1);
        const double a = warp_agg_sums(G, Ia, Ib, sh[threadIdx.x >> 5], [&](int i) {
            const double pi = r[i] + beta * (p[i] - omega * v[i]);
            p[i] = pi;
            return pi;
        });
        if (Ia + lane < Ib) G.r1[Ia + lane] = (float)a;
    }
}

// s = r - alpha v, |s|, and r1 = P^T s in one pass (grid at most RGRID blocks: one partial
// sum of |s|^2 per block).
__global__ void __launch_bounds__(RB) k_bcg_s_agg(MgFine G, const double* __restrict__ r,
                                                  const double* __restrict__ v, double* __restrict__ s,
                                                  BcgScalars* S, Partials P) {
    pdl_begin();
    if (S->done) return;
    __shared__ double sh[RB / 32][AGG_W];
    const double alpha = S->alpha;
    const int lane = threadIdx.x & 31;
    const long long nt = (G.n1 + AGG_W - 1) / AGG_W;
    double acc = 0;
    for (long long task = (blockIdx.x * (long long)RB + threadIdx.x) >> 5; task < nt;
         task += ((long long)gridDim.x * RB) >> 5) {
        const long long Ia = task * AGG_W, Ib = min(Ia + AGG_W, G.n1);
        const double a = warp_agg_sums(G, Ia, Ib, sh[threadIdx.x >> 5], [&](int i) {
            const double si = r[i] - alpha * v[i];
            s[i] = si;
            acc += si * si;
            return si;
        });
        if (Ia + lane < Ib) G.r1[Ia + lane] = (float)a;
    }
    if (block_partials(acc, 0.0, P, &S->counter[1])) {
        double ss, unused;
        final_sum(P, &ss, &unused);
        if (threadIdx.x == 0) {
            S->counter[1] = 0;
            S->sn = sqrt(ss);
            if (S->sn <= S->thresh) { S->s_conv = 1; S->iters = S->it + 1; }
        }
    }
}

// t = A sv; omega = (t, s) / (t, t), with sv = s, or the preconditioned M s when a
// preconditioner is applied (s then only enters the dot)
template <class T, class TM = T, bool C16 = false>
__global__ void __launch_bounds__(RB, spmv_blocks_per_sm<TM, C16>()) k_bcg_t(Sell<TM> A, const T* __restrict__ sv, T* __restrict__ t,
                                              BcgScalars* S, Partials P, const T* __restrict__ sd) {
    pdl_begin();
    if (S->done || S->s_conv) return;
    double ats = 0, att = 0;
    SELL_LOOP(A) {
        double y = sell_pipe<TM, C16>() ? sell_row16_pipe(A, s, lane, sv) : sell_row<C16>(A, s, lane, sv);
        long long i = (s << 5) + lane;
        if (i < A.n) {
            T ti = (T)y;
            t[i] = ti;
            ats += (double)ti * (double)sd[i];
            att += (double)ti * (double)ti;
        }
    }
    if (block_partials(ats, att, P, &S->counter[2])) {
        double ts, tt;
        final_sum(P, &ts, &tt);
        if (threadIdx.x == 0) {
            S->counter[2] = 0;
            S->tt = tt;
            if (!isfinite(tt) || !isfinite(ts)) { S->nonfinite = 1; S->done = 2; }
            else if (tt < 1e-30) S->done = 2;
            else S->omega = ts / tt;
        }
    }
}

// x += alpha p + omega s; r = s - omega t; |r|, rho' = (r0, r); beta
// (or, when the |s| test passed: x += alpha p and finish). PRE: the x update takes the
// preconditioned directions ph = M p and sh = M s instead of p and s.
template <class T, bool PRE = false>
__global__ void __launch_bounds__(RB) k_bcg_x(long long n, T* __restrict__ x, T* __restrict__ r,
                                              const T* __restrict__ p, const T* __restrict__ s,
                                              const T* __restrict__ t, const T* __restrict__ r0,
                                              BcgScalars* S, Partials P, const T* __restrict__ ph = nullptr,
                                              const T* __restrict__ sh = nullptr) {
    pdl_begin();
    if (S->done) return;
    const T alpha = (T)S->alpha, omega = (T)S->omega;
    const T* __restrict__ xp = PRE ? ph : p;
    const T* __restrict__ xs = PRE ? sh : s;
    if (S->s_conv) {
        for (long long i = blockIdx.x * (long long)RB + threadIdx.x; i < n; i += (long long)gridDim.x * RB) {
            x[i] += alpha * xp[i];
            r[i] = s[i];
        }
        __syncthreads();
        if (block_partials(0.0, 0.0, P, &S->counter[3]) && threadIdx.x == 0) {
            S->counter[3] = 0;
            S->rn = S->sn;
            S->done = 1;
        }
        return;
    }
    double arr = 0, ar0r = 0;
    vec_loop(n, [&](long long i) {
        V4<T> xx = ld_v4(x + i), pp = ld_v4(xp + i), ss = ld_v4(s + i), tt = ld_v4(t + i), q0 = ld_v4(r0 + i), rr;
        V4<T> xsv = PRE ? ld_v4(xs + i) : ss;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            xx.a[j] += alpha * pp.a[j] + omega * xsv.a[j];
            rr.a[j] = ss.a[j] - omega * tt.a[j];
            arr += (double)rr.a[j] * (double)rr.a[j];
            ar0r += (double)q0.a[j] * (double)rr.a[j];
        }
        st_v4(x + i, xx);
        st_v4(r + i, rr);
    }, [&](long long i) {
        T si = s[i];
        x[i] += alpha * xp[i] + omega * (PRE ? xs[i] : si);
        T ri = si - omega * t[i];
        r[i] = ri;
        arr += (double)ri * (double)ri;
        ar0r += (double)r0[i] * (double)ri;
    });
    if (block_partials(arr, ar0r, P, &S->counter[3])) {
        double rr, rho;
        final_sum(P, &rr, &rho);
        if (threadIdx.x == 0) {
            S->counter[3] = 0;
            S->iters = S->it + 1;
            S->it += 1;
            double rn = sqrt(rr);
            S->rn = rn;
            if (!isfinite(rn)) { S->nonfinite = 1; S->done = 2; return; }
            if (rn <= S->thresh) { S->done = 1; return; }
            // stall bookkeeping (learned solver fallback rule)
            if (rn < 0.99 * S->best_rn) { S->best_rn = rn; S->since_best = 0; }
            else if (++S->since_best >= S->stall_window && S->stall_window > 0) { S->done = 4; return; }
            if (fabs(S->omega) < 1e-30) { S->done = 2; return; }
            if (S->it >= S->max_iter) { S->done = 3; return; }
            if (fabs(rho) < 1e-30) { S->done = 2; return; }
            S->beta = (rho / S->rho) * (S->alpha / S->omega);
            S->rho0 = S->rho;
            S->rho = rho;
        }
    }
}

// Initialisation: r = b - A x (or r = b when x = 0), r0 = r, p = v = 0, |b|, rho = (r0, r).
template <class T, class TM = T, bool C16 = false>
__global__ void __launch_bounds__(RB, 6) k_bcg_init(Sell<TM> A, const T* __restrict__ b, const T* __restrict__ x,
                                                 int use_x, T* __restrict__ r, T* __restrict__ r0,
                                                 T* __restrict__ p, T* __restrict__ v, BcgScalars* S,
                                                 Partials P, double tol, double bnorm_override,
                                                 const int* gate = nullptr, int want = 0) {
    if (gate && *gate != want) return;  // device-driven loop: runs only when the control chose it
    double abb = 0, arr = 0;
    SELL_LOOP(A) {
        double ax = use_x ? sell_row<C16>(A, s, lane, x) : 0.0;
        long long i = (s << 5) + lane;
        if (i < A.n) {
            T bi = b[i];
            T ri = use_x ? (T)((double)bi - ax) : bi;
            r[i] = ri;
            r0[i] = ri;
            p[i] = 0;
            v[i] = 0;
            abb += (double)bi * (double)bi;
            arr += (double)ri * (double)ri;
        }
    }
    if (block_partials(abb, arr, P, &S->counter[4])) {
        double bb, rr;
        final_sum(P, &bb, &rr);
        if (threadIdx.x == 0) {
            S->counter[4] = 0;
            double bnorm = bnorm_override >= 0 ? bnorm_override : sqrt(bb);
            S->bnorm = sqrt(bb);
            S->thresh = tol * fmax(1.0, bnorm);
            S->rho0 = S->alpha = S->omega = 1.0;
            S->rho = rr;
            S->beta = rr;  // (rho / rho0) (alpha / omega) with rho0 = alpha = omega = 1
            S->rn = sqrt(rr);
            S->best_rn = S->rn;
            S->since_best = 0;
            S->it = 0;
            S->iters = 0;
            S->s_conv = 0;
            S->nonfinite = !isfinite(rr) ? 1 : 0;
            S->done = 0;
            if (S->nonfinite) S->done = 2;
            else if (S->rn <= S->thresh) S->done = 1;  // already converged
            else if (fabs(rr) < 1e-30) S->done = 2;
            else if (S->max_iter <= 0) S->done = 3;
        }
    }
}

// r = b - A x (FP64), |r|^2 and |b|^2 into out2 (fixed-order partials).
template <bool C16 = false>
__global__ void __launch_bounds__(RB, 6) k_residual64(Sell<double> A, const double* __restrict__ b,
                                                   const double* __restrict__ x, double* __restrict__ r,
                                                   double* out2, Partials P, unsigned int* counter) {
    double arr = 0, abb = 0;
    SELL_LOOP(A) {
        double ax = sell_row<C16>(A, s, lane, x);
        long long i = (s << 5) + lane;
        if (i < A.n) {
            double ri = b[i] - ax;
            r[i] = ri;
            arr += ri * ri;
            abb += b[i] * b[i];
        }
    }
    if (block_partials(arr, abb, P, counter)) {
        double rr, bb;
        final_sum(P, &rr, &bb);
        if (threadIdx.x == 0) {
            *counter = 0;
            out2[0] = rr;
            out2[1] = bb;
        }
    }
}

// ---- SELL-32 construction from the CSR rows ----
// slice lengths: one warp per slice
__global__ void k_sell_len(long long n, long long nslices, const int* __restrict__ row, int* __restrict__ slen,
                           int* __restrict__ ssize) {
    const int lane = threadIdx.x & 31;
    long long s = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    if (s >= nslices) return;
    long long i = (s << 5) + lane;
    int len = i < n ? row[i + 1] - row[i] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) len = max(len, __shfl_xor_sync(0xffffffffu, len, o));
    len = (len + 3) & ~3;  // chunks of four entries
    if (lane == 0) {
        slen[s] = len;
        ssize[s] = len * 32;
    }
}

// All SELL arrays of a slice in one pass, one warp per slice of 32 rows: the slice's CSR entries
// (one contiguous range) are staged in shared memory with coalesced loads, then each lane writes
// its row four entries at a time with 16-byte stores: columns (the diagonal moved to its place
// in column order, padding repeating the last column), values A (padding 0), the column steps
// and the row's first column (any row that does not ascend or steps by more than 65535 sets
// *bad), and the column-scaled copies A D^-1 in FP64 and FP32. Slices of more than SB_CAP
// entries read their rows from global memory instead. Same values as a per-row fill followed
// by the column-scaling passes (each scaled value is the same single product, rounded once).
constexpr int SB_CAP = 1024;
__global__ void __launch_bounds__(128) k_sell_build(long long n, long long nslices, const int* __restrict__ row,
                                                    const int* __restrict__ acol, const double* __restrict__ aval,
                                                    const double* __restrict__ dinv, const int* __restrict__ sptr,
                                                    const int* __restrict__ slen, int* __restrict__ col,
                                                    double* __restrict__ val, unsigned short* __restrict__ dcol,
                                                    int* __restrict__ rbase, double* __restrict__ vals,
                                                    float* __restrict__ valf, int* bad, int raw) {
    __shared__ int scol[4][SB_CAP];
    __shared__ double sval[4][SB_CAP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long s = blockIdx.x * 4LL + w;
    if (s >= nslices) return;  // whole warp
    const long long u0 = s << 5, i = u0 + lane;
    const int b0 = row[u0], b1 = row[min(u0 + 32, n)];
    const bool staged = b1 - b0 <= SB_CAP;
    if (staged) {
        for (int t = lane; t < b1 - b0; t += 32) {
            scol[w][t] = acol[b0 + t];
            sval[w][t] = aval[b0 + t];
        }
    }
    __syncwarp();
    int e0 = 0, len = 0;
    if (i < n) {
        e0 = row[i];
        len = row[i + 1] - e0;
    }
    auto C = [&](int e) { return staged ? scol[w][e - b0] : acol[e]; };
    auto V = [&](int e) { return staged ? sval[w][e - b0] : aval[e]; };
    // the CSR row's last entry is its diagonal: it goes where it belongs in column order
    int pos = 0;
    if (len > 0)
        while (pos < len - 1 && C(e0 + pos) < (int)i) ++pos;
    int last = i < n ? (int)i : 0, prev = 0;
    bool ok = true;
    const int L = slen[s];
    const long long base = (long long)sptr[s] + 4 * lane;
    for (int k4 = 0; k4 < L; k4 += 4) {
        int cc[4];
        double vv[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k = k4 + j;
            if (k < len) {
                const int src = k < pos ? e0 + k : (k == pos ? e0 + len - 1 : e0 + k - 1);
                cc[j] = C(src);
                vv[j] = V(src);
                last = cc[j];
            } else {
                cc[j] = last;
                vv[j] = 0.0;
            }
        }
        if (k4 == 0) {
            prev = cc[0];
            rbase[i] = cc[0];
        }
        unsigned short dd[4];
        double sv[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int d = cc[j] - prev;
            ok = ok && d >= 0 && d <= 65535;
            dd[j] = (unsigned short)(d >= 0 && d <= 65535 ? d : 0);
            prev = cc[j];
            sv[j] = vv[j] * dinv[cc[j]];
        }
        const long long e = base + 128LL * (k4 >> 2);
        if (raw) {  // unscaled values and 32-bit columns: only the plain FP64 solver reads them
            *reinterpret_cast<int4*>(col + e) = make_int4(cc[0], cc[1], cc[2], cc[3]);
            *reinterpret_cast<double2*>(val + e) = make_double2(vv[0], vv[1]);
            *reinterpret_cast<double2*>(val + e + 2) = make_double2(vv[2], vv[3]);
        }
        *reinterpret_cast<ushort4*>(dcol + e) = make_ushort4(dd[0], dd[1], dd[2], dd[3]);
        *reinterpret_cast<double2*>(vals + e) = make_double2(sv[0], sv[1]);
        *reinterpret_cast<double2*>(vals + e + 2) = make_double2(sv[2], sv[3]);
        *reinterpret_cast<float4*>(valf + e) =
            make_float4((float)sv[0], (float)sv[1], (float)sv[2], (float)sv[3]);
    }
    if (!ok) atomicOr(bad, 1);
}



// ---------------------------------------------------------------------------------------
// Mixed-precision helpers
// ---------------------------------------------------------------------------------------
template <class T>
__global__ void k_fill(long long n, T* __restrict__ x, T v) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = v;
}

__global__ void k_unscale(long long n, double* __restrict__ x, const double* __restrict__ dinv) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] *= dinv[i];
}

__global__ void k_scale_by_diag(long long n, double* __restrict__ x, const double* __restrict__ dinv) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        x[i] = dinv[i] != 0 ? x[i] / dinv[i] : x[i];
}

// error statistics against p*: |x - p*|^2, |p*|^2, max |x - p*| (fixed-order partials)
__global__ void __launch_bounds__(RB) k_error_stats(long long n, const double* __restrict__ x,
                                                    const double* __restrict__ xe, double* out3, Partials P,
                                                    unsigned int* counter, unsigned long long* maxbits) {
    double se = 0, ee = 0, mx = 0;
    for (long long i = blockIdx.x * (long long)RB + threadIdx.x; i < n; i += (long long)gridDim.x * RB) {
        double e = x[i] - xe[i];
        se += e * e;
        ee += xe[i] * xe[i];
        mx = fmax(mx, fabs(e));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(maxbits, (unsigned long long)__double_as_longlong(mx));
    if (block_partials(se, ee, P, counter)) {
        double a, b;
        final_sum(P, &a, &b);
        if (threadIdx.x == 0) {
            *counter = 0;
            out3[0] = a;
            out3[1] = b;
        }
    }
}

// ---- reliable updates of the mixed-precision solver ----
// x_hi += sigma D^-1 y_lo (FP64), y_lo = 0
__global__ void k_reliable_x(long long n, double* __restrict__ x, float* __restrict__ y,
                             const double* __restrict__ dinv, const double* sigma) {
    const double sg = *sigma;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        x[i] += sg * dinv[i] * (double)y[i];
        y[i] = 0.f;
    }
}

// r = r64 / sigma in FP32 replaces the recursive residual; rho' = (r0, r) and the next
// beta follow, so the iteration continues with its search direction (van der Vorst & Ye
// residual replacement).
__global__ void __launch_bounds__(RB) k_reliable_r(long long n, const double* __restrict__ r64,
                                                   const double* sigma, float* __restrict__ r,
                                                   const float* __restrict__ r0, BcgScalars* S, Partials P) {
    const double inv = 1.0 / *sigma;
    double arr = 0, ar0r = 0;
    for (long long i = blockIdx.x * (long long)RB + threadIdx.x; i < n; i += (long long)gridDim.x * RB) {
        float ri = (float)(r64[i] * inv);
        r[i] = ri;
        arr += (double)ri * (double)ri;
        ar0r += (double)r0[i] * (double)ri;
    }
    if (block_partials(arr, ar0r, P, &S->counter[7])) {
        double rr, rho;
        final_sum(P, &rr, &rho);
        if (threadIdx.x == 0) {
            S->counter[7] = 0;
            S->rn = sqrt(rr);
            if (S->rn < S->best_rn) S->best_rn = S->rn;
            S->beta = (rho / S->rho0) * (S->alpha / S->omega);
            S->rho = rho;
            S->done = 0;
            S->s_conv = 0;
            if (!isfinite(rho) || fabs(rho) < 1e-30) S->done = 2;
        }
    }
}

// rf = r64 / sigma (start of an FP32 run), sigma = |r64| given as its square in scal[0]
__global__ void k_start_rhs(long long n, const double* __restrict__ r64, const double* scal, double* sigma,
                            float* __restrict__ rf, float* __restrict__ y) {
    const double sg = sqrt(scal[0]);
    if (blockIdx.x == 0 && threadIdx.x == 0) *sigma = sg;
    const double inv = sg > 0 ? 1.0 / sg : 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        rf[i] = (float)(r64[i] * inv);
        y[i] = 0.f;
    }
}

// Residual replacement of the mixed solver (FP64 vectors, FP32 matrix in the iteration):
// r = b - (A D^-1) y with the FP64 matrix; rho' = (r0, r) and the next beta follow, so the
// iteration continues with its search direction (van der Vorst & Ye). |r| goes to S->rn.
template <bool C16 = false>
__global__ void __launch_bounds__(RB, 6) k_replace_residual(Sell<double> A, const double* __restrict__ b,
                                                            const double* __restrict__ y, double* __restrict__ r,
                                                            const double* __restrict__ r0, BcgScalars* S,
                                                            Partials P, const int* gate = nullptr, int want = 0) {
    if (gate && *gate != want) return;  // device-driven loop: runs only when the control chose it
    double arr = 0, ar0r = 0;
    SELL_LOOP(A) {
        double ay = sell_row<C16>(A, s, lane, y);
        long long i = (s << 5) + lane;
        if (i < A.n) {
            double ri = b[i] - ay;
            r[i] = ri;
            arr += ri * ri;
            ar0r += r0[i] * ri;
        }
    }
    if (block_partials(arr, ar0r, P, &S->counter[7])) {
        double rr, rho;
        final_sum(P, &rr, &rho);
        if (threadIdx.x == 0) {
            S->counter[7] = 0;
            S->rn = sqrt(rr);
            if (S->rn < S->best_rn) S->best_rn = S->rn;
            S->beta = (rho / S->rho0) * (S->alpha / S->omega);
            S->rho = rho;
            S->done = 0;
            S->s_conv = 0;
            if (!isfinite(rr)) { S->nonfinite = 1; S->done = 2; }
            else if (S->rn <= S->thresh) S->done = 1;
            else if (!isfinite(rho) || fabs(rho) < 1e-30) S->done = 2;
        }
    }
}

// |b|^2 into scal[0], fixed-order partials (once per learned solve)
__global__ void __launch_bounds__(RB) k_norm2(long long n, const double* __restrict__ b, double* scal, Partials P,
                                              unsigned int* counter) {
    double acc = 0;
    for (long long i = blockIdx.x * (long long)RB + threadIdx.x; i < n; i += (long long)gridDim.x * RB)
        acc += b[i] * b[i];
    if (block_partials(acc, 0.0, P, counter)) {
        double tot, unused;
        final_sum(P, &tot, &unused);
        if (threadIdx.x == 0) {
            *counter = 0;
            scal[0] = tot;
        }
    }
}

// network input b / |b| (FP32)
__global__ void k_rhs_unit(long long n, const double* __restrict__ b, float* __restrict__ rf, const double* scal) {
    const double inv = scal[0] > 0 ? 1.0 / sqrt(scal[0]) : 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        rf[i] = (float)(b[i] * inv);
}

// y0 = |b| net(b / |b|)
__global__ void k_y_from_net(long long n, const float* __restrict__ yf, const double* scal, double* __restrict__ y) {
    const double nb = sqrt(scal[0]);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = nb * (double)yf[i];
}

// y += |r0| net(r0 / |r0|) (network correction of a warm start), keeping y in keep
__global__ void k_y_add_net(long long n, const float* __restrict__ yf, const double* scal, double* __restrict__ y,
                            double* __restrict__ keep) {
    const double nr = sqrt(scal[0]);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        keep[i] = y[i];
        y[i] += nr * (double)yf[i];
    }
}

// initial guess of the unknowns from a per-particle field (caller order): unknown u is
// particle perm[sorted_of_u[u]]
__global__ void k_guess_from_particles(long long U, const int* __restrict__ sorted_of_u, const int* __restrict__ perm,
                                       const double* __restrict__ pp, double* __restrict__ x) {
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < U; u += (long long)gridDim.x * blockDim.x)
        x[u] = pp[perm[sorted_of_u[u]]];
}

__global__ void k_fill_value(size_t n, double v, double* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) out[i] = v;
}

__global__ void k_solution_to_particles(long long U, const int* __restrict__ sorted_of_u, const int* __restrict__ perm,
                                        const double* __restrict__ x, double* __restrict__ pp) {
    for (long long u = blockIdx.x * (long long)blockDim.x + threadIdx.x; u < U; u += (long long)gridDim.x * blockDim.x)
        pp[perm[sorted_of_u[u]]] = x[u];
}

// ---------------------------------------------------------------------------------------
// device-driven solve loop: the host loop's decisions (residual replacement, restart, stop)
// made by single-thread kernels between the iteration chunks of a conditional WHILE graph
// node, so that a whole solve is one graph launch with no host round trip
// ---------------------------------------------------------------------------------------
struct LoopCtl {
    double rn_upd;      // |r| at the last replacement or restart
    double delta;       // replacement when |r| fell below delta rn_upd
    int total;          // iterations so far (over restarts)
    int base;           // S->iters at the last accounting
    int replacements, restarts, fallback;
    int act;            // 0 none, 1 replace, 2 restart: gates the replacement and init kernels
    int final_replace;  // the pending replacement ends the solve (iteration cap)
    int state;          // 0 running, 1 converged, 2 failed, 3 iteration cap, 4 multigrid gave up
    int trips, max_trips, max_iter, use_nn;
    int use_mg;         // the body applies the multigrid: a breakdown or stall ends it (state 4)
    int stall;          // stall window of the restarted runs (multigrid only)
};

// as set_scalar_caps on the host: a fresh scalar block with the remaining iteration budget
__device__ void restart_caps(BcgScalars* S, int max_iter, int stall) {
    BcgScalars z{};
    z.max_iter = max_iter;
    z.stall_window = stall;
    *S = z;
}

__global__ void k_mix_after_chunk(BcgScalars* S, LoopCtl* C) {
    C->total += S->iters - C->base;
    C->base = S->iters;
    C->act = 0;
    if (!S->done && S->rn > C->delta * C->rn_upd) return;  // keep iterating
    const int why = S->done;
    if (why == 3 || C->total >= C->max_iter) {
        C->act = 1;
        C->final_replace = 1;
        return;
    }
    if (why == 0) {
        C->act = 1;
        C->final_replace = 0;
        return;
    }
    if (C->use_mg && (why == 2 || why == 4)) {  // the multigrid broke down or stalled: host falls back
        C->state = 4;
        return;
    }
    if (why == 4 && C->use_nn) C->fallback = 1;
    if (S->nonfinite) {
        C->state = 2;
        return;
    }
    restart_caps(S, C->max_iter - C->total, C->stall);
    C->act = 2;
}

__global__ void k_mix_after_replace(BcgScalars* S, LoopCtl* C) {
    if (C->act != 1) return;
    C->act = 0;
    if (C->final_replace) {
        C->state = S->done == 1 ? 1 : 3;
        return;
    }
    C->replacements += 1;
    C->rn_upd = S->rn;
    if (S->done == 1) {
        C->state = 1;
        return;
    }
    if (S->done == 0) return;
    if (C->use_mg) {  // breakdown after the replacement with the multigrid: host falls back
        C->state = 4;
        return;
    }
    if (S->nonfinite) {  // breakdown after the replacement: restart, unless non-finite
        C->state = 2;
        return;
    }
    restart_caps(S, C->max_iter - C->total, C->stall);
    C->act = 2;
}

__global__ void k_mix_after_restart(BcgScalars* S, LoopCtl* C) {
    if (C->act != 2) return;
    C->act = 0;
    C->restarts += 1;
    C->base = 0;
    C->rn_upd = S->rn;
    if (S->done == 1) C->state = 1;
    else if (S->done) C->state = 2;
}

// plain loop (FP64 / Jacobi): stop when the iteration stopped
__global__ void k_plain_after_chunk(const BcgScalars* S, LoopCtl* C) {
    if (S->done) C->state = S->done == 1 ? 1 : 2;
}

// the WHILE condition; trips are bounded whatever the control state says
__global__ void k_loop_continue(LoopCtl* C, cudaGraphConditionalHandle h) {
    C->trips += 1;
    cudaGraphSetConditional(h, (C->state == 0 && C->trips < C->max_trips) ? 1u : 0u);
}

// ---------------------------------------------------------------------------------------
// host side of the engine
// ---------------------------------------------------------------------------------------
struct Engine {
    lsmps_ctx* ctx;
    cudaStream_t s;
    BcgScalars* S;
    Partials P;
};

template <class T>
struct Vecs {
    T *x, *r, *r0, *p, *v, *s, *t;
    T *ph = nullptr, *sh = nullptr;  // preconditioned directions M p, M s (multigrid)
};

Engine make_engine(lsmps_ctx* ctx) {
    Engine E{ctx, ctx->stream, nullptr, {}};
    double* red = ctx->red.ensure<double>(2 * RGRID + 256);
    E.P = Partials{red, red + RGRID};
    E.S = reinterpret_cast<BcgScalars*>(red + 2 * RGRID);
    return E;
}

double* engine_scalars(lsmps_ctx* ctx) { return ctx->red.get<double>() + 2 * RGRID + 128; }

LoopCtl* engine_loop_ctl(lsmps_ctx* ctx) {
    return reinterpret_cast<LoopCtl*>(ctx->red.get<double>() + 2 * RGRID + 160);
}
static_assert(sizeof(BcgScalars) <= 128 * sizeof(double) && sizeof(LoopCtl) <= 96 * sizeof(double),
              "engine scalar layout");

// A graph whose one node is a WHILE conditional: its body (captured from stream s by `body`,
// then k_loop_continue) runs until the control clears the condition.
template <class F>
cudaGraphExec_t build_while_graph(cudaStream_t s, LoopCtl* C, F&& body) {
    cudaGraph_t g = nullptr;
    LSMPS_CUDA(cudaGraphCreate(&g, 0));
    cudaGraphExec_t exec = nullptr;
    try {
        cudaGraphConditionalHandle h;
        LSMPS_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        LSMPS_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &np));
        LSMPS_CUDA(cudaStreamBeginCaptureToGraph(s, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                 cudaStreamCaptureModeThreadLocal));
        body();
        k_loop_continue<<<1, 1, 0, s>>>(C, h);
        cudaGraph_t captured = nullptr;
        LSMPS_CUDA(cudaStreamEndCapture(s, &captured));
        LSMPS_CUDA(cudaGraphInstantiate(&exec, g, 0));
    } catch (...) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
            cudaGraph_t tmp = nullptr;
            cudaStreamEndCapture(s, &tmp);
            if (tmp) cudaGraphDestroy(tmp);
        }
        cudaGetLastError();
        cudaGraphDestroy(g);
        throw;
    }
    cudaGraphDestroy(g);
    return exec;
}

// One BiCGStab iteration; with `mg` (FP64 vectors only) the multigrid V-cycle is the right
// preconditioner: ph = D M p before v = A ph, sh = D M s before t = A sh.
template <class T, class TM = T>
void iteration(Engine& E, const Sell<TM>& A, const Vecs<T>& V, bool mg = false) {
    note_launches(5);
    const T* pv = V.p;
    const T* sv = V.s;
    if constexpr (std::is_same<T, double>::value) {
        if (mg) {  // p and its level-1 restriction in one pass, then the rest of the V-cycle
            const MgFine G = mg_fine(E.ctx);
            launch_pdl(k_bcg_p_agg, agg_blocks(G.n1), RB, 0, E.s, G, V.r, V.p, V.v, E.S);
            mg_apply(E.ctx, V.p, V.ph, E.S, 0, true);
            pv = V.ph;
        }
    }
    if (!mg) launch_pdl(k_bcg_p<T>, RGRID, RB, 0, E.s, A.n, V.r, V.p, V.v, E.S);
    if (A.dcol) launch_pdl(k_bcg_v<T, TM, true>, spmv_grid<TM, true>(), RB, 0, E.s, A, pv, V.v, V.r0, E.S, E.P);
    else launch_pdl(k_bcg_v<T, TM, false>, RGRID, RB, 0, E.s, A, pv, V.v, V.r0, E.S, E.P);
    if constexpr (std::is_same<T, double>::value) {
        if (mg) {
            const MgFine G = mg_fine(E.ctx);
            launch_pdl(k_bcg_s_agg, std::min<unsigned>(RGRID, agg_blocks(G.n1)), RB, 0, E.s, G, V.r, V.v, V.s, E.S,
                       E.P);
            mg_apply(E.ctx, V.s, V.sh, E.S, 1, true);
            sv = V.sh;
        }
    }
    if (!mg) launch_pdl(k_bcg_s<T>, RGRID, RB, 0, E.s, A.n, V.r, V.v, V.s, E.S, E.P);
    if (A.dcol) launch_pdl(k_bcg_t<T, TM, true>, spmv_grid<TM, true>(), RB, 0, E.s, A, sv, V.t, E.S, E.P, V.s);
    else launch_pdl(k_bcg_t<T, TM, false>, RGRID, RB, 0, E.s, A, sv, V.t, E.S, E.P, V.s);
    if (mg)
        launch_pdl(k_bcg_x<T, true>, RGRID, RB, 0, E.s, A.n, V.x, V.r, V.p, V.s, V.t, V.r0, E.S, E.P, V.ph, V.sh);
    else
        launch_pdl(k_bcg_x<T, false>, RGRID, RB, 0, E.s, A.n, V.x, V.r, V.p, V.s, V.t, V.r0, E.S, E.P,
                   (const T*)nullptr, (const T*)nullptr);
}

// kernel launches of one iteration
int launches_per_iteration(lsmps_ctx* ctx, bool mg) { return 5 + (mg ? 2 * mg_launches_per_apply(ctx, true) : 0); }

template <class T, class TM = T>
void init(Engine& E, const Sell<TM>& A, const T* b, const Vecs<T>& V, bool use_x, double tol, double bnorm_override) {
    if (A.dcol)
        k_bcg_init<T, TM, true><<<RGRID, RB, 0, E.s>>>(A, b, V.x, use_x, V.r, V.r0, V.p, V.v, E.S, E.P, tol,
                                                       bnorm_override);
    else
        k_bcg_init<T, TM, false><<<RGRID, RB, 0, E.s>>>(A, b, V.x, use_x, V.r, V.r0, V.p, V.v, E.S, E.P, tol,
                                                        bnorm_override);
    LSMPS_CHECK_LAUNCH();
}

// the mixed solver's FP64 residual replacement (gated by the device-driven loop's control)
void launch_replace(cudaStream_t s, const Sell<double>& As, const double* b, const Vecs<double>& V, Engine& E,
                    const int* gate, int want) {
    if (As.dcol) k_replace_residual<true><<<RGRID, RB, 0, s>>>(As, b, V.x, V.r, V.r0, E.S, E.P, gate, want);
    else k_replace_residual<false><<<RGRID, RB, 0, s>>>(As, b, V.x, V.r, V.r0, E.S, E.P, gate, want);
}

void residual64(Engine& E, const Sell<double>& A, const double* b, const double* x, double* r, double* out2) {
    if (A.dcol) k_residual64<true><<<RGRID, RB, 0, E.s>>>(A, b, x, r, out2, E.P, &E.S->counter[5]);
    else k_residual64<false><<<RGRID, RB, 0, E.s>>>(A, b, x, r, out2, E.P, &E.S->counter[5]);
    LSMPS_CHECK_LAUNCH();
}

// Runs the iteration until done. mode 1: one graph whose WHILE node repeats `chunk`
// iterations until the scalars say done (no host round trip); mode 2: a graph of `chunk`
// iterations launched from a host loop that reads the scalars after each; mode 0: eager
// launches with the same host loop. Returns the final scalars.
template <class T>
BcgScalars run_loop(Engine& E, const Sell<T>& A, const Vecs<T>& V, int chunk, int mode) {
    BcgScalars h{};
    LSMPS_CUDA(cudaMemcpyAsync(&h, E.S, sizeof(h), cudaMemcpyDeviceToHost, E.s));
    LSMPS_CUDA(cudaStreamSynchronize(E.s));
    // the iteration cap bounds the loop; two extra chunks cover the final no-op kernels
    const long long max_chunks = (h.max_iter + chunk - 1) / chunk + 2;
    if (h.done) return h;
    if (mode == 1) {
        LoopCtl* C = engine_loop_ctl(E.ctx);
        LoopCtl c0{};
        c0.max_trips = (int)std::min<long long>(max_chunks, INT_MAX);
        LSMPS_CUDA(cudaMemcpyAsync(C, &c0, sizeof(c0), cudaMemcpyHostToDevice, E.s));
        cudaGraphExec_t exec = build_while_graph(E.s, C, [&] {
            for (int c = 0; c < chunk; ++c) iteration<T>(E, A, V);
            k_plain_after_chunk<<<1, 1, 0, E.s>>>(E.S, C);
        });
        note_launches(0 - (uint64_t)(5 * chunk));  // captured, not launched
        cudaError_t e = cudaGraphLaunch(exec, E.s);
        LoopCtl hc{};
        if (e == cudaSuccess) e = cudaMemcpyAsync(&hc, C, sizeof(hc), cudaMemcpyDeviceToHost, E.s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&h, E.S, sizeof(h), cudaMemcpyDeviceToHost, E.s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(E.s);
        cudaGraphExecDestroy(exec);
        LSMPS_CUDA(e);
        note_launches((uint64_t)hc.trips * (5 * (uint64_t)chunk + 2));
        return h;
    }
    cudaGraphExec_t exec = nullptr;
    if (mode == 2) {
        cudaGraph_t graph;
        LSMPS_CUDA(cudaStreamBeginCapture(E.s, cudaStreamCaptureModeThreadLocal));
        for (int c = 0; c < chunk; ++c) iteration<T>(E, A, V);
        note_launches(0 - (uint64_t)(5 * chunk));  // captured, not launched
        cudaError_t e = cudaStreamEndCapture(E.s, &graph);
        LSMPS_CUDA(e);
        LSMPS_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        cudaGraphDestroy(graph);
    }
    for (long long c = 0; c < max_chunks && !h.done; ++c) {
        if (exec) {
            LSMPS_CUDA(cudaGraphLaunch(exec, E.s));
            note_launches(5 * (uint64_t)chunk);
        } else {
            for (int k = 0; k < chunk; ++k) iteration<T>(E, A, V);
            LSMPS_CHECK_LAUNCH();
        }
        LSMPS_CUDA(cudaMemcpyAsync(&h, E.S, sizeof(h), cudaMemcpyDeviceToHost, E.s));
        LSMPS_CUDA(cudaStreamSynchronize(E.s));
    }
    if (exec) cudaGraphExecDestroy(exec);
    return h;
}

void set_scalar_caps(Engine& E, int max_iter, int stall_window) {
    BcgScalars init{};
    init.max_iter = max_iter;
    init.stall_window = stall_window;
    LSMPS_CUDA(cudaMemcpyAsync(E.S, &init, sizeof(init), cudaMemcpyHostToDevice, E.s));
}

}  // namespace

// ---------------------------------------------------------------------------------------
static void solve_exact(lsmps_ctx* ctx, const lsmps_solver_opts* o, lsmps_ppe_stats* ps) {
    cudaStream_t s = ctx->stream;
    long long U = ctx->U;
    double* x = ctx->vx.ensure<double>(U + 1);
    double* r = ctx->vr.ensure<double>(U + 1);
    double* r0 = ctx->vr0.ensure<double>(U + 1);
    double* p = ctx->vp.ensure<double>(U + 1);
    double* v = ctx->vv.ensure<double>(U + 1);
    double* sv = ctx->vs.ensure<double>(U + 1);
    double* t = ctx->vt.ensure<double>(U + 1);
    double* prod = ctx->vph.ensure<double>(U + 1);
    ExactState* st = reinterpret_cast<ExactState*>(ctx->red.ensure<double>(64));
    const double* b = ctx->A_b.get<double>();
    const int* uref = ctx->u_of_ref.get<int>();
    const int* row = ctx->A_row.get<int>();
    const int* col = ctx->A_col.get<int>();
    const double* val = ctx->A_val.get<double>();
    LSMPS_CUDA(cudaMemsetAsync(st, 0, sizeof(ExactState), s));
    LSMPS_CUDA(cudaMemsetAsync(x, 0, U * sizeof(double), s));
    LSMPS_CUDA(cudaMemsetAsync(p, 0, U * sizeof(double), s));
    LSMPS_CUDA(cudaMemsetAsync(v, 0, U * sizeof(double), s));
    LSMPS_CUDA(cudaMemcpyAsync(r, b, U * sizeof(double), cudaMemcpyDeviceToDevice, s));
    LSMPS_CUDA(cudaMemcpyAsync(r0, b, U * sizeof(double), cudaMemcpyDeviceToDevice, s));
    const unsigned G = 148 * 4, B = 256;
    const int max_iter = o->max_iter;
    const double tol = o->tol;
    auto dot = [&](const double* a, const double* c, int op) {
        k_x_prod<<<G, B, 0, s>>>(a, c, uref, U, prod, st);
        k_x_tail<<<1, 32, 0, s>>>(prod, U, st, op, tol, max_iter);
    };
    ev_record(ctx, 10);
    if (U > 0) {
        dot(b, b, OP_BNORM);
        const int check = std::max(1, o->check_every > 0 ? o->check_every : 16);
        for (int it = 0; it < max_iter; ++it) {
            dot(r0, r, OP_RHO);
            k_x_vec<<<G, B, 0, s>>>(U, 0, x, r, p, v, sv, t, st);
            k_x_spmv<<<G, B, 0, s>>>(U, row, col, val, p, v, st, 1);
            dot(r0, v, OP_DEN);
            k_x_vec<<<G, B, 0, s>>>(U, 1, x, r, p, v, sv, t, st);
            dot(sv, sv, OP_SN);
            k_x_vec<<<G, B, 0, s>>>(U, 2, x, r, p, v, sv, t, st);
            k_x_finish_sconv<<<1, 1, 0, s>>>(st);
            k_x_spmv<<<G, B, 0, s>>>(U, row, col, val, sv, t, st, 1);
            dot(t, t, OP_TT);
            dot(t, sv, OP_TS);
            k_x_vec<<<G, B, 0, s>>>(U, 3, x, r, p, v, sv, t, st);
            dot(r, r, OP_RN);
            LSMPS_CHECK_LAUNCH();
            note_launches(18);
            if ((it + 1) % check == 0) {
                int done = 0;
                LSMPS_CUDA(cudaMemcpyAsync(&done, &st->done, sizeof(int), cudaMemcpyDeviceToHost, s));
                LSMPS_CUDA(cudaStreamSynchronize(s));
                if (done) break;
            }
        }
    }
    ev_record(ctx, 11);
    ExactState h{};
    LSMPS_CUDA(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, s));
    double fin[3] = {0, 0, 0};
    if (U > 0) {
        k_x_spmv<<<G, B, 0, s>>>(U, row, col, val, x, t, st, 0);
        double* out = reinterpret_cast<double*>(st + 1);
        k_x_final<<<1, 32, 0, s>>>(t, b, x, ctx->A_xexact.get<double>(), uref, U, out);
        LSMPS_CHECK_LAUNCH();
        LSMPS_CUDA(cudaMemcpyAsync(fin, out, sizeof(fin), cudaMemcpyDeviceToHost, s));
    }
    LSMPS_CUDA(cudaStreamSynchronize(s));
    ps->iterations = h.iters;
    ps->converged = h.converged;
    ps->initial_residual = h.bnorm;
    ps->final_residual = fin[0];
    ps->relative_l2_error = fin[1];
    ps->max_error = fin[2];
    ps->relative_residual = fin[0] / std::max(h.bnorm, 1e-300);
    ps->solve_ms = ev_elapsed(ctx, 10, 11);
}


// ---- SELL-32 copies of the assembled matrix (built on first use after an assembly) ----
static void sell_raw(lsmps_ctx* ctx);
// kind 0: A (FP64), 1: A D^-1 (FP64), 2: A D^-1 (FP32)
static void sell_structure(lsmps_ctx* ctx) {
    if (ctx->have_sell) return;
    cudaStream_t s = ctx->stream;
    const long long U = ctx->U;
    const long long ns = (U + 31) / 32;
    int* slen = ctx->S_len.ensure<int>(ns + 1);
    int* ssize = ctx->vtmp.ensure<int>(ns + 1);
    int* sptr = ctx->S_ptr.ensure<int>(ns + 1);
    if (ns) {
        k_sell_len<<<blocks_for(ns * 32, 256), 256, 0, s>>>(U, ns, ctx->A_row.get<int>(), slen, ssize);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<int>(ssize, sptr, ns, s, ctx->scan_tmp, ctx->dflags.get<int>());
    int total = 0;
    read_back(ctx, {{sptr + ns, &total, sizeof(int)}}, "SELL layout");
    ctx->sell_nslices = ns;
    ctx->sell_entries = total;
    int* col = ctx->S_col.ensure<int>((size_t)total + 8);
    double* val = ctx->S_val.ensure<double>((size_t)total + 8);
    double* vals = ctx->S_vals.ensure<double>((size_t)total + 8);
    float* valf = ctx->S_valf.ensure<float>((size_t)total + 8);
    unsigned short* dcol = ctx->S_dcol.ensure<unsigned short>((size_t)total + 8);
    int* rbase = ctx->S_rbase.ensure<int>(ns * 32 + 1);
    ctx->have_steps = false;
    if (ns) {
        int* bad = ctx->scratch.get<int>() + 46;
        LSMPS_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), s));
        k_sell_build<<<(unsigned)((ns + 3) / 4), 128, 0, s>>>(U, ns, ctx->A_row.get<int>(), ctx->A_col.get<int>(),
                                                              ctx->A_val.get<double>(), ctx->A_dinv.get<double>(), sptr,
                                                              slen, col, val, dcol, rbase, vals, valf, bad, 0);
        LSMPS_CHECK_LAUNCH();
        int hbad = 1;
        read_back(ctx, {{bad, &hbad, sizeof(int)}}, nullptr);
        ctx->have_steps = hbad == 0 && ctx->sell_steps_enabled;
    }
    ctx->have_sell_s = ctx->have_sell_f = true;  // the scaled copies come with the structure
    ctx->have_sell = true;
    ctx->have_sell_raw = ns == 0;
    if (!ctx->have_steps) sell_raw(ctx);  // every view then reads the 32-bit columns
}

// The unscaled FP64 values and 32-bit columns (the plain FP64 solver's matrix, and the columns
// of every view when the copies have no 16-bit steps): the same build again, writing them too.
static void sell_raw(lsmps_ctx* ctx) {
    if (ctx->have_sell_raw) return;
    const long long U = ctx->U, ns = ctx->sell_nslices;
    if (ns) {
        int* bad = ctx->scratch.get<int>() + 46;
        k_sell_build<<<(unsigned)((ns + 3) / 4), 128, 0, ctx->stream>>>(
            U, ns, ctx->A_row.get<int>(), ctx->A_col.get<int>(), ctx->A_val.get<double>(), ctx->A_dinv.get<double>(),
            ctx->S_ptr.get<int>(), ctx->S_len.get<int>(), ctx->S_col.get<int>(), ctx->S_val.get<double>(),
            ctx->S_dcol.get<unsigned short>(), ctx->S_rbase.get<int>(), ctx->S_vals.get<double>(),
            ctx->S_valf.get<float>(), bad, 1);
        LSMPS_CHECK_LAUNCH();
    }
    ctx->have_sell_raw = true;
}

template <class T>
static Sell<T> sell_view(lsmps_ctx* ctx, const T* val) {
    Sell<T> A{ctx->U, ctx->sell_nslices, ctx->S_ptr.get<int>(), ctx->S_len.get<int>(), ctx->S_col.get<int>(), val};
    if (ctx->have_steps) {
        A.dcol = ctx->S_dcol.get<unsigned short>();
        A.rbase = ctx->S_rbase.get<int>();
    }
    return A;
}

static Sell<double> sell_a64(lsmps_ctx* ctx) {
    sell_structure(ctx);
    sell_raw(ctx);
    return sell_view<double>(ctx, ctx->S_val.get<double>());
}

Sell<double> sell_a64_view(lsmps_ctx* ctx) { return sell_a64(ctx); }

static Sell<double> sell_scaled64(lsmps_ctx* ctx) {  // A D^-1 in FP64 (built with the structure)
    sell_structure(ctx);
    return sell_view<double>(ctx, ctx->S_vals.get<double>());
}

static Sell<float> sell_scaled32(lsmps_ctx* ctx) {  // A D^-1 in FP32 (built with the structure)
    sell_structure(ctx);
    return sell_view<float>(ctx, ctx->S_valf.get<float>());
}

Sell<float> sell_scaled32_view(lsmps_ctx* ctx) { return sell_scaled32(ctx); }

// Fast FP64 / Jacobi: BiCGStab on A (or A D^-1) in FP64.
static void solve_fast64(lsmps_ctx* ctx, const lsmps_solver_opts* o, lsmps_ppe_stats* ps, bool jacobi) {
    cudaStream_t s = ctx->stream;
    long long U = ctx->U;
    Engine E = make_engine(ctx);
    Vecs<double> V{ctx->vx.ensure<double>(U + 1), ctx->vr.ensure<double>(U + 1), ctx->vr0.ensure<double>(U + 1),
                   ctx->vp.ensure<double>(U + 1), ctx->vv.ensure<double>(U + 1), ctx->vs.ensure<double>(U + 1),
                   ctx->vt.ensure<double>(U + 1)};
    const double* dinv = ctx->A_dinv.get<double>();
    bool warm = o->warm_start && ctx->have_solution;
    ev_record(ctx, 10);
    Sell<double> Aop = jacobi ? sell_scaled64(ctx) : sell_a64(ctx);
    set_scalar_caps(E, o->max_iter, 0);
    if (warm && jacobi) {  // the iteration works on y = D x
        k_scale_by_diag<<<1184, 256, 0, s>>>(U, V.x, dinv);
        LSMPS_CHECK_LAUNCH();
    } else if (!warm) {
        LSMPS_CUDA(cudaMemsetAsync(V.x, 0, U * sizeof(double), s));
    }
    init<double>(E, Aop, ctx->A_b.get<double>(), V, warm, o->tol, -1.0);
    int chunk = std::max(1, o->check_every > 0 ? o->check_every : 8);
    BcgScalars h = run_loop<double>(E, Aop, V, chunk, o->use_graph);
    if (jacobi) {
        k_unscale<<<1184, 256, 0, s>>>(U, V.x, dinv);
        LSMPS_CHECK_LAUNCH();
    }
    ev_record(ctx, 11);
    LSMPS_CUDA(cudaStreamSynchronize(s));
    ps->iterations = h.iters;
    ps->converged = h.done == 1;
    ps->solve_ms = ev_elapsed(ctx, 10, 11);
    if (h.nonfinite) ps->converged = 0;
}

// Mixed precision with FP32 vectors (MIXED_F32). One FP32 Jacobi-BiCGStab on A D^-1 y = r0 / sigma (sigma =
// |r0|, so FP32 values start at O(1)) accumulates y_lo; whenever its recursive residual has
// dropped by a factor `inner_tol` since the last update (checked every `check_every`
// iterations), a reliable update folds y_lo into the FP64 solution x_hi, recomputes the
// true residual b - A x_hi with the FP64 matrix, and replaces the FP32 residual with it,
// keeping the search direction. Convergence is always decided on the FP64 residual. A
// breakdown, a stall (LEARNED: no 1 % progress in `stall_window` iterations) or an FP32
// residual that claims convergence the FP64 one does not confirm restarts the Krylov space
// from the true residual; LEARNED starts the first run from the network's guess and, after
// a stall, continues as plain Jacobi-BiCGStab (fallback).
static void solve_mixed_f32(lsmps_ctx* ctx, const lsmps_solver_opts* o, lsmps_ppe_stats* ps, bool learned) {
    cudaStream_t s = ctx->stream;
    long long U = ctx->U;
    Engine E = make_engine(ctx);
    double* scal = engine_scalars(ctx);  // [0] |r|^2, [1] |b|^2, [6] sigma
    double* sigma = scal + 6;
    const double* dinv = ctx->A_dinv.get<double>();
    double* x = ctx->vx.ensure<double>(U + 1);
    double* r64 = ctx->vr.ensure<double>(U + 1);
    float* rhs = ctx->fph.ensure<float>(U + 1);
    Vecs<float> V{ctx->fx.ensure<float>(U + 1), ctx->fr.ensure<float>(U + 1), ctx->fr0.ensure<float>(U + 1),
                  ctx->fp.ensure<float>(U + 1), ctx->fv.ensure<float>(U + 1), ctx->fs.ensure<float>(U + 1),
                  ctx->ft.ensure<float>(U + 1)};
    const bool use_nn = learned && mpnn_ready(ctx);
    const bool warm = o->warm_start && ctx->have_solution;
    const double delta = o->inner_tol > 0 ? o->inner_tol : 0.1;  // residual drop between updates
    const int chunk = std::max(1, o->check_every > 0 ? o->check_every : 8);
    const int stall = o->stall_window > 0 ? o->stall_window : 20;
    ev_record(ctx, 10);
    Sell<double> A = sell_a64(ctx);
    Sell<float> Af = sell_scaled32(ctx);
    set_scalar_caps(E, 0, 0);  // zero the reduction tickets
    if (!warm) LSMPS_CUDA(cudaMemsetAsync(x, 0, U * sizeof(double), s));
    auto true_residual = [&]() {
        residual64(E, A, ctx->A_b.get<double>(), x, r64, scal);
        double h2[2];
        LSMPS_CUDA(cudaMemcpyAsync(h2, scal, sizeof(h2), cudaMemcpyDeviceToHost, s));
        LSMPS_CUDA(cudaStreamSynchronize(s));
        return std::make_pair(std::sqrt(h2[0]), std::sqrt(h2[1]));
    };
    auto [rnorm, bnorm] = true_residual();
    const double thresh = o->tol * std::max(1.0, bnorm);
    int total = 0, runs = 0, updates = 0, fallback = 0;
    bool converged = rnorm <= thresh;
    bool nonfinite = !std::isfinite(rnorm);
    cudaGraphExec_t exec = nullptr;
    auto read_scalars = [&](BcgScalars& h) {
        LSMPS_CUDA(cudaMemcpyAsync(&h, E.S, sizeof(h), cudaMemcpyDeviceToHost, s));
        LSMPS_CUDA(cudaStreamSynchronize(s));
    };
    while (!converged && !nonfinite && total < o->max_iter) {
        // ---- an FP32 run from the true residual: sigma = |r|, rhs = r / sigma ----
        k_start_rhs<<<1184, 256, 0, s>>>(U, r64, scal, sigma, rhs, V.x);
        LSMPS_CHECK_LAUNCH();
        const bool nn_now = use_nn && !fallback && runs == 0;
        if (nn_now) mpnn_warm_start(ctx, rhs, V.x);
        set_scalar_caps(E, o->max_iter - total, nn_now ? stall : 0);
        // FP32 threshold in the scaled system's units: |r| / sigma <= thresh / sigma
        init<float>(E, Af, rhs, V, nn_now, thresh / std::max(rnorm, 1e-300), 1.0);
        ++runs;
        if (!exec && o->use_graph) {
            cudaGraph_t graph;
            LSMPS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            for (int c = 0; c < chunk; ++c) iteration<float>(E, Af, V);
            note_launches(0 - (uint64_t)(5 * chunk));  // captured, not launched
            cudaError_t e = cudaStreamEndCapture(s, &graph);
            LSMPS_CUDA(e);
            LSMPS_CUDA(cudaGraphInstantiate(&exec, graph, 0));
            cudaGraphDestroy(graph);
        }
        BcgScalars h{};
        read_scalars(h);
        double rn_upd = h.rn;  // FP32 residual at the last update of this run
        int run_base = 0;      // iterations of this run already counted
        while (true) {
            if (!h.done) {
                if (exec) {
                    LSMPS_CUDA(cudaGraphLaunch(exec, s));
                    note_launches(5 * (uint64_t)chunk);
                } else {
                    for (int k = 0; k < chunk; ++k) iteration<float>(E, Af, V);
                    LSMPS_CHECK_LAUNCH();
                }
                read_scalars(h);
            }
            total += h.iters - run_base;
            run_base = h.iters;
            if (!h.done && h.rn > delta * rn_upd) continue;
            // ---- reliable update: fold y_lo into x_hi, true FP64 residual ----
            k_reliable_x<<<1184, 256, 0, s>>>(U, x, V.x, dinv, sigma);
            LSMPS_CHECK_LAUNCH();
            std::tie(rnorm, bnorm) = true_residual();
            ++updates;
            if (!std::isfinite(rnorm)) { nonfinite = true; break; }
            if (rnorm <= thresh) { converged = true; break; }
            if (total >= o->max_iter || h.done == 3) break;
            if (h.done) {  // breakdown, stall, or an FP32 convergence the FP64 residual denies
                if (h.done == 4 && nn_now) fallback = 1;
                break;     // restart from the true residual
            }
            k_reliable_r<<<RGRID, RB, 0, s>>>(U, r64, sigma, V.r, V.r0, E.S, E.P);
            LSMPS_CHECK_LAUNCH();
            read_scalars(h);
            rn_upd = h.rn;
            if (h.done) break;  // rho breakdown after the replacement: restart
        }
        if (h.done == 3) break;
    }
    if (exec) cudaGraphExecDestroy(exec);
    ev_record(ctx, 11);
    LSMPS_CUDA(cudaStreamSynchronize(s));
    ps->iterations = total;
    ps->outer_iterations = updates;
    ps->converged = converged && !nonfinite;
    ps->fallback = fallback;
    ps->solve_ms = ev_elapsed(ctx, 10, 11);
}

// The multigrid hierarchy set-up on the context's side stream (created at first use with the
// device's highest priority), ordered after everything the context stream held when `fork`
// was recorded; the context stream then waits for it. The set-up reads each level's size back
// to the host, so work queued on the context stream meanwhile (the network's inference) fills
// the GPU during those round trips, and the set-up's kernels take the SMs first when both wait.
static void mg_setup_on_side(lsmps_ctx* ctx) {
    cudaStream_t main = ctx->stream;
    LSMPS_CUDA(cudaStreamWaitEvent(ctx->side_stream, ctx->side_fork, 0));
    ctx->stream = ctx->side_stream;
    try {
        mg_setup(ctx);
    } catch (...) {
        ctx->stream = main;
        cudaStreamSynchronize(ctx->side_stream);
        throw;
    }
    ctx->stream = main;
    LSMPS_CUDA(cudaEventRecord(ctx->side_join, ctx->side_stream));
    LSMPS_CUDA(cudaStreamWaitEvent(main, ctx->side_join, 0));
}

static void side_stream_fork(lsmps_ctx* ctx) {
    if (!ctx->side_stream) {
        int least = 0, greatest = 0;
        LSMPS_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        LSMPS_CUDA(cudaStreamCreateWithPriority(&ctx->side_stream, cudaStreamNonBlocking, greatest));
        LSMPS_CUDA(cudaEventCreateWithFlags(&ctx->side_fork, cudaEventDisableTiming));
        LSMPS_CUDA(cudaEventCreateWithFlags(&ctx->side_join, cudaEventDisableTiming));
    }
    LSMPS_CUDA(cudaEventRecord(ctx->side_fork, ctx->stream));
}

// Mixed precision (MIXED, and LEARNED): Jacobi-BiCGStab with FP64 vectors and recurrences
// whose two SpMVs per iteration read the FP32 copy of A D^-1 (8 bytes per entry instead
// of 12: the matrix is the bandwidth). The FP32 matrix perturbs each product at ~6e-8
// relative, so the recursive residual drifts from the true one; whenever it has fallen by
// `inner_tol` (default 0.01: measured best on the 1M WLS system) since the last replacement, or the iteration stops, the true
// residual b - A D^-1 y is recomputed with the FP64 matrix and replaces it, keeping the
// search direction. Convergence is decided on that FP64 residual only. A breakdown, a
// stall (LEARNED: no 1 % progress in `stall_window` iterations) or an FP32-driven
// convergence claim the FP64 residual denies restarts the Krylov space from the current
// iterate; LEARNED starts from the network's guess and, after a stall, continues as plain
// Jacobi-BiCGStab (fallback). With the multigrid preconditioner a stall (no 1 % progress in
// `stall_window` iterations) or a breakdown ends the multigrid phase, and the solve continues
// as Jacobi MIXED from the current iterate (from zero when it is no longer finite; fallback).
// exit_res (optional): {|b - A D^-1 y|, |b|} of the returned iterate when the solve converged
// (the convergence test's own FP64 residual), else {-1, -1}.
static void solve_mixed(lsmps_ctx* ctx, const lsmps_solver_opts* o, lsmps_ppe_stats* ps, bool learned,
                        double* exit_res = nullptr) {
    cudaStream_t s = ctx->stream;
    const long long U = ctx->U;
    Engine E = make_engine(ctx);
    const double* dinv = ctx->A_dinv.get<double>();
    const double* b = ctx->A_b.get<double>();
    Vecs<double> V{ctx->vx.ensure<double>(U + 1), ctx->vr.ensure<double>(U + 1), ctx->vr0.ensure<double>(U + 1),
                   ctx->vp.ensure<double>(U + 1), ctx->vv.ensure<double>(U + 1), ctx->vs.ensure<double>(U + 1),
                   ctx->vt.ensure<double>(U + 1)};
    const bool use_nn = learned && mpnn_ready(ctx);
    const bool warm = o->warm_start && ctx->have_solution;
    const double delta = o->inner_tol > 0 ? o->inner_tol : 0.01;
    const int chunk = std::max(1, o->check_every > 0 ? o->check_every : 8);
    const int stall = o->stall_window > 0 ? o->stall_window : 20;
    ev_record(ctx, 10);
    const bool mg = o->precond == LSMPS_PRECOND_MULTIGRID;
    // y0 = |b| net(b / |b|): launches only (no host round trip)
    auto net_guess = [&] {
        float* rhs = ctx->fph.ensure<float>(U + 1);
        float* yf = ctx->fx.ensure<float>(U + 1);
        double* scal = engine_scalars(ctx);
        k_norm2<<<RGRID, RB, 0, s>>>(U, b, scal, E.P, &E.S->counter[5]);
        k_rhs_unit<<<1184, 256, 0, s>>>(U, b, rhs, scal);  // network input: b / |b| in FP32
        LSMPS_CHECK_LAUNCH();
        mpnn_warm_start(ctx, rhs, yf);
        k_y_from_net<<<1184, 256, 0, s>>>(U, yf, scal, V.x);
        LSMPS_CHECK_LAUNCH();
    };
    // LEARNED with the multigrid from a cold start: the network's guess (context stream) and
    // the hierarchy set-up (side stream) run at the same time; they read the assembled system
    // and write disjoint buffers
    const bool overlap = mg && use_nn && !warm;
    if (mg) {
        if (overlap) {
            side_stream_fork(ctx);
            net_guess();
            mg_setup_on_side(ctx);
        } else {
            mg_setup(ctx);
        }
        V.ph = ctx->vph.ensure<double>(U + 1);
        V.sh = ctx->vsh.ensure<double>(U + 1);
    }
    Sell<double> As = sell_scaled64(ctx);
    Sell<float> Af = sell_scaled32(ctx);
    set_scalar_caps(E, o->max_iter, (use_nn || mg) ? stall : 0);
    bool have_start = warm;
    double warm_rn = 0;  // |b - A x0| of a warm start the network corrected
    if (warm) {  // the iteration works on y = D x
        k_scale_by_diag<<<1184, 256, 0, s>>>(U, V.x, dinv);
        LSMPS_CHECK_LAUNCH();
        if (use_nn) {  // the network corrects the warm start: y += |r0| net(r0 / |r0|), r0 = b - A D^-1 y
            float* rhs = ctx->fph.ensure<float>(U + 1);
            float* yf = ctx->fx.ensure<float>(U + 1);
            double* scal = engine_scalars(ctx);
            residual64(E, As, b, V.x, V.r, scal);
            k_rhs_unit<<<1184, 256, 0, s>>>(U, V.r, rhs, scal);
            LSMPS_CHECK_LAUNCH();
            mpnn_warm_start(ctx, rhs, yf);
            k_y_add_net<<<1184, 256, 0, s>>>(U, yf, scal, V.x, V.p);  // the warm start kept in p
            LSMPS_CHECK_LAUNCH();
            double r2 = 0;
            LSMPS_CUDA(cudaMemcpyAsync(&r2, scal, sizeof(double), cudaMemcpyDeviceToHost, s));
            LSMPS_CUDA(cudaStreamSynchronize(s));
            warm_rn = std::sqrt(r2);
        }
    } else if (use_nn) {
        if (!overlap) net_guess();
        have_start = true;
    } else {
        LSMPS_CUDA(cudaMemsetAsync(V.x, 0, U * sizeof(double), s));
    }
    init<double, double>(E, As, b, V, have_start, o->tol, -1.0);
    auto read = [&](BcgScalars& h) {
        LSMPS_CUDA(cudaMemcpyAsync(&h, E.S, sizeof(h), cudaMemcpyDeviceToHost, s));
        LSMPS_CUDA(cudaStreamSynchronize(s));
    };
    BcgScalars h{};
    read(h);
    int total = 0, replacements = 0, restarts = 0, fallback = 0;
    if (use_nn && !warm && (!std::isfinite(h.rn) || h.rn >= h.bnorm)) {
        // the network's guess is worse than zero: discard it and run plain Jacobi-BiCGStab
        fallback = 1;
        LSMPS_CUDA(cudaMemsetAsync(V.x, 0, U * sizeof(double), s));
        set_scalar_caps(E, o->max_iter, mg ? stall : 0);
        init<double, double>(E, As, b, V, false, o->tol, -1.0);
        read(h);
    } else if (use_nn && warm && (!std::isfinite(h.rn) || h.rn >= warm_rn)) {
        // the correction made the warm start worse: go back to it
        fallback = 1;
        LSMPS_CUDA(cudaMemcpyAsync(V.x, V.p, U * sizeof(double), cudaMemcpyDeviceToDevice, s));
        set_scalar_caps(E, o->max_iter, mg ? stall : 0);
        init<double, double>(E, As, b, V, true, o->tol, -1.0);
        read(h);
    }
    bool converged = h.done == 1, failed = h.done == 2 && h.nonfinite;
    const long long max_chunks = (long long)o->max_iter / chunk + 4 + o->max_iter;  // bounded loop
    // Iterates from the scalars in h until converged, failed or the iteration cap; with the
    // multigrid (mgp), a breakdown or a stall ends the phase early and returns true instead
    // (the caller then continues without it).
    auto phase = [&](bool mgp) -> bool {
        const uint64_t kpi = (uint64_t)launches_per_iteration(ctx, mgp);
        const int restart_stall = mgp ? stall : 0;
        double rn_upd = h.rn;
        if (o->use_graph == 1) {
            if (converged || failed) return false;
            // the loop below, decided on the device: one graph launch for the whole solve
            LoopCtl* C = engine_loop_ctl(ctx);
            LoopCtl c0{};
            c0.rn_upd = rn_upd;
            c0.delta = delta;
            c0.fallback = fallback;
            c0.max_trips = (int)std::min<long long>(max_chunks, INT_MAX);
            c0.max_iter = o->max_iter;
            c0.total = total;
            c0.use_nn = use_nn ? 1 : 0;
            c0.use_mg = mgp ? 1 : 0;
            c0.stall = restart_stall;
            LSMPS_CUDA(cudaMemcpyAsync(C, &c0, sizeof(c0), cudaMemcpyHostToDevice, s));
            cudaGraphExec_t wexec = build_while_graph(s, C, [&] {
                for (int c = 0; c < chunk; ++c) iteration<double, float>(E, Af, V, mgp);
                k_mix_after_chunk<<<1, 1, 0, s>>>(E.S, C);
                launch_replace(s, As, b, V, E, &C->act, 1);
                k_mix_after_replace<<<1, 1, 0, s>>>(E.S, C);
                if (As.dcol)
                    k_bcg_init<double, double, true><<<RGRID, RB, 0, s>>>(As, b, V.x, 1, V.r, V.r0, V.p, V.v, E.S,
                                                                          E.P, o->tol, -1.0, &C->act, 2);
                else
                    k_bcg_init<double, double, false><<<RGRID, RB, 0, s>>>(As, b, V.x, 1, V.r, V.r0, V.p, V.v, E.S,
                                                                           E.P, o->tol, -1.0, &C->act, 2);
                k_mix_after_restart<<<1, 1, 0, s>>>(E.S, C);
            });
            note_launches(0 - kpi * (uint64_t)chunk);  // captured, not launched
            cudaError_t e = cudaGraphLaunch(wexec, s);
            LoopCtl hc{};
            if (e == cudaSuccess) e = cudaMemcpyAsync(&hc, C, sizeof(hc), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaMemcpyAsync(&h, E.S, sizeof(h), cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            cudaGraphExecDestroy(wexec);
            LSMPS_CUDA(e);
            note_launches((uint64_t)hc.trips * (kpi * (uint64_t)chunk + 6));
            total = hc.total;
            replacements += hc.replacements;
            restarts += hc.restarts;
            fallback = hc.fallback;
            converged = hc.state == 1;
            failed = hc.state == 2;
            return hc.state == 4;
        }
        cudaGraphExec_t exec = nullptr;
        if (o->use_graph == 2) {
            cudaGraph_t graph;
            LSMPS_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
            for (int c = 0; c < chunk; ++c) iteration<double, float>(E, Af, V, mgp);
            note_launches(0 - kpi * (uint64_t)chunk);  // captured, not launched
            cudaError_t e = cudaStreamEndCapture(s, &graph);
            LSMPS_CUDA(e);
            LSMPS_CUDA(cudaGraphInstantiate(&exec, graph, 0));
            cudaGraphDestroy(graph);
        }
        bool give_up = false;
        int base = h.iters;
        for (long long guard = 0; !converged && !failed && guard < max_chunks; ++guard) {
            if (!h.done) {
                if (exec) {
                    LSMPS_CUDA(cudaGraphLaunch(exec, s));
                    note_launches(kpi * (uint64_t)chunk);
                } else {
                    for (int k = 0; k < chunk; ++k) iteration<double, float>(E, Af, V, mgp);
                    LSMPS_CHECK_LAUNCH();
                }
                read(h);
            }
            total += h.iters - base;
            base = h.iters;
            if (!h.done && h.rn > delta * rn_upd) continue;
            const int why = h.done;  // 0: drop by delta; else the iteration stopped
            if (why == 3 || total >= o->max_iter) {
                // iteration cap: report the true residual of the last iterate
                launch_replace(s, As, b, V, E, nullptr, 0);
                LSMPS_CHECK_LAUNCH();
                read(h);
                converged = h.done == 1;
                break;
            }
            if (why == 0) {
                launch_replace(s, As, b, V, E, nullptr, 0);
                LSMPS_CHECK_LAUNCH();
                ++replacements;
                read(h);
                rn_upd = h.rn;
                if (h.done == 1) { converged = true; break; }
                if (h.done == 0) continue;
                // rho breakdown after the replacement: fall through to a restart
            }
            if (mgp && (h.done == 2 || h.done == 4)) { give_up = true; break; }
            if (why == 4 && use_nn) fallback = 1;
            if (h.nonfinite) { failed = true; break; }
            // restart from the current iterate with the FP64 matrix (true residual)
            set_scalar_caps(E, o->max_iter - total, restart_stall);
            init<double, double>(E, As, b, V, true, o->tol, -1.0);
            ++restarts;
            read(h);
            base = 0;
            rn_upd = h.rn;
            if (h.done == 1) { converged = true; break; }
            if (h.done) { failed = true; break; }
        }
        if (exec) cudaGraphExecDestroy(exec);
        return give_up;
    };
    if (phase(mg)) {
        // The multigrid broke down or stalled (near-singular aggregates can do this): continue
        // as Jacobi MIXED from the current iterate, or from zero if it is no longer finite.
        fallback = 1;
        const bool keep_x = !h.nonfinite;
        if (!keep_x) LSMPS_CUDA(cudaMemsetAsync(V.x, 0, U * sizeof(double), s));
        set_scalar_caps(E, o->max_iter - total, 0);
        init<double, double>(E, As, b, V, keep_x, o->tol, -1.0);
        ++restarts;
        read(h);
        converged = h.done == 1;
        failed = h.done == 2;
        if (total < o->max_iter) phase(false);
    }
    k_unscale<<<1184, 256, 0, s>>>(U, V.x, dinv);
    LSMPS_CHECK_LAUNCH();
    ev_record(ctx, 11);
    LSMPS_CUDA(cudaStreamSynchronize(s));
    ps->iterations = total;
    ps->outer_iterations = replacements + restarts;
    ps->converged = converged;
    ps->fallback = fallback;
    ps->solve_ms = ev_elapsed(ctx, 10, 11);
    if (exit_res) {
        // convergence is only declared right after a residual replacement or a (re)start (in
        // the device-driven loop too, which runs the same kernels in the same order), whose
        // FP64 residual b - A D^-1 y of the final iterate h holds
        const bool exact = converged && std::isfinite(h.rn);
        exit_res[0] = exact ? h.rn : -1.0;
        exit_res[1] = exact ? h.bnorm : -1.0;
    }
}

void ppe_set_initial_particles(lsmps_ctx* ctx, const double* pp, size_t n, bool device) {
    LSMPS_REQUIRE(ctx->have_ppe && !ctx->ppe_loaded, LSMPS_ERR_STATE,
                  "per-particle initial guesses need an assembled particle system");
    LSMPS_REQUIRE(n == ctx->n && (n == 0 || pp), LSMPS_ERR_ARG, "initial guess must hold one value per particle");
    cudaStream_t s = ctx->stream;
    const long long U = ctx->U;
    double* x = ctx->vx.ensure<double>(U + 1);
    const double* src = pp;
    if (!device && n) {
        double* tmp = ctx->vtmp.ensure<double>(n + 1);
        LSMPS_CUDA(cudaMemcpyAsync(tmp, pp, n * sizeof(double), cudaMemcpyHostToDevice, s));
        src = tmp;
    }
    if (U) {
        k_guess_from_particles<<<1184, 256, 0, s>>>(U, ctx->sorted_of_u.get<int>(), ctx->perm.get<int>(), src, x);
        LSMPS_CHECK_LAUNCH();
    }
    LSMPS_CUDA(cudaStreamSynchronize(s));
    ctx->have_solution = true;
}

void ppe_pressure_particles(lsmps_ctx* ctx, double* pp, size_t n, double fill, bool device) {
    LSMPS_REQUIRE(ctx->have_solution, LSMPS_ERR_STATE, "no solution: lsmps_ppe_solve first");
    LSMPS_REQUIRE(!ctx->ppe_loaded, LSMPS_ERR_STATE, "per-particle pressure needs an assembled particle system");
    LSMPS_REQUIRE(n == ctx->n && (n == 0 || pp), LSMPS_ERR_ARG, "output must hold one value per particle");
    cudaStream_t s = ctx->stream;
    const long long U = ctx->U;
    double* dst = device ? pp : ctx->vtmp.ensure<double>(n + 1);
    if (n && std::isnan(fill)) {  // keep the other particles' values
        if (!device) LSMPS_CUDA(cudaMemcpyAsync(dst, pp, n * sizeof(double), cudaMemcpyHostToDevice, s));
    } else if (n) {
        k_fill_value<<<std::min<unsigned>(blocks_for(n, 256), 1184), 256, 0, s>>>(n, fill, dst);
        LSMPS_CHECK_LAUNCH();
    }
    if (U) {
        k_solution_to_particles<<<1184, 256, 0, s>>>(U, ctx->sorted_of_u.get<int>(), ctx->perm.get<int>(),
                                                     ctx->vx.get<double>(), dst);
        LSMPS_CHECK_LAUNCH();
    }
    if (!device && n) LSMPS_CUDA(cudaMemcpyAsync(pp, dst, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    LSMPS_CUDA(cudaStreamSynchronize(s));
}

void ppe_solve(lsmps_ctx* ctx, const lsmps_solver_opts* o, lsmps_ppe_stats* out) {
    LSMPS_REQUIRE(ctx->have_ppe, LSMPS_ERR_STATE, "PPE solve needs lsmps_ppe_assemble first");
    LSMPS_REQUIRE(o && o->solver >= 0 && o->solver <= 5, LSMPS_ERR_ARG, "unknown solver");
    LSMPS_REQUIRE(o->solver != LSMPS_SOLVER_LEARNED || mpnn_ready(ctx), LSMPS_ERR_STATE,
                  "learned solver needs lsmps_mpnn_init / lsmps_mpnn_load first");
    LSMPS_REQUIRE(o->solver != LSMPS_SOLVER_LEARNED || !ctx->ppe_loaded, LSMPS_ERR_STATE,
                  "the learned solver needs an assembled particle system (its features are per particle)");
    LSMPS_REQUIRE(o->precond == LSMPS_PRECOND_JACOBI ||
                      (o->precond == LSMPS_PRECOND_MULTIGRID &&
                       (o->solver == LSMPS_SOLVER_MIXED || o->solver == LSMPS_SOLVER_LEARNED)),
                  LSMPS_ERR_ARG, "the multigrid preconditioner is for the MIXED and LEARNED solvers");
    LSMPS_REQUIRE(o->precond != LSMPS_PRECOND_MULTIGRID || !ctx->ppe_loaded, LSMPS_ERR_STATE,
                  "the multigrid preconditioner aggregates particle cells: a loaded CSR system has none");
    lsmps_ppe_stats ps = ctx->ppe_assembly;
    ps.iterations = 0;
    ps.converged = 0;
    long long U = ctx->U;
    if (U == 0) {  // src/lsmps.cpp:67: if(!n) return st;
        if (out) *out = ps;
        return;
    }
    if (o->solver == LSMPS_SOLVER_REFERENCE) {
        solve_exact(ctx, o, &ps);
    } else {
        double exit_res[2] = {-1.0, -1.0};
        if (o->solver == LSMPS_SOLVER_FP64) solve_fast64(ctx, o, &ps, false);
        else if (o->solver == LSMPS_SOLVER_JACOBI) solve_fast64(ctx, o, &ps, true);
        else if (o->solver == LSMPS_SOLVER_MIXED_F32) solve_mixed_f32(ctx, o, &ps, false);
        else solve_mixed(ctx, o, &ps, o->solver == LSMPS_SOLVER_LEARNED, exit_res);
        // final statistics in FP64: |Ax - b|, |b| (for a converged MIXED / LEARNED solve the
        // convergence test's own FP64 residual of the final iterate, |b - A D^-1 y| with
        // y = D x), error against p*
        cudaStream_t s = ctx->stream;
        Engine E = make_engine(ctx);
        double* scal = engine_scalars(ctx);
        double* x = ctx->vx.get<double>();
        double* tmp = ctx->vt.ensure<double>(U + 1);
        if (exit_res[0] < 0) residual64(E, sell_a64(ctx), ctx->A_b.get<double>(), x, tmp, scal);
        auto* maxbits = reinterpret_cast<unsigned long long*>(scal + 4);
        LSMPS_CUDA(cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long), s));
        k_error_stats<<<RGRID, RB, 0, s>>>(U, x, ctx->A_xexact.get<double>(), scal + 2, E.P, &E.S->counter[6],
                                            maxbits);
        LSMPS_CHECK_LAUNCH();
        double h[5];
        LSMPS_CUDA(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, s));
        LSMPS_CUDA(cudaStreamSynchronize(s));
        ps.initial_residual = exit_res[0] < 0 ? std::sqrt(h[1]) : exit_res[1];
        ps.final_residual = exit_res[0] < 0 ? std::sqrt(h[0]) : exit_res[0];
        ps.relative_residual = ps.final_residual / std::max(ps.initial_residual, 1e-300);
        ps.relative_l2_error = std::sqrt(h[2] / std::max(h[3], 1e-30));
        unsigned long long mb;
        std::memcpy(&mb, &h[4], sizeof(mb));
        double mx;
        std::memcpy(&mx, &mb, sizeof(mx));
        ps.max_error = mx;
        if (!std::isfinite(ps.final_residual)) ps.converged = 0;
    }
    ctx->have_solution = true;
    ctx->timings[5] = ps.solve_ms;
    if (out) *out = ps;
}

// The solver's SpMV as the iterations run it: LSMPS_KB_SPMV32 is the MIXED solver's kernel
// (FP32 A D^-1 values, FP64 vectors), LSMPS_KB_SPMV64 the plain FP64 solver's (FP64 A).
void solver_kernel_bench(lsmps_ctx* ctx, int kernel, int reps, double* ms, double* bytes) {
    LSMPS_REQUIRE(ctx->have_ppe, LSMPS_ERR_STATE, "SpMV bench needs an assembled PPE");
    cudaStream_t s = ctx->stream;
    const long long U = ctx->U;
    Engine E = make_engine(ctx);
    BcgScalars init{};
    init.max_iter = 1 << 30;
    init.rho = 1.0;
    LSMPS_CUDA(cudaMemcpyAsync(E.S, &init, sizeof(init), cudaMemcpyHostToDevice, s));
    const bool f32 = kernel == LSMPS_KB_SPMV32;
    // operands of ones: the fused dot is then nonzero, so no breakdown guard stops the kernel
    double* x = ctx->vp.ensure<double>(U + 1);
    double* r0 = ctx->vr0.ensure<double>(U + 1);
    double* y = ctx->vv.ensure<double>(U + 1);
    k_fill<double><<<1184, 256, 0, s>>>(U, x, 1.0);
    k_fill<double><<<1184, 256, 0, s>>>(U, r0, 1.0);
    LSMPS_CHECK_LAUNCH();
    Sell<float> Af{};
    Sell<double> Ad{};
    if (f32) Af = sell_scaled32(ctx);
    else Ad = sell_a64(ctx);
    auto launch = [&] {
        if (f32 && Af.dcol) k_bcg_v<double, float, true><<<spmv_grid<float, true>(), RB, 0, s>>>(Af, x, y, r0, E.S, E.P);
        else if (f32) k_bcg_v<double, float, false><<<RGRID, RB, 0, s>>>(Af, x, y, r0, E.S, E.P);
        else if (Ad.dcol) k_bcg_v<double, double, true><<<RGRID, RB, 0, s>>>(Ad, x, y, r0, E.S, E.P);
        else k_bcg_v<double, double, false><<<RGRID, RB, 0, s>>>(Ad, x, y, r0, E.S, E.P);
        LSMPS_CHECK_LAUNCH();
    };
    launch();
    ev_record(ctx, 14);
    for (int r = 0; r < reps; ++r) launch();
    ev_record(ctx, 15);
    *ms = ev_elapsed(ctx, 14, 15) / reps;
    // algorithmic bytes: values + columns of the nonzeros (not the padding), the x gathers
    // counted once, y written, r0 read (FP64 vectors), slice pointers and lengths
    const double nnz = (double)ctx->nnz;
    // values + columns (2 bytes as steps, plus a 4-byte first column per row) per entry
    *bytes = ((f32 ? 4.0 : 8.0) + (ctx->have_steps ? 2.0 : 4.0)) * nnz + (ctx->have_steps ? 28.25 : 24.25) * U;
    // the bench overwrote solver vectors: a warm start from them is no longer valid
    ctx->have_solution = false;
}

__global__ void k_to_ref(const double* __restrict__ x, const int* __restrict__ u_of_ref, long long U,
                         double* __restrict__ out) {
    long long rr = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (rr < U) out[rr] = x[u_of_ref[rr]];
}

void ppe_download_pressure(lsmps_ctx* ctx, double* p, size_t u) {
    LSMPS_REQUIRE(ctx->have_solution, LSMPS_ERR_STATE, "no PPE solution");
    LSMPS_REQUIRE((long long)u == ctx->U, LSMPS_ERR_ARG, "pressure buffer size differs from the unknown count");
    if (!u) return;
    double* tmp = ctx->vtmp.ensure<double>(u + 1);
    k_to_ref<<<blocks_for(u, 256), 256, 0, ctx->stream>>>(ctx->vx.get<double>(), ctx->u_of_ref.get<int>(),
                                                          (long long)u, tmp);
    LSMPS_CHECK_LAUNCH();
    LSMPS_CUDA(cudaMemcpyAsync(p, tmp, u * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    LSMPS_CUDA(cudaStreamSynchronize(ctx->stream));
}

// The same values without waiting: reordered into a staging buffer on the context stream,
// then copied to the host on the context's copy stream, so the next step's kernels run while
// the copy is in flight. The staging buffer is reused by the next call, which therefore first
// orders the context stream after the previous copy.
void ppe_download_pressure_async(lsmps_ctx* ctx, double* p, size_t u) {
    LSMPS_REQUIRE(ctx->have_solution, LSMPS_ERR_STATE, "no PPE solution");
    LSMPS_REQUIRE((long long)u == ctx->U, LSMPS_ERR_ARG, "pressure buffer size differs from the unknown count");
    if (!u) return;
    if (!ctx->copy_stream) LSMPS_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    if (!ctx->dl_ready) {
        LSMPS_CUDA(cudaEventCreateWithFlags(&ctx->dl_ready, cudaEventDisableTiming));
        LSMPS_CUDA(cudaEventCreateWithFlags(&ctx->dl_done, cudaEventDisableTiming));
    }
    if (ctx->dl_pending) {
        if (ctx->dl_stage.bytes < (u + 1) * sizeof(double)) {  // growing frees the copy's source
            LSMPS_CUDA(cudaEventSynchronize(ctx->dl_done));
            ctx->dl_pending = false;
        } else {
            LSMPS_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->dl_done, 0));
        }
    }
    double* st = ctx->dl_stage.ensure<double>(u + 1);
    k_to_ref<<<blocks_for(u, 256), 256, 0, ctx->stream>>>(ctx->vx.get<double>(), ctx->u_of_ref.get<int>(),
                                                          (long long)u, st);
    LSMPS_CHECK_LAUNCH();
    LSMPS_CUDA(cudaEventRecord(ctx->dl_ready, ctx->stream));
    LSMPS_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->dl_ready, 0));
    LSMPS_CUDA(cudaMemcpyAsync(p, st, u * sizeof(double), cudaMemcpyDeviceToHost, ctx->copy_stream));
    LSMPS_CUDA(cudaEventRecord(ctx->dl_done, ctx->copy_stream));
    ctx->dl_pending = true;
}

void ppe_download_wait(lsmps_ctx* ctx) {
    if (!ctx->dl_pending) return;
    LSMPS_CUDA(cudaEventSynchronize(ctx->dl_done));
    ctx->dl_pending = false;
}

}  // namespace lsmps_gpu
