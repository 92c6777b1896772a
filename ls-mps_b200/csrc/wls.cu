// Second-order 3-D WLS on sm_100a: the 9x9 moment matrix M = sum w q q^T / sum w over a
// particle's neighbor row, its Cholesky factor (with the reference's regularisation
// retries) and multi-RHS solves.
//
// Mode 0 reproduces the reference's wls_test (src/lsmps.cpp:22-25,28) bit for bit: the
// strided sample is evaluated one thread per candidate with exactly rounded FP64
// operations in the reference's order, then one thread replays the reference's
// sequential bookkeeping (stop after wls_samples successes, error sums in sample order).
//
// Mode 1 is the batched form over every particle: one thread per particle in cell-sorted
// order (neighbors of adjacent threads share cells, so the position gathers hit L1),
// the packed lower triangle of M in registers, in-place Cholesky, solves for up to three
// quadratic fields plus the Laplacian vector z = M^-1 (e3 + e4 + e5) that the WLS-Laplacian
// PPE rows use. Precision 1 factors in FP32 and refines each solve against the FP64 M;
// a system whose FP32 factorisation fails or that needed regularisation is refactored
// in FP64.
#include <cmath>
#include <vector>

#include "ops.cuh"

namespace lsmps_gpu {
namespace {

constexpr int NT = 45;  // packed lower triangle of a 9x9 matrix
__host__ __device__ constexpr int tri(int a, int c) { return a * (a + 1) / 2 + c; }  // c <= a

enum WlsStatus : int { W_OK = 0, W_REG = 1, W_SKIP = 2, W_NOWEIGHT = 3, W_CHOLFAIL = 4 };

// ---------------- exact (reference-identical) helpers -----------------------------------
// The reference's test field (src/lsmps.cpp:28), accumulated left to right.
__device__ double xquad(const double* c, double x, double y, double z) {
    double t = xadd(c[0], xmul(c[1], x));
    t = xadd(t, xmul(c[2], y));
    t = xadd(t, xmul(c[3], z));
    t = xadd(t, xmul(xmul(c[4], x), x));
    t = xadd(t, xmul(xmul(c[5], y), y));
    t = xadd(t, xmul(xmul(c[6], z), z));
    t = xadd(t, xmul(xmul(c[7], x), y));
    t = xadd(t, xmul(xmul(c[8], x), z));
    t = xadd(t, xmul(xmul(c[9], y), z));
    return t;
}

__constant__ double kRefQuad[10] = {1, 2, -3, 0.5, 0.7, -0.2, 0.4, 0.3, -0.1, 0.25};

// basis (src/lsmps.cpp:23), exact operation order.
__device__ void xbasis(double dx, double dy, double dz, double r, double l0, double* q) {
    double ir = xdiv(1.0, r);
    q[0] = xmul(dx, ir);
    q[1] = xmul(dy, ir);
    q[2] = xmul(dz, ir);
    double two_l0_r = xmul(xmul(2.0, l0), r), l0_r = xmul(l0, r);
    q[3] = xdiv(xmul(dx, dx), two_l0_r);
    q[4] = xdiv(xmul(dy, dy), two_l0_r);
    q[5] = xdiv(xmul(dz, dz), two_l0_r);
    q[6] = xdiv(xmul(dx, dy), l0_r);
    q[7] = xdiv(xmul(dx, dz), l0_r);
    q[8] = xdiv(xmul(dy, dz), l0_r);
}

// cholesky (src/lsmps.cpp:24) on a full row-major 9x9 (only the lower triangle is read).
__device__ bool xcholesky(double* a, double reg, bool& used) {
    used = false;
    double m[K * K];
    for (int at = 0; at < 5; ++at) {
        for (int t = 0; t < K * K; ++t) m[t] = a[t];
        // reg * pow(10, at - 1): the powers 1, 10, 100, 1000 are exact
        double add = at ? xmul(reg, at == 1 ? 1.0 : at == 2 ? 10.0 : at == 3 ? 100.0 : 1000.0) : 0.0;
        if (add != 0.0) {
            used = true;
            for (int i = 0; i < K; ++i) m[i * K + i] = xadd(m[i * K + i], add);
        }
        bool ok = true;
        for (int i = 0; i < K && ok; ++i) {
            for (int j = 0; j <= i; ++j) {
                double s = m[i * K + j];
                for (int k = 0; k < j; ++k) s = xsub(s, xmul(m[i * K + k], m[j * K + k]));
                if (i == j) {
                    if (!(s > 1e-14) || !isfinite(s)) { ok = false; break; }
                    m[i * K + j] = __dsqrt_rn(s);
                } else {
                    m[i * K + j] = xdiv(s, m[j * K + j]);
                }
            }
            for (int j = i + 1; j < K; ++j) m[i * K + j] = 0;
        }
        if (ok) {
            for (int t = 0; t < K * K; ++t) a[t] = m[t];
            return true;
        }
    }
    return false;
}

// solve (src/lsmps.cpp:25).
__device__ void xsolve(const double* l, const double* b, double* x) {
    double y[K];
    for (int i = 0; i < K; ++i) {
        double s = b[i];
        for (int k = 0; k < i; ++k) s = xsub(s, xmul(l[i * K + k], y[k]));
        y[i] = xdiv(s, l[i * K + i]);
    }
    for (int i = K - 1; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < K; ++k) s = xsub(s, xmul(l[k * K + i], x[k]));
        x[i] = xdiv(s, l[i * K + i]);
    }
}

struct SampleOut {
    int status;   // WlsStatus
    int virt;     // NearWall / FreeSurface with sum w > 0
    double ge, le;
};

// Mode 0: one thread per strided candidate i = c * stride (caller order).
__global__ void k_wls_sample(const int* __restrict__ iperm, const uint8_t* __restrict__ cls,
                             const double* __restrict__ sx, const double* __restrict__ sy,
                             const double* __restrict__ sz, const int* __restrict__ row,
                             const int* __restrict__ col, long long ncand, long long stride, double re,
                             double l0, double reg, SampleOut* __restrict__ out) {
    long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= ncand) return;
    long long i = c * stride;
    int k = iperm[i];
    uint8_t t = cls[k];
    SampleOut o{W_SKIP, 0, 0.0, 0.0};
    if (t == LSMPS_WALL || t == LSMPS_SPLASH) { out[c] = o; return; }
    double M[K * K];
    double b[K];
    for (int a = 0; a < K * K; ++a) M[a] = 0;
    for (int a = 0; a < K; ++a) b[a] = 0;
    double xi = sx[k], yi = sy[k], zi = sz[k];
    double ws = 0, fi = xquad(kRefQuad, xi, yi, zi);
    for (int e = row[k]; e < row[k + 1]; ++e) {
        int m = col[e];
        double dx = xsub(sx[m], xi), dy = xsub(sy[m], yi), dz = xsub(sz[m], zi);
        double r = __dsqrt_rn(xnorm2(dx, dy, dz)), w = xweight(r, re);
        if (w == 0.0) continue;
        double q[K];
        xbasis(dx, dy, dz, r, l0, q);
        double df = xsub(xquad(kRefQuad, sx[m], sy[m], sz[m]), fi);
        ws = xadd(ws, w);
        for (int a = 0; a < K; ++a) {
            double wq = xmul(w, q[a]);
            b[a] = xadd(b[a], xdiv(xmul(wq, df), r));
            for (int cc = 0; cc <= a; ++cc) M[a * K + cc] = xadd(M[a * K + cc], xmul(wq, q[cc]));
        }
    }
    if (ws <= 0) { o.status = W_NOWEIGHT; out[c] = o; return; }
    for (int a = 0; a < K * K; ++a) M[a] = xdiv(M[a], ws);
    for (int a = 0; a < K; ++a) b[a] = xdiv(b[a], ws);
    o.virt = (t == LSMPS_NEAR_WALL || t == LSMPS_FREE_SURFACE) ? 1 : 0;
    bool used = false;
    if (!xcholesky(M, reg, used)) { o.status = W_CHOLFAIL; out[c] = o; return; }
    double x[K];
    xsolve(M, b, x);
    // analytic gradient of the test field, in the reference's expression order
    double ex = xsub(xadd(xadd(2.0, xmul(1.4, xi)), xmul(.3, yi)), xmul(.1, zi));
    double ey = xadd(xadd(xsub(-3.0, xmul(.4, yi)), xmul(.3, xi)), xmul(.25, zi));
    double ez = xadd(xsub(xadd(.5, xmul(.8, zi)), xmul(.1, xi)), xmul(.25, yi));
    o.ge = __dsqrt_rn(xnorm2(xsub(x[0], ex), xsub(x[1], ey), xsub(x[2], ez)));
    o.le = fabs(xsub(xdiv(xadd(xadd(x[3], x[4]), x[5]), l0), 1.8));
    o.status = used ? W_REG : W_OK;
    out[c] = o;
}

// Sequential bookkeeping of wls_test over the candidates in order.
// res: sampled, ok, regularized, failed, virtual (as doubles), max_g, rms_g, max_l, rms_l.
__global__ void k_wls_sample_reduce(const SampleOut* __restrict__ in, long long ncand,
                                    unsigned long long cap, double* res) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long sampled = 0, ok = 0, regd = 0, failed = 0, virt = 0;
    double mg = 0, ml = 0, seG = 0, seL = 0;
    for (long long c = 0; c < ncand && sampled < cap; ++c) {
        SampleOut o = in[c];
        if (o.status == W_SKIP) continue;
        if (o.status == W_NOWEIGHT) { failed++; continue; }
        if (o.virt) virt++;
        if (o.status == W_CHOLFAIL) { failed++; continue; }
        sampled++;
        if (o.status == W_REG) regd++; else ok++;
        mg = fmax(mg, o.ge);
        ml = fmax(ml, o.le);
        seG = xadd(seG, xmul(o.ge, o.ge));
        seL = xadd(seL, xmul(o.le, o.le));
    }
    res[0] = (double)sampled; res[1] = (double)ok; res[2] = (double)regd; res[3] = (double)failed;
    res[4] = (double)virt;
    res[5] = mg;
    res[6] = sampled ? __dsqrt_rn(xdiv(seG, (double)sampled)) : 0.0;
    res[7] = ml;
    res[8] = sampled ? __dsqrt_rn(xdiv(seL, (double)sampled)) : 0.0;
}

// ---------------- mode 1: batched over every particle ------------------------------------
struct WlsParams {
    double re, l0, reg;
    int nrhs;
    int precision;
    int store;
    int mirror_walls;  // wall neighbors take the particle's own field values (zero normal gradient)
    double coef[30];  // nrhs x 10
};

__device__ __forceinline__ double quad_fast(const double* c, double x, double y, double z) {
    return c[0] + c[1] * x + c[2] * y + c[3] * z + c[4] * x * x + c[5] * y * y + c[6] * z * z + c[7] * x * y +
           c[8] * x * z + c[9] * y * z;
}

// Every basis function of the reference (src/lsmps.cpp:23) is one power of 1/r times a monomial
// of (dx, dy, dz) times a constant: q_a = c_a mono_a(d) / r with mono = x, y, z, xx, yy, zz,
// xy, xz, yz and c = 1, 1, 1, 1/(2 l0) x 3, 1/l0 x 3. So M_ac = sum w q_a q_c = c_a c_c
// sum (w / r^2) mono_a mono_c, and the 45 moments are 31 distinct sums T over the monomials of
// degree 2 to 4 of W d, W = w / r^2 (degree 2 xx xy xz yy yz zz, then degree 3 and 4 in the
// same order: descending x exponent, then descending y exponent). A neighbor costs 43 FP64
// operations for the moments instead of 9 basis products, 9 weight products and 45 FMAs.
constexpr int NMONO = 31;
__host__ __device__ constexpr int basis_exp(int a, int axis) {  // exponent of axis in mono_a
    return a < 3 ? (a == axis) : a < 6 ? 2 * (a - 3 == axis) : (a == 6 ? axis != 2 : a == 7 ? axis != 1 : axis != 0);
}
__host__ __device__ constexpr int mono_index(int ex, int ey, int ez) {  // position among T
    const int d = ex + ey + ez;
    int pos = d == 2 ? 0 : d == 3 ? 6 : 16;
    for (int e = d; e > ex; --e) pos += d - e + 1;  // monomials with a larger x exponent
    return pos + (d - ex - ey);
}
__host__ __device__ constexpr int moment_mono(int a, int c) {
    return mono_index(basis_exp(a, 0) + basis_exp(c, 0), basis_exp(a, 1) + basis_exp(c, 1),
                      basis_exp(a, 2) + basis_exp(c, 2));
}
static_assert(moment_mono(0, 0) == 0 && moment_mono(1, 2) == 4 && moment_mono(5, 5) == 30 &&
                  moment_mono(3, 4) == 19 && moment_mono(6, 6) == 19 && moment_mono(8, 0) == 10 &&
                  moment_mono(7, 2) == 11 && moment_mono(4, 8) == 27,
              "monomial numbering");
__device__ __forceinline__ double basis_const(int a, double l0inv) {
    return a < 3 ? 1.0 : a < 6 ? 0.5 * l0inv : l0inv;
}

// Adds one neighbor's W d-monomials to T; p = (xx, xy, xz, yy, yz, zz) of d.
__device__ __forceinline__ void add_monomials(double W, double dx, double dy, double dz, const double* p,
                                              double* T) {
    const double bxx = W * p[0], bxy = W * p[1], bxz = W * p[2], byy = W * p[3], byz = W * p[4], bzz = W * p[5];
    T[0] += bxx, T[1] += bxy, T[2] += bxz, T[3] += byy, T[4] += byz, T[5] += bzz;
    T[6] += bxx * dx, T[7] += bxx * dy, T[8] += bxx * dz, T[9] += byy * dx, T[10] += bxy * dz;
    T[11] += bzz * dx, T[12] += byy * dy, T[13] += byy * dz, T[14] += bzz * dy, T[15] += bzz * dz;
    T[16] += bxx * p[0], T[17] += bxx * p[1], T[18] += bxx * p[2], T[19] += bxx * p[3], T[20] += bxx * p[4];
    T[21] += bxx * p[5], T[22] += byy * p[1], T[23] += byy * p[2], T[24] += bzz * p[1], T[25] += bzz * p[2];
    T[26] += byy * p[3], T[27] += byy * p[4], T[28] += byy * p[5], T[29] += bzz * p[4], T[30] += bzz * p[5];
}

// The packed normalised moments from the monomial sums (M = 0 where sum w is 0).
__device__ __forceinline__ void moments_from_sums(const double* T, double ws, double l0inv, double* M) {
    const double inv = ws > 0 ? 1.0 / ws : 0.0;
#pragma unroll
    for (int a = 0; a < K; ++a)
#pragma unroll
        for (int c = 0; c <= a; ++c)
            M[tri(a, c)] = basis_const(a, l0inv) * basis_const(c, l0inv) * inv * T[moment_mono(a, c)];
}

// Accumulates the normalised packed moment matrix of particle k; returns sum w.
__device__ __forceinline__ double accumulate_moments(int k, const double* __restrict__ sx,
                                                     const double* __restrict__ sy,
                                                     const double* __restrict__ sz,
                                                     const int* __restrict__ row,
                                                     const int* __restrict__ col, double re, double l0inv,
                                                     double* M) {
    double T[NMONO];
#pragma unroll
    for (int t = 0; t < NMONO; ++t) T[t] = 0;
    const double xi = sx[k], yi = sy[k], zi = sz[k];
    double ws = 0;
    for (int e = row[k]; e < row[k + 1]; ++e) {
        const int m = col[e];
        const double dx = sx[m] - xi, dy = sy[m] - yi, dz = sz[m] - zi;
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 > 1e-24) || r2 >= re * re) continue;  // r <= 1e-12 or r >= re: weight 0
        const double ir = rsqrt(r2);                     // 1 / r without a square root and a division
        const double qq = re * ir - 1.0;
        const double w = qq * qq;
        const double p[6] = {dx * dx, dx * dy, dx * dz, dy * dy, dy * dz, dz * dz};
        ws += w;
        add_monomials(w * (ir * ir), dx, dy, dz, p, T);
    }
    moments_from_sums(T, ws, l0inv, M);
    return ws;
}

// One pass over the neighbors for both the moments (as accumulate_moments) and the
// right-hand sides B[f]_a = sum w q_a (f_m - f_k) / r = c_a sum W (f_m - f_k) mono_a, in the
// neighbor order. Returns sum w.
template <int NRHS>
__device__ __forceinline__ double accumulate_moments_rhs(int k, const double* __restrict__ sx,
                                                         const double* __restrict__ sy,
                                                         const double* __restrict__ sz,
                                                         const int* __restrict__ row, const int* __restrict__ col,
                                                         const uint8_t* __restrict__ cls, const WlsParams& P,
                                                         double l0inv, const double* __restrict__ fvals,
                                                         const double* fi, double* M, double (*B)[K]) {
    double T[NMONO];
#pragma unroll
    for (int t = 0; t < NMONO; ++t) T[t] = 0;
#pragma unroll
    for (int f = 0; f < NRHS; ++f)
#pragma unroll
        for (int a = 0; a < K; ++a) B[f][a] = 0;
    const double xi = sx[k], yi = sy[k], zi = sz[k];
    double ws = 0;
    for (int e = row[k]; e < row[k + 1]; ++e) {
        const int m = col[e];
        const double xm = sx[m], ym = sy[m], zm = sz[m];
        const double dx = xm - xi, dy = ym - yi, dz = zm - zi;
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 > 1e-24) || r2 >= P.re * P.re) continue;  // r <= 1e-12 or r >= re: weight 0
        const double ir = rsqrt(r2);                         // 1 / r without a square root and a division
        const double qq = P.re * ir - 1.0;
        const double w = qq * qq;
        const double W = w * (ir * ir);
        const double p[6] = {dx * dx, dx * dy, dx * dz, dy * dy, dy * dz, dz * dz};
        ws += w;
        add_monomials(W, dx, dy, dz, p, T);
        if (P.mirror_walls && cls[m] == LSMPS_WALL) continue;  // f_m = f_k: no right-hand-side term
#pragma unroll
        for (int f = 0; f < NRHS; ++f) {
            const double fm = fvals ? fvals[(size_t)m * NRHS + f] : quad_fast(P.coef + 10 * f, xm, ym, zm);
            const double g = (fm - fi[f]) * W;
            B[f][0] += g * dx, B[f][1] += g * dy, B[f][2] += g * dz;
            B[f][3] += g * p[0], B[f][4] += g * p[3], B[f][5] += g * p[5];
            B[f][6] += g * p[1], B[f][7] += g * p[2], B[f][8] += g * p[4];
        }
    }
#pragma unroll
    for (int f = 0; f < NRHS; ++f)
#pragma unroll
        for (int a = 0; a < K; ++a) B[f][a] *= basis_const(a, l0inv);
    moments_from_sums(T, ws, l0inv, M);
    return ws;
}

// In-place packed Cholesky (reference pivot rule: > 1e-14 and finite) with diagonal add. The
// diagonal slots receive the reciprocals 1 / L_ii (one reciprocal square root per pivot), so
// the factor and both triangular solves multiply instead of dividing.
__device__ __forceinline__ double recip_sqrt(double s) { return rsqrt(s); }
__device__ __forceinline__ float recip_sqrt(float s) { return rsqrtf(s); }
template <class T>
__device__ __forceinline__ bool chol_packed(T* L, T add) {
#pragma unroll
    for (int i = 0; i < K; ++i) {
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            T s = L[tri(i, j)];
            if (i == j) s += add;
#pragma unroll
            for (int k = 0; k < j; ++k) s -= L[tri(i, k)] * L[tri(j, k)];
            if (i == j) {
                if (!(s > (T)1e-14) || !isfinite(s)) return false;
                L[tri(i, i)] = recip_sqrt(s);
            } else {
                L[tri(i, j)] = s * L[tri(j, j)];
            }
        }
    }
    return true;
}

template <class T>
__device__ __forceinline__ void solve_packed(const T* L, T* x) {  // x holds b on entry
#pragma unroll
    for (int i = 0; i < K; ++i) {
        T s = x[i];
#pragma unroll
        for (int k = 0; k < i; ++k) s -= L[tri(i, k)] * x[k];
        x[i] = s * L[tri(i, i)];
    }
#pragma unroll
    for (int i = K - 1; i >= 0; --i) {
        T s = x[i];
#pragma unroll
        for (int k = i + 1; k < K; ++k) s -= L[tri(k, i)] * x[k];
        x[i] = s * L[tri(i, i)];
    }
}

// Per-block statistics: counts (u64) [0] ok [1] reg [2] skip [3] noweight [4] cholfail
// [5] virtual [6] fp64 fallback; sums (f64) [0] se_grad [1] se_lap [2] max_grad [3] max_lap
struct WlsAccum {
    unsigned long long cnt[8];
    double se_g, se_l, mx_g, mx_l;
};

__device__ void atomic_max_nonneg(double* addr, double v) {
    atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// The right-hand sides accumulate in the moments' neighbor pass (one pass over the neighbors;
// measured 22 % faster at 1M particles than a second right-hand-side pass, for 2 more registers).
// MINB > 1 caps the registers so that MINB blocks of 128 threads fit an SM (the Cholesky's
// values spill to L1; the neighbor pass stays in registers).
template <int NRHS, int PREC, int MINB>
__global__ void __launch_bounds__(128, MINB) k_wls_all(WlsParams P, int n, const uint8_t* __restrict__ cls,
                                                 const double* __restrict__ sx, const double* __restrict__ sy,
                                                 const double* __restrict__ sz, const int* __restrict__ row,
                                                 const int* __restrict__ col, int* __restrict__ status,
                                                 double* __restrict__ zout, double* __restrict__ wsum,
                                                 double* __restrict__ xout, unsigned long long* gcnt,
                                                 double* gsum, const double* __restrict__ fvals) {
    __shared__ unsigned long long s_cnt[8];
    __shared__ double s_sum[4];
    if (threadIdx.x < 8) s_cnt[threadIdx.x] = 0;
    if (threadIdx.x < 4) s_sum[threadIdx.x] = 0;
    __syncthreads();
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    int my_status = -1, my_virt = 0, my_fb = 0;
    double se_g = 0, se_l = 0, mx_g = 0, mx_l = 0;
    if (k < n) {
        uint8_t t = cls[k];
        const double l0inv = 1.0 / P.l0;
        if (t == LSMPS_WALL || t == LSMPS_SPLASH) {
            my_status = W_SKIP;
            wsum[k] = 0;
#pragma unroll
            for (int a = 0; a < K; ++a) zout[(size_t)k * K + a] = 0;
        } else {
            double L[NT];
            const double xi = sx[k], yi = sy[k], zi = sz[k];
            // right-hand sides: the quadratic fields (the Laplacian vector is solved separately)
            double B[NRHS][K];
            // field values: per-particle array (sorted order, NRHS per particle) or the
            // analytic quadratics
            double fi[NRHS];
#pragma unroll
            for (int f = 0; f < NRHS; ++f)
                fi[f] = fvals ? fvals[(size_t)k * NRHS + f] : quad_fast(P.coef + 10 * f, xi, yi, zi);
            double ws = accumulate_moments_rhs<NRHS>(k, sx, sy, sz, row, col, cls, P, l0inv, fvals, fi, L, B);
            wsum[k] = ws;
            if (!(ws > 0)) {
                my_status = W_NOWEIGHT;
#pragma unroll
                for (int a = 0; a < K; ++a) zout[(size_t)k * K + a] = 0;
            } else {
                my_virt = (t == LSMPS_NEAR_WALL || t == LSMPS_FREE_SURFACE) ? 1 : 0;
                bool ok = false, used = false, fp32 = false;
                float Lf[PREC ? NT : 1];
                if (PREC) {
#pragma unroll
                    for (int a = 0; a < NT; ++a) Lf[a] = (float)L[a];
                    fp32 = chol_packed<float>(Lf, 0.0f);
                    if (fp32) {
                        // ill-conditioned systems go to FP64: squared pivot ratio below 1e-3
                        // (the factor holds the pivots' reciprocals: the smallest pivot is the
                        // reciprocal of the largest one stored)
                        float rmin = Lf[0], rmax = Lf[0];
#pragma unroll
                        for (int a = 1; a < K; ++a) {
                            rmin = fminf(rmin, Lf[tri(a, a)]);
                            rmax = fmaxf(rmax, Lf[tri(a, a)]);
                        }
                        if (rmin * rmin < 1e-3f * rmax * rmax) fp32 = false;
                    }
                }
                if (fp32) {
                    ok = true;
                } else {
                    // FP64 factorisation with the reference's retries (re-accumulating M, whose
                    // packed storage the failed attempt overwrote).
                    for (int at = 0; at < 5 && !ok; ++at) {
                        if (at > 0 || PREC) accumulate_moments(k, sx, sy, sz, row, col, P.re, l0inv, L);
                        double add = at ? P.reg * (at == 1 ? 1.0 : at == 2 ? 10.0 : at == 3 ? 100.0 : 1000.0) : 0.0;
                        used = at > 0;
                        ok = chol_packed<double>(L, add);
                    }
                    if (PREC) my_fb = 1;
                }
                if (!ok) {
                    my_status = W_CHOLFAIL;
#pragma unroll
                    for (int a = 0; a < K; ++a) zout[(size_t)k * K + a] = 0;
                } else {
                    my_status = used ? W_REG : W_OK;
                    double inv = 1.0 / ws;
                    double z[K] = {0, 0, 0, 1, 1, 1, 0, 0, 0};
                    if (PREC && fp32) {
                        // FP32 solves refined against the FP64 moments (three sweeps); L still
                        // holds the FP64 moments because the FP32 factor lives in Lf.
                        const double* Md = L;
                        auto refine = [&](double* x) {
                            double bb[K];
#pragma unroll
                            for (int a = 0; a < K; ++a) bb[a] = x[a];
                            float xf[K];
#pragma unroll
                            for (int a = 0; a < K; ++a) xf[a] = (float)bb[a];
                            solve_packed<float>(Lf, xf);
#pragma unroll
                            for (int a = 0; a < K; ++a) x[a] = xf[a];
#pragma unroll
                            for (int sweep = 0; sweep < 3; ++sweep) {
                                float rf[K];
#pragma unroll
                                for (int a = 0; a < K; ++a) {
                                    double s = bb[a];
#pragma unroll
                                    for (int c = 0; c < K; ++c)
                                        s -= Md[a >= c ? tri(a, c) : tri(c, a)] * x[c];
                                    rf[a] = (float)s;
                                }
                                solve_packed<float>(Lf, rf);
#pragma unroll
                                for (int a = 0; a < K; ++a) x[a] += (double)rf[a];
                            }
                        };
                        refine(z);
#pragma unroll
                        for (int f = 0; f < NRHS; ++f) {
#pragma unroll
                            for (int a = 0; a < K; ++a) B[f][a] *= inv;
                            refine(B[f]);
                        }
                    } else {
                        solve_packed<double>(L, z);
#pragma unroll
                        for (int f = 0; f < NRHS; ++f) {
#pragma unroll
                            for (int a = 0; a < K; ++a) B[f][a] *= inv;
                            solve_packed<double>(L, B[f]);
                        }
                    }
#pragma unroll
                    for (int a = 0; a < K; ++a) zout[(size_t)k * K + a] = z[a];
#pragma unroll
                    for (int f = 0; f < NRHS; ++f) {
                        if (P.store)
#pragma unroll
                            for (int a = 0; a < K; ++a) xout[((size_t)k * NRHS + f) * K + a] = B[f][a];
                        if (fvals) continue;  // no analytic field to measure against
                        const double* c = P.coef + 10 * f;
                        double gx = c[1] + 2 * c[4] * xi + c[7] * yi + c[8] * zi;
                        double gy = c[2] + 2 * c[5] * yi + c[7] * xi + c[9] * zi;
                        double gz = c[3] + 2 * c[6] * zi + c[8] * xi + c[9] * yi;
                        double lap = 2 * (c[4] + c[5] + c[6]);
                        double ex = B[f][0] - gx, ey = B[f][1] - gy, ez = B[f][2] - gz;
                        double ge = sqrt(ex * ex + ey * ey + ez * ez);
                        double le = fabs((B[f][3] + B[f][4] + B[f][5]) * l0inv - lap);
                        se_g += ge * ge;
                        se_l += le * le;
                        mx_g = fmax(mx_g, ge);
                        mx_l = fmax(mx_l, le);
                    }
                }
            }
        }
        status[k] = my_status;
    }
    // block reduction of the statistics
    if (my_status >= 0) atomicAdd(&s_cnt[my_status], 1ull);
    if (my_virt) atomicAdd(&s_cnt[5], 1ull);
    if (my_fb) atomicAdd(&s_cnt[6], 1ull);
    se_g = warp_sum(se_g);
    se_l = warp_sum(se_l);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx_g = fmax(mx_g, __shfl_xor_sync(0xffffffffu, mx_g, o));
        mx_l = fmax(mx_l, __shfl_xor_sync(0xffffffffu, mx_l, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&s_sum[0], se_g);
        atomicAdd(&s_sum[1], se_l);
        atomic_max_nonneg(&s_sum[2], mx_g);
        atomic_max_nonneg(&s_sum[3], mx_l);
    }
    __syncthreads();
    if (threadIdx.x < 7 && s_cnt[threadIdx.x]) atomicAdd(&gcnt[threadIdx.x], s_cnt[threadIdx.x]);
    if (threadIdx.x == 0) {
        atomicAdd(&gsum[0], s_sum[0]);
        atomicAdd(&gsum[1], s_sum[1]);
        atomic_max_nonneg(&gsum[2], s_sum[2]);
        atomic_max_nonneg(&gsum[3], s_sum[3]);
    }
}

// Launch shapes the autotuner chooses from (one particle per thread: same bits for each):
// blocks of 32, 64 or 128 threads with the compiler's register count, and (single field) 128
// threads capped at 128 registers for four blocks per SM.
constexpr int WLS_BLOCK[4] = {32, 64, 128, 128};

// Outputs of one all-particle WLS launch (sorted order).
struct WlsOut {
    int* status;
    double *z, *wsum, *x;
};

template <int NRHS, int PREC>
void launch_all(lsmps_ctx* ctx, const WlsParams& P, unsigned long long* gcnt, double* gsum,
                const double* fvals = nullptr, const WlsOut* dst = nullptr) {
    int n = (int)ctx->n;
    if (!n) return;
    const WlsOut o = dst ? *dst
                         : WlsOut{ctx->wls_status.get<int>(), ctx->wls_z.get<double>(), ctx->wls_wsum.get<double>(),
                                  ctx->wls_x.get<double>()};
    constexpr bool capped = NRHS == 1;  // the register-capped shape exists for one field
    auto go = [&](int c) {
        const int t = WLS_BLOCK[c];
        if (capped && c == 3)
            k_wls_all<NRHS, PREC, capped ? 4 : 1><<<blocks_for(n, t), t, 0, ctx->stream>>>(
                P, n, ctx->cls.get<uint8_t>(), ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(),
                ctx->nbr_row.get<int>(), ctx->nbr_col.get<int>(), o.status, o.z, o.wsum, o.x, gcnt, gsum, fvals);
        else
            k_wls_all<NRHS, PREC, 1><<<blocks_for(n, t), t, 0, ctx->stream>>>(
                P, n, ctx->cls.get<uint8_t>(), ctx->sx.get<double>(), ctx->sy.get<double>(), ctx->sz.get<double>(),
                ctx->nbr_row.get<int>(), ctx->nbr_col.get<int>(), o.status, o.z, o.wsum, o.x, gcnt, gsum, fvals);
        LSMPS_CHECK_LAUNCH();
    };
    static const std::vector<std::string> names3 = {"block32", "block64", "block128"};
    static const std::vector<std::string> names4 = {"block32", "block64", "block128", "block128 regs128"};
    const std::string key = "wls_all nrhs" + std::to_string(NRHS) + (PREC ? " mixed" : " fp64");
    const size_t tuned_before = ctx->tuner.table.size();
    // without tuning: the capped shape for one field (fastest at 1M), else 128 threads
    const int c = autotune(ctx, key.c_str(), n, capped ? names4 : names3, capped ? 3 : 2, go);
    if (ctx->tuner.table.size() != tuned_before)  // the timed launches added to the statistics
        LSMPS_CUDA(cudaMemsetAsync(gcnt, 0, 16 * sizeof(double), ctx->stream));
    go(c);
}

// Back to caller order (wls arrays are kept in sorted order).
__global__ void k_wls_unsort(const int* __restrict__ iperm, size_t n, int nrhs, const int* __restrict__ st,
                             const double* __restrict__ z, const double* __restrict__ ws,
                             const double* __restrict__ x, int* __restrict__ ost, double* __restrict__ oz,
                             double* __restrict__ ows, double* __restrict__ ox) {
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    int k = iperm[i];
    if (ost) ost[i] = st[k];
    if (ows) ows[i] = ws[k];
    if (oz)
        for (int a = 0; a < K; ++a) oz[i * K + a] = z[(size_t)k * K + a];
    if (ox)
        for (int a = 0; a < nrhs * K; ++a) ox[i * nrhs * K + a] = x[(size_t)k * nrhs * K + a];
}

}  // namespace

void wls_run(lsmps_ctx* ctx, const lsmps_wls_opts* o, lsmps_wls_stats* out) {
    LSMPS_REQUIRE(ctx->have_neighbors && ctx->have_classes, LSMPS_ERR_STATE,
                  "WLS needs neighbor lists and classification first");
    LSMPS_REQUIRE(o && o->re > 0 && o->l0 > 0, LSMPS_ERR_ARG, "WLS options need re > 0 and l0 > 0");
    cudaStream_t s = ctx->stream;
    size_t n = ctx->n;
    lsmps_wls_stats st{};
    if (o->mode == 0) {
        // wls_test: stride = max(1, N / max(1, wls_samples)) (src/lsmps.cpp:28)
        long long samples = o->wls_samples;
        size_t stride = std::max<size_t>(1, n / (size_t)std::max<long long>(1, samples));
        long long ncand = n ? (long long)((n + stride - 1) / stride) : 0;
        auto* so = ctx->wls_sample.ensure<SampleOut>(ncand + 1);
        double* res = ctx->wls_stats.ensure<double>(16);
        if (ncand) {
            k_wls_sample<<<blocks_for(ncand, 64), 64, 0, s>>>(ctx->iperm.get<int>(), ctx->cls.get<uint8_t>(),
                                                              ctx->sx.get<double>(), ctx->sy.get<double>(),
                                                              ctx->sz.get<double>(), ctx->nbr_row.get<int>(),
                                                              ctx->nbr_col.get<int>(), ncand, (long long)stride,
                                                              o->re, o->l0, o->regularization, so);
            LSMPS_CHECK_LAUNCH();
        }
        k_wls_sample_reduce<<<1, 32, 0, s>>>(so, ncand, (unsigned long long)(long long)o->wls_samples, res);
        LSMPS_CHECK_LAUNCH();
        double h[9];
        LSMPS_CUDA(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, s));
        LSMPS_CUDA(cudaStreamSynchronize(s));
        st.sampled = (uint64_t)h[0]; st.ok = (uint64_t)h[1]; st.regularized = (uint64_t)h[2];
        st.failed = (uint64_t)h[3]; st.virtual_points = (uint64_t)h[4];
        st.max_gradient_error = h[5]; st.rms_gradient_error = h[6];
        st.max_laplacian_error = h[7]; st.rms_laplacian_error = h[8];
        if (out) *out = st;
        return;
    }
    LSMPS_REQUIRE(o->mode == 1, LSMPS_ERR_ARG, "WLS mode must be 0 or 1");
    LSMPS_REQUIRE(o->nrhs >= 1 && o->nrhs <= 3 && o->quad_coef, LSMPS_ERR_ARG,
                  "WLS mode 1 needs 1..3 fields and their coefficients");
    LSMPS_REQUIRE(o->precision == 0 || o->precision == 1, LSMPS_ERR_ARG, "WLS precision must be 0 or 1");
    WlsParams P{};
    P.re = o->re; P.l0 = o->l0; P.reg = o->regularization; P.nrhs = o->nrhs; P.precision = o->precision;
    P.store = o->store_solutions ? 1 : 0;
    for (int a = 0; a < 10 * o->nrhs; ++a) P.coef[a] = o->quad_coef[a];
    ctx->wls_status.ensure<int>(n + 1);
    ctx->wls_z.ensure<double>(n * K + 1);
    ctx->wls_wsum.ensure<double>(n + 1);
    ctx->wls_x.ensure<double>(P.store ? n * o->nrhs * K + 1 : 1);
    auto* gcnt = reinterpret_cast<unsigned long long*>(ctx->wls_stats.ensure<double>(16));
    double* gsum = reinterpret_cast<double*>(gcnt + 8);
    LSMPS_CUDA(cudaMemsetAsync(gcnt, 0, 16 * sizeof(double), s));
    if (P.precision == 0) {
        if (P.nrhs == 1) launch_all<1, 0>(ctx, P, gcnt, gsum);
        else if (P.nrhs == 2) launch_all<2, 0>(ctx, P, gcnt, gsum);
        else launch_all<3, 0>(ctx, P, gcnt, gsum);
    } else {
        if (P.nrhs == 1) launch_all<1, 1>(ctx, P, gcnt, gsum);
        else if (P.nrhs == 2) launch_all<2, 1>(ctx, P, gcnt, gsum);
        else launch_all<3, 1>(ctx, P, gcnt, gsum);
    }
    ctx->have_wls = true;
    ctx->wls_nrhs = o->nrhs;
    ctx->wls_stored = P.store != 0;
    ctx->have_ppe = ctx->have_solution = false;
    if (!out) return;  // no statistics wanted: no read-back, the host does not wait
    unsigned long long hc[8];
    double hs[4];
    read_back(ctx, {{gcnt, hc, sizeof(hc)}, {gsum, hs, sizeof(hs)}}, nullptr);
    st.ok = hc[W_OK];
    st.regularized = hc[W_REG];
    st.skipped = hc[W_SKIP];
    st.failed = hc[W_NOWEIGHT] + hc[W_CHOLFAIL];
    st.virtual_points = hc[5];
    st.fp64_fallback = hc[6];
    st.sampled = st.ok + st.regularized;
    double nsol = (double)st.sampled * o->nrhs;
    st.rms_gradient_error = nsol > 0 ? std::sqrt(hs[0] / nsol) : 0;
    st.rms_laplacian_error = nsol > 0 ? std::sqrt(hs[1] / nsol) : 0;
    st.max_gradient_error = hs[2];
    st.max_laplacian_error = hs[3];
    *out = st;
}

namespace {
// caller order (n x nrhs) -> sorted order, and the solutions back
__global__ void k_fields_to_sorted(const int* __restrict__ perm, size_t n, int nrhs, const double* __restrict__ in,
                                   double* __restrict__ out) {
    for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const size_t i = (size_t)perm[k];
        for (int f = 0; f < nrhs; ++f) out[k * nrhs + f] = in[i * nrhs + f];
    }
}
__global__ void k_solutions_to_caller(const int* __restrict__ iperm, size_t n, int nrhs, const double* __restrict__ x,
                                      double* __restrict__ out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t k = (size_t)iperm[i];
        for (int a = 0; a < nrhs * K; ++a) out[i * nrhs * K + a] = x[k * nrhs * K + a];
    }
}
}  // namespace

void wls_fields(lsmps_ctx* ctx, const double* d_fields, int nrhs, double* d_out, bool mirror_walls) {
    LSMPS_REQUIRE(ctx->have_neighbors && ctx->have_classes, LSMPS_ERR_STATE,
                  "WLS of fields needs neighbor lists and classification first");
    LSMPS_REQUIRE(nrhs >= 1 && nrhs <= 3, LSMPS_ERR_ARG, "WLS of fields takes 1..3 fields");
    const size_t n = ctx->n;
    LSMPS_REQUIRE(n == 0 || (d_fields && d_out), LSMPS_ERR_ARG, "null field or output buffer");
    cudaStream_t s = ctx->stream;
    WlsParams P{};
    P.re = ctx->re;
    P.l0 = ctx->l0;
    P.reg = 1e-8;
    P.nrhs = nrhs;
    P.precision = 0;
    P.store = 1;
    P.mirror_walls = mirror_walls ? 1 : 0;
    double* fs = ctx->wf_in.ensure<double>(n * nrhs + 1);
    WlsOut o{ctx->wf_status.ensure<int>(n + 1), ctx->wf_z.ensure<double>(n * K + 1), ctx->wf_wsum.ensure<double>(n + 1),
             ctx->wf_x.ensure<double>(n * nrhs * K + 1)};
    auto* gcnt = reinterpret_cast<unsigned long long*>(ctx->wf_stats.ensure<double>(16));
    double* gsum = reinterpret_cast<double*>(gcnt + 8);
    LSMPS_CUDA(cudaMemsetAsync(gcnt, 0, 16 * sizeof(double), s));
    if (n) {
        LSMPS_CUDA(cudaMemsetAsync(o.x, 0, n * nrhs * K * sizeof(double), s));  // failed rows stay 0
        k_fields_to_sorted<<<std::min<unsigned>(blocks_for(n, 256), 1184), 256, 0, s>>>(ctx->perm.get<int>(), n, nrhs,
                                                                                      d_fields, fs);
        LSMPS_CHECK_LAUNCH();
    }
    if (nrhs == 1) launch_all<1, 0>(ctx, P, gcnt, gsum, fs, &o);
    else if (nrhs == 2) launch_all<2, 0>(ctx, P, gcnt, gsum, fs, &o);
    else launch_all<3, 0>(ctx, P, gcnt, gsum, fs, &o);
    if (n) {
        k_solutions_to_caller<<<std::min<unsigned>(blocks_for(n, 256), 1184), 256, 0, s>>>(ctx->iperm.get<int>(), n,
                                                                                         nrhs, o.x, d_out);
        LSMPS_CHECK_LAUNCH();
    }
}

void wls_kernel_bench(lsmps_ctx* ctx, int reps, double* ms, double* bytes) {
    LSMPS_REQUIRE(ctx->have_wls, LSMPS_ERR_STATE, "kernel bench needs the all-particle WLS first");
    WlsParams P{};
    P.re = ctx->re;
    P.l0 = ctx->l0;
    P.reg = 1e-8;
    P.nrhs = 1;
    const double q[10] = {1, 2, -3, 0.5, 0.7, -0.2, 0.4, 0.3, -0.1, 0.25};
    for (int a = 0; a < 10; ++a) P.coef[a] = q[a];
    auto* gcnt = reinterpret_cast<unsigned long long*>(ctx->wls_stats.ensure<double>(16));
    double* gsum = reinterpret_cast<double*>(gcnt + 8);
    ctx->wls_x.ensure<double>(1);
    launch_all<1, 0>(ctx, P, gcnt, gsum);
    ev_record(ctx, 14);
    for (int r = 0; r < reps; ++r) launch_all<1, 0>(ctx, P, gcnt, gsum);
    ev_record(ctx, 15);
    *ms = ev_elapsed(ctx, 14, 15) / reps;
    double N = (double)ctx->n, Pp = (double)ctx->pairs;
    *bytes = 113.0 * N + 4.0 * Pp;
}

void wls_download(lsmps_ctx* ctx, double* x, int32_t* status, double* z, double* wsum) {
    LSMPS_REQUIRE(ctx->have_wls, LSMPS_ERR_STATE, "no all-particle WLS computed");
    LSMPS_REQUIRE(!x || ctx->wls_stored, LSMPS_ERR_STATE, "WLS solutions were not stored");
    cudaStream_t s = ctx->stream;
    size_t n = ctx->n;
    int nrhs = ctx->wls_nrhs;
    // staging in the general temporary buffer: status | wsum | z | x
    size_t bytes = n * (sizeof(int) + sizeof(double) * (1 + K + (x ? nrhs * K : 0))) + 64;
    char* base = ctx->vtmp.ensure<char>(bytes);
    int* dst = reinterpret_cast<int*>(base);
    double* dws = reinterpret_cast<double*>(base + ((n * sizeof(int) + 15) / 16) * 16);
    double* dz = dws + n;
    double* dx = dz + n * K;
    if (n) {
        k_wls_unsort<<<blocks_for(n, 256), 256, 0, s>>>(ctx->iperm.get<int>(), n, nrhs, ctx->wls_status.get<int>(),
                                                        ctx->wls_z.get<double>(), ctx->wls_wsum.get<double>(),
                                                        ctx->wls_x.get<double>(), dst, dz, dws, x ? dx : nullptr);
        LSMPS_CHECK_LAUNCH();
        if (status) LSMPS_CUDA(cudaMemcpyAsync(status, dst, n * sizeof(int), cudaMemcpyDeviceToHost, s));
        if (wsum) LSMPS_CUDA(cudaMemcpyAsync(wsum, dws, n * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (z) LSMPS_CUDA(cudaMemcpyAsync(z, dz, n * K * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (x) LSMPS_CUDA(cudaMemcpyAsync(x, dx, n * nrhs * K * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    LSMPS_CUDA(cudaStreamSynchronize(s));
}

}  // namespace lsmps_gpu
