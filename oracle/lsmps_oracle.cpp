// ORACLE — test infrastructure, not product code.
//
// A plain CPU restatement of the LS-MPS per-step path of the reference
// (lilux618/LS-MPS, src/lsmps.cpp), written for this repository, plus the variants
// the reference does not implement (all-particle multi-RHS WLS, the WLS-Laplacian and
// shifted graph-Laplacian PPE rows, Jacobi-preconditioned and warm-started BiCGStab).
// Only tests, the smoke check and bench.py's CPU-baseline / reference arm call it; the
// product library never links or loads it.
//
// Floating-point expressions that the reference evaluates are written in the same
// operation order, and the file is built with -ffp-contract=off, so that on inputs the
// reference also handles the results are bit-identical to the reference compiled with
// its own flags (pinned by tests/test_oracle.py against oracle/_ref/libref.so).
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <unordered_map>
#include <vector>

#include <thread>

namespace {

constexpr int K = 9;
enum : uint8_t { INTERIOR = 0, FREE_SURFACE = 1, SPLASH = 2, NEAR_WALL = 3, WALL = 4 };

struct CellKey {
    int x, y, z;
    bool operator==(const CellKey& o) const { return x == o.x && y == o.y && z == o.z; }
};
struct CellKeyHash {
    size_t operator()(const CellKey& c) const {
        uint64_t h = (uint64_t)(uint32_t)c.x * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)(uint32_t)c.y * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
        h ^= (uint64_t)(uint32_t)c.z * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};

inline double sq3(double dx, double dy, double dz) { return dx * dx + dy * dy + dz * dz; }

// weight (src/lsmps.cpp:22): (re/r - 1)^2 inside (1e-12, re), else 0.
inline double weight(double r, double re) {
    if (r <= 1e-12 || r >= re) return 0;
    double q = re / r - 1;
    return q * q;
}

// basis (src/lsmps.cpp:23): normalised second-order Taylor terms.
inline void basis(double dx, double dy, double dz, double r, double l0, double* q) {
    double ir = 1 / r;
    q[0] = dx * ir; q[1] = dy * ir; q[2] = dz * ir;
    q[3] = dx * dx / (2 * l0 * r); q[4] = dy * dy / (2 * l0 * r); q[5] = dz * dz / (2 * l0 * r);
    q[6] = dx * dy / (l0 * r); q[7] = dx * dz / (l0 * r); q[8] = dy * dz / (l0 * r);
}

// cholesky (src/lsmps.cpp:24): row-wise LL^T on the lower triangle, pivot > 1e-14 and
// finite, five attempts adding 0, reg, 10 reg, 100 reg, 1000 reg to the diagonal.
bool cholesky(double* a, double reg, bool& used) {
    used = false;
    double m[K * K];
    for (int at = 0; at < 5; ++at) {
        std::memcpy(m, a, sizeof(m));
        double add = at ? reg * std::pow(10.0, at - 1) : 0;
        if (add) {
            used = true;
            for (int i = 0; i < K; ++i) m[i * K + i] += add;
        }
        bool ok = true;
        for (int i = 0; i < K && ok; ++i) {
            for (int j = 0; j <= i; ++j) {
                double s = m[i * K + j];
                for (int k = 0; k < j; ++k) s -= m[i * K + k] * m[j * K + k];
                if (i == j) {
                    if (!(s > 1e-14) || !std::isfinite(s)) { ok = false; break; }
                    m[i * K + j] = std::sqrt(s);
                } else {
                    m[i * K + j] = s / m[j * K + j];
                }
            }
            for (int j = i + 1; j < K; ++j) m[i * K + j] = 0;
        }
        if (ok) { std::memcpy(a, m, sizeof(m)); return true; }
    }
    return false;
}

// solve (src/lsmps.cpp:25): forward then backward substitution with L and L^T.
void chol_solve(const double* l, const double* b, double* x) {
    double y[K];
    for (int i = 0; i < K; ++i) {
        double s = b[i];
        for (int k = 0; k < i; ++k) s -= l[i * K + k] * y[k];
        y[i] = s / l[i * K + i];
    }
    for (int i = K - 1; i >= 0; --i) {
        double s = y[i];
        for (int k = i + 1; k < K; ++k) s -= l[k * K + i] * x[k];
        x[i] = s / l[i * K + i];
    }
}

// A quadratic field f = c0 + c1 x + c2 y + c3 z + c4 x^2 + c5 y^2 + c6 z^2 + c7 xy + c8 xz
// + c9 yz, accumulated left to right as the reference's fixed test field is
// (src/lsmps.cpp:28), so the reference's coefficients reproduce its values exactly.
inline double quad_eval(const double* c, double x, double y, double z) {
    double t = c[0] + c[1] * x;
    t = t + c[2] * y;
    t = t + c[3] * z;
    t = t + c[4] * x * x;
    t = t + c[5] * y * y;
    t = t + c[6] * z * z;
    t = t + c[7] * x * y;
    t = t + c[8] * x * z;
    t = t + c[9] * y * z;
    return t;
}

// Runs fn(lo, hi, t) over nt contiguous blocks of [0, n) on nt threads (nt <= 1: inline).
template <class F>
void par_blocks(size_t n, int nt, F&& fn) {
    if (nt <= 1) { fn((size_t)0, n, 0); return; }
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t)
        th.emplace_back([&, t] { fn(n * t / nt, n * (t + 1) / nt, t); });
    for (auto& x : th) x.join();
}

double now_ms() {
    using C = std::chrono::steady_clock;
    return std::chrono::duration<double, std::milli>(C::now().time_since_epoch()).count();
}

}  // namespace

extern "C" {

// Uniform-grid neighbor lists (src/lsmps.cpp:16-18,26). Cell = floor(r/re) per axis;
// the 27 cells are visited dz outer, dy, dx inner, each from -1 to +1; within a cell in
// ascending particle index; accept j != i with |rj - ri|^2 < re^2; keep the first maxn
// and count the dropped pairs in *truncated. Returns the kept pair count. row_ptr has
// n+1 entries; col is filled only when col_cap is large enough.
long long orc_neighbors(const double* xyz, size_t n, double re, int maxn, int* row_ptr,
                        int* col, size_t col_cap, unsigned long long* truncated) {
    std::vector<CellKey> cell(n);
    std::unordered_map<CellKey, std::vector<int>, CellKeyHash> grid;
    grid.reserve(n * 2 + 1);
    for (size_t i = 0; i < n; ++i) {
        cell[i] = {(int)std::floor(xyz[3 * i] / re), (int)std::floor(xyz[3 * i + 1] / re),
                   (int)std::floor(xyz[3 * i + 2] / re)};
        grid[cell[i]].push_back((int)i);  // insertion in index order keeps cells ascending
    }
    const double re2 = re * re;
    size_t off = 0;
    unsigned long long trunc = 0;
    if (row_ptr) row_ptr[0] = 0;
    for (size_t i = 0; i < n; ++i) {
        int kept = 0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    auto it = grid.find({cell[i].x + dx, cell[i].y + dy, cell[i].z + dz});
                    if (it == grid.end()) continue;
                    for (int j : it->second) {
                        if ((size_t)j == i) continue;
                        double ddx = xyz[3 * j] - xyz[3 * i], ddy = xyz[3 * j + 1] - xyz[3 * i + 1],
                               ddz = xyz[3 * j + 2] - xyz[3 * i + 2];
                        if (sq3(ddx, ddy, ddz) < re2) {
                            if (kept < maxn) {
                                if (col && off + kept < col_cap) col[off + kept] = j;
                                ++kept;
                            } else {
                                ++trunc;
                            }
                        }
                    }
                }
        off += kept;
        if (row_ptr) row_ptr[i + 1] = (int)off;
    }
    if (truncated) *truncated = trunc;
    return (long long)off;
}

// 14-direction coverage classification (src/lsmps.cpp:27): Wall stays Wall; fewer than
// 10 kept neighbors -> Splash; sectors = 6 dominant-axis bins (ties to x, then y; sign
// d >= 0) + 8 octants; z < 1.5 l0 -> NearWall (tested before coverage); fewer than 11
// sectors -> FreeSurface; otherwise Interior. Only the particle's own input type is
// read, so the in-place update of the reference is order independent.
void orc_classify(const double* xyz, const uint8_t* type_in, size_t n, const int* row_ptr,
                  const int* col, double l0, uint8_t* type_out) {
    for (size_t i = 0; i < n; ++i) {
        if (type_in[i] == WALL) { type_out[i] = WALL; continue; }
        int deg = row_ptr[i + 1] - row_ptr[i];
        if (deg < 10) { type_out[i] = SPLASH; continue; }
        bool seen[14] = {};
        for (int e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
            int j = col[e];
            double dx = xyz[3 * j] - xyz[3 * i], dy = xyz[3 * j + 1] - xyz[3 * i + 1],
                   dz = xyz[3 * j + 2] - xyz[3 * i + 2];
            double ax = std::abs(dx), ay = std::abs(dy), az = std::abs(dz);
            int s = (ax >= ay && ax >= az) ? (dx >= 0 ? 0 : 1)
                                           : ((ay >= ax && ay >= az) ? (dy >= 0 ? 2 : 3) : (dz >= 0 ? 4 : 5));
            seen[s] = true;
            seen[6 + (dx >= 0) + 2 * (dy >= 0) + 4 * (dz >= 0)] = true;
        }
        int sectors = 0;
        for (bool b : seen) sectors += b;
        if (xyz[3 * i + 2] < 1.5 * l0) type_out[i] = NEAR_WALL;
        else if (sectors < 11) type_out[i] = FREE_SURFACE;
        else type_out[i] = INTERIOR;
    }
}

// All-particle second-order WLS (src/lsmps.cpp:22-25,28) for nrhs quadratic fields.
// For particle i (Wall and Splash skipped, status 2): M = sum w q q^T / sum w and
// b_k = sum w q (f_k(j) - f_k(i)) / r / sum w, Cholesky with regularisation retries, then
// x_k = M^-1 b_k (x_out[(i*nrhs+k)*9 ..]). Also z_i = M^-1 (e3+e4+e5) (z_out[i*9 ..])
// and sum w (wsum_out[i]), from which the WLS Laplacian operator is
//   lap_i(f) = sum_j c_ij (f_j - f_i),  c_ij = w_ij q_ij . z_i / (r_ij sum_w l0).
// status: 0 ok, 1 regularised, 2 skipped type, 3 sum w <= 0, 4 Cholesky failed.
// Field values either from the quadratics coef (nrhs x 10) or from the array fields
// (n x nrhs, per particle).
// mirror_walls: Wall neighbors take the particle's own value (f_j = f_i, a zero normal
// gradient; python/rain_plate_lsmps_cpu.py:179), so they shape the moments but add nothing
// to the right-hand sides.
static void wls_impl(const double* xyz, const uint8_t* type, size_t n, const int* row_ptr, const int* col,
                     double re, double l0, double reg, int nrhs, const double* coef, const double* fields,
                     double* x_out, int* status, double* z_out, double* wsum_out, int mirror_walls = 0) {
    auto fval = [&](int k, size_t p) {
        return fields ? fields[p * nrhs + k]
                      : quad_eval(coef + 10 * k, xyz[3 * p], xyz[3 * p + 1], xyz[3 * p + 2]);
    };
    std::vector<double> bb((size_t)nrhs * K);
    for (size_t i = 0; i < n; ++i) {
        if (x_out) std::fill(x_out + i * nrhs * K, x_out + (i + 1) * nrhs * K, 0.0);
        if (z_out) std::fill(z_out + i * K, z_out + (i + 1) * K, 0.0);
        if (wsum_out) wsum_out[i] = 0;
        if (type[i] == WALL || type[i] == SPLASH) { status[i] = 2; continue; }
        double M[K * K] = {};
        std::fill(bb.begin(), bb.end(), 0.0);
        double ws = 0;
        const double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
        for (int e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
            int j = col[e];
            double dx = xyz[3 * j] - xi, dy = xyz[3 * j + 1] - yi, dz = xyz[3 * j + 2] - zi;
            double r = std::sqrt(sq3(dx, dy, dz)), w = weight(r, re);
            if (!w) continue;
            double q[K];
            basis(dx, dy, dz, r, l0, q);
            ws += w;
            for (int k = 0; k < nrhs && !(mirror_walls && type[j] == WALL); ++k) {
                double df = fval(k, (size_t)j) - fval(k, i);
                for (int a = 0; a < K; ++a) bb[k * K + a] += w * q[a] * df / r;
            }
            for (int a = 0; a < K; ++a)
                for (int c = 0; c <= a; ++c) M[a * K + c] += w * q[a] * q[c];
        }
        if (wsum_out) wsum_out[i] = ws;
        if (ws <= 0) { status[i] = 3; continue; }
        for (double& v : M) v /= ws;
        for (double& v : bb) v /= ws;
        bool used = false;
        if (!cholesky(M, reg, used)) { status[i] = 4; continue; }
        status[i] = used ? 1 : 0;
        for (int k = 0; k < nrhs; ++k)
            if (x_out) chol_solve(M, &bb[k * K], x_out + (i * nrhs + k) * K);
        if (z_out) {
            double e[K] = {0, 0, 0, 1, 1, 1, 0, 0, 0};
            chol_solve(M, e, z_out + i * K);
        }
    }
}

void orc_wls(const double* xyz, const uint8_t* type, size_t n, const int* row_ptr,
             const int* col, double re, double l0, double reg, int nrhs, const double* coef,
             double* x_out, int* status, double* z_out, double* wsum_out) {
    wls_impl(xyz, type, n, row_ptr, col, re, l0, reg, nrhs, coef, nullptr, x_out, status, z_out, wsum_out);
}

// The same WLS for per-particle fields (n x nrhs): the solutions a projection step's
// gradients come from (lsmps_wls_fields).
void orc_wls_fields(const double* xyz, const uint8_t* type, size_t n, const int* row_ptr, const int* col,
                    double re, double l0, double reg, int nrhs, const double* fields, double* x_out,
                    int* status, int mirror_walls) {
    wls_impl(xyz, type, n, row_ptr, col, re, l0, reg, nrhs, nullptr, fields, x_out, status, nullptr, nullptr,
             mirror_walls);
}

// Pressure-Poisson assembly. Unknowns are Interior or NearWall particles in index order,
// capped at max_unknowns (src/lsmps.cpp:33-36). For each unknown row the neighbors that
// are unknowns with w > 0 are appended in list order and the diagonal last
// (src/lsmps.cpp:40-57). Variants:
//  0 reference: off-diagonal -w/r^2, diagonal sum w/r^2, row 0 pinned to the identity,
//    p* = x^2 + y^2 (src/lsmps.cpp:29,43-55).
//  1 shifted graph Laplacian: off-diagonal -w, diagonal sum w * (1 + diag_shift),
//    p* = sin(0.3x) cos(0.2y) + 0.1 z, no pinned row.
//  2 WLS Laplacian: c_ij = w_ij q_ij . z_i / (r_ij sum_w l0); entries with c_ij <= 0 are
//    dropped (clipped);
//    off-diagonal -c_ij, diagonal sum over all neighbors with w > 0 of c_ij (Dirichlet
//    neighbors move to the right-hand side through b = A p*), times (1 + diag_shift); a
//    row whose WLS failed or whose diagonal is not positive becomes an identity row
//    (failed_rows). p* as in variant 1. Unclipped second-order WLS rows are not
//    diagonally dominant near one-sided (wall, surface) stencils and BiCGStab breaks
//    down on them; with the clip every row is an M-matrix row.
//  3 WLS Laplacian with Neumann walls: as 2, but Wall neighbors take the row particle's
//    own pressure (zero normal gradient, the mirrored wall value of
//    python/rain_plate_lsmps_cpu.py:90-100,179), so their coefficients c_ij (p_i - p_i)
//    vanish: they add neither an entry nor to the diagonal. Free-surface and splash
//    neighbors stay Dirichlet.
// Row diagonals that are <= 0 or non-finite count as failed rows and are set to 1
// (src/lsmps.cpp:52). b = A p* in row order (src/lsmps.cpp:59-61).
// stats: unknowns, nnz, dirichlet, neumann, failed_rows. Call with row == nullptr first
// for the sizes. unknown_particle[u] gives the particle of unknown u.
long long orc_ppe_assemble(int variant, const double* xyz, const uint8_t* type, size_t n,
                           const int* row_ptr, const int* col, double re, double l0,
                           long long max_unknowns, double diag_shift, const double* z,
                           const double* wsum, const int* wls_status, int* row, int* ocol,
                           double* val, double* b, double* xexact, int* unknown_particle,
                           long long* stats) {
    const size_t cap = std::min(n, (size_t)max_unknowns);
    std::vector<int> map(n, -1), rev;
    for (size_t i = 0; i < n && rev.size() < cap; ++i)
        if (type[i] == INTERIOR || type[i] == NEAR_WALL) { map[i] = (int)rev.size(); rev.push_back((int)i); }
    std::vector<int> rw{0}, cl;
    std::vector<double> vl;
    long long neumann = 0, failed = 0;
    for (size_t rr = 0; rr < rev.size(); ++rr) {
        int i = rev[rr];
        const double xi = xyz[3 * i], yi = xyz[3 * i + 1], zi = xyz[3 * i + 2];
        if (variant == 0 && rr == 0) {
            cl.push_back(0); vl.push_back(1.0); rw.push_back((int)cl.size());
            continue;
        }
        size_t row_begin = cl.size();
        double diag = 0.0;
        bool identity = false;
        const bool wls_rows = variant == 2 || variant == 3;
        if (wls_rows && !(wls_status[i] == 0 || wls_status[i] == 1)) identity = true;
        if (!identity) {
            for (int e = row_ptr[i]; e < row_ptr[i + 1]; ++e) {
                int j = col[e];
                int cj = map[j];
                if (!wls_rows && cj < 0) continue;
                if (variant == 3 && type[j] == WALL) continue;
                double dx = xyz[3 * j] - xi, dy = xyz[3 * j + 1] - yi, dz = xyz[3 * j + 2] - zi;
                double r = std::sqrt(sq3(dx, dy, dz)), w = weight(r, re);
                if (w <= 0) continue;
                double a;
                if (variant == 0) {
                    a = w / (r * r);
                } else if (variant == 1) {
                    a = w;
                } else {
                    double q[K];
                    basis(dx, dy, dz, r, l0, q);
                    double s = 0;
                    for (int k = 0; k < K; ++k) s += q[k] * z[(size_t)i * K + k];
                    a = w * s / (r * wsum[i] * l0);
                    if (!(a > 0)) continue;  // clip: keeps the row diagonally dominant
                }
                diag += a;
                if (cj >= 0) { cl.push_back(cj); vl.push_back(-a); }
            }
            if (variant != 0) diag = diag * (1.0 + diag_shift);
        }
        if (wls_rows && (identity || !(diag > 0) || !std::isfinite(diag))) {
            cl.resize(row_begin); vl.resize(row_begin);
            failed++;
            diag = 1.0;
        } else if (diag <= 0 || !std::isfinite(diag)) {
            failed++;
            diag = 1.0;
        }
        cl.push_back((int)rr); vl.push_back(diag);
        rw.push_back((int)cl.size());
        if (type[i] == NEAR_WALL) neumann++;
    }
    if (stats) {
        stats[0] = (long long)rev.size(); stats[1] = (long long)vl.size();
        stats[2] = (long long)(n - rev.size()); stats[3] = neumann; stats[4] = failed;
    }
    if (row) {
        std::memcpy(row, rw.data(), rw.size() * sizeof(int));
        std::memcpy(ocol, cl.data(), cl.size() * sizeof(int));
        std::memcpy(val, vl.data(), vl.size() * sizeof(double));
        std::vector<double> xs(rev.size());
        for (size_t rr = 0; rr < rev.size(); ++rr) {
            int i = rev[rr];
            double x = xyz[3 * i], y = xyz[3 * i + 1], zz = xyz[3 * i + 2];
            xs[rr] = variant == 0 ? x * x + y * y : std::sin(0.3 * x) * std::cos(0.2 * y) + 0.1 * zz;
        }
        for (size_t rr = 0; rr < rev.size(); ++rr) {
            double sum = 0;
            for (int k = rw[rr]; k < rw[rr + 1]; ++k) sum += vl[k] * xs[cl[k]];
            b[rr] = sum;
        }
        if (xexact) std::memcpy(xexact, xs.data(), xs.size() * sizeof(double));
        if (unknown_particle) std::memcpy(unknown_particle, rev.data(), rev.size() * sizeof(int));
    }
    return (long long)vl.size();
}

// y = A x for CSR A, row by row in stored order (src/lsmps.cpp:65).
void orc_spmv(size_t n, const int* row, const int* col, const double* val, const double* x,
              double* y, int nthreads) {
    par_blocks(n, nthreads, [&](size_t lo, size_t hi, int) {
        for (size_t i = lo; i < hi; ++i) {
            double s = 0;
            for (int k = row[i]; k < row[i + 1]; ++k) s += val[k] * x[col[k]];
            y[i] = s;
        }
    });
}

namespace {
// Dot product: one thread sums in index order as the reference does (src/lsmps.cpp:66);
// several threads sum contiguous blocks and combine the block sums in order.
double dotp(const double* a, const double* b, size_t n, int nt) {
    if (nt <= 1) {
        double s = 0;
        for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
        return s;
    }
    std::vector<double> part(nt, 0.0);
    par_blocks(n, nt, [&](size_t lo, size_t hi, int t) {
        double s = 0;
        for (size_t i = lo; i < hi; ++i) s += a[i] * b[i];
        part[t] = s;
    });
    double s = 0;
    for (double v : part) s += v;
    return s;
}
}  // namespace

// BiCGStab (src/lsmps.cpp:67): x0 = 0 (or the caller's x0), r_hat = r = b - A x0,
// rho0 = alpha = omega = 1, p = v = 0, breakdown guards at 1e-30, convergence when
// |s| or |r| <= tol * max(1, |b|). precond = 1 applies Jacobi (diagonal) preconditioning
// on the right; precond = 0 with x0 == nullptr and nthreads = 1 is the reference
// iteration operation for operation.
// out: iterations, converged, |Ax - b| at exit, ms.
void orc_bicgstab(size_t n, const int* row, const int* col, const double* val, const double* b,
                  const double* x0, int max_iter, double tol, int precond, int nthreads,
                  double* x, double* out4) {
    double t0 = now_ms();
    int nt = nthreads > 0 ? nthreads : 1;
    std::vector<double> r(n), r0, p(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n), dinv(n, 1.0), Ax(n);
    if (precond == 1)
        for (size_t i = 0; i < n; ++i)
            for (int k = row[i]; k < row[i + 1]; ++k)
                if ((size_t)col[k] == i) dinv[i] = val[k] != 0 ? 1.0 / val[k] : 1.0;
    if (x0) {
        std::memcpy(x, x0, n * sizeof(double));
        orc_spmv(n, row, col, val, x, Ax.data(), nt);
        for (size_t i = 0; i < n; ++i) r[i] = b[i] - Ax[i];
    } else {
        std::fill(x, x + n, 0.0);
        std::memcpy(r.data(), b, n * sizeof(double));
    }
    r0 = r;
    double bnorm = std::sqrt(dotp(b, b, n, nt));
    double thresh = tol * std::max(1.0, bnorm);
    double rho0 = 1, alpha = 1, omega = 1;
    int iters = 0;
    bool conv = false;
    for (int it = 0; it < max_iter; ++it) {
        double rho = dotp(r0.data(), r.data(), n, nt);
        if (std::abs(rho) < 1e-30) break;
        double beta = (rho / rho0) * (alpha / omega);
        for (size_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        const double* pp = p.data();
        if (precond == 1) { for (size_t i = 0; i < n; ++i) ph[i] = dinv[i] * p[i]; pp = ph.data(); }
        orc_spmv(n, row, col, val, pp, v.data(), nt);
        double den = dotp(r0.data(), v.data(), n, nt);
        if (std::abs(den) < 1e-30) break;
        alpha = rho / den;
        for (size_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        double sn = std::sqrt(dotp(s.data(), s.data(), n, nt));
        if (sn <= thresh) {
            for (size_t i = 0; i < n; ++i) x[i] += alpha * pp[i];
            iters = it + 1; conv = true; break;
        }
        const double* ss = s.data();
        if (precond == 1) { for (size_t i = 0; i < n; ++i) sh[i] = dinv[i] * s[i]; ss = sh.data(); }
        orc_spmv(n, row, col, val, ss, t.data(), nt);
        double tt = dotp(t.data(), t.data(), n, nt);
        if (tt < 1e-30) break;
        omega = dotp(t.data(), s.data(), n, nt) / tt;
        for (size_t i = 0; i < n; ++i) x[i] += alpha * pp[i] + omega * ss[i];
        for (size_t i = 0; i < n; ++i) r[i] = s[i] - omega * t[i];
        double rn = std::sqrt(dotp(r.data(), r.data(), n, nt));
        iters = it + 1;
        if (rn <= thresh) { conv = true; break; }
        if (std::abs(omega) < 1e-30) break;
        rho0 = rho;
    }
    orc_spmv(n, row, col, val, x, Ax.data(), nt);
    double res = 0;
    for (size_t i = 0; i < n; ++i) { double d = Ax[i] - b[i]; res += d * d; }
    out4[0] = iters; out4[1] = conv ? 1.0 : 0.0; out4[2] = std::sqrt(res); out4[3] = now_ms() - t0;
}

// Particle-set generators of the bench and the tests, restated for the CPU side so that the
// reference arm of bench.py builds its inputs without the product library. Positions must be
// bit-identical to the library's generate_case (ls-mps_b200/csrc/host.cpp), so the draws come
// from std::mt19937 + uniform_real_distribution<double> in the same order: that order is the
// contract, pinned by tests/test_oracle.py against the library's positions.
//   kind 0: the reference's default jittered lattice (src/lsmps.cpp:68,72; jitter .03)
//   kind 1: rain on a 20-degree plate (3 wall layers, 4 film layers holding 70 % of the
//           fluid, radius-3 droplets 10-40 l0 above; jitter .1)
//   kind 2: 80 % jittered bulk lattice + 20 % rain on a plate 25 l0 beyond it (jitter .1)
// jitter < 0 selects the kind's default. Returns the particle count written (n).
size_t orc_generate(int kind, size_t n, double l0, double jitter, unsigned seed, double* xyz, uint8_t* type) {
    std::mt19937 rng(seed);
    size_t w = 0;
    auto put = [&](double x, double y, double z, uint8_t t) {
        xyz[3 * w] = x; xyz[3 * w + 1] = y; xyz[3 * w + 2] = z; type[w] = t; ++w;
    };
    auto grid = [&](size_t upto, int nx, int ny, int nz, double jit) {
        std::uniform_real_distribution<double> u(-jit, jit);
        for (int k = 0; k < nz && w < upto; ++k)
            for (int j = 0; j < ny && w < upto; ++j)
                for (int i = 0; i < nx && w < upto; ++i) {
                    const double a = u(rng), b = u(rng), c = u(rng);
                    put((i + .5 + a) * l0, (j + .5 + b) * l0, (k + .5 + c) * l0, INTERIOR);
                }
    };
    auto plate = [&](size_t count, double jit, double x0) {
        const double th = 20.0 * 3.14159265358979323846 / 180.0;
        const double c = std::cos(th), sn = std::sin(th);
        // a point at plate coordinates (s, y) and height h: s t1 + y t2 + h nrm
        auto at = [&](double s, double y, double h, double* o) {
            o[0] = (c * s + 0.0 * y) + -sn * h;
            o[1] = (0.0 * s + 1.0 * y) + 0.0 * h;
            o[2] = (sn * s + 0.0 * y) + c * h;
        };
        const int wall = 3, film = 4;
        const int m = std::max(4, (int)std::floor(std::sqrt((double)count / (wall + film / 0.7))));
        std::uniform_real_distribution<double> u(-jit, jit);
        const size_t end = w + count;
        auto layer = [&](double h, uint8_t t) {
            for (int b = 0; b < m && w < end; ++b)
                for (int a = 0; a < m && w < end; ++a) {
                    const double ds = u(rng), dy = u(rng), dh = u(rng);
                    double o[3];
                    at((a + .5 + ds) * l0, (b + .5 + dy) * l0, (h + dh) * l0, o);
                    put(o[0] + x0, o[1], o[2], t);
                }
        };
        for (int k = 0; k < wall; ++k) layer(-(k + .5), WALL);
        for (int k = 0; k < film; ++k) layer(k + .5, INTERIOR);
        std::vector<std::array<int, 3>> ball;
        for (int k = -3; k <= 3; ++k)
            for (int j = -3; j <= 3; ++j)
                for (int i = -3; i <= 3; ++i)
                    if (i * i + j * j + k * k <= 9.0) ball.push_back({i, j, k});
        std::uniform_real_distribution<double> us(0.0, m * l0), uh(10.0 * l0, 40.0 * l0);
        while (w < end) {
            const double s0 = us(rng), y0 = us(rng), h0 = uh(rng);
            double ctr[3];
            at(s0, y0, h0, ctr);
            ctr[0] += x0;
            for (const auto& o : ball) {
                if (w >= end) break;
                const double a = u(rng), b = u(rng), d = u(rng);
                put(ctr[0] + (o[0] + a) * l0, ctr[1] + (o[1] + b) * l0, ctr[2] + (o[2] + d) * l0, INTERIOR);
            }
        }
    };
    if (kind == 1) {
        plate(n, jitter >= 0 ? jitter : .1, 0.0);
    } else if (kind == 2) {
        const size_t nbulk = (size_t)(0.8 * (double)n);
        const int nb = std::max(4, (int)std::ceil(std::cbrt((double)nbulk)));
        grid(nbulk, nb, nb, nb, jitter >= 0 ? jitter : .1);
        plate(n - w, jitter >= 0 ? jitter : .1, (nb + 25) * l0);
    } else {
        const int nx = std::max(4, (int)std::ceil(std::cbrt((double)n)));
        grid(n, nx, nx, nx, jitter >= 0 ? jitter : .03);
    }
    return w;
}

}  // extern "C"
