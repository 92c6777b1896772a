// Test infrastructure only: a C-ABI shim over the reference implementation of
// LS-MPS (lilux618/LS-MPS), compiled from the reference's own source file where it
// lies (the path is given to the compiler by oracle/Makefile; nothing is copied).
// Its internal functions live in an anonymous namespace of src/lsmps.cpp, so this
// translation unit includes that file and re-exports them with plain pointers.
//
// Only tests, the smoke check and bench.py's CPU-baseline / reference arm load the
// resulting oracle/_ref/libref.so; the product never does.
#include LSMPS_REF_SOURCE   // "<reference>/src/lsmps.cpp", set by oracle/Makefile

#include <cstring>
#include <memory>

namespace {
struct RefCase {
    lsmps::Config cfg;
    std::vector<lsmps::Particle> ps;
    lsmps::NeighborData nd;
    bool have_nd = false;
    lsmps::CSR A;
    lsmps::PpeStats ppe_assembly;
    lsmps::Metrics metrics;
};
}  // namespace

extern "C" {

// Config from a .cfg file (src/lsmps.cpp:71). Returns nullptr on error.
void* ref_case_from_cfg(const char* path) {
    try {
        auto* h = new RefCase();
        h->cfg = lsmps::load_config(path);
        return h;
    } catch (...) {
        return nullptr;
    }
}

void ref_case_free(void* h) { delete static_cast<RefCase*>(h); }

// Read back the parsed config fields as doubles (for load_config parity tests).
int ref_cfg_get(void* hv, const char* key, double* out, char* strbuf, size_t strcap) {
    auto& c = static_cast<RefCase*>(hv)->cfg;
    std::string k(key);
    if (k == "case") { std::snprintf(strbuf, strcap, "%s", c.case_name.c_str()); return 0; }
    if (k == "particles") { *out = (double)c.particles; return 0; }
    if (k == "seed") { *out = (double)c.seed; return 0; }
    if (k == "l0") { *out = c.l0; return 0; }
    if (k == "re_ratio") { *out = c.re_ratio; return 0; }
    if (k == "film_layers") { *out = c.film_layers; return 0; }
    if (k == "max_neighbors") { *out = c.max_neighbors; return 0; }
    if (k == "wls_samples") { *out = c.wls_samples; return 0; }
    if (k == "steps") { *out = c.steps; return 0; }
    if (k == "injected_per_step") { *out = c.injected_per_step; return 0; }
    if (k == "cnl_rebuild_interval") { *out = c.cnl_rebuild_interval; return 0; }
    if (k == "ppe_max_unknowns") { *out = c.ppe_max_unknowns; return 0; }
    if (k == "ppe_max_iter") { *out = c.ppe_max_iter; return 0; }
    if (k == "ppe_tol") { *out = c.ppe_tol; return 0; }
    if (k == "wls_regularization") { *out = c.wls_regularization; return 0; }
    if (k == "boundary_constraint_weight") { *out = c.boundary_constraint_weight; return 0; }
    if (k == "virtual_weight") { *out = c.virtual_weight; return 0; }
    if (k == "write_csv") { *out = c.write_csv ? 1.0 : 0.0; return 0; }
    return -1;
}

// Override numeric config fields (used to run the reference on the same inputs).
int ref_cfg_set(void* hv, const char* key, double v) {
    auto& c = static_cast<RefCase*>(hv)->cfg;
    std::string k(key);
    if (k == "particles") c.particles = (size_t)v;
    else if (k == "seed") c.seed = (uint32_t)v;
    else if (k == "l0") c.l0 = v;
    else if (k == "re_ratio") c.re_ratio = v;
    else if (k == "film_layers") c.film_layers = (int)v;
    else if (k == "max_neighbors") c.max_neighbors = (int)v;
    else if (k == "wls_samples") c.wls_samples = (int)v;
    else if (k == "ppe_max_unknowns") c.ppe_max_unknowns = (int)v;
    else if (k == "ppe_max_iter") c.ppe_max_iter = (int)v;
    else if (k == "ppe_tol") c.ppe_tol = v;
    else return -1;
    return 0;
}

int ref_cfg_set_case(void* hv, const char* name) {
    static_cast<RefCase*>(hv)->cfg.case_name = name;
    return 0;
}

// generate_case (src/lsmps.cpp:72); returns the particle count.
size_t ref_generate(void* hv) {
    auto* h = static_cast<RefCase*>(hv);
    h->ps = lsmps::generate_case(h->cfg);
    h->have_nd = false;
    return h->ps.size();
}

// Replace the particle set with caller data (xyz interleaved, types as uint8).
void ref_set_particles(void* hv, const double* xyz, const uint8_t* type, size_t n) {
    auto* h = static_cast<RefCase*>(hv);
    h->ps.assign(n, lsmps::Particle{});
    for (size_t i = 0; i < n; ++i) {
        h->ps[i].r = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
        h->ps[i].type = static_cast<lsmps::ParticleType>(type[i]);
    }
    h->have_nd = false;
}

void ref_get_particles(void* hv, double* xyz, uint8_t* type, double* uvw) {
    auto* h = static_cast<RefCase*>(hv);
    for (size_t i = 0; i < h->ps.size(); ++i) {
        const auto& p = h->ps[i];
        if (xyz) { xyz[3 * i] = p.r.x; xyz[3 * i + 1] = p.r.y; xyz[3 * i + 2] = p.r.z; }
        if (type) type[i] = static_cast<uint8_t>(p.type);
        if (uvw) { uvw[3 * i] = p.u.x; uvw[3 * i + 1] = p.u.y; uvw[3 * i + 2] = p.u.z; }
    }
}

// neighbors (src/lsmps.cpp:26) with re = re_ratio*l0 as run_benchmark passes it (:73).
// Returns total kept pairs; fills row_ptr (n+1) and col (if col_cap suffices).
long long ref_neighbors(void* hv, int* row_ptr, int* col, size_t col_cap,
                        unsigned long long* truncated) {
    auto* h = static_cast<RefCase*>(hv);
    h->nd = lsmps::neighbors(h->ps, h->cfg.re_ratio * h->cfg.l0, h->cfg.max_neighbors);
    h->have_nd = true;
    if (truncated) *truncated = h->nd.truncated;
    size_t off = 0;
    if (row_ptr) row_ptr[0] = 0;
    for (size_t i = 0; i < h->ps.size(); ++i) {
        const auto& v = h->nd.list[i];
        if (col && off + v.size() <= col_cap) std::memcpy(col + off, v.data(), v.size() * sizeof(int));
        off += v.size();
        if (row_ptr) row_ptr[i + 1] = (int)off;
    }
    return (long long)h->nd.pairs;
}

// classify in place, exactly as run_benchmark does (src/lsmps.cpp:27,73).
void ref_classify(void* hv, uint8_t* types_out) {
    auto* h = static_cast<RefCase*>(hv);
    for (size_t i = 0; i < h->ps.size(); ++i)
        h->ps[i].type = lsmps::classify(h->ps[i], h->nd.list[i], h->ps, h->cfg.l0);
    if (types_out)
        for (size_t i = 0; i < h->ps.size(); ++i) types_out[i] = static_cast<uint8_t>(h->ps[i].type);
}

// wls_test (src/lsmps.cpp:28). out: sampled, ok, regularized, failed, virtual_points,
// max_grad, rms_grad, max_lap, rms_lap.
void ref_wls_test(void* hv, double* out9) {
    auto* h = static_cast<RefCase*>(hv);
    auto st = lsmps::wls_test(h->cfg, h->ps, h->nd);
    double o[9] = {(double)st.sampled, (double)st.ok, (double)st.regularized, (double)st.failed,
                   (double)st.virtual_points, st.max_gradient_error, st.rms_gradient_error,
                   st.max_laplacian_error, st.rms_laplacian_error};
    std::memcpy(out9, o, sizeof(o));
}

// One particle's WLS solve for the fixed quadratic of wls_test: x[9], returns
// 0 ok, 1 regularized, -1 sum of weights <= 0, -2 Cholesky failure.
int ref_wls_particle(void* hv, size_t i, double* x9) {
    auto* h = static_cast<RefCase*>(hv);
    const auto& ps = h->ps;
    const auto& cfg = h->cfg;
    using namespace lsmps;
    double re = cfg.re_ratio * cfg.l0;
    auto f = [](Vec3 r) {
        return 1 + 2 * r.x - 3 * r.y + .5 * r.z + .7 * r.x * r.x - .2 * r.y * r.y + .4 * r.z * r.z +
               .3 * r.x * r.y - .1 * r.x * r.z + .25 * r.y * r.z;
    };
    std::array<double, K * K> M{};
    std::array<double, K> b{};
    double ws = 0, fi = f(ps[i].r);
    for (int j : h->nd.list[i]) {
        auto d = ps[j].r - ps[i].r;
        double r = norm(d), w = weight(r, re);
        if (!w) continue;
        auto q = basis(d, r, cfg.l0);
        double df = f(ps[j].r) - fi;
        ws += w;
        for (int a = 0; a < K; ++a) {
            b[a] += w * q[a] * df / r;
            for (int c = 0; c < K; ++c) M[a * K + c] += w * q[a] * q[c];
        }
    }
    if (ws <= 0) return -1;
    for (double& x : M) x /= ws;
    for (double& x : b) x /= ws;
    bool reg = false;
    if (!cholesky(M, cfg.wls_regularization, reg)) return -2;
    auto x = solve(M, b);
    for (int a = 0; a < K; ++a) x9[a] = x[a];
    return reg ? 1 : 0;
}

// assemble_ppe (src/lsmps.cpp:30-64). First call with col == nullptr to get sizes.
// sizes[0]=unknowns, [1]=nnz, [2]=dirichlet, [3]=neumann, [4]=failed_rows.
void ref_assemble_ppe(void* hv, long long* sizes, int* row, int* col, double* val, double* b,
                      double* x_exact) {
    auto* h = static_cast<RefCase*>(hv);
    h->ppe_assembly = lsmps::PpeStats{};
    h->A = lsmps::assemble_ppe(h->cfg, h->ps, h->nd, h->ppe_assembly);
    const auto& st = h->ppe_assembly;
    sizes[0] = (long long)st.unknowns; sizes[1] = (long long)st.nnz; sizes[2] = (long long)st.dirichlet;
    sizes[3] = (long long)st.neumann; sizes[4] = (long long)st.failed_rows;
    if (row) std::memcpy(row, h->A.row.data(), h->A.row.size() * sizeof(int));
    if (col) std::memcpy(col, h->A.col.data(), h->A.col.size() * sizeof(int));
    if (val) std::memcpy(val, h->A.val.data(), h->A.val.size() * sizeof(double));
    if (b) std::memcpy(b, h->A.b.data(), h->A.b.size() * sizeof(double));
    if (x_exact) std::memcpy(x_exact, h->A.x_exact.data(), h->A.x_exact.size() * sizeof(double));
}

// solve_ppe (src/lsmps.cpp:67): assembly + BiCGStab. out: iterations, converged,
// initial_residual, final_residual, relative_l2_error, max_error, assembly_ms, solve_ms,
// unknowns, nnz.
void ref_solve_ppe(void* hv, double* out10) {
    auto* h = static_cast<RefCase*>(hv);
    auto st = lsmps::solve_ppe(h->cfg, h->ps, h->nd);
    double o[10] = {(double)st.iterations, st.converged ? 1.0 : 0.0, st.initial_residual,
                    st.final_residual, st.relative_l2_error, st.max_error, st.assembly_ms,
                    st.solve_ms, (double)st.unknowns, (double)st.nnz};
    std::memcpy(out10, o, sizeof(o));
}

// The reference's BiCGStab on caller-provided CSR data (src/lsmps.cpp:65-67), used to
// time the reference's solver on matrices it does not assemble itself.
// out: iterations, converged, final_residual(|Ax-b|), rel_l2 vs x_exact, max_error, solve_ms.
void ref_bicgstab_csr(size_t n, const int* row, const int* col, const double* val,
                      const double* b, const double* x_exact, int max_iter, double tol,
                      double* x_out, double* out6) {
    lsmps::CSR A;
    A.row.assign(row, row + n + 1);
    A.col.assign(col, col + row[n]);
    A.val.assign(val, val + row[n]);
    A.b.assign(b, b + n);
    A.x_exact.assign(x_exact, x_exact + n);
    auto t0 = lsmps::Clock::now();
    std::vector<double> x(n, 0), r = A.b, r0 = r, p(n), v(n), s(n), t(n), Ax;
    double bnorm = std::sqrt(lsmps::dot(A.b, A.b));
    double rho0 = 1, alpha = 1, omega = 1;
    int iters = 0;
    bool conv = false;
    // Same iteration as solve_ppe (src/lsmps.cpp:67), restated over a caller CSR.
    for (int it = 0; it < max_iter; ++it) {
        double rho = lsmps::dot(r0, r);
        if (std::abs(rho) < 1e-30) break;
        double beta = (rho / rho0) * (alpha / omega);
        for (size_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
        lsmps::spmv(A, p, v);
        double den = lsmps::dot(r0, v);
        if (std::abs(den) < 1e-30) break;
        alpha = rho / den;
        for (size_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        double sn = std::sqrt(lsmps::dot(s, s));
        if (sn <= tol * std::max(1.0, bnorm)) {
            for (size_t i = 0; i < n; ++i) x[i] += alpha * p[i];
            iters = it + 1; conv = true; r = s; break;
        }
        lsmps::spmv(A, s, t);
        double tt = lsmps::dot(t, t);
        if (tt < 1e-30) break;
        omega = lsmps::dot(t, s) / tt;
        for (size_t i = 0; i < n; ++i) x[i] += alpha * p[i] + omega * s[i];
        for (size_t i = 0; i < n; ++i) r[i] = s[i] - omega * t[i];
        double rn = std::sqrt(lsmps::dot(r, r));
        iters = it + 1;
        if (rn <= tol * std::max(1.0, bnorm)) { conv = true; break; }
        if (std::abs(omega) < 1e-30) break;
        rho0 = rho;
    }
    lsmps::spmv(A, x, Ax);
    double res = 0, se = 0, mx = 0, exn = 0;
    for (size_t i = 0; i < n; ++i) {
        double d = Ax[i] - A.b[i]; res += d * d;
        double e = x[i] - A.x_exact[i]; se += e * e;
        exn += A.x_exact[i] * A.x_exact[i];
        mx = std::max(mx, std::abs(e));
    }
    double ms = std::chrono::duration<double, std::milli>(lsmps::Clock::now() - t0).count();
    double o[6] = {(double)iters, conv ? 1.0 : 0.0, std::sqrt(res),
                   std::sqrt(se / std::max(exn, 1e-30)), mx, ms};
    std::memcpy(out6, o, sizeof(o));
    if (x_out) std::memcpy(x_out, x.data(), n * sizeof(double));
}

// run_benchmark (src/lsmps.cpp:73) + writers (:74-75). out (22 doubles): particles,
// interior, free_surface, splash, near_wall, wall, pairs, truncated, mean, p50, p90, p99,
// neighbor_ms, classify_ms, wls_ms, wls.sampled, wls.failed, ppe.unknowns, ppe.nnz,
// ppe.iterations, ppe.converged, ppe.rel_l2.
void ref_run_benchmark(void* hv, double* out22) {
    auto* h = static_cast<RefCase*>(hv);
    h->metrics = lsmps::run_benchmark(h->cfg, h->ps);
    const auto& m = h->metrics;
    double o[22] = {(double)m.particles, (double)m.interior, (double)m.free_surface,
                    (double)m.splash, (double)m.near_wall, (double)m.wall,
                    (double)m.neighbor_pairs, (double)m.truncated_particles, m.neighbor_mean,
                    (double)m.neighbor_p50, (double)m.neighbor_p90, (double)m.neighbor_p99,
                    m.neighbor_ms, m.classify_ms, m.wls_ms, (double)m.wls.sampled,
                    (double)m.wls.failed, (double)m.ppe.unknowns, (double)m.ppe.nnz,
                    (double)m.ppe.iterations, m.ppe.converged ? 1.0 : 0.0,
                    m.ppe.relative_l2_error};
    std::memcpy(out22, o, sizeof(o));
}

void ref_write_outputs(void* hv, const char* json_path, const char* csv_path) {
    auto* h = static_cast<RefCase*>(hv);
    if (json_path) lsmps::write_json(json_path, h->cfg, h->metrics);
    if (csv_path) lsmps::write_csv(csv_path, h->cfg, h->metrics);
}

}  // extern "C"
