// Host side of the drop-in: include/lsmps.hpp implemented over the sm_100a C ABI.
//
// load_config keeps the reference's .cfg grammar (src/lsmps.cpp:20,71); generate_case
// draws the reference's cases with the same std::mt19937 / uniform_real_distribution
// call sequence, so positions are bit-identical (src/lsmps.cpp:68,72), and adds the
// rain-on-plate and mixed generators; run_benchmark (src/lsmps.cpp:73) runs neighbor build
// + classification, WLS, PPE assembly and solve on the GPU; write_json / write_csv emit
// the reference's bytes (src/lsmps.cpp:74-75).
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "lsmps.hpp"
#include "lsmps_gpu.h"

namespace lsmps {
namespace {

std::string strip(const std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) ++b;
    while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
    return s.substr(b, e - b);
}

// Applies one key=value pair. The reference's keys are parsed exactly as the reference
// does (std::stoull / stoul / stod / stoi); the others are this library's extensions,
// which the reference's parser ignores. Returns false for an unknown key.
bool apply_key(Config& c, const std::string& k, const std::string& v) {
    // reference keys (src/lsmps.cpp:71)
    if (k == "case") c.case_name = v;
    else if (k == "particles") c.particles = std::stoull(v);
    else if (k == "seed") c.seed = (uint32_t)std::stoul(v);
    else if (k == "l0") c.l0 = std::stod(v);
    else if (k == "re_ratio") c.re_ratio = std::stod(v);
    else if (k == "film_layers") c.film_layers = std::stoi(v);
    else if (k == "max_neighbors") c.max_neighbors = std::stoi(v);
    else if (k == "wls_samples") c.wls_samples = std::stoi(v);
    else if (k == "ppe_max_unknowns") c.ppe_max_unknowns = std::stoi(v);
    else if (k == "ppe_max_iter") c.ppe_max_iter = std::stoi(v);
    else if (k == "ppe_tol") c.ppe_tol = std::stod(v);
    else if (k == "boundary_constraint_weight") c.boundary_constraint_weight = std::stod(v);
    else if (k == "virtual_weight") c.virtual_weight = std::stod(v);
    // extensions
    else if (k == "jitter") c.jitter = std::stod(v);
    else if (k == "ppe_variant") c.ppe_variant = v;
    else if (k == "ppe_diag_shift") c.ppe_diag_shift = std::stod(v);
    else if (k == "solver") c.solver = v;
    else if (k == "wls_mode") c.wls_mode = v;
    else if (k == "wls_precision") c.wls_precision = v;
    else if (k == "device") c.device = std::stoi(v);
    else if (k == "mpnn_weights") c.mpnn_weights = v;
    else if (k == "precond") c.precond = v;
    else return false;
    return true;
}

// lattice (src/lsmps.cpp:68): k, j, i loops, positions ((i + .5 + u) l0, ...) with u drawn
// for x, y, z in that order; the bottom layer is Wall when requested.
void lattice(std::vector<Particle>& out, size_t target, int nx, int ny, int nz, double l0, double jit,
             std::mt19937& rng, bool bottom_wall) {
    std::uniform_real_distribution<double> u(-jit, jit);
    for (int k = 0; k < nz && out.size() < target; ++k)
        for (int j = 0; j < ny && out.size() < target; ++j)
            for (int i = 0; i < nx && out.size() < target; ++i) {
                Particle q;
                double dx = u(rng);
                double dy = u(rng);
                double dz = u(rng);
                q.r = {(i + .5 + dx) * l0, (j + .5 + dy) * l0, (k + .5 + dz) * l0};
                if (bottom_wall && k == 0) q.type = ParticleType::Wall;
                out.push_back(q);
            }
}

double jitter_or(const Config& c, double dflt) { return c.jitter >= 0 ? c.jitter : dflt; }

// Rain on an inclined plate (this library's generator; the reference has none in 3-D):
// a plate through the origin rising along +x at angle theta, `wall_layers` layers of Wall
// particles below its surface and `film_layers` fluid layers above it (square m x m sites
// per layer, spacing l0, jittered), holding film_fraction of the fluid; the remaining
// fluid falls as droplets: jittered cubic-lattice spheres of radius R l0 whose centres
// sit at uniform random plate coordinates and heights h in [hmin, hmax] l0 above the
// plate, with velocity (0, 0, -v l0) per step. Droplets may overlap one another, which is
// what skews the neighbor counts.
struct RainPlate {
    double theta_deg = 20.0;
    int wall_layers = 3;
    int film_layers = 4;
    double film_fraction = 0.7;
    double radius = 3.0, hmin = 10.0, hmax = 40.0, speed = 5.0;
};

void rain_plate(std::vector<Particle>& out, size_t count, double l0, double jit, const RainPlate& rp,
                double x_offset, std::mt19937& rng) {
    const double th = rp.theta_deg * 3.14159265358979323846 / 180.0;
    const Vec3 t1{std::cos(th), 0, std::sin(th)}, t2{0, 1, 0}, nrm{-std::sin(th), 0, std::cos(th)};
    const double per_site = rp.wall_layers + rp.film_layers / rp.film_fraction;
    int m = std::max(4, (int)std::floor(std::sqrt((double)count / per_site)));
    std::uniform_real_distribution<double> u(-jit, jit);
    const size_t start = out.size();
    auto emit_layer = [&](double h, ParticleType type) {
        for (int b = 0; b < m && out.size() - start < count; ++b)
            for (int a = 0; a < m && out.size() - start < count; ++a) {
                double ds = u(rng), dy = u(rng), dh = u(rng);
                double s = (a + .5 + ds) * l0, y = (b + .5 + dy) * l0, hh = (h + dh) * l0;
                Particle q;
                q.r = t1 * s + t2 * y + nrm * hh;
                q.r.x += x_offset;
                q.type = type;
                out.push_back(q);
            }
    };
    for (int k = 0; k < rp.wall_layers; ++k) emit_layer(-(k + .5), ParticleType::Wall);
    for (int k = 0; k < rp.film_layers; ++k) emit_layer(k + .5, ParticleType::Interior);
    // droplet template: integer lattice points within the radius
    std::vector<Vec3> tmpl;
    int R = (int)std::ceil(rp.radius);
    for (int k = -R; k <= R; ++k)
        for (int j = -R; j <= R; ++j)
            for (int i = -R; i <= R; ++i)
                if (i * i + j * j + k * k <= rp.radius * rp.radius) tmpl.push_back({(double)i, (double)j, (double)k});
    std::uniform_real_distribution<double> us(0.0, m * l0), uh(rp.hmin * l0, rp.hmax * l0);
    while (out.size() - start < count) {
        double s = us(rng), y = us(rng), h = uh(rng);
        Vec3 c = t1 * s + t2 * y + nrm * h;
        c.x += x_offset;
        for (const auto& o : tmpl) {
            if (out.size() - start >= count) break;
            double dx = u(rng), dy = u(rng), dz = u(rng);
            Particle q;
            q.r = {c.x + (o.x + dx) * l0, c.y + (o.y + dy) * l0, c.z + (o.z + dz) * l0};
            q.u = {0, 0, -rp.speed * l0};
            q.type = ParticleType::Interior;
            out.push_back(q);
        }
    }
}

}  // namespace

const char* type_name(ParticleType t) {
    switch (t) {
        case ParticleType::Interior: return "interior";
        case ParticleType::FreeSurface: return "free_surface";
        case ParticleType::Splash: return "splash";
        case ParticleType::NearWall: return "near_wall";
        case ParticleType::Wall: return "wall";
    }
    return "unknown";
}

Config load_config(const std::string& path) {
    std::ifstream in(path);
    if (!in) throw std::runtime_error("cannot open config: " + path);
    Config c;
    std::string line;
    while (std::getline(in, line)) {
        size_t hash = line.find('#');
        if (hash != std::string::npos) line.erase(hash);
        size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        apply_key(c, strip(line.substr(0, eq)), strip(line.substr(eq + 1)));
    }
    return c;
}

std::vector<Particle> generate_case(const Config& c) {
    std::mt19937 rng(c.seed);
    std::vector<Particle> p;
    p.reserve(c.particles);
    int nx = std::max(4, (int)std::ceil(std::cbrt((double)c.particles)));
    int ny = nx, nz = nx;
    const std::string& cs = c.case_name;
    if (cs == "wall_film") {
        nz = std::max(3, c.film_layers + 1);
        nx = std::max(8, (int)std::ceil(std::sqrt((double)c.particles / nz)));
        ny = nx;
        lattice(p, c.particles, nx, ny, nz, c.l0, jitter_or(c, .04), rng, true);
    } else if (cs == "narrow_gap") {
        nz = std::max(4, c.film_layers + 2);
        nx = std::max(8, (int)std::ceil(std::sqrt((double)c.particles / nz)));
        ny = nx;
        lattice(p, c.particles, nx, ny, nz, c.l0, jitter_or(c, .02), rng, true);
        for (auto& q : p)
            if (q.r.z > (nz - 1.5) * c.l0) q.type = ParticleType::Wall;
    } else if (cs == "rain_injection") {
        size_t film = (size_t)(.75 * c.particles);
        nz = std::max(3, c.film_layers + 1);
        nx = std::max(8, (int)std::ceil(std::sqrt((double)film / nz)));
        ny = nx;
        lattice(p, film, nx, ny, nz, c.l0, jitter_or(c, .05), rng, true);
        std::uniform_real_distribution<double> ux(0, nx * c.l0), uy(0, ny * c.l0), uz(4 * c.l0, 20 * c.l0);
        while (p.size() < c.particles) {
            Particle q;
            double x = ux(rng);
            double y = uy(rng);
            double z = uz(rng);
            q.r = {x, y, z};
            q.u = {0, 0, -5};
            q.type = ParticleType::Splash;
            p.push_back(q);
        }
    } else if (cs == "rain_plate") {
        rain_plate(p, c.particles, c.l0, jitter_or(c, .1), RainPlate{}, 0.0, rng);
    } else if (cs == "mixed") {
        // 80 % bulk jittered lattice, 20 % rain on a plate placed beside it; the plate starts
        // 25 l0 past the block so that droplets (up to 40 l0 above the 20-degree plate, which
        // shifts them by up to 14 l0 in -x) stay clear of it
        size_t nbulk = (size_t)(0.8 * (double)c.particles);
        int nb = std::max(4, (int)std::ceil(std::cbrt((double)nbulk)));
        lattice(p, nbulk, nb, nb, nb, c.l0, jitter_or(c, .1), rng, false);
        rain_plate(p, c.particles - p.size(), c.l0, jitter_or(c, .1), RainPlate{}, (nb + 25) * c.l0, rng);
    } else {
        lattice(p, c.particles, nx, ny, nz, c.l0, jitter_or(c, .03), rng, false);
    }
    return p;
}

namespace {
struct Ctx {
    lsmps_ctx* p = nullptr;
    explicit Ctx(int device) {
        int rc = lsmps_ctx_create(device, &p);
        if (rc != LSMPS_OK) throw std::runtime_error("cannot create GPU context on device " + std::to_string(device) +
                                                     " (status " + std::to_string(rc) + ")");
    }
    ~Ctx() { lsmps_ctx_destroy(p); }
    void check(int rc, const char* what) const {
        if (rc != LSMPS_OK)
            throw std::runtime_error(std::string(what) + " failed (status " + std::to_string(rc) + "): " +
                                     lsmps_last_error(p));
    }
};

int solver_id(const std::string& s) {
    if (s == "reference") return LSMPS_SOLVER_REFERENCE;
    if (s == "fp64") return LSMPS_SOLVER_FP64;
    if (s == "jacobi") return LSMPS_SOLVER_JACOBI;
    if (s == "mixed") return LSMPS_SOLVER_MIXED;
    if (s == "learned") return LSMPS_SOLVER_LEARNED;
    if (s == "mixed_f32") return LSMPS_SOLVER_MIXED_F32;
    throw std::runtime_error("unknown solver: " + s);
}

int precond_id(const std::string& s) {
    if (s == "jacobi") return LSMPS_PRECOND_JACOBI;
    if (s == "multigrid") return LSMPS_PRECOND_MULTIGRID;
    throw std::runtime_error("unknown precond: " + s);
}

int variant_id(const std::string& s) {
    if (s == "reference") return LSMPS_PPE_REFERENCE;
    if (s == "shifted") return LSMPS_PPE_SHIFTED;
    if (s == "wls") return LSMPS_PPE_WLS;
    throw std::runtime_error("unknown ppe_variant: " + s);
}
}  // namespace

Metrics run_benchmark(const Config& c, std::vector<Particle>& ps) {
    Metrics m;
    m.particles = ps.size();
    const size_t n = ps.size();
    const double re = c.re_ratio * c.l0;  // as src/lsmps.cpp:73 passes it
    Ctx ctx(c.device);
    std::vector<double> xyz(3 * n);
    std::vector<uint8_t> type(n);
    for (size_t i = 0; i < n; ++i) {
        xyz[3 * i] = ps[i].r.x;
        xyz[3 * i + 1] = ps[i].r.y;
        xyz[3 * i + 2] = ps[i].r.z;
        type[i] = static_cast<uint8_t>(ps[i].type);
    }
    ctx.check(lsmps_upload_particles(ctx.p, xyz.data(), type.data(), n), "upload");
    lsmps_neighbor_stats ns{};
    ctx.check(lsmps_build_neighbors(ctx.p, re, c.max_neighbors, c.l0, LSMPS_NBR_CLASSIFY, &ns), "neighbor build");
    ctx.check(lsmps_download_types(ctx.p, type.data(), n), "type download");
    for (size_t i = 0; i < n; ++i) ps[i].type = static_cast<ParticleType>(type[i]);  // in place, as the reference
    double tm[8];
    lsmps_get_timings(ctx.p, tm);
    m.upload_ms = tm[0];
    m.neighbor_ms = tm[1];  // neighbor build with the classification fused into its fill pass
    m.classify_ms = 0.0;
    m.neighbor_pairs = ns.pairs;
    m.truncated_particles = ns.truncated;
    m.neighbor_mean = ns.mean;
    m.neighbor_p50 = ns.p50;
    m.neighbor_p90 = ns.p90;
    m.neighbor_p99 = ns.p99;
    m.interior = ns.type_count[LSMPS_INTERIOR];
    m.free_surface = ns.type_count[LSMPS_FREE_SURFACE];
    m.splash = ns.type_count[LSMPS_SPLASH];
    m.near_wall = ns.type_count[LSMPS_NEAR_WALL];
    m.wall = ns.type_count[LSMPS_WALL];

    // WLS: the reference's sampled test, or every particle
    const int variant = variant_id(c.ppe_variant);
    static const double kRefQuad[10] = {1, 2, -3, 0.5, 0.7, -0.2, 0.4, 0.3, -0.1, 0.25};
    lsmps_wls_stats ws{};
    lsmps_wls_opts wo{};
    wo.re = re;
    wo.l0 = c.l0;
    wo.regularization = c.wls_regularization;
    wo.wls_samples = c.wls_samples;
    wo.nrhs = 1;
    wo.quad_coef = kRefQuad;
    wo.precision = c.wls_precision == "mixed" ? 1 : 0;
    double wls_ms = 0;
    if (c.wls_mode == "all") {
        wo.mode = 1;
        ctx.check(lsmps_wls(ctx.p, &wo, &ws), "WLS");
        lsmps_get_timings(ctx.p, tm);
        wls_ms += tm[3];
    } else {
        wo.mode = 0;
        ctx.check(lsmps_wls(ctx.p, &wo, &ws), "WLS");
        lsmps_get_timings(ctx.p, tm);
        wls_ms += tm[3];
        if (variant == LSMPS_PPE_WLS) {  // the WLS PPE needs every particle's operator
            lsmps_wls_stats tmp{};
            wo.mode = 1;
            ctx.check(lsmps_wls(ctx.p, &wo, &tmp), "WLS");
            lsmps_get_timings(ctx.p, tm);
            wls_ms += tm[3];
        }
    }
    m.wls_ms = wls_ms;
    m.wls.sampled = ws.sampled;
    m.wls.ok = ws.ok;
    m.wls.regularized = ws.regularized;
    m.wls.failed = ws.failed;
    m.wls.virtual_points = ws.virtual_points;
    m.wls.max_gradient_error = ws.max_gradient_error;
    m.wls.rms_gradient_error = ws.rms_gradient_error;
    m.wls.max_laplacian_error = ws.max_laplacian_error;
    m.wls.rms_laplacian_error = ws.rms_laplacian_error;

    // PPE (src/lsmps.cpp:67 solve_ppe = assemble + BiCGStab)
    lsmps_ppe_opts po{};
    po.variant = variant;
    po.max_unknowns = c.ppe_max_unknowns;
    po.re = re;
    po.l0 = c.l0;
    po.diag_shift = c.ppe_diag_shift;
    lsmps_ppe_stats pst{};
    ctx.check(lsmps_ppe_assemble(ctx.p, &po, &pst), "PPE assembly");
    lsmps_solver_opts so{};
    so.solver = solver_id(c.solver);
    so.precond = precond_id(c.precond);
    so.max_iter = c.ppe_max_iter;
    so.tol = c.ppe_tol;
    so.use_graph = 1;
    if (so.solver == LSMPS_SOLVER_LEARNED) {
        if (c.mpnn_weights.empty()) throw std::runtime_error("solver=learned needs mpnn_weights=<file>");
        ctx.check(lsmps_mpnn_load(ctx.p, c.mpnn_weights.c_str()), "network load");
    }
    double assembly_ms = pst.assembly_ms;
    ctx.check(lsmps_ppe_solve(ctx.p, &so, &pst), "PPE solve");
    m.ppe.unknowns = pst.unknowns;
    m.ppe.nnz = pst.nnz;
    m.ppe.dirichlet = pst.dirichlet;
    m.ppe.neumann = pst.neumann;
    m.ppe.failed_rows = pst.failed_rows;
    m.ppe.iterations = pst.iterations;
    m.ppe.initial_residual = pst.initial_residual;
    m.ppe.final_residual = pst.final_residual;
    m.ppe.relative_l2_error = pst.relative_l2_error;
    m.ppe.max_error = pst.max_error;
    m.ppe.assembly_ms = assembly_ms;
    m.ppe.solve_ms = pst.solve_ms;
    m.ppe.converged = pst.converged != 0;
    m.outer_iterations = pst.outer_iterations;
    m.fallback = pst.fallback;
    return m;
}

// write_json (src/lsmps.cpp:74): fixed notation, 8 decimals, fixed field order.
void write_json(const std::string& path, const Config& c, const Metrics& m) {
    std::ofstream o(path);
    if (!o) throw std::runtime_error("cannot write " + path);
    o << std::fixed << std::setprecision(8);
    o << "{\n";
    o << "  \"case\": \"" << c.case_name << "\",\n";
    o << "  \"particles\": " << m.particles << ",\n";
    o << "  \"types\": {\"interior\": " << m.interior << ", \"free_surface\": " << m.free_surface
      << ", \"splash\": " << m.splash << ", \"near_wall\": " << m.near_wall << ", \"wall\": " << m.wall << "},\n";
    o << "  \"neighbors\": {\"pairs\": " << m.neighbor_pairs << ", \"mean\": " << m.neighbor_mean
      << ", \"p50\": " << m.neighbor_p50 << ", \"p90\": " << m.neighbor_p90 << ", \"p99\": " << m.neighbor_p99
      << ", \"truncated\": " << m.truncated_particles << "},\n";
    o << "  \"wls\": {\"sampled\": " << m.wls.sampled << ", \"regularized\": " << m.wls.regularized
      << ", \"failed\": " << m.wls.failed << ", \"virtual_points\": " << m.wls.virtual_points
      << ", \"gradient_rms_error\": " << m.wls.rms_gradient_error
      << ", \"laplacian_rms_error\": " << m.wls.rms_laplacian_error << "},\n";
    o << "  \"ppe\": {\"unknowns\": " << m.ppe.unknowns << ", \"nnz\": " << m.ppe.nnz
      << ", \"dirichlet\": " << m.ppe.dirichlet << ", \"neumann\": " << m.ppe.neumann
      << ", \"failed_rows\": " << m.ppe.failed_rows << ", \"iterations\": " << m.ppe.iterations
      << ", \"converged\": " << (m.ppe.converged ? "true" : "false")
      << ", \"final_residual\": " << m.ppe.final_residual
      << ", \"relative_l2_error\": " << m.ppe.relative_l2_error << ", \"assembly_ms\": " << m.ppe.assembly_ms
      << ", \"solve_ms\": " << m.ppe.solve_ms << "}\n";
    o << "}\n";
}

// write_csv (src/lsmps.cpp:75): header line and one row, default stream formatting.
void write_csv(const std::string& path, const Config& c, const Metrics& m) {
    std::ofstream o(path);
    if (!o) throw std::runtime_error("cannot write " + path);
    o << "case,particles,interior,free_surface,splash,near_wall,wall,neighbor_mean,p50,p90,p99,wls_failed,"
         "wls_virtual,ppe_unknowns,ppe_nnz,ppe_iterations,ppe_converged,ppe_residual,ppe_rel_l2,"
         "ppe_assembly_ms,ppe_solve_ms\n";
    const char s = ',';
    o << c.case_name << s << m.particles << s << m.interior << s << m.free_surface << s << m.splash << s
      << m.near_wall << s << m.wall << s << m.neighbor_mean << s << m.neighbor_p50 << s << m.neighbor_p90 << s
      << m.neighbor_p99 << s << m.wls.failed << s << m.wls.virtual_points << s << m.ppe.unknowns << s
      << m.ppe.nnz << s << m.ppe.iterations << s << m.ppe.converged << s << m.ppe.final_residual << s
      << m.ppe.relative_l2_error << s << m.ppe.assembly_ms << s << m.ppe.solve_ms << '\n';
}

}  // namespace lsmps

// ---- C host helpers ------------------------------------------------------------------
extern "C" int lsmps_host_generate(const char* cfg_path, const char* overrides, double* xyz, uint8_t* type,
                                   double* uvw, size_t* n) {
    if (!n) return LSMPS_ERR_ARG;
    try {
        lsmps::Config c = cfg_path && *cfg_path ? lsmps::load_config(cfg_path) : lsmps::Config{};
        if (overrides) {
            std::stringstream ss(overrides);
            std::string kv;
            while (std::getline(ss, kv, ';')) {
                size_t eq = kv.find('=');
                if (eq == std::string::npos) continue;
                std::string k = lsmps::strip(kv.substr(0, eq)), v = lsmps::strip(kv.substr(eq + 1));
                if (!lsmps::apply_key(c, k, v)) return LSMPS_ERR_ARG;
            }
        }
        auto p = lsmps::generate_case(c);
        if (!xyz) {
            *n = p.size();
            return LSMPS_OK;
        }
        if (*n < p.size()) return LSMPS_ERR_ARG;
        for (size_t i = 0; i < p.size(); ++i) {
            xyz[3 * i] = p[i].r.x;
            xyz[3 * i + 1] = p[i].r.y;
            xyz[3 * i + 2] = p[i].r.z;
            if (type) type[i] = static_cast<uint8_t>(p[i].type);
            if (uvw) {
                uvw[3 * i] = p[i].u.x;
                uvw[3 * i + 1] = p[i].u.y;
                uvw[3 * i + 2] = p[i].u.z;
            }
        }
        *n = p.size();
        return LSMPS_OK;
    } catch (const std::exception&) {
        return LSMPS_ERR_IO;
    }
}
