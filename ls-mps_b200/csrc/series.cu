// Step series of a 3-D rain-on-plate proxy on one context. Particles move with fixed
// kinematics (wall fixed, droplets fall, film slides down the plate); droplets are injected
// above the plate every step; particles past the plate's lower edge (the outflow plane) leave.
// Every step runs the full per-step path: neighbor lists (candidate lists of radius re + skin
// rebuilt every cnl_rebuild_interval steps, filtered in between), classification, all-particle
// WLS, WLS-Laplacian PPE assembly, and the PPE solve warm-started from the previous step's
// pressure per particle. The particle set the PPE sees is fixed between rebuilds: injected
// droplets wait in flight and flagged outflow particles stay until the next rebuild, where
// they join or leave. The fluid particle count is taken on the device every step and checked
// against the injection/outflow bookkeeping (mass balance).
//
// The reference's step series is the 2-D penalty-force baseline python/rain_plate_cpu.py
// (inject:67-87, remove_outflow:146-154) and the keys steps / injected_per_step /
// cnl_rebuild_interval of config/rain_injection.cfg, which its C++ benchmark does not parse.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <vector>

#include "ops.cuh"
#include "scan.cuh"

namespace lsmps_gpu {
namespace {

enum : uint8_t { MAT_WALL = 0, MAT_FILM = 1, MAT_DROP = 2 };

struct Frame {
    double t1x, t1z;    // down-slope is -t1 (t1 = (cos a, 0, sin a))
    double nx, nz;      // plate normal (-sin a, 0, cos a)
    double vd, vf;      // droplet fall and film slide per step (length units)
    double film_top;    // normal coordinate where a droplet joins the film
    double plate_len;   // L: u = 1 - s / L
};

// sections of the validation outputs, as the advance kernel counts them
struct Sections {
    int n;
    double u[LSMPS_RAIN_MAX_SECTIONS], maxd[LSMPS_RAIN_MAX_SECTIONS];
};

__device__ __forceinline__ double plate_u(const Frame& F, double x, double z) {
    return 1.0 - (x * F.t1x + z * F.t1z) / F.plate_len;
}

__global__ void k_advance(size_t n, double* __restrict__ pos, uint8_t* __restrict__ mat, uint8_t* __restrict__ del,
                          Frame F, Sections SC, unsigned long long* __restrict__ crossings) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        uint8_t m = mat[i];
        if (m == MAT_WALL) continue;
        double x = pos[3 * i], z = pos[3 * i + 2];
        const double u0 = plate_u(F, x, z);
        if (m == MAT_DROP) {
            z -= F.vd;
            if (x * F.nx + z * F.nz <= F.film_top) {
                m = MAT_FILM;
                mat[i] = m;
            }
        } else {
            x -= F.vf * F.t1x;
            z -= F.vf * F.t1z;
        }
        pos[3 * i] = x;
        pos[3 * i + 2] = z;
        if (x * F.t1x + z * F.t1z < 0.0) del[i] = 1;  // past the outflow edge
        const double u1 = plate_u(F, x, z), d = x * F.nx + z * F.nz;
        for (int c = 0; c < SC.n; ++c)
            if (u0 < SC.u[c] && u1 >= SC.u[c] && d >= 0.0 && d <= SC.maxd[c]) atomicAdd(&crossings[c], 1ull);
    }
}

// windows of the validation outputs: per window and cell along u, the fluid particle count
// and the largest thickness d + l0 (non-negative doubles order as their bits)
struct Windows {
    int n, cells;
    double wet, l0;
    double lo[LSMPS_RAIN_MAX_WINDOWS], hi[LSMPS_RAIN_MAX_WINDOWS];
};

__global__ void k_rain_windows(size_t n, const double* __restrict__ pos, const uint8_t* __restrict__ mat, Frame F,
                               Windows W, unsigned long long* __restrict__ count,
                               unsigned long long* __restrict__ thick) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        if (mat[i] == MAT_WALL) continue;
        const double x = pos[3 * i], z = pos[3 * i + 2];
        const double u = plate_u(F, x, z), d = x * F.nx + z * F.nz;
        if (d < 0.0 || d > W.wet) continue;
        for (int w = 0; w < W.n; ++w) {
            if (u < W.lo[w] || u >= W.hi[w]) continue;
            const int c = min(W.cells - 1, (int)((u - W.lo[w]) / (W.hi[w] - W.lo[w]) * W.cells));
            const size_t slot = (size_t)w * LSMPS_RAIN_MAX_CELLS + c;
            atomicAdd(&count[slot], 1ull);
            atomicMax(&thick[slot], (unsigned long long)__double_as_longlong(d + W.l0));
        }
    }
}

// keep[i] = 1 - del[i] over the particle set followed by the in-flight set
__global__ void k_keep_flags(size_t n, const uint8_t* __restrict__ del, size_t nq, const uint8_t* __restrict__ qdel,
                             int* __restrict__ keep) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n + nq; i += (size_t)gridDim.x * blockDim.x)
        keep[i] = i < n ? !del[i] : !qdel[i - n];
}

__global__ void k_compact(size_t n, size_t nq, const int* __restrict__ keep, const int* __restrict__ dest,
                          const double* __restrict__ pos, const uint8_t* __restrict__ mat,
                          const double* __restrict__ pres, const double* __restrict__ qpos,
                          const uint8_t* __restrict__ qmat, double* __restrict__ opos, uint8_t* __restrict__ omat,
                          uint8_t* __restrict__ otype, double* __restrict__ opres) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n + nq; i += (size_t)gridDim.x * blockDim.x) {
        if (!keep[i]) continue;
        const size_t d = (size_t)dest[i];
        const bool act = i < n;
        const size_t k = act ? i : i - n;
        const double* src = act ? pos : qpos;
        opos[3 * d] = src[3 * k];
        opos[3 * d + 1] = src[3 * k + 1];
        opos[3 * d + 2] = src[3 * k + 2];
        const uint8_t m = act ? mat[k] : qmat[k];
        omat[d] = m;
        otype[d] = m == MAT_WALL ? (uint8_t)LSMPS_WALL : (uint8_t)LSMPS_INTERIOR;
        opres[d] = act ? pres[k] : 0.0;
    }
}

// counts[0] += fluid particles, counts[1] += flagged particles
__global__ void k_count(size_t n, const uint8_t* __restrict__ mat, const uint8_t* __restrict__ del,
                        unsigned long long* counts) {
    unsigned long long f = 0, d = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        f += mat[i] != MAT_WALL;
        d += del[i] != 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        f += __shfl_xor_sync(0xffffffffu, f, o);
        d += __shfl_xor_sync(0xffffffffu, d, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (f) atomicAdd(&counts[0], f);
        if (d) atomicAdd(&counts[1], d);
    }
}

unsigned grid_for(size_t n) { return std::max(1u, std::min<unsigned>(blocks_for(n, 256), 148 * 8)); }

// the reference's wls_test field (src/lsmps.cpp:28); the PPE rows do not depend on it
const double kQuadratic[10] = {1, 2, -3, 0.5, 0.7, -0.2, 0.4, 0.3, -0.1, 0.25};

}  // namespace
}  // namespace lsmps_gpu

using namespace lsmps_gpu;

struct lsmps_series {
    lsmps_ctx* ctx = nullptr;
    lsmps_series_params p{};
    Frame F{};
    double plate_len = 0, plate_wid = 0;
    // the context's particle set (caller order): positions, material, type, pressure, outflow flag
    DevBuf pos, mat, type, pres, del;
    size_t n = 0;
    // injected, waiting for the next rebuild
    DevBuf qpos, qmat, qdel;
    size_t nq = 0, qcap = 0;
    DevBuf keep, dest, opos, omat, otype, opres, counts;
    uint64_t fluid0 = 0, injected_total = 0, deleted_total = 0;
    int step = 0;
    bool have_pressure = false;
    std::mt19937 rng;
    std::vector<double> tmpl;  // droplet lattice offsets (x, y, z) in l0
    cudaEvent_t ev[6] = {};
    lsmps_rain_validation vcfg{};
    lsmps_rain_outputs vout{};
    DevBuf vbuf;  // crossings [8], window counts [8 x 64], window thickness bits [8 x 64]
    ~lsmps_series() {
        DevBuf* bufs[] = {&pos, &mat, &type, &pres, &del, &qpos, &qmat, &qdel, &keep, &dest,
                          &opos, &omat, &otype, &opres, &counts, &vbuf};
        for (auto* b : bufs) b->release();
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
};

namespace lsmps_gpu {

void series_create(lsmps_ctx* ctx, const lsmps_series_params* pp, const double* xyz, const uint8_t* type, size_t n,
                   lsmps_series** out) {
    LSMPS_REQUIRE(pp && out && (n == 0 || (xyz && type)), LSMPS_ERR_ARG, "series arguments");
    const lsmps_series_params& p = *pp;
    LSMPS_REQUIRE(p.l0 > 0 && p.re > 0 && p.skin >= 0 && p.cnl_rebuild_interval >= 1 && p.injected_per_step >= 0,
                  LSMPS_ERR_ARG, "series parameters: l0, re > 0, skin >= 0, interval >= 1, injection >= 0");
    LSMPS_REQUIRE(p.solver >= LSMPS_SOLVER_FP64 && p.solver <= LSMPS_SOLVER_MIXED_F32, LSMPS_ERR_ARG,
                  "series solver must be one of the GPU solvers");
    LSMPS_REQUIRE(p.precond == LSMPS_PRECOND_JACOBI ||
                      (p.precond == LSMPS_PRECOND_MULTIGRID &&
                       (p.solver == LSMPS_SOLVER_MIXED || p.solver == LSMPS_SOLVER_LEARNED)),
                  LSMPS_ERR_ARG, "the multigrid preconditioner is for the MIXED and LEARNED solvers");
    LSMPS_REQUIRE(p.droplet_radius >= 0 && p.inject_hmax >= p.inject_hmin, LSMPS_ERR_ARG, "injection band");
    LSMPS_REQUIRE(p.max_candidates >= p.max_neighbors && p.max_neighbors >= 0, LSMPS_ERR_ARG,
                  "max_candidates must be at least max_neighbors");
    // the skin must cover the motion between rebuilds, else every refresh would force a rebuild
    const double per_step = std::max(p.droplet_speed, p.film_speed);
    LSMPS_REQUIRE(per_step * (p.cnl_rebuild_interval - 1) <= 0.5 * p.skin * (1.0 - 1e-9) || p.cnl_rebuild_interval == 1,
                  LSMPS_ERR_ARG, "skin / 2 must cover (interval - 1) steps of the fastest motion");
    auto S = std::make_unique<lsmps_series>();
    S->ctx = ctx;
    S->p = p;
    const double a = p.theta_deg * 3.14159265358979323846 / 180.0;
    S->F = Frame{std::cos(a), std::sin(a), -std::sin(a), std::cos(a), p.droplet_speed * p.l0, p.film_speed * p.l0,
                 p.film_thickness * p.l0};
    // plate extent from the wall particles (tangential coordinate s, span y); materials
    std::vector<uint8_t> m(n);
    double smax = 0, ymax = 0;
    for (size_t i = 0; i < n; ++i) {
        const double x = xyz[3 * i], y = xyz[3 * i + 1], z = xyz[3 * i + 2];
        if (type[i] == LSMPS_WALL) {
            m[i] = MAT_WALL;
            smax = std::max(smax, x * S->F.t1x + z * S->F.t1z);
            ymax = std::max(ymax, y);
        } else {
            const double h = x * S->F.nx + z * S->F.nz;
            m[i] = h > S->F.film_top + 0.5 * p.l0 ? MAT_DROP : MAT_FILM;
            S->fluid0 += 1;
        }
    }
    S->plate_len = smax;
    S->plate_wid = ymax;
    S->F.plate_len = std::max(smax, p.l0);
    // the reference's config/rain_plate_validation.json
    lsmps_rain_validation& v = S->vcfg;
    v.nwindows = 3;
    v.nsections = 2;
    v.coverage_cells = 32;
    v.min_particles_per_cell = 1;
    v.wet_distance_factor = 3.0;
    const double wl[3] = {0.1, 0.4, 0.75}, wh[3] = {0.35, 0.7, 0.95};
    for (int w = 0; w < 3; ++w) { v.window_lo[w] = wl[w]; v.window_hi[w] = wh[w]; }
    v.section_u[0] = 0.55; v.section_u[1] = 0.9;
    v.section_max_normal[0] = v.section_max_normal[1] = 5.0;
    S->vbuf.ensure<unsigned long long>(LSMPS_RAIN_MAX_SECTIONS + 2 * LSMPS_RAIN_MAX_WINDOWS * LSMPS_RAIN_MAX_CELLS);
    const int R = (int)std::ceil(p.droplet_radius);
    for (int k = -R; k <= R; ++k)
        for (int j = -R; j <= R; ++j)
            for (int i = -R; i <= R; ++i)
                if (i * i + j * j + k * k <= p.droplet_radius * p.droplet_radius) {
                    S->tmpl.push_back(i);
                    S->tmpl.push_back(j);
                    S->tmpl.push_back(k);
                }
    LSMPS_REQUIRE(!S->tmpl.empty() || p.injected_per_step == 0, LSMPS_ERR_ARG, "empty droplet template");
    S->rng.seed(p.seed);
    cudaStream_t s = ctx->stream;
    S->n = n;
    std::vector<uint8_t> t(n);
    for (size_t i = 0; i < n; ++i) t[i] = m[i] == MAT_WALL ? (uint8_t)LSMPS_WALL : (uint8_t)LSMPS_INTERIOR;
    double* dpos = S->pos.ensure<double>(3 * n + 3);
    uint8_t* dmat = S->mat.ensure<uint8_t>(n + 1);
    uint8_t* dtype = S->type.ensure<uint8_t>(n + 1);
    double* dpres = S->pres.ensure<double>(n + 1);
    uint8_t* ddel = S->del.ensure<uint8_t>(n + 1);
    if (n) {
        LSMPS_CUDA(cudaMemcpyAsync(dpos, xyz, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
        LSMPS_CUDA(cudaMemcpyAsync(dmat, m.data(), n, cudaMemcpyHostToDevice, s));
        LSMPS_CUDA(cudaMemcpyAsync(dtype, t.data(), n, cudaMemcpyHostToDevice, s));
        LSMPS_CUDA(cudaMemsetAsync(dpres, 0, n * sizeof(double), s));
        LSMPS_CUDA(cudaMemsetAsync(ddel, 0, n, s));
    }
    S->qcap = (size_t)p.injected_per_step * (size_t)(p.cnl_rebuild_interval + 1) + 1;
    S->qpos.ensure<double>(3 * S->qcap);
    S->qmat.ensure<uint8_t>(S->qcap);
    S->qdel.ensure<uint8_t>(S->qcap);
    S->counts.ensure<unsigned long long>(4);
    for (auto& e : S->ev) LSMPS_CUDA(cudaEventCreate(&e));
    LSMPS_CUDA(cudaStreamSynchronize(s));
    *out = S.release();
}

namespace {

// Droplets of the template at uniform positions over the plate, at heights in the band.
void inject(lsmps_series& S) {
    const lsmps_series_params& p = S.p;
    const size_t k = (size_t)p.injected_per_step;
    if (!k) return;
    LSMPS_REQUIRE(S.nq + k <= S.qcap, LSMPS_ERR_STATE, "in-flight buffer full: rebuild more often");
    const double l0 = p.l0, r = p.droplet_radius * l0;
    std::uniform_real_distribution<double> us(r, std::max(r, S.plate_len - r)), uy(r, std::max(r, S.plate_wid - r)),
        uh(p.inject_hmin * l0, p.inject_hmax * l0), jit(-0.1 * l0, 0.1 * l0);
    std::vector<double> xyz(3 * k);
    size_t c = 0;
    const size_t nt = S.tmpl.size() / 3;
    while (c < k) {
        const double s_ = us(S.rng), y = uy(S.rng), h = uh(S.rng);
        const double cx = S.F.t1x * s_ + S.F.nx * h, cy = y, cz = S.F.t1z * s_ + S.F.nz * h;
        for (size_t t = 0; t < nt && c < k; ++t, ++c) {
            xyz[3 * c] = cx + S.tmpl[3 * t] * l0 + jit(S.rng);
            xyz[3 * c + 1] = cy + S.tmpl[3 * t + 1] * l0 + jit(S.rng);
            xyz[3 * c + 2] = cz + S.tmpl[3 * t + 2] * l0 + jit(S.rng);
        }
    }
    cudaStream_t s = S.ctx->stream;
    LSMPS_CUDA(cudaMemcpyAsync(S.qpos.get<double>() + 3 * S.nq, xyz.data(), 3 * k * sizeof(double),
                               cudaMemcpyHostToDevice, s));
    LSMPS_CUDA(cudaMemsetAsync(S.qmat.get<uint8_t>() + S.nq, MAT_DROP, k, s));
    LSMPS_CUDA(cudaMemsetAsync(S.qdel.get<uint8_t>() + S.nq, 0, k, s));
    LSMPS_CUDA(cudaStreamSynchronize(s));  // the host vector goes out of scope
    S.nq += k;
    S.injected_total += k;
}

// Drop flagged particles and append the in-flight ones (stable order).
void merge(lsmps_series& S) {
    lsmps_ctx* ctx = S.ctx;
    cudaStream_t s = ctx->stream;
    const size_t tot = S.n + S.nq;
    int* keep = S.keep.ensure<int>(tot + 1);
    int* dest = S.dest.ensure<int>(tot + 1);
    if (tot) {
        k_keep_flags<<<grid_for(tot), 256, 0, s>>>(S.n, S.del.get<uint8_t>(), S.nq, S.qdel.get<uint8_t>(), keep);
        LSMPS_CHECK_LAUNCH();
    }
    scan_exclusive<int>(keep, dest, (long long)tot, s, ctx->scan_tmp, ctx->dflags.get<int>());
    int kept = 0;
    LSMPS_CUDA(cudaMemcpyAsync(&kept, dest + tot, sizeof(int), cudaMemcpyDeviceToHost, s));
    LSMPS_CUDA(cudaStreamSynchronize(s));
    double* opos = S.opos.ensure<double>(3 * (size_t)kept + 3);
    uint8_t* omat = S.omat.ensure<uint8_t>((size_t)kept + 1);
    uint8_t* otype = S.otype.ensure<uint8_t>((size_t)kept + 1);
    double* opres = S.opres.ensure<double>((size_t)kept + 1);
    if (tot) {
        k_compact<<<grid_for(tot), 256, 0, s>>>(S.n, S.nq, keep, dest, S.pos.get<double>(), S.mat.get<uint8_t>(),
                                                S.pres.get<double>(), S.qpos.get<double>(), S.qmat.get<uint8_t>(),
                                                opos, omat, otype, opres);
        LSMPS_CHECK_LAUNCH();
    }
    std::swap(S.pos, S.opos);
    std::swap(S.mat, S.omat);
    std::swap(S.type, S.otype);
    std::swap(S.pres, S.opres);
    uint8_t* del = S.del.ensure<uint8_t>((size_t)kept + 1);
    LSMPS_CUDA(cudaMemsetAsync(del, 0, (size_t)kept + 1, s));
    S.deleted_total += tot - (size_t)kept;
    S.n = (size_t)kept;
    S.nq = 0;
    LSMPS_CUDA(cudaStreamSynchronize(s));
}

}  // namespace

// Window and section outputs from the step's device histograms (host side: at most 8 x 64 cells).
static void rain_outputs_from(lsmps_series& S, const std::vector<unsigned long long>& hv) {
    const lsmps_rain_validation& vc = S.vcfg;
    lsmps_rain_outputs o{};
    for (int c = 0; c < vc.nsections; ++c) o.section_crossings[c] = hv[c];
    const unsigned long long* cnt = hv.data() + LSMPS_RAIN_MAX_SECTIONS;
    const unsigned long long* thk = cnt + LSMPS_RAIN_MAX_WINDOWS * LSMPS_RAIN_MAX_CELLS;
    for (int w = 0; w < vc.nwindows; ++w) {
        std::vector<double> t;
        int covered = 0;
        uint64_t np = 0;
        for (int c = 0; c < vc.coverage_cells; ++c) {
            const size_t slot = (size_t)w * LSMPS_RAIN_MAX_CELLS + c;
            np += cnt[slot];
            if (cnt[slot] >= (unsigned long long)vc.min_particles_per_cell) ++covered;
            if (cnt[slot]) {
                double d;
                std::memcpy(&d, &thk[slot], sizeof(d));
                t.push_back(d);
            }
        }
        o.window_particles[w] = np;
        o.window_coverage[w] = vc.coverage_cells ? (double)covered / vc.coverage_cells : 0.0;
        if (!t.empty()) {
            std::sort(t.begin(), t.end());
            double sum = 0;
            for (double v : t) sum += v;
            o.film_mean[w] = sum / t.size();
            const double q = 0.9 * (t.size() - 1);  // linear interpolation between order statistics
            const size_t lo = (size_t)std::floor(q);
            const size_t hi = std::min(lo + 1, t.size() - 1);
            o.film_p90[w] = t[lo] + (t[hi] - t[lo]) * (q - lo);
            o.film_max[w] = t.back();
        }
    }
    S.vout = o;
}

void series_set_validation(lsmps_series* S, const lsmps_rain_validation* v) {
    LSMPS_REQUIRE(S && v, LSMPS_ERR_ARG, "null series or validation config");
    LSMPS_REQUIRE(v->nwindows >= 0 && v->nwindows <= LSMPS_RAIN_MAX_WINDOWS && v->nsections >= 0 &&
                      v->nsections <= LSMPS_RAIN_MAX_SECTIONS && v->coverage_cells >= 1 &&
                      v->coverage_cells <= LSMPS_RAIN_MAX_CELLS && v->min_particles_per_cell >= 0,
                  LSMPS_ERR_ARG, "validation config: at most 8 windows, 8 sections, 1..64 cells");
    for (int w = 0; w < v->nwindows; ++w)
        LSMPS_REQUIRE(v->window_hi[w] > v->window_lo[w], LSMPS_ERR_ARG, "validation window with hi <= lo");
    S->vcfg = *v;
}

void series_rain_outputs(lsmps_series* S, lsmps_rain_outputs* out) {
    LSMPS_REQUIRE(S && out, LSMPS_ERR_ARG, "null series or output");
    *out = S->vout;
}

void series_step(lsmps_series* Sp, lsmps_series_stats* out) {
    LSMPS_REQUIRE(Sp, LSMPS_ERR_ARG, "null series");
    lsmps_series& S = *Sp;
    lsmps_ctx* ctx = S.ctx;
    const lsmps_series_params& p = S.p;
    cudaStream_t s = ctx->stream;
    lsmps_series_stats st{};
    S.step += 1;
    st.step = S.step;
    LSMPS_CUDA(cudaEventRecord(S.ev[0], s));
    // validation accumulators of this step
    const lsmps_rain_validation& vc = S.vcfg;
    Sections SC{};
    SC.n = vc.nsections;
    for (int c = 0; c < vc.nsections; ++c) {
        SC.u[c] = vc.section_u[c];
        SC.maxd[c] = vc.section_max_normal[c] * p.l0;
    }
    auto* vb = S.vbuf.get<unsigned long long>();
    LSMPS_CUDA(cudaMemsetAsync(vb, 0, S.vbuf.bytes, s));
    // 1. kinematics of the particle set and of the droplets in flight; 2. injection
    if (S.n) {
        k_advance<<<grid_for(S.n), 256, 0, s>>>(S.n, S.pos.get<double>(), S.mat.get<uint8_t>(), S.del.get<uint8_t>(),
                                                S.F, SC, vb);
        LSMPS_CHECK_LAUNCH();
    }
    if (S.nq) {
        k_advance<<<grid_for(S.nq), 256, 0, s>>>(S.nq, S.qpos.get<double>(), S.qmat.get<uint8_t>(),
                                                 S.qdel.get<uint8_t>(), S.F, SC, vb);
        LSMPS_CHECK_LAUNCH();
    }
    inject(S);
    // 3. neighbor lists: rebuild every interval steps (and when the skin no longer covers the
    // motion), else refresh from the candidates
    lsmps_neighbor_stats ns{};
    bool rebuild = S.step == 1 || S.step % p.cnl_rebuild_interval == 0 || !ctx->have_candidates;
    LSMPS_CUDA(cudaEventRecord(S.ev[1], s));
    if (!rebuild) {
        nb_update_positions(ctx, S.pos.get<double>(), S.n, true);
        st.max_displacement = nb_max_displacement(ctx);
        if (st.max_displacement > 0.5 * p.skin * p.l0 * (1.0 - 1e-9)) {
            rebuild = true;
            st.forced_rebuild = 1;
        } else {
            nb_refresh(ctx, LSMPS_NBR_CLASSIFY, &ns);
        }
    }
    if (rebuild) {
        merge(S);
        particles_upload(ctx, S.pos.get<double>(), S.type.get<uint8_t>(), S.n, true);
        nb_build_skin(ctx, p.re * p.l0, p.skin * p.l0, p.max_neighbors, p.max_candidates, p.l0, LSMPS_NBR_CLASSIFY,
                      &ns);
        st.max_displacement = 0;
    }
    st.rebuilt = rebuild ? 1 : 0;
    LSMPS_CUDA(cudaEventRecord(S.ev[2], s));
    // 4. WLS over every particle; 5. WLS-Laplacian PPE
    lsmps_wls_opts wo{};
    wo.re = p.re * p.l0;
    wo.l0 = p.l0;
    wo.regularization = 1e-8;
    wo.mode = 1;
    wo.nrhs = 1;
    wo.precision = p.wls_precision;
    wo.quad_coef = kQuadratic;
    lsmps_wls_stats ws{};
    wls_run(ctx, &wo, &ws);
    LSMPS_CUDA(cudaEventRecord(S.ev[3], s));
    lsmps_ppe_opts po{};
    po.variant = LSMPS_PPE_WLS;
    po.max_unknowns = (int64_t)1 << 40;
    po.re = p.re * p.l0;
    po.l0 = p.l0;
    po.diag_shift = 0.0;
    lsmps_ppe_stats ps{};
    ppe_assemble(ctx, &po, &ps);
    LSMPS_CUDA(cudaEventRecord(S.ev[4], s));
    // 6. solve, warm-started from the previous pressure of the same particles
    const bool warm = p.warm_start && S.have_pressure;
    if (warm) ppe_set_initial_particles(ctx, S.pres.get<double>(), S.n, true);
    lsmps_solver_opts so{};
    so.solver = p.solver;
    so.precond = p.precond;
    so.max_iter = p.max_iter;
    so.tol = p.tol;
    so.warm_start = warm ? 1 : 0;
    so.use_graph = 1;
    ppe_solve(ctx, &so, &ps);
    if (ctx->U) ppe_pressure_particles(ctx, S.pres.get<double>(), S.n, std::nan(""), true);
    S.have_pressure = true;
    LSMPS_CUDA(cudaEventRecord(S.ev[5], s));
    // 7. accounting on the device: fluid particles of the set and in flight, flagged outflow
    auto* cnt = S.counts.get<unsigned long long>();
    LSMPS_CUDA(cudaMemsetAsync(cnt, 0, 4 * sizeof(unsigned long long), s));
    if (S.n) {
        k_count<<<grid_for(S.n), 256, 0, s>>>(S.n, S.mat.get<uint8_t>(), S.del.get<uint8_t>(), cnt);
        LSMPS_CHECK_LAUNCH();
    }
    if (S.nq) {
        k_count<<<grid_for(S.nq), 256, 0, s>>>(S.nq, S.qmat.get<uint8_t>(), S.qdel.get<uint8_t>(), cnt + 2);
        LSMPS_CHECK_LAUNCH();
    }
    // validation windows over the fluid of the set and in flight (the domain's fluid)
    Windows W{};
    W.n = vc.nwindows;
    W.cells = vc.coverage_cells;
    W.wet = vc.wet_distance_factor * p.l0;
    W.l0 = p.l0;
    for (int w = 0; w < vc.nwindows; ++w) {
        W.lo[w] = vc.window_lo[w];
        W.hi[w] = vc.window_hi[w];
    }
    unsigned long long* wcount = vb + LSMPS_RAIN_MAX_SECTIONS;
    unsigned long long* wthick = wcount + LSMPS_RAIN_MAX_WINDOWS * LSMPS_RAIN_MAX_CELLS;
    if (S.n) k_rain_windows<<<grid_for(S.n), 256, 0, s>>>(S.n, S.pos.get<double>(), S.mat.get<uint8_t>(), S.F, W,
                                                         wcount, wthick);
    if (S.nq) k_rain_windows<<<grid_for(S.nq), 256, 0, s>>>(S.nq, S.qpos.get<double>(), S.qmat.get<uint8_t>(), S.F, W,
                                                           wcount, wthick);
    LSMPS_CHECK_LAUNCH();
    unsigned long long hc[4];
    std::vector<unsigned long long> hv(LSMPS_RAIN_MAX_SECTIONS + 2 * LSMPS_RAIN_MAX_WINDOWS * LSMPS_RAIN_MAX_CELLS);
    LSMPS_CUDA(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, s));
    LSMPS_CUDA(cudaMemcpyAsync(hv.data(), vb, hv.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    LSMPS_CUDA(cudaStreamSynchronize(s));
    rain_outputs_from(S, hv);
    float ms[4];  // neighbor lists, WLS, assembly, whole step
    LSMPS_CUDA(cudaEventElapsedTime(&ms[0], S.ev[1], S.ev[2]));
    LSMPS_CUDA(cudaEventElapsedTime(&ms[1], S.ev[2], S.ev[3]));
    LSMPS_CUDA(cudaEventElapsedTime(&ms[2], S.ev[3], S.ev[4]));
    LSMPS_CUDA(cudaEventElapsedTime(&ms[3], S.ev[0], S.ev[5]));
    st.particles = S.n;
    st.in_flight = S.nq;
    st.flagged = hc[1] + hc[3];
    st.injected_total = S.injected_total;
    st.deleted_total = S.deleted_total;
    st.fluid_particles = hc[0] + hc[2];
    st.mass_balance = (int64_t)st.fluid_particles - (int64_t)(S.fluid0 + S.injected_total - S.deleted_total);
    st.fluid_volume = (double)st.fluid_particles * p.l0 * p.l0 * p.l0;
    st.pairs = ns.pairs;
    st.unknowns = ps.unknowns;
    st.nnz = ps.nnz;
    st.iterations = ps.iterations;
    st.outer_iterations = ps.outer_iterations;
    st.fallback = ps.fallback;
    st.converged = ps.converged;
    st.relative_l2_error = ps.relative_l2_error;
    st.relative_residual = ps.relative_residual;
    st.neighbor_ms = ms[0];
    st.wls_ms = ms[1];
    st.assembly_ms = ms[2];
    st.solve_ms = ps.solve_ms;
    st.step_ms = ms[3];
    if (out) *out = st;
}

void series_particles(lsmps_series* S, double* xyz, uint8_t* material, double* pressure, size_t cap, size_t* n) {
    LSMPS_REQUIRE(S, LSMPS_ERR_ARG, "null series");
    if (n) *n = S->n;
    if (!xyz && !material && !pressure) return;
    LSMPS_REQUIRE(cap >= S->n, LSMPS_ERR_ARG, "buffer smaller than the particle set");
    cudaStream_t s = S->ctx->stream;
    if (S->n) {
        if (xyz)
            LSMPS_CUDA(cudaMemcpyAsync(xyz, S->pos.get<double>(), 3 * S->n * sizeof(double), cudaMemcpyDeviceToHost, s));
        if (material) LSMPS_CUDA(cudaMemcpyAsync(material, S->mat.get<uint8_t>(), S->n, cudaMemcpyDeviceToHost, s));
        if (pressure)
            LSMPS_CUDA(cudaMemcpyAsync(pressure, S->pres.get<double>(), S->n * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    LSMPS_CUDA(cudaStreamSynchronize(s));
}

void series_destroy(lsmps_series* S) { delete S; }

lsmps_ctx* series_context(lsmps_series* S) { return S ? S->ctx : nullptr; }

}  // namespace lsmps_gpu
