// LS-MPS per-step path — the C++ interface of the reference benchmark, kept so that this
// library is a drop-in for it. Every declaration of the reference's include/lsmps.hpp
// (lines 8-32) is present with the same name, field order, defaults and meaning; the
// implementation (ls-mps_b200/csrc/host.cpp) runs the path on an sm_100a GPU through the
// C ABI of lsmps_gpu.h.
//
// Additions, all placed after the reference's fields so existing aggregate initialisers
// and field accesses keep compiling: Config gains keys that the reference's parser would
// ignore (jitter, ppe_variant, solver, ...), Metrics gains the GPU timings and the
// extended solver statistics. With the additions at their defaults, run_benchmark
// reproduces the reference's results and write_json / write_csv its bytes (timings
// aside).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace lsmps {

// Particle classes (reference include/lsmps.hpp:8).
enum class ParticleType : uint8_t { Interior = 0, FreeSurface = 1, Splash = 2, NearWall = 3, Wall = 4 };

// (reference include/lsmps.hpp:9)
struct Vec3 {
    double x{}, y{}, z{};
    Vec3 operator+(const Vec3& o) const { return {x + o.x, y + o.y, z + o.z}; }
    Vec3 operator-(const Vec3& o) const { return {x - o.x, y - o.y, z - o.z}; }
    Vec3 operator*(double s) const { return {x * s, y * s, z * s}; }
};

// (reference include/lsmps.hpp:10)
struct Particle {
    Vec3 r, u;
    ParticleType type{ParticleType::Interior};
    double pressure{};
};

// Benchmark configuration (reference include/lsmps.hpp:12-19), parsed from key=value
// .cfg files by load_config.
struct Config {
    std::string case_name{"wall_film"};
    size_t particles{20000};
    uint32_t seed{7};
    double l0{0.01}, re_ratio{2.1};
    int film_layers{4}, max_neighbors{96}, wls_samples{4096};
    int steps{5}, injected_per_step{0}, cnl_rebuild_interval{1};
    int ppe_max_unknowns{12000}, ppe_max_iter{400};
    double ppe_tol{1e-9};
    double wls_regularization{1e-8}, boundary_constraint_weight{8.0}, virtual_weight{0.25};
    bool write_csv{true};

    // ---- extensions (keys the reference's parser ignores) ----
    double jitter{-1.0};           // lattice jitter / l0; < 0 keeps each case's own value
    std::string ppe_variant{"reference"};  // reference | shifted | wls
    double ppe_diag_shift{1e-3};   // diagonal factor (1 + shift) of the shifted / wls rows
    std::string solver{"reference"};  // reference | fp64 | jacobi | mixed | learned
    std::string wls_mode{"sampled"};  // sampled (reference statistics) | all
    std::string wls_precision{"fp64"};  // fp64 | mixed (fp32 Cholesky + fp64 refinement)
    int device{0};                 // CUDA device ordinal
    std::string mpnn_weights{};    // learned preconditioner weights file (solver=learned)
    std::string precond{"jacobi"};  // jacobi | multigrid (the mixed and learned solvers)
};

// (reference include/lsmps.hpp:20)
struct WlsStats {
    size_t sampled{}, ok{}, regularized{}, failed{}, virtual_points{};
    double max_gradient_error{}, rms_gradient_error{}, max_laplacian_error{}, rms_laplacian_error{};
};

// (reference include/lsmps.hpp:21)
struct PpeStats {
    size_t unknowns{}, nnz{}, dirichlet{}, neumann{}, failed_rows{};
    int iterations{};
    double initial_residual{}, final_residual{}, relative_l2_error{}, max_error{}, assembly_ms{}, solve_ms{};
    bool converged{};
};

// (reference include/lsmps.hpp:22-26)
struct Metrics {
    size_t particles{}, interior{}, free_surface{}, splash{}, near_wall{}, wall{}, neighbor_pairs{},
        truncated_particles{};
    double neighbor_mean{};
    int neighbor_p50{}, neighbor_p90{}, neighbor_p99{};
    double classify_ms{}, neighbor_ms{}, wls_ms{};
    WlsStats wls;
    PpeStats ppe;

    // ---- extensions ----
    double upload_ms{};            // host -> device particle copy
    int outer_iterations{};        // mixed / learned solvers: FP64 refinement sweeps
    int fallback{};                // learned solver fell back to Jacobi BiCGStab
};

// (reference include/lsmps.hpp:27-32)
Config load_config(const std::string& path);
std::vector<Particle> generate_case(const Config& cfg);
Metrics run_benchmark(const Config& cfg, std::vector<Particle>& particles);
void write_json(const std::string& path, const Config& cfg, const Metrics& m);
void write_csv(const std::string& path, const Config& cfg, const Metrics& m);
const char* type_name(ParticleType t);

}  // namespace lsmps
