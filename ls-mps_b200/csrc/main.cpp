// lsmps-bench: the reference's CLI (src/main.cpp:5) over the sm_100a library.
// Usage: lsmps-bench [cfg] [outdir]; writes <outdir>/<case>.json and .csv with the
// reference's bytes (timings aside), prints the reference's summary, and returns 0, 2
// when the PPE did not converge or WLS failures exceed a fifth of the sample, 1 on error.
// It also writes <outdir>/<case>.gpu.json with the extended solver statistics.
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>

#include "lsmps.hpp"

int main(int argc, char** argv) {
    try {
        std::string cfg_path = argc > 1 ? argv[1] : "config/wall_film.cfg";
        std::string out_dir = argc > 2 ? argv[2] : "results";
        lsmps::Config cfg = lsmps::load_config(cfg_path);
        std::vector<lsmps::Particle> particles = lsmps::generate_case(cfg);
        lsmps::Metrics m = lsmps::run_benchmark(cfg, particles);
        std::filesystem::create_directories(out_dir);
        const std::string base = out_dir + "/" + cfg.case_name;
        lsmps::write_json(base + ".json", cfg, m);
        lsmps::write_csv(base + ".csv", cfg, m);
        {
            std::ofstream o(base + ".gpu.json");
            o << std::setprecision(10) << "{\"solver\": \"" << cfg.solver << "\", \"precond\": \"" << cfg.precond
              << "\", \"ppe_variant\": \"" << cfg.ppe_variant
              << "\", \"wls_mode\": \"" << cfg.wls_mode << "\", \"upload_ms\": " << m.upload_ms
              << ", \"neighbor_ms\": " << m.neighbor_ms << ", \"wls_ms\": " << m.wls_ms
              << ", \"assembly_ms\": " << m.ppe.assembly_ms << ", \"solve_ms\": " << m.ppe.solve_ms
              << ", \"iterations\": " << m.ppe.iterations << ", \"outer_iterations\": " << m.outer_iterations
              << ", \"fallback\": " << m.fallback << ", \"relative_l2_error\": " << m.ppe.relative_l2_error
              << ", \"max_error\": " << m.ppe.max_error << ", \"final_residual\": " << m.ppe.final_residual
              << ", \"initial_residual\": " << m.ppe.initial_residual << "}\n";
        }
        std::cout << "LS-MPS industrial benchmark v0.2\ncase=" << cfg.case_name << " particles=" << m.particles
                  << "\ntypes interior=" << m.interior << " surface=" << m.free_surface << " splash=" << m.splash
                  << " near_wall=" << m.near_wall << " wall=" << m.wall << "\n"
                  << std::fixed << std::setprecision(2) << "neighbors mean=" << m.neighbor_mean
                  << " p50=" << m.neighbor_p50 << " p90=" << m.neighbor_p90 << " p99=" << m.neighbor_p99
                  << "\nWLS sampled=" << m.wls.sampled << " regularized=" << m.wls.regularized
                  << " failed=" << m.wls.failed << " virtual=" << m.wls.virtual_points
                  << " grad_rms=" << std::scientific << m.wls.rms_gradient_error
                  << " lap_rms=" << m.wls.rms_laplacian_error << "\nPPE unknowns=" << m.ppe.unknowns
                  << " nnz=" << m.ppe.nnz << " iterations=" << m.ppe.iterations
                  << " converged=" << m.ppe.converged << " residual=" << m.ppe.final_residual
                  << " rel_l2=" << m.ppe.relative_l2_error << "\nPPE timing(ms) assembly=" << std::fixed
                  << m.ppe.assembly_ms << " solve=" << m.ppe.solve_ms << "\noutput=" << base << ".{json,csv}\n";
        return (!m.ppe.converged || m.wls.failed > m.wls.sampled / 5) ? 2 : 0;
    } catch (const std::exception& e) {
        std::cerr << "error: " << e.what() << '\n';
        return 1;
    }
}
