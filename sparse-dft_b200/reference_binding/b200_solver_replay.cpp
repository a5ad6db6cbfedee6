// sdft_b200_solver_replay: the reference's solver replay (src/solver_replay_cli.cpp)
// with the solve on the B200 (b200_solver.hpp) and the check on the host.
//
//   sdft_b200_solver_replay snapshot.pwop report.json [max_iterations] [fp64|mixed]
//
// Same arguments (except the warm-snapshot output) and the same report schema
// as the reference's tool, plus "solver" and "precision". The returned
// vectors are checked exactly as the reference's tool checks them: a fresh
// FP64 application of the reference's own CPU operator (loaded from the same
// snapshot), fma residuals and long-double sums; the report passes only for a
// converged solve with max residual <= tolerance and S-normalisation within
// 1e-12. Search guard files (.guards) are not read: the device route seeds
// its own guards.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>

#include "b200_solver.hpp"

int main(int argc, char** argv) {
  try {
    if (argc < 3 || argc > 5)
      throw std::invalid_argument("usage: sdft_b200_solver_replay snapshot.pwop report.json [max_iterations] [fp64|mixed]");
    if (std::filesystem::exists(argv[2])) throw std::runtime_error("refusing to overwrite replay report");
    std::size_t roots, iterations;
    double tolerance;
    std::vector<std::complex<double>> initial;
    auto op = sdft::PlaneWaveOperator::load_solver_snapshot(argv[1], roots, iterations, tolerance, initial);
    const auto stored_iterations = iterations;
    if (argc >= 4) {
      std::size_t end;
      const std::string value = argv[3];
      iterations = std::stoull(value, &end);
      if (end != value.size() || !iterations || iterations > 1000000 || value[0] == '-')
        throw std::invalid_argument("invalid replay iteration limit");
    }
    sdft::b200::DeviceSolveSettings settings;
    std::string precision = "mixed";
    if (argc == 5) {
      precision = argv[4];
      if (precision != "fp64" && precision != "mixed") throw std::invalid_argument("precision must be fp64 or mixed");
    }
    settings.precision = precision == "fp64" ? SDFT_B200_PRECISION_FP64 : SDFT_B200_PRECISION_MIXED;
    if (const char* device = std::getenv("SDFT_B200_DEVICE")) settings.device = std::atoi(device);
    const auto start = std::chrono::steady_clock::now();
    const auto result = sdft::b200::solve_snapshot_davidson_device(argv[1], iterations, settings);
    const double seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
    // The reference tool's independent check (src/solver_replay_cli.cpp:28-45).
    auto h = op->hamiltonian();
    const auto s = op->overlap();
    std::vector<std::complex<double>> hx, sx;
    h.apply_block(result.eigenvectors, roots, hx, true);
    s.apply_block(result.eigenvectors, roots, sx, true);
    double maximum = 0, normalization_error = 0;
    for (std::size_t band = 0; band < roots; ++band) {
      long double square = 0, metric = 0;
      for (std::size_t g = 0; g < h.dimension; ++g) {
        const auto i = band * h.dimension + g;
        const double re = std::fma(-result.eigenvalues[band], sx[i].real(), hx[i].real());
        const double im = std::fma(-result.eigenvalues[band], sx[i].imag(), hx[i].imag());
        square += static_cast<long double>(re) * re + static_cast<long double>(im) * im;
        metric += static_cast<long double>(result.eigenvectors[i].real()) * sx[i].real() +
                  static_cast<long double>(result.eigenvectors[i].imag()) * sx[i].imag();
      }
      maximum = std::max(maximum, std::sqrt(static_cast<double>(square)));
      normalization_error = std::max(normalization_error, std::abs(static_cast<double>(metric) - 1));
    }
    const bool passed = result.converged && maximum <= tolerance && normalization_error <= 1e-12;
    std::ofstream f(argv[2]);
    f << std::setprecision(17) << "{\"schema_version\":\"sparse-dft-solver-replay-1\",\"scientific_scf_result\":false"
      << ",\"solver\":\"b200\",\"precision\":\"" << precision << "\",\"passed\":" << (passed ? "true" : "false")
      << ",\"dimension\":" << h.dimension << ",\"roots\":" << roots << ",\"stored_max_iterations\":"
      << stored_iterations << ",\"max_iterations\":" << iterations << ",\"iterations\":" << result.iterations
      << ",\"tolerance\":" << tolerance << ",\"solver_converged\":" << (result.converged ? "true" : "false")
      << ",\"fresh_max_residual\":" << maximum << ",\"s_normalization_error\":" << normalization_error
      << ",\"seconds\":" << seconds << ",\"residuals\":[";
    for (std::size_t i = 0; i < roots; ++i) f << (i ? "," : "") << result.residual_norms[i];
    f << "],\"eigenvalues_hartree\":[";
    for (std::size_t i = 0; i < roots; ++i) f << (i ? "," : "") << result.eigenvalues[i];
    f << "]}\n";
    f.close();
    if (!f) throw std::runtime_error("replay report write failed");
    return passed ? 0 : 2;
  } catch (const std::exception& e) {
    std::cerr << "sdft_b200_solver_replay: " << e.what() << "\n";
    return 1;
  }
}
