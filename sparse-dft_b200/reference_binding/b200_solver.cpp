// Device-resident solve in the reference's types (see b200_solver.hpp).
#include "b200_solver.hpp"

#include <cstdint>
#include <stdexcept>
#include <string>

namespace sdft::b200 {

void throw_on_error(sdft_b200_status status) {
  if (status == SDFT_B200_OK) return;
  char message[1024];
  sdft_b200_last_error(message, sizeof(message));
  switch (status) {
    case SDFT_B200_INVALID_ARGUMENT: throw std::invalid_argument(message);
    case SDFT_B200_OVERFLOW: throw std::overflow_error(message);
    case SDFT_B200_CUDA_ERROR: throw std::runtime_error(std::string("CUDA: ") + message);
    default: throw std::runtime_error(message);
  }
}

namespace {

// One context and one operator, released in reverse order.
struct DeviceSession {
  sdft_b200_context* context = nullptr;
  sdft_b200_operator* op = nullptr;
  explicit DeviceSession(int device) { throw_on_error(sdft_b200_context_create(device, nullptr, &context)); }
  ~DeviceSession() {
    if (op) sdft_b200_operator_destroy(op);
    if (context) sdft_b200_context_destroy(context);
  }
  DeviceSession(const DeviceSession&) = delete;
  DeviceSession& operator=(const DeviceSession&) = delete;
};

ComplexGeneralizedEigenResult solve(DeviceSession& session, std::size_t npw, std::size_t roots,
                                    std::size_t max_iterations, double tolerance,
                                    const std::vector<std::complex<double>>& initial,
                                    const DeviceSolveSettings& settings) {
  if (!initial.empty() && initial.size() != npw * roots)
    throw std::invalid_argument("invalid matrix-free Davidson problem");
  sdft_b200_davidson_options options{};
  options.roots = roots;
  options.max_iterations = max_iterations;
  options.tolerance = tolerance;
  options.precision = settings.precision;
  options.subspace_factor = settings.subspace_factor;
  options.handoff = 0.0;
  options.correction_steps = settings.correction_steps;
  ComplexGeneralizedEigenResult result;
  result.dimension = npw;
  result.eigenvalues.assign(roots, 0.0);
  result.residual_norms.assign(roots, 0.0);
  result.eigenvectors.assign(npw * roots, {});
  sdft_b200_davidson_stats stats{};
  throw_on_error(sdft_b200_davidson(session.op, &options,
                                    initial.empty() ? nullptr : reinterpret_cast<const double*>(initial.data()),
                                    result.eigenvalues.data(), reinterpret_cast<double*>(result.eigenvectors.data()),
                                    result.residual_norms.data(), &stats, SDFT_B200_MEMORY_HOST));
  result.converged = stats.converged != 0;
  result.iterations = stats.iterations;
  return result;
}

}  // namespace

ComplexGeneralizedEigenResult solve_generalized_hermitian_davidson_device(
    const std::vector<GVector>& basis, const FourierDensity& potential, const std::vector<ComplexPawOperator>& paw,
    double hartree_to_ev, double regularization, std::size_t n_roots, std::size_t max_iterations, double tolerance,
    const std::vector<std::complex<double>>& initial, const DeviceSolveSettings& settings) {
  const std::size_t npw = basis.size();
  std::vector<std::int32_t> hkl(3 * npw);
  std::vector<double> kinetic(npw);
  for (std::size_t g = 0; g < npw; ++g) {
    hkl[3 * g] = basis[g].h;
    hkl[3 * g + 1] = basis[g].k;
    hkl[3 * g + 2] = basis[g].l;
    kinetic[g] = basis[g].kinetic_ev;
  }
  std::vector<std::int32_t> keys;
  std::vector<std::complex<double>> values;
  keys.reserve(3 * potential.size());
  values.reserve(potential.size());
  for (const auto& [key, value] : potential) {
    keys.push_back(std::get<0>(key));
    keys.push_back(std::get<1>(key));
    keys.push_back(std::get<2>(key));
    values.push_back(value);
  }
  std::vector<std::uint64_t> projectors;
  std::vector<std::complex<double>> amplitudes, d, q;
  for (const auto& atom : paw) {
    if (atom.amplitudes.size() != atom.projectors * npw || atom.d.size() != atom.projectors * atom.projectors ||
        atom.q.size() != atom.projectors * atom.projectors)
      throw std::invalid_argument("invalid PAW operator dimensions");
    projectors.push_back(atom.projectors);
    amplitudes.insert(amplitudes.end(), atom.amplitudes.begin(), atom.amplitudes.end());
    d.insert(d.end(), atom.d.begin(), atom.d.end());
    q.insert(q.end(), atom.q.begin(), atom.q.end());
  }
  DeviceSession session(settings.device);
  throw_on_error(sdft_b200_operator_create(
      session.context, npw, hkl.data(), kinetic.data(), values.size(), keys.data(),
      reinterpret_cast<const double*>(values.data()), projectors.size(), projectors.data(),
      reinterpret_cast<const double*>(amplitudes.data()), reinterpret_cast<const double*>(d.data()),
      reinterpret_cast<const double*>(q.data()), hartree_to_ev, regularization, &session.op));
  return solve(session, npw, n_roots, max_iterations, tolerance, initial, settings);
}

ComplexGeneralizedEigenResult solve_snapshot_davidson_device(const std::string& path, std::size_t max_iterations,
                                                             const DeviceSolveSettings& settings) {
  sdft_b200_snapshot_info info{};
  throw_on_error(sdft_b200_snapshot_read_info(path.c_str(), &info));
  std::vector<std::complex<double>> initial(info.initial_values);
  DeviceSession session(settings.device);
  throw_on_error(sdft_b200_operator_from_snapshot(session.context, path.c_str(), &session.op,
                                                  initial.empty() ? nullptr : reinterpret_cast<double*>(initial.data())));
  return solve(session, info.npw, info.roots, max_iterations ? max_iterations : info.iterations, info.tolerance,
               initial, settings);
}

}  // namespace sdft::b200
