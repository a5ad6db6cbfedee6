// C entry points over the reference's own C++ API, so that Python tests can
// call the unmodified reference code (built with the shims beside this file)
// as an oracle. Test infrastructure only: nothing in the product links this.
//
// Each function converts flat arrays into the reference's types and calls:
//   enumerate_g_vectors                 src/pw_core.cpp:140-171
//   PlaneWaveOperator ctor              src/plane_wave_operator.cpp:393-516
//   hamiltonian()/overlap() callbacks   src/plane_wave_operator.cpp:672-719
//   solve_generalized_hermitian_davidson src/pw_core.cpp:532-1437
//   solve_generalized_hermitian_rmm_trial src/rmm_trial.cpp:128-206
//   solve_generalized_hermitian_band_groups src/band_group_solver.cpp:55-212
//   kinetic_preconditioner              src/pw_core.cpp:33-47
//   save/load_solver_snapshot           src/plane_wave_operator.cpp:542-653
//   plane_wave_density_fft              src/density_functionals.cpp:407-460
//   pbe_unpolarized                     src/pbe_xc.cpp:116-140
//   pbe_collinear                       src/spin_pbe_xc.cpp:54-107
//   onsite_density_from_amplitudes      src/onsite_density.hpp:10-36
//   paw_lm_moments_from_density         src/paw_augmentation.cpp:490-525
//   PawCompensationOperator ctor/density_sum src/paw_compensation.cpp:185-342,465-524
//   evaluate_density_functionals        src/density_functionals.cpp:462-729
//   evaluate_collinear_density_functionals src/density_functionals.cpp:732-806
// Complex arrays are interleaved (re, im) doubles, column-major blocks.
#include "plane_wave_operator.hpp"
#include "pw_core.hpp"
#include "compute_backend.hpp"
#include "density_functionals.hpp"
#include "pbe_xc.hpp"
#include "spin_pbe_xc.hpp"
#include "env_cache.hpp"
#include "onsite_density.hpp"
#include "paw_augmentation.hpp"
#include "paw_compensation.hpp"

#include <algorithm>
#include <array>
#include <complex>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

namespace {
using C = std::complex<double>;

void set_error(char* buffer, long length, const std::exception& e) {
  if (!buffer || length <= 0) return;
  std::string text = std::string(typeid(e).name()) + ": " + e.what();
  const auto count = std::min<std::size_t>(text.size(), static_cast<std::size_t>(length - 1));
  std::memcpy(buffer, text.data(), count);
  buffer[count] = 0;
}

struct Handle {
  std::unique_ptr<sdft::PlaneWaveOperator> op;
};
}  // namespace

extern "C" {

long ref_enumerate_g_vectors(const double* reciprocal, double cutoff_ev, const double* kpoint,
                             double hartree_to_ev, int* hkl, double* cartesian,
                             double* kinetic_ev, long capacity) {
  std::array<sdft::Vec3, 3> recip{};
  for (int a = 0; a < 3; ++a) recip[a] = {reciprocal[3 * a], reciprocal[3 * a + 1], reciprocal[3 * a + 2]};
  const sdft::Vec3 k{kpoint[0], kpoint[1], kpoint[2]};
  const auto g = sdft::enumerate_g_vectors(recip, cutoff_ev, k, hartree_to_ev);
  if (hkl && static_cast<long>(g.size()) <= capacity) {
    for (std::size_t i = 0; i < g.size(); ++i) {
      hkl[3 * i] = g[i].h;
      hkl[3 * i + 1] = g[i].k;
      hkl[3 * i + 2] = g[i].l;
      cartesian[3 * i] = g[i].cartesian.x;
      cartesian[3 * i + 1] = g[i].cartesian.y;
      cartesian[3 * i + 2] = g[i].cartesian.z;
      kinetic_ev[i] = g[i].kinetic_ev;
    }
  }
  return static_cast<long>(g.size());
}

void* ref_operator_create(long n, const int* hkl, const double* cartesian, const double* kinetic_ev,
                          long nv, const int* v_hkl, const double* v_values, long atoms,
                          const long* projectors, const double* amplitudes, const double* d,
                          const double* q, double hartree_to_ev, double regularization,
                          unsigned long long projector_identity, char* error, long error_length) {
  try {
    std::vector<sdft::GVector> basis(static_cast<std::size_t>(n));
    for (long i = 0; i < n; ++i)
      basis[i] = {hkl[3 * i], hkl[3 * i + 1], hkl[3 * i + 2],
                  {cartesian[3 * i], cartesian[3 * i + 1], cartesian[3 * i + 2]}, kinetic_ev[i]};
    sdft::FourierDensity potential;
    for (long i = 0; i < nv; ++i)
      potential[{v_hkl[3 * i], v_hkl[3 * i + 1], v_hkl[3 * i + 2]}] = C(v_values[2 * i], v_values[2 * i + 1]);
    std::vector<sdft::ComplexPawOperator> paw;
    std::size_t amp_offset = 0, block_offset = 0;
    for (long a = 0; a < atoms; ++a) {
      sdft::ComplexPawOperator p;
      p.projectors = static_cast<std::size_t>(projectors[a]);
      const std::size_t np = p.projectors;
      p.amplitudes.resize(np * n);
      for (std::size_t i = 0; i < np * static_cast<std::size_t>(n); ++i)
        p.amplitudes[i] = C(amplitudes[2 * (amp_offset + i)], amplitudes[2 * (amp_offset + i) + 1]);
      p.d.resize(np * np);
      p.q.resize(np * np);
      for (std::size_t i = 0; i < np * np; ++i) {
        p.d[i] = C(d[2 * (block_offset + i)], d[2 * (block_offset + i) + 1]);
        p.q[i] = C(q[2 * (block_offset + i)], q[2 * (block_offset + i) + 1]);
      }
      amp_offset += np * n;
      block_offset += np * np;
      paw.push_back(std::move(p));
    }
    auto handle = std::make_unique<Handle>();
    handle->op = std::make_unique<sdft::PlaneWaveOperator>(basis, potential, std::move(paw), hartree_to_ev,
                                                           regularization, projector_identity);
    return handle.release();
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return nullptr;
  }
}

void ref_operator_destroy(void* handle) { delete static_cast<Handle*>(handle); }

long ref_operator_grid(void* handle) { return static_cast<long>(static_cast<Handle*>(handle)->op->fft_grid_points()); }

int ref_apply(void* handle, int overlap, const double* x, long columns, double* y, int exact,
              char* error, long error_length) {
  try {
    auto* h = static_cast<Handle*>(handle);
    auto op = overlap ? h->op->overlap() : h->op->hamiltonian();
    op.apply_block_into(reinterpret_cast<const C*>(x), static_cast<std::size_t>(columns),
                        reinterpret_cast<C*>(y), exact != 0);
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

int ref_apply_pair(void* handle, const double* x, long columns, double* hy, double* sy, int exact,
                   char* error, long error_length) {
  try {
    auto* h = static_cast<Handle*>(handle);
    auto op = h->op->hamiltonian();
    op.apply_pair_into(reinterpret_cast<const C*>(x), static_cast<std::size_t>(columns),
                       reinterpret_cast<C*>(hy), reinterpret_cast<C*>(sy), exact != 0);
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

int ref_project(void* handle, const double* x, long columns, double* p, char* error, long error_length) {
  try {
    auto op = static_cast<Handle*>(handle)->op->hamiltonian();
    op.project_into(reinterpret_cast<const C*>(x), static_cast<std::size_t>(columns), reinterpret_cast<C*>(p), true);
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

long ref_projector_rows(void* handle) {
  return static_cast<long>(static_cast<Handle*>(handle)->op->hamiltonian().projector_rows);
}

int ref_davidson(void* handle, long roots, long max_iterations, double tolerance, const double* initial,
                 double* eigenvalues, double* vectors, double* residuals, int* converged,
                 long* iterations, char* error, long error_length) {
  try {
    auto* h = static_cast<Handle*>(handle);
    auto ham = h->op->hamiltonian();
    auto ovl = h->op->overlap();
    std::vector<C> warm;
    if (initial) warm.assign(reinterpret_cast<const C*>(initial), reinterpret_cast<const C*>(initial) + roots * ham.dimension);
    const auto result = sdft::solve_generalized_hermitian_davidson(ham, ovl, static_cast<std::size_t>(roots),
                                                                   static_cast<std::size_t>(max_iterations), tolerance, warm);
    std::copy(result.eigenvalues.begin(), result.eigenvalues.end(), eigenvalues);
    std::copy(result.residual_norms.begin(), result.residual_norms.end(), residuals);
    std::memcpy(vectors, result.eigenvectors.data(), result.eigenvectors.size() * sizeof(C));
    *converged = result.converged ? 1 : 0;
    *iterations = static_cast<long>(result.iterations);
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

// The signature PlaneWaveOperator::overlap() determines
// (src/plane_wave_operator.cpp:702-717): *indefinite = indefinite_metric;
// a numerically singular S~ is its runtime_error (returns 1 with the message).
int ref_overlap_signature(void* handle, int* indefinite, char* error, long error_length) {
  try {
    auto* h = static_cast<Handle*>(handle);
    const auto ovl = h->op->overlap();
    *indefinite = ovl.indefinite_metric ? 1 : 0;
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

// solve_generalized_hermitian_rmm_trial (src/rmm_trial.cpp:128-206) on the
// operator's callbacks marked as an SCF warm request (scf_trial_update).
int ref_rmm_trial(void* handle, long roots, long max_iterations, double tolerance, const double* initial,
                  double* eigenvalues, double* vectors, double* residuals, int* converged, long* iterations,
                  int* trial_manifold, char* error, long error_length) {
  try {
    auto* h = static_cast<Handle*>(handle);
    auto ham = h->op->hamiltonian();
    auto ovl = h->op->overlap();
    ham.scf_trial_update = true;
    std::vector<C> warm(reinterpret_cast<const C*>(initial), reinterpret_cast<const C*>(initial) + roots * ham.dimension);
    const auto result = sdft::solve_generalized_hermitian_rmm_trial(ham, ovl, static_cast<std::size_t>(roots),
                                                                    static_cast<std::size_t>(max_iterations),
                                                                    tolerance, warm);
    std::copy(result.eigenvalues.begin(), result.eigenvalues.end(), eigenvalues);
    std::copy(result.residual_norms.begin(), result.residual_norms.end(), residuals);
    std::memcpy(vectors, result.eigenvectors.data(), result.eigenvectors.size() * sizeof(C));
    *converged = result.converged ? 1 : 0;
    *iterations = static_cast<long>(result.iterations);
    *trial_manifold = result.trial_manifold ? 1 : 0;
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

// solve_generalized_hermitian_band_groups (src/band_group_solver.cpp:55-212).
int ref_band_groups(void* handle, long roots, long max_iterations, double tolerance, const double* initial,
                    double* eigenvalues, double* vectors, double* residuals, int* converged, long* iterations,
                    char* error, long error_length) {
  try {
    auto* h = static_cast<Handle*>(handle);
    auto ham = h->op->hamiltonian();
    auto ovl = h->op->overlap();
    std::vector<C> warm;
    if (initial) warm.assign(reinterpret_cast<const C*>(initial), reinterpret_cast<const C*>(initial) + roots * ham.dimension);
    const auto result = sdft::solve_generalized_hermitian_band_groups(ham, ovl, static_cast<std::size_t>(roots),
                                                                      static_cast<std::size_t>(max_iterations),
                                                                      tolerance, warm);
    std::copy(result.eigenvalues.begin(), result.eigenvalues.end(), eigenvalues);
    std::copy(result.residual_norms.begin(), result.residual_norms.end(), residuals);
    std::memcpy(vectors, result.eigenvectors.data(), result.eigenvectors.size() * sizeof(C));
    *converged = result.converged ? 1 : 0;
    *iterations = static_cast<long>(result.iterations);
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

double ref_kinetic_preconditioner(double kinetic, double wavefunction_kinetic) {
  return sdft::kinetic_preconditioner(kinetic, wavefunction_kinetic);
}

int ref_save_snapshot(void* handle, const char* path, long roots, long iterations, double tolerance,
                      const double* initial, long initial_count, char* error, long error_length) {
  try {
    std::vector<C> warm;
    if (initial && initial_count)
      warm.assign(reinterpret_cast<const C*>(initial), reinterpret_cast<const C*>(initial) + initial_count);
    static_cast<Handle*>(handle)->op->save_solver_snapshot(path, static_cast<std::size_t>(roots),
                                                           static_cast<std::size_t>(iterations), tolerance, warm);
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

void* ref_load_snapshot(const char* path, long* roots, long* iterations, double* tolerance,
                        char* error, long error_length) {
  try {
    std::size_t r = 0, it = 0;
    std::vector<C> initial;
    auto handle = std::make_unique<Handle>();
    handle->op = sdft::PlaneWaveOperator::load_solver_snapshot(path, r, it, *tolerance, initial);
    *roots = static_cast<long>(r);
    *iterations = static_cast<long>(it);
    return handle.release();
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return nullptr;
  }
}

// Band density on the support keys (h,k,l); output interleaved complex per key.
int ref_plane_wave_density_fft(long n, const int* hkl, long bands, const double* coefficients,
                               const double* occupations, double volume, long support_count,
                               const int* support_hkl, double* density, char* error, long error_length) {
  try {
    std::vector<std::tuple<int, int, int>> g(static_cast<std::size_t>(n));
    for (long i = 0; i < n; ++i) g[i] = {hkl[3 * i], hkl[3 * i + 1], hkl[3 * i + 2]};
    std::vector<C> coeff(reinterpret_cast<const C*>(coefficients), reinterpret_cast<const C*>(coefficients) + n * bands);
    std::vector<double> occ(occupations, occupations + bands);
    sdft::FourierDensity support;
    for (long i = 0; i < support_count; ++i) support[{support_hkl[3 * i], support_hkl[3 * i + 1], support_hkl[3 * i + 2]}] = C(0, 0);
    const auto result = sdft::plane_wave_density_fft(g, coeff, occ, volume, support);
    for (long i = 0; i < support_count; ++i) {
      const auto found = result.find({support_hkl[3 * i], support_hkl[3 * i + 1], support_hkl[3 * i + 2]});
      const C v = found == result.end() ? C(0, 0) : found->second;
      density[2 * i] = v.real();
      density[2 * i + 1] = v.imag();
    }
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

// Per point: energy_density, energy_per_particle, exchange_energy_density,
// correlation_energy_density, exchange_potential, correlation_potential,
// gradient_squared_coefficient.
void ref_pbe_unpolarized(long count, const double* density, const double* gradient, double* out) {
  for (long i = 0; i < count; ++i) {
    const auto p = sdft::pbe_unpolarized(density[i], gradient[i]);
    double* o = out + 7 * i;
    o[0] = p.energy_density;
    o[1] = p.energy_per_particle;
    o[2] = p.exchange_energy_density;
    o[3] = p.correlation_energy_density;
    o[4] = p.exchange_potential;
    o[5] = p.correlation_potential;
    o[6] = p.gradient_squared_coefficient;
  }
}

// pbe_collinear (src/spin_pbe_xc.cpp:54-107) per point: out[9 i ..] =
// energy density, v_up, v_down, gradient responses up (3) and down (3).
int ref_pbe_collinear(long count, const double* up, const double* down, const double* gradient_up,
                      const double* gradient_down, double* out, char* error, long error_length) {
  try {
    for (long i = 0; i < count; ++i) {
      const std::array<double, 3> gu{gradient_up[3 * i], gradient_up[3 * i + 1], gradient_up[3 * i + 2]};
      const std::array<double, 3> gd{gradient_down[3 * i], gradient_down[3 * i + 1], gradient_down[3 * i + 2]};
      const auto p = sdft::pbe_collinear(up[i], down[i], gu, gd);
      double* o = out + 9 * i;
      o[0] = p.energy_density;
      o[1] = p.density_potential[0];
      o[2] = p.density_potential[1];
      for (int a = 0; a < 3; ++a) {
        o[3 + a] = p.gradient_response[0][a];
        o[6 + a] = p.gradient_response[1][a];
      }
    }
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

void ref_refresh_environment() { sdft::refresh_environment_cache(); }

// rho_ij (row-major rows x rows) of one atom from amplitudes (rows x bands, column stride `stride`).
int ref_onsite_density(long rows, long bands, const double* amplitudes, long stride, const double* occupations,
                       double* out, char* error, long error_length) {
  try {
    const auto rho = sdft::onsite_density_from_amplitudes(
        static_cast<std::size_t>(rows), static_cast<std::size_t>(bands), reinterpret_cast<const C*>(amplitudes),
        static_cast<std::size_t>(stride), occupations);
    std::memcpy(out, rho.data(), sizeof(C) * rho.size());
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}
}

namespace {
sdft::PawAugmentationData augmentation(long channels, const int* channel_l, int max_l, long radial,
                                       const double* radial_grid, const double* aug_moment,
                                       const double* compensation_r2) {
  sdft::PawAugmentationData a;
  a.channel_l.assign(channel_l, channel_l + channels);
  a.max_l = max_l;
  a.radial_grid.assign(radial_grid, radial_grid + radial);
  a.rmax = a.radial_grid.back();
  a.rdep = a.radial_grid.back();
  a.aug_moment.assign(aug_moment, aug_moment + channels * channels * (max_l + 1));
  a.overlap_correction.assign(static_cast<std::size_t>(channels * channels), 0.0);
  for (long i = 0; i < channels; ++i)
    for (long j = 0; j < channels; ++j)
      if (channel_l[i] == channel_l[j]) a.overlap_correction[i * channels + j] = a.moment(i, j, 0);
  for (int l = 0; l <= max_l; ++l)
    a.compensation_r2.emplace_back(compensation_r2 + l * radial, compensation_r2 + (l + 1) * radial);
  a.compensation_q.assign(max_l + 1, {0.0, 0.0});
  a.compensation_amplitudes.assign(max_l + 1, {0.0, 0.0});
  return a;
}
}  // namespace

extern "C" {

// (L,M) moments transform [lm][i*dim+j]: paw_lm_moments_from_density of each unit matrix.
int ref_lm_transform(long channels, const int* channel_l, int max_l, long radial, const double* radial_grid,
                     const double* aug_moment, const double* compensation_r2, double* out, char* error,
                     long error_length) {
  try {
    const auto a = augmentation(channels, channel_l, max_l, radial, radial_grid, aug_moment, compensation_r2);
    std::size_t dim = 0;
    for (int l : a.channel_l) dim += 2 * l + 1;
    const std::size_t entries = dim * dim, lms = (max_l + 1) * (max_l + 1);
    std::vector<C> unit(entries);
    auto* o = reinterpret_cast<C*>(out);
    for (std::size_t e = 0; e < entries; ++e) {
      unit[e] = 1.0;
      const auto m = sdft::paw_lm_moments_from_density(a, unit, dim);
      unit[e] = 0.0;
      for (std::size_t lm = 0; lm < lms; ++lm) o[lm * entries + e] = m[lm];
    }
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

// Compensation charge on `count` reciprocal keys for `atoms` atoms sharing one
// geometry; onsite: atoms x dim^2 complex row-major; out: count complex.
int ref_compensation_density(const double* lattice, long atoms, const double* fractional, long count,
                             const int* keys, long channels, const int* channel_l, int max_l, long radial,
                             const double* radial_grid, const double* aug_moment, const double* compensation_r2,
                             const double* onsite, double* out, char* error, long error_length) {
  try {
    const auto a = augmentation(channels, channel_l, max_l, radial, radial_grid, aug_moment, compensation_r2);
    std::array<sdft::Vec3, 3> cell{};
    for (int r = 0; r < 3; ++r) cell[r] = {lattice[3 * r], lattice[3 * r + 1], lattice[3 * r + 2]};
    std::vector<std::tuple<int, int, int>> support(static_cast<std::size_t>(count));
    for (long i = 0; i < count; ++i) support[i] = {keys[3 * i], keys[3 * i + 1], keys[3 * i + 2]};
    std::size_t dim = 0;
    for (int l : a.channel_l) dim += 2 * l + 1;
    std::vector<sdft::PawCompensationOperator> ops;
    ops.reserve(static_cast<std::size_t>(atoms));
    std::vector<std::vector<C>> rho(static_cast<std::size_t>(atoms));
    for (long i = 0; i < atoms; ++i) {
      const sdft::Vec3 f{fractional[3 * i], fractional[3 * i + 1], fractional[3 * i + 2]};
      ops.emplace_back(a, cell, f, support, sdft::AtomicUnitConvention::Codata, i ? &ops.front() : nullptr);
      const auto* p = reinterpret_cast<const C*>(onsite) + i * dim * dim;
      rho[i].assign(p, p + dim * dim);
    }
    const auto charge = sdft::PawCompensationOperator::density_sum(ops, rho);
    auto* o = reinterpret_cast<C*>(out);
    for (long i = 0; i < count; ++i) o[i] = charge.at(support[i]);
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}

// PawCompensationOperator::project_potential_batch (src/paw_compensation.cpp:552)
// of a potential given on `potential_count` keys; out: atoms x dim^2 complex.
int ref_compensation_project(const double* lattice, long atoms, const double* fractional, long count,
                             const int* keys, long channels, const int* channel_l, int max_l, long radial,
                             const double* radial_grid, const double* aug_moment, const double* compensation_r2,
                             long potential_count, const int* potential_keys, const double* potential, double* out,
                             char* error, long error_length) {
  try {
    const auto a = augmentation(channels, channel_l, max_l, radial, radial_grid, aug_moment, compensation_r2);
    std::array<sdft::Vec3, 3> cell{};
    for (int r = 0; r < 3; ++r) cell[r] = {lattice[3 * r], lattice[3 * r + 1], lattice[3 * r + 2]};
    std::vector<std::tuple<int, int, int>> support(static_cast<std::size_t>(count));
    for (long i = 0; i < count; ++i) support[i] = {keys[3 * i], keys[3 * i + 1], keys[3 * i + 2]};
    std::size_t dim = 0;
    for (int l : a.channel_l) dim += 2 * l + 1;
    std::vector<sdft::PawCompensationOperator> ops;
    ops.reserve(static_cast<std::size_t>(atoms));
    for (long i = 0; i < atoms; ++i) {
      const sdft::Vec3 f{fractional[3 * i], fractional[3 * i + 1], fractional[3 * i + 2]};
      ops.emplace_back(a, cell, f, support, sdft::AtomicUnitConvention::Codata, i ? &ops.front() : nullptr);
    }
    sdft::FourierDensity v;
    const auto* pv = reinterpret_cast<const C*>(potential);
    for (long i = 0; i < potential_count; ++i)
      v[{potential_keys[3 * i], potential_keys[3 * i + 1], potential_keys[3 * i + 2]}] = pv[i];
    const auto projected = sdft::PawCompensationOperator::project_potential_batch(ops, v);
    auto* o = reinterpret_cast<C*>(out);
    for (long i = 0; i < atoms; ++i)
      for (std::size_t e = 0; e < dim * dim; ++e) o[i * dim * dim + e] = projected[i][e];
    return 0;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return 1;
  }
}
}

extern "C" {

// evaluate_density_functionals on a density (and optional frozen core) given
// as key/value arrays. Returns the support size (the potential's keys, in map
// order) or -1 with the error text. With capacity >= that size it writes the
// keys, potential, xc_potential and scalars = [hartree_energy, xc_energy,
// vxc_density, sampled_electrons, minimum_density, clipped_density_points,
// grid_points, hartree_stress (9, row-major), xc_stress (9)].
long ref_density_functionals(const double* lattice, long count, const int* keys, const double* values,
                             long core_count, const int* core_keys, const double* core, int padding, long capacity,
                             int* out_keys, double* potential, double* xc_potential, double* scalars, char* error,
                             long error_length) {
  try {
    std::array<sdft::Vec3, 3> cell{};
    for (int r = 0; r < 3; ++r) cell[r] = {lattice[3 * r], lattice[3 * r + 1], lattice[3 * r + 2]};
    sdft::FourierDensity density, frozen;
    const auto* pv = reinterpret_cast<const C*>(values);
    for (long i = 0; i < count; ++i) density[{keys[3 * i], keys[3 * i + 1], keys[3 * i + 2]}] = pv[i];
    const auto* pc = reinterpret_cast<const C*>(core);
    for (long i = 0; i < core_count; ++i)
      frozen[{core_keys[3 * i], core_keys[3 * i + 1], core_keys[3 * i + 2]}] = pc[i];
    const auto result = sdft::evaluate_density_functionals(density, cell, core_count ? &frozen : nullptr, padding,
                                                           false);
    const long size = static_cast<long>(result.potential.size());
    if (capacity < size) return size;
    long i = 0;
    auto* po = reinterpret_cast<C*>(potential);
    auto* xo = reinterpret_cast<C*>(xc_potential);
    for (const auto& [key, value] : result.potential) {
      out_keys[3 * i] = std::get<0>(key);
      out_keys[3 * i + 1] = std::get<1>(key);
      out_keys[3 * i + 2] = std::get<2>(key);
      po[i] = value;
      const auto found = result.xc_potential.find(key);
      xo[i] = found == result.xc_potential.end() ? C{} : found->second;
      ++i;
    }
    scalars[0] = result.hartree_energy;
    scalars[1] = result.xc_energy;
    scalars[2] = result.vxc_density;
    scalars[3] = result.sampled_electrons;
    scalars[4] = result.minimum_density;
    scalars[5] = static_cast<double>(result.clipped_density_points);
    scalars[6] = static_cast<double>(result.grid_points);
    for (int a = 0; a < 3; ++a) {
      const auto& h = result.hartree_stress[a];
      const auto& x = result.xc_stress[a];
      scalars[7 + 3 * a] = h.x;
      scalars[8 + 3 * a] = h.y;
      scalars[9 + 3 * a] = h.z;
      scalars[16 + 3 * a] = x.x;
      scalars[17 + 3 * a] = x.y;
      scalars[18 + 3 * a] = x.z;
    }
    return size;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return -1;
  }
}
}

extern "C" {

// evaluate_collinear_density_functionals on up/down densities and an
// optional frozen core. Returns the support size (map order) or -1 with the
// error text; with capacity >= that size it writes the keys, per channel the
// potential and xc_potential (up then down, capacity entries each) and
// scalars[25 * channel + ...] in ref_density_functionals' order.
long ref_collinear_functionals(const double* lattice, long count_up, const int* keys_up, const double* up,
                               long count_down, const int* keys_down, const double* down, long core_count,
                               const int* core_keys, const double* core, int padding, long capacity, int* out_keys,
                               double* potential, double* xc_potential, double* scalars, char* error,
                               long error_length) {
  try {
    std::array<sdft::Vec3, 3> cell{};
    for (int r = 0; r < 3; ++r) cell[r] = {lattice[3 * r], lattice[3 * r + 1], lattice[3 * r + 2]};
    std::array<sdft::FourierDensity, 2> density;
    sdft::FourierDensity frozen;
    const auto fill = [](sdft::FourierDensity& map, long count, const int* keys, const double* values) {
      const auto* v = reinterpret_cast<const C*>(values);
      for (long i = 0; i < count; ++i) map[{keys[3 * i], keys[3 * i + 1], keys[3 * i + 2]}] = v[i];
    };
    fill(density[0], count_up, keys_up, up);
    fill(density[1], count_down, keys_down, down);
    fill(frozen, core_count, core_keys, core);
    const auto result = sdft::evaluate_collinear_density_functionals(density, cell, core_count ? &frozen : nullptr,
                                                                      padding);
    const long size = static_cast<long>(result[0].potential.size());
    if (capacity < size) return size;
    for (int s = 0; s < 2; ++s) {
      long i = 0;
      auto* po = reinterpret_cast<C*>(potential) + s * capacity;
      auto* xo = reinterpret_cast<C*>(xc_potential) + s * capacity;
      for (const auto& [key, value] : result[s].potential) {
        if (s == 0) {
          out_keys[3 * i] = std::get<0>(key);
          out_keys[3 * i + 1] = std::get<1>(key);
          out_keys[3 * i + 2] = std::get<2>(key);
        }
        po[i] = value;
        const auto found = result[s].xc_potential.find(key);
        xo[i] = found == result[s].xc_potential.end() ? C{} : found->second;
        ++i;
      }
      double* o = scalars + 25 * s;
      const auto& r = result[s];
      o[0] = r.hartree_energy;
      o[1] = r.xc_energy;
      o[2] = r.vxc_density;
      o[3] = r.sampled_electrons;
      o[4] = r.minimum_density;
      o[5] = static_cast<double>(r.clipped_density_points);
      o[6] = static_cast<double>(r.grid_points);
      for (int a = 0; a < 3; ++a) {
        o[7 + 3 * a] = r.hartree_stress[a].x;
        o[8 + 3 * a] = r.hartree_stress[a].y;
        o[9 + 3 * a] = r.hartree_stress[a].z;
        o[16 + 3 * a] = r.xc_stress[a].x;
        o[17 + 3 * a] = r.xc_stress[a].y;
        o[18 + 3 * a] = r.xc_stress[a].z;
      }
    }
    return size;
  } catch (const std::exception& e) {
    set_error(error, error_length, e);
    return -1;
  }
}
}
