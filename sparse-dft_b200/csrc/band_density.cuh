// Band density on the device: n(G) on a Fourier support from band-major
// plane-wave coefficients, the reference's plane_wave_density_fft
// (src/density_functionals.cpp:407-460) with FourierGrid::add_wavefunction_density
// (:71-77) and to_fourier (:269-284).
#pragma once
#include <cstdint>
#include <vector>

#include "local_hamiltonian.cuh"

namespace sdft_b200 {

struct Context;

// Density grid of the reference's rule, N_a = max(3, 2 m_a + 1) with
// m_a = max(max |support_a|, max_g - min_g) (min/max seeded at 0), rounded up
// to a 2/3/5/7-smooth length (the reference's SDFT_FAST_DENSITY_GRID=1
// option; every retained mode is unchanged and the grid stays alias-free).
void density_grid_shape(const std::int32_t* hkl, std::size_t npw, const std::int32_t* support, std::size_t count,
                        int shape[3]);

// out[j] = sum_b occupations[b]/volume |FFT_bwd(scatter psi_b)|^2 transformed
// forward and divided by N, at support key j. psi: `bands` columns of npw
// complex values, band-major (device). out: `count` complex values (device).
// Occupations (host) must lie in [0, 2]; zero bands are skipped.
void band_density(Context& ctx, const std::int32_t* hkl, std::size_t npw, const Cx<double>* psi,
                  const double* occupations, std::size_t bands, double volume, const std::int32_t* support,
                  std::size_t count, Cx<double>* out);

}  // namespace sdft_b200
