// Hartree + PBE exchange-correlation functional of a Fourier density
// (xc_functional.cu): the reference's evaluate_density_functionals,
// src/density_functionals.hpp:40-47 (src/density_functionals.cpp:462-729).
#pragma once
#include <array>
#include <cstdint>
#include <vector>

#include "operator.cuh"

namespace sdft_b200 {

// The union support of the density and the frozen core in the reference's
// map order, with what the device passes need per key.
struct FunctionalSupport {
  double volume = 0;
  bool with_core = false;
  int shape[3] = {0, 0, 0};
  long long points = 0;
  bool collinear = false;                // two spin channels: valence = up, down = down
  std::vector<std::array<int, 3>> keys;  // sorted lexicographically
  std::vector<Cx<double>> valence, core, down;  // 0 where the key is absent
  std::vector<unsigned char> flags;      // bit 0: density (up) key, bit 1: core key, bit 2: down key
  std::vector<long long> index, opposite;  // wrapped grid index of +G, -G
  std::vector<int> opposite_key;           // union position of -G, or -1
  std::vector<double> q;                   // G per key, 3 values
};

// Scalars of the reference's DensityFunctionals (stresses row-major 3 x 3).
struct FunctionalResult {
  double hartree_energy = 0, xc_energy = 0, vxc_density = 0;
  double hartree_stress[9] = {}, xc_stress[9] = {};
  double sampled_electrons = 0, minimum_density = 0;
  std::uint64_t clipped_density_points = 0, grid_points = 0;
  int grid[3] = {0, 0, 0};
};

// Host part: the reference's checks (singular lattice, empty or nonfinite
// density, nonfinite density plus core, padding range, SDFT_FFT_OVERSAMPLING,
// SDFT_FAST_DENSITY_GRID), duplicate keys rejected, the XC grid
// padding * max(3, 2 m_a + 1) per axis (at most 512).
// lattice: rows a1, a2, a3 in bohr; values interleaved complex.
FunctionalSupport functional_support(const double lattice[9], std::size_t count, const int* hkl,
                                     const double* density, std::size_t core_count, const int* core_hkl,
                                     const double* core, int quadrature_padding);

// Device part: potential (Hartree + v_xc) and v_xc on the support's keys, in
// its order, into host arrays; the scalars into result.
void density_functionals(Context& ctx, const FunctionalSupport& support, Cx<double>* potential,
                         Cx<double>* xc_potential, FunctionalResult& result);

// Collinear spin form (the reference's evaluate_collinear_density_functionals,
// src/density_functionals.hpp:52-56, src/density_functionals.cpp:732-806):
// host checks and support (union of both channels and the core, which each
// channel receives with weight 1/2), then per channel the potential
// (Hartree of the total density + the channel's v_xc), v_xc and the scalars
// (Hartree and XC energies and stresses split equally, <n_s, v_xc,s>,
// electrons Omega Re n_s(0), minimum and count of negative samples).
FunctionalSupport collinear_support(const double lattice[9], const std::size_t count[2], const int* const hkl[2],
                                    const double* const density[2], std::size_t core_count, const int* core_hkl,
                                    const double* core, int padding);
void collinear_functionals(Context& ctx, const FunctionalSupport& support, Cx<double>* const potential[2],
                           Cx<double>* const xc_potential[2], FunctionalResult result[2]);

}  // namespace sdft_b200
