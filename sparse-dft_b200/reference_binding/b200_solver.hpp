// Device-resident route for the reference's solve_generalized_hermitian_davidson
// (src/pw_core.hpp:184-188), in the reference's own types.
//
// The accelerator plugin (compute_b200.cpp) keeps the reference's Davidson on
// the host and sends it per-call products. This route instead hands the whole
// solve to libsdft_b200: the operator (B, D, Q, V(r), maps) is uploaded once
// and every NPW-long array of the Davidson stays in HBM; only eigenvalues,
// band-major eigenvectors and fresh FP64 residuals come back, in a
// ComplexGeneralizedEigenResult. A caller that builds a PlaneWaveOperator from
// (basis, potential, paw) -- the SCF k-loop, src/scf_core.cpp:2312-2313 and
// :3043 -- or replays a solver snapshot (src/solver_replay_cli.cpp:18-27)
// calls one of the two functions below in its place.
#pragma once

#include <complex>
#include <cstddef>
#include <string>
#include <vector>

#include "plane_wave_operator.hpp"
#include "pw_core.hpp"
#include "sdft_b200.h"

namespace sdft::b200 {

// Maps a library status to the reference's exception classes.
void throw_on_error(sdft_b200_status status);

struct DeviceSolveSettings {
  int device = 0;
  int precision = SDFT_B200_PRECISION_MIXED;  // FP64 runs the plain form throughout
  int subspace_factor = 8;
  int correction_steps = 0;                   // library default (see sdft_b200_davidson_options)
};

// The operator of PlaneWaveOperator(basis, potential, paw, hartree_to_ev,
// regularization) (src/plane_wave_operator.hpp:27-30) solved on the device.
// initial: band-major n_roots x NPW warm vectors, or empty.
ComplexGeneralizedEigenResult solve_generalized_hermitian_davidson_device(
    const std::vector<GVector>& basis, const FourierDensity& potential, const std::vector<ComplexPawOperator>& paw,
    double hartree_to_ev, double regularization, std::size_t n_roots, std::size_t max_iterations, double tolerance,
    const std::vector<std::complex<double>>& initial = {}, const DeviceSolveSettings& settings = {});

// The operator stored in a solver snapshot (save_solver_snapshot's SDFTPWO3
// file) solved on the device with the snapshot's roots, iteration limit,
// tolerance and warm vectors unless overridden (0 keeps the stored value).
ComplexGeneralizedEigenResult solve_snapshot_davidson_device(const std::string& path, std::size_t max_iterations = 0,
                                                             const DeviceSolveSettings& settings = {});

}  // namespace sdft::b200
