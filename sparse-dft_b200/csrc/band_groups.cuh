// Band-group solver (band_groups.cu): the reference's
// solve_generalized_hermitian_band_groups, src/pw_core.hpp:179-182
// (src/band_group_solver.cpp:55-212), on the device operator with the
// device Davidson solver for the local solves and the final refinement.
#pragma once
#include <vector>

#include "davidson.cuh"

namespace sdft_b200 {

struct BandGroupResult {
  std::vector<double> eigenvalues, residuals;
  int iterations = 0;
  bool converged = false;
  int sweeps = 0;
  bool refined = false;  // swept mode handed the block to a global Davidson solve
};

class BandGroupSolver {
 public:
  BandGroupSolver(DeviceOperator& op, DavidsonSolver& davidson) : op_(op), davidson_(davidson) {}
  // initial: device n x roots warm vectors or null.
  BandGroupResult solve(const DavidsonOptions& options, const Cx<double>* initial);
  const Cx<double>* vectors() const { return vectors_; }

 private:
  DeviceOperator& op_;
  DavidsonSolver& davidson_;
  Scratch x_, images_, small_, scalars_;
  EigenWorkspace eigen_;
  const Cx<double>* vectors_ = nullptr;
};

}  // namespace sdft_b200
