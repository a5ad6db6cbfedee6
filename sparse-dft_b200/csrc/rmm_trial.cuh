// Residual-minimisation trial for SCF warm solves (rmm_trial.cu): the
// reference's solve_generalized_hermitian_rmm_trial, src/pw_core.hpp:170-178
// (src/rmm_trial.cpp:128-206), on the device operator and the device
// Davidson solver (its fallback).
#pragma once
#include <vector>

#include "davidson.cuh"

namespace sdft_b200 {

struct RmmResult {
  std::vector<double> eigenvalues, residuals;
  int iterations = 0;          // trial steps plus the fallback's iterations
  int trial_steps = 0;
  bool converged = false;      // only a fallback solve can converge
  bool trial_manifold = false; // residual-checked trial, explicitly not converged
  bool fell_back = false;
  DavidsonStats fallback_stats;
};

class RmmTrial {
 public:
  RmmTrial(DeviceOperator& op, DavidsonSolver& fallback) : op_(op), fallback_(fallback) {}
  // initial: device n x roots warm vectors (required). options.tolerance must
  // be coarse (> 1e-9). vectors() holds the result afterwards.
  RmmResult solve(const DavidsonOptions& options, const Cx<double>* initial);
  const Cx<double>* vectors() const { return vectors_; }

 private:
  struct Images {
    Cx<double>* x = nullptr;
    Cx<double>* h = nullptr;
    Cx<double>* s = nullptr;
  };
  void apply(Images& v, bool exact);
  bool full_rank(const Images& v);
  void rotate(Images& v, const Cx<double>* u, Images& spare);
  void project(Images& d, const Images& x);
  void normalize(Images& v);
  double residual(const Images& v);

  DeviceOperator& op_;
  DavidsonSolver& fallback_;
  int n_ = 0, k_ = 0;
  Scratch blocks_, small_, scalars_;
  EigenWorkspace eigen_;
  Cx<double>* r_ = nullptr;
  Cx<double>* hs_ = nullptr;
  Cx<double>* ss_ = nullptr;
  Cx<double>* u_ = nullptr;
  Cx<double>* coeff_ = nullptr;
  double* values_ = nullptr;
  double* metric_ = nullptr;
  double* norms_ = nullptr;
  int* flags_ = nullptr;
  const Cx<double>* vectors_ = nullptr;
  std::vector<double> host_values_, host_norms_;
};

}  // namespace sdft_b200
