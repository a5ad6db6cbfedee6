// Device-resident generalized block Davidson in the S~ metric.
#pragma once
#include <vector>

#include "eigensolver.cuh"
#include "operator.cuh"
#include "umma_gemm.cuh"

namespace sdft_b200 {

struct DavidsonOptions {
  int roots = 0;
  int max_iterations = 256;
  double tolerance = 1e-10;
  Precision precision = Precision::FP64;  // search precision; certification is always FP64
  int subspace_factor = 8;                // capacity = min(n, max(factor*roots, 64)), in [4,16]
  double handoff = 1e-8;                  // search residual that hands the basis to FP64
  // Mixed form: CG steps on each unconverged root's Jacobi-Davidson
  // correction equation (correction.cuh) in place of the reference's single
  // kinetic-preconditioner step; 0 keeps the reference's step.
  int correction_steps = 0;
  // Band-group local solves (src/band_group_solver.cpp:95-107): an explicit
  // subspace capacity (0 = the factor rule) and completed lower bands, device
  // n x excluded_count, S-orthonormal, projected out of every search
  // direction (the reference's excluded_vectors, src/pw_core.cpp:675-712).
  int capacity = 0;
  const Cx<double>* excluded = nullptr;
  int excluded_count = 0;
};

struct DavidsonStats {
  int iterations = 0;
  bool converged = false;
  double max_residual = 0.0;
  long long h_columns_search = 0, h_columns_fp64 = 0, s_columns_search = 0, s_columns_fp64 = 0;
  int rayleigh_ritz = 0, restarts = 0, fp64_refreshes = 0, certifications = 0, handoff_iteration = -1;
  int block_rank_fallbacks = 0;
  long long correction_columns = 0;
  // Strict FP64 refinements (tangent polish and root-manifold steps), tried / accepted.
  int polish_steps = 0, polish_accepted = 0, manifold_steps = 0, manifold_accepted = 0;
  double seconds = 0.0, rr_seconds = 0.0;  // rr_seconds: device time of the Rayleigh-Ritz steps
};

class DavidsonSolver {
 public:
  // The solver's device state lives in the operator's context (reused by
  // the solves of later operators on that context).
  explicit DavidsonSolver(DeviceOperator& op)
      : op_(op), b_(op.context().davidson), basis_(b_.basis), hbasis_(b_.hbasis), sbasis_(b_.sbasis),
        cached_h_(b_.cached_h), cached_s_(b_.cached_s), rr_a_(b_.rr_a), rr_b_(b_.rr_b), rr_w_(b_.rr_w),
        rr_work_(b_.rr_work), info_(b_.info), eigen_(b_.eigen), xs_(b_.xs), sxs_(b_.sxs), hxs_(b_.hxs),
        res_(b_.res), block_(b_.block), metric_(b_.metric), original_(b_.original), projections_(b_.projections),
        gram_(b_.gram), small_(b_.small), order_(b_.order), select_(b_.select), pack_vc_(b_.pack_vc),
        pack_vn_(b_.pack_vn), pack_hn_(b_.pack_hn), pack_sn_(b_.pack_sn), pack_hb_(b_.pack_hb),
        pack_sb_(b_.pack_sb) {}
  ~DavidsonSolver();
  DavidsonSolver(const DavidsonSolver&) = delete;
  DavidsonSolver& operator=(const DavidsonSolver&) = delete;
  // initial: device n x roots (column-major) warm vectors, or null for a cold start.
  void solve(const DavidsonOptions& options, const Cx<double>* initial);

  const std::vector<double>& eigenvalues() const { return values_; }
  const std::vector<double>& residuals() const { return residual_norms_; }
  const Cx<double>* vectors() const { return x_; }  // n x roots, S-normalised, on the device
  const DavidsonStats& stats() const { return stats_; }

 private:
  Precision mode() const { return exact_mode_ ? Precision::FP64 : Precision::Mixed; }
  void gemm(Op aop, int m, int n, int k, const Cx<double>* a, long long lda, const Cx<double>* b, long long ldb,
            Cx<double>* c, long long ldc, bool add, double alpha, bool exact);
  void apply_h(const Cx<double>* x, int cols, Cx<double>* y, bool exact);
  void apply_s(const Cx<double>* x, int cols, Cx<double>* y, bool exact);
  void apply_pair(const Cx<double>* x, int cols, Cx<double>* hy, Cx<double>* sy, bool exact);
  bool append_block(Cx<double>* vectors, int k);
  bool append_single(const Cx<double>* v);
  void update_projected(const Cx<double>* applied, Cx<double>* cached, const std::uint16_t* packed_applied);
  // Mixed search: BF16-split copies of the basis V and its images HV, SV,
  // written once per column as the column is formed, in the layouts the
  // tensor-core products read (A rows for V^H, K entries for V, HV, SV as
  // left factors, B rows for HV, SV as right factors).
  bool searching() const { return !exact_mode_ && packs_; }
  void pack_basis(int first, int count);
  void pack_images(int first, int count);
  PackedA basis_rows(int first, int rows) const;                    // V^H rows [first, first+rows), K = n
  PackedA left_factor(const std::uint16_t* base, int k) const;      // n x k left factor (V, HV or SV)
  void gemm_left(const std::uint16_t* packed, int n, int k, const Cx<double>* b, long long ldb, Cx<double>* c,
                 long long ldc, bool add, double alpha);
  void remove_excluded(Cx<double>* vectors, int cols);
  void rayleigh_ritz();
  void certify();
  // Strict FP64 refinements of a certified block that Davidson no longer
  // improves (src/strict_residual_polish.hpp:70-197): a generalized Ritz
  // problem inside span(X) and a per-root tangent line search along the
  // projected, preconditioned residual. Each replaces X only with a fresh,
  // improved FP64 certificate and S-orthonormality within 1e-12.
  bool root_manifold_step();
  bool tangent_polish_step();
  // Keeps the polished X and the rest of the search space (its S-orthogonal
  // complement in the basis, or the guard Ritz vectors at capacity) as the
  // new basis (src/pw_core.cpp:1337-1356).
  void preserve_search_subspace();
  bool commit_trial(Cx<double>* trial, Cx<double>* th, Cx<double>* ts, Cx<double>* errors, double old_max);
  double max_residual() const;
  void refresh_images();
  std::vector<double> download(const double* device, int count);

  DeviceOperator& op_;
  DavidsonStats stats_;
  int n_ = 0, roots_ = 0, capacity_ = 0, kmax_ = 0, correction_steps_ = 0;
  int size_ = 0, computed_h_ = 0, projected_size_ = 0;
  const Cx<double>* excluded_ = nullptr;  // completed bands of a band-group local solve
  Cx<double>* excluded_s_ = nullptr;      // their S images
  int excluded_count_ = 0;
  bool exact_mode_ = true, incremental_ = true, strict_projection_ = false;
  bool polish_enabled_ = true, manifold_enabled_ = true;
  int polish_attempts_ = 0, manifold_attempts_ = 0;
  double strict_entry_ = 0.0;
  double tolerance_ = 1e-10;
  DavidsonBuffers& b_;
  Scratch &basis_, &hbasis_, &sbasis_, &cached_h_, &cached_s_, &rr_a_, &rr_b_, &rr_w_, &rr_work_, &info_;
  EigenWorkspace& eigen_;
  Scratch &xs_, &sxs_, &hxs_, &res_, &block_, &metric_, &original_, &projections_, &gram_, &small_, &order_,
      &select_;
  Scratch &pack_vc_, &pack_vn_, &pack_hn_, &pack_sn_, &pack_hb_, &pack_sb_;
  bool packs_ = false;
  Split split_ = Split::BF16x6;
  long long ld_rows_ = 0, ld_cols_ = 0;  // packed row lengths: K = n (rows of V^H, HV, SV) and K = capacity
  Cx<double>* v_ = nullptr;
  Cx<double>* hv_ = nullptr;
  Cx<double>* sv_ = nullptr;
  Cx<double>* ch_ = nullptr;
  Cx<double>* cs_ = nullptr;
  Cx<double>* x_ = nullptr;
  Cx<double>* sx_ = nullptr;
  Cx<double>* hx_ = nullptr;
  Cx<double>* r_ = nullptr;
  double* w_ = nullptr;       // RR eigenvalues (device)
  double* dsmall_ = nullptr;  // per-column device scalars (norms, metric, values)
  std::vector<double> values_, residual_norms_;
  std::vector<double> residual_history_;
  cudaEvent_t rr_events_[2] = {nullptr, nullptr};  // Rayleigh-Ritz step start / end on the solver's stream
};

}  // namespace sdft_b200
