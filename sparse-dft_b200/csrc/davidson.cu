// Device-resident generalized block Davidson (restates the control flow of the
// reference's solve_generalized_hermitian_davidson, src/pw_core.cpp:532-1437,
// with its default flags: joint H/S, block CGS2 in the S metric, incremental
// Galerkin slabs, kinetic preconditioner, thick restart to 2*roots, FP64
// refresh when the approximate search converges, fresh FP64 certification).
//
// Every NPW-long array (basis, H/S images, Ritz block, residuals) stays in HBM
// for the whole solve; the host sees only per-column scalars (residual norms,
// Ritz values) to take the same branch decisions as the reference.
#include <cusolverDn.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <limits>
#include <numeric>
#include <string>

#include "correction.cuh"
#include "davidson.cuh"
#include "dense.cuh"
#include "umma_gemm.cuh"

namespace sdft_b200 {

namespace {
void check_solver(cusolverStatus_t status, const char* what) {
  if (status != CUSOLVER_STATUS_SUCCESS)
    throw CudaError(std::string("cuSOLVER error ") + std::to_string(static_cast<int>(status)) + " in " + what);
}
void check_blas(cublasStatus_t status, const char* what) {
  if (status != CUBLAS_STATUS_SUCCESS)
    throw CudaError(std::string("cuBLAS error ") + std::to_string(static_cast<int>(status)) + " in " + what);
}
// The reference's 0/1 environment switches (src/pw_core.cpp:598-603).
bool boolean_control(const char* name, bool fallback) {
  const char* flag = std::getenv(name);
  if (!flag) return fallback;
  const std::string value(flag);
  if (value != "0" && value != "1") throw InvalidArgument(std::string(name) + " must be 0 or 1");
  return value == "1";
}
double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}
template <typename T>
T* as(Scratch& s, std::size_t count) {
  return static_cast<T*>(s.reserve(sizeof(T) * std::max<std::size_t>(count, 1)));
}
}  // namespace

std::vector<double> DavidsonSolver::download(const double* device, int count) {
  std::vector<double> host(std::max(count, 0));
  if (count > 0) {
    SDFT_CUDA(cudaMemcpyAsync(host.data(), device, sizeof(double) * count, cudaMemcpyDeviceToHost,
                              op_.context().stream));
    op_.context().synchronize();
    if (umma_error_flag()) throw CudaError("tensor-core GEMM wait limit exceeded");
  }
  return host;
}

void DavidsonSolver::gemm(Op aop, int m, int n, int k, const Cx<double>* a, long long lda, const Cx<double>* b,
                          long long ldb, Cx<double>* c, long long ldc, bool add, double alpha, bool exact) {
  auto& ctx = op_.context();
  if (exact) zgemm(ctx.blas, aop, Op::N, m, n, k, a, lda, b, ldb, c, ldc, add, alpha);
  else gemm_tc(aop, m, n, k, a, lda, nullptr, b, ldb, c, ldc, add, alpha, search_split(), ctx.tc, ctx.stream);
}

PackedA DavidsonSolver::basis_rows(int first, int rows) const {
  PackedA p;
  p.data = static_cast<std::uint16_t*>(pack_vc_.ptr) + first * ld_rows_;
  p.ld = ld_rows_;
  p.rows = rows;
  p.k = n_;
  p.split = split_;
  return p;
}

PackedA DavidsonSolver::left_factor(const std::uint16_t* base, int k) const {
  PackedA p;
  p.data = const_cast<std::uint16_t*>(base);
  p.ld = ld_cols_;
  p.rows = n_;
  p.k = k;
  p.split = split_;
  return p;
}

// C (n x cols) = alpha L B (+ C): L one of the packed n x k left factors.
void DavidsonSolver::gemm_left(const std::uint16_t* packed, int n, int k, const Cx<double>* b, long long ldb,
                               Cx<double>* c, long long ldc, bool add, double alpha) {
  auto& ctx = op_.context();
  const PackedA a = left_factor(packed, k);
  gemm_tc(Op::N, n_, n, k, nullptr, 0, &a, b, ldb, c, ldc, add, alpha, split_, ctx.tc, ctx.stream);
}

void DavidsonSolver::pack_basis(int first, int count) {
  if (!packs_ || count <= 0) return;
  const cudaStream_t st = op_.context().stream;
  const Cx<double>* v = v_ + static_cast<long long>(first) * n_;
  pack_a(Op::C, v, n_, count, n_, split_, static_cast<std::uint16_t*>(pack_vc_.ptr) + first * ld_rows_, ld_rows_, st);
  pack_a_columns(v_, n_, n_, first, count, split_, static_cast<std::uint16_t*>(pack_vn_.ptr), ld_cols_, st);
  pack_a_columns(sv_, n_, n_, first, count, split_, static_cast<std::uint16_t*>(pack_sn_.ptr), ld_cols_, st);
  pack_b(sv_ + static_cast<long long>(first) * n_, n_, n_, count, split_,
         static_cast<std::uint16_t*>(pack_sb_.ptr) + 2LL * first * ld_rows_, ld_rows_, st);
}

void DavidsonSolver::pack_images(int first, int count) {
  if (!packs_ || count <= 0) return;
  const cudaStream_t st = op_.context().stream;
  pack_a_columns(hv_, n_, n_, first, count, split_, static_cast<std::uint16_t*>(pack_hn_.ptr), ld_cols_, st);
  pack_b(hv_ + static_cast<long long>(first) * n_, n_, n_, count, split_,
         static_cast<std::uint16_t*>(pack_hb_.ptr) + 2LL * first * ld_rows_, ld_rows_, st);
}

void DavidsonSolver::apply_h(const Cx<double>* x, int cols, Cx<double>* y, bool exact) {
  op_.apply_hamiltonian(x, cols, y, exact ? Precision::FP64 : Precision::Mixed);
  (exact ? stats_.h_columns_fp64 : stats_.h_columns_search) += cols;
}

void DavidsonSolver::apply_s(const Cx<double>* x, int cols, Cx<double>* y, bool exact) {
  op_.apply_overlap(x, cols, y, exact ? Precision::FP64 : Precision::Mixed);
  (exact ? stats_.s_columns_fp64 : stats_.s_columns_search) += cols;
}

void DavidsonSolver::apply_pair(const Cx<double>* x, int cols, Cx<double>* hy, Cx<double>* sy, bool exact) {
  op_.apply_pair(x, cols, hy, sy, exact ? Precision::FP64 : Precision::Mixed);
  (exact ? stats_.h_columns_fp64 : stats_.h_columns_search) += cols;
  (exact ? stats_.s_columns_fp64 : stats_.s_columns_search) += cols;
}

// vectors -= E (SE^H vectors) for the completed bands E of a band-group local
// solve, FP64 (the reference's remove_excluded, src/pw_core.cpp:701-712).
// The coefficients use the region after the S images that solve() reserved
// (excluded_count x max(excluded_count, kmax) entries; cols <= kmax).
void DavidsonSolver::remove_excluded(Cx<double>* vectors, int cols) {
  if (cols > std::max(excluded_count_, kmax_)) throw InvalidArgument("completed-band projection block too wide");
  Cx<double>* coefficients = excluded_s_ + static_cast<std::size_t>(n_) * excluded_count_;
  gemm(Op::C, excluded_count_, cols, n_, excluded_s_, n_, vectors, n_, coefficients, excluded_count_, false, 1.0, true);
  gemm(Op::N, n_, cols, excluded_count_, excluded_, n_, coefficients, excluded_count_, vectors, n_, true, -1.0, true);
}

// One direction at a time (src/pw_core.cpp:796-853): CGS2 in the S metric with
// FP64 operators, reject norm^2 < 1e-24.
bool DavidsonSolver::append_single(const Cx<double>* source) {
  if (size_ >= capacity_) return false;
  auto& ctx = op_.context();
  const cudaStream_t st = ctx.stream;
  Cx<double>* v = as<Cx<double>>(original_, static_cast<std::size_t>(n_) * kmax_);
  Cx<double>* sv = as<Cx<double>>(metric_, static_cast<std::size_t>(n_) * kmax_);
  Cx<double>* proj = as<Cx<double>>(projections_, static_cast<std::size_t>(capacity_) * kmax_);
  if (source != v) copy_block(source, n_, v, n_, n_, 1, st);
  column_norms(v, n_, n_, 1, dsmall_, st);
  const double norm = download(dsmall_, 1)[0];
  if (!std::isfinite(norm)) throw std::runtime_error("nonfinite Davidson direction");
  if (norm == 0) return false;
  unit_columns(v, n_, n_, 1, dsmall_, st);
  for (int pass = 0; pass < 2 && (size_ || excluded_count_); ++pass) {
    if (excluded_count_) remove_excluded(v, 1);
    if (!size_) continue;
    apply_s(v, 1, sv, true);
    gemm(Op::C, size_, 1, n_, v_, n_, sv, n_, proj, size_, false, 1.0, true);
    gemm(Op::N, n_, 1, size_, v_, n_, proj, size_, v, n_, true, -1.0, true);
  }
  apply_s(v, 1, sv, true);
  metric_norms(v, sv, n_, n_, 1, dsmall_, st);
  const double norm2 = download(dsmall_, 1)[0];
  if (!std::isfinite(norm2) || norm2 < -1e-10) throw std::runtime_error("Davidson encountered non-positive overlap direction");
  if (norm2 < 1e-24) return false;
  scale_columns(v, n_, n_, 1, dsmall_, true, st);
  scale_columns(sv, n_, n_, 1, dsmall_, true, st);
  copy_block(v, n_, v_ + static_cast<long long>(size_) * n_, n_, n_, 1, st);
  copy_block(sv, n_, sv_ + static_cast<long long>(size_) * n_, n_, n_, 1, st);
  if (searching()) pack_basis(size_, 1);
  ++size_;
  return true;
}

// Block CGS2 in the S metric (src/pw_core.cpp:871-1013). `vectors` is an
// n x k workspace block that this call may overwrite.
bool DavidsonSolver::append_block(Cx<double>* vectors, int k) {
  auto& ctx = op_.context();
  const cudaStream_t st = ctx.stream;
  const int before = size_;
  k = std::min(k, capacity_ - size_);
  if (k <= 0) return false;
  auto serial = [&]() {
    for (int j = 0; j < k; ++j) append_single(vectors + static_cast<long long>(j) * n_);
    return size_ > before;
  };
  if (k == 1) return serial();
  const bool exact = exact_mode_;
  column_norms(vectors, n_, n_, k, dsmall_, st);
  const auto norms = download(dsmall_, k);
  for (double v : norms)
    if (!(v > 0) || !std::isfinite(v)) return serial();
  unit_columns(vectors, n_, n_, k, dsmall_, st);
  Cx<double>* original = as<Cx<double>>(original_, static_cast<std::size_t>(n_) * kmax_);
  Cx<double>* metric = as<Cx<double>>(metric_, static_cast<std::size_t>(n_) * kmax_);
  Cx<double>* proj = as<Cx<double>>(projections_, static_cast<std::size_t>(capacity_) * kmax_);
  copy_block(vectors, n_, original, n_, n_, k, st);
  apply_s(vectors, k, metric, exact);
  for (int pass = 0; (size_ || excluded_count_) && pass < 2; ++pass) {
    if (excluded_count_) {
      remove_excluded(vectors, k);
      if (!size_) {
        apply_s(vectors, k, metric, exact);
        continue;
      }
      apply_s(vectors, k, metric, exact);
    }
    if (!exact && searching()) {
      const PackedA vh = basis_rows(0, size_);
      gemm_tc(Op::C, size_, k, n_, nullptr, 0, &vh, metric, n_, proj, size_, false, 1.0, split_, ctx.tc, st);
      gemm_left(static_cast<std::uint16_t*>(pack_vn_.ptr), k, size_, proj, size_, vectors, n_, true, -1.0);
    } else {
      gemm(Op::C, size_, k, n_, v_, n_, metric, n_, proj, size_, false, 1.0, exact);
      gemm(Op::N, n_, k, size_, v_, n_, proj, size_, vectors, n_, true, -1.0, exact);
    }
    apply_s(vectors, k, metric, exact);
  }
  // Gram matrix and its normalisation.
  const std::size_t kk = static_cast<std::size_t>(kmax_) * kmax_;
  Cx<double>* gram = as<Cx<double>>(gram_, kk * 4);
  Cx<double>* herm = gram + kk;
  gemm(Op::C, k, k, n_, vectors, n_, metric, n_, gram, k, false, 1.0, exact);
  hermitian_part(gram, k, herm, k, k, st);
  // Well-conditioned blocks: G = U^H U (Cholesky) and the normalisation
  // U^-1, accepted when U^-H G U^-1 is the identity within 1e-8 (condition
  // numbers up to ~1e8, two orders inside the eigenvalue test's 1e10). The
  // span, and with it the next Rayleigh-Ritz step, is the one the
  // eigendecomposition's U diag(1/sqrt(l)) gives.
  {
    Cx<double>* factor = gram;  // the raw Gram is no longer needed
    Cx<double>* inverse = gram + 2 * kk;
    Cx<double>* check = gram + 3 * kk;
    copy_block(herm, k, factor, k, k, k, st);
    int lwork = 0;
    check_solver(cusolverDnZpotrf_bufferSize(ctx.solver, CUBLAS_FILL_MODE_UPPER, k,
                                             reinterpret_cast<cuDoubleComplex*>(factor), k, &lwork),
                 "zpotrf_bufferSize");
    auto* work = as<cuDoubleComplex>(rr_work_, static_cast<std::size_t>(std::max(1, lwork)));
    int* info = as<int>(info_, 4);
    check_solver(cusolverDnZpotrf(ctx.solver, CUBLAS_FILL_MODE_UPPER, k, reinterpret_cast<cuDoubleComplex*>(factor), k,
                                  work, lwork, info),
                 "zpotrf");
    int host_info = 0;
    SDFT_CUDA(cudaMemcpyAsync(&host_info, info, sizeof(int), cudaMemcpyDeviceToHost, st));
    SDFT_CUDA(cudaStreamSynchronize(st));
    if (host_info == 0) {
      zero_block(inverse, k, k, k, st);
      add_identity(inverse, k, st);
      const cuDoubleComplex one{1.0, 0.0};
      check_blas(cublasZtrsm(ctx.blas, CUBLAS_SIDE_LEFT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, k, k,
                             &one, reinterpret_cast<const cuDoubleComplex*>(factor), k,
                             reinterpret_cast<cuDoubleComplex*>(inverse), k),
                 "ztrsm");
      zgemm(ctx.blas, Op::N, Op::N, k, k, k, herm, k, inverse, k, factor, k, false);
      zgemm(ctx.blas, Op::C, Op::N, k, k, k, inverse, k, factor, k, check, k, false);
      const double deviation = identity_deviation(check, k, eigen_, st);
      static const bool trace = std::getenv("SDFT_B200_TRACE") != nullptr;
      if (trace)
        std::fprintf(stderr, "block-normalisation k=%d cholesky deviation=%.3e%s\n", k, deviation,
                     deviation <= 1e-8 ? "" : " (eigendecomposition)");
      if (deviation <= 1e-8) {
        gemm(Op::N, n_, k, k, vectors, n_, inverse, k, v_ + static_cast<long long>(size_) * n_, n_, false, 1.0, exact);
        gemm(Op::N, n_, k, k, metric, n_, inverse, k, sv_ + static_cast<long long>(size_) * n_, n_, false, 1.0, exact);
        if (searching()) pack_basis(size_, k);
        size_ += k;
        return true;
      }
    }
  }
  // Otherwise the reference's metric eigendecomposition, rank test and
  // normalisation U diag(1/sqrt(l)).
  double* lam = as<double>(small_, static_cast<std::size_t>(kmax_) * 2);
  int lwork = 0;
  check_solver(cusolverDnZheevd_bufferSize(ctx.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, k,
                                           reinterpret_cast<cuDoubleComplex*>(herm), k, lam, &lwork),
               "zheevd_bufferSize");
  auto* work = as<cuDoubleComplex>(rr_work_, static_cast<std::size_t>(lwork));
  int* info = as<int>(info_, 4);
  check_solver(cusolverDnZheevd(ctx.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, k,
                                reinterpret_cast<cuDoubleComplex*>(herm), k, lam, work, lwork, info),
               "zheevd");
  int host_info = 0;
  SDFT_CUDA(cudaMemcpyAsync(&host_info, info, sizeof(int), cudaMemcpyDeviceToHost, st));
  const auto eig = download(lam, k);
  if (host_info) throw std::runtime_error("block Davidson metric decomposition failed");
  const double smallest = *std::min_element(eig.begin(), eig.end());
  const double largest = *std::max_element(eig.begin(), eig.end());
  if (smallest < -1e-10) throw std::runtime_error("block Davidson encountered non-positive overlap");
  if (!(largest > 0) || smallest < 1e-10 * largest) {
    ++stats_.block_rank_fallbacks;
    copy_block(original, n_, vectors, n_, n_, k, st);
    return serial();
  }
  scale_columns(herm, k, k, k, lam, true, st);  // U diag(1/sqrt(lambda))
  gemm(Op::N, n_, k, k, vectors, n_, herm, k, v_ + static_cast<long long>(size_) * n_, n_, false, 1.0, exact);
  gemm(Op::N, n_, k, k, metric, n_, herm, k, sv_ + static_cast<long long>(size_) * n_, n_, false, 1.0, exact);
  if (searching()) pack_basis(size_, k);
  size_ += k;
  return true;
}

// Galerkin slabs for the new columns (src/pw_core.cpp:771-785).
void DavidsonSolver::update_projected(const Cx<double>* applied, Cx<double>* cached,
                                      const std::uint16_t* packed_applied) {
  const int first = incremental_ ? projected_size_ : 0;
  if (first == size_) return;
  const int columns = size_ - first;
  if (searching()) {
    // V^H (A new columns) and V_new^H (A old columns) from the packed copies.
    auto& ctx = op_.context();
    const long long kexp = expanded_k(n_, split_);
    umma_complex_gemm(static_cast<std::uint16_t*>(pack_vc_.ptr), ld_rows_, packed_applied + 2LL * first * ld_rows_,
                      ld_rows_, size_, columns, kexp, cached + static_cast<long long>(first) * capacity_, capacity_,
                      false, 1.0, ctx.tc.partial, ctx.stream);
    if (first)
      umma_complex_gemm(static_cast<std::uint16_t*>(pack_vc_.ptr) + first * ld_rows_, ld_rows_, packed_applied,
                        ld_rows_, columns, first, kexp, cached + first, capacity_, false, 1.0, ctx.tc.partial,
                        ctx.stream);
    return;
  }
  gemm(Op::C, size_, columns, n_, v_, n_, applied + static_cast<long long>(first) * n_, n_,
       cached + static_cast<long long>(first) * capacity_, capacity_, false, 1.0, exact_mode_);
  if (first)
    gemm(Op::C, columns, first, n_, v_ + static_cast<long long>(first) * n_, n_, applied, n_, cached + first,
         capacity_, false, 1.0, exact_mode_);
}

// Generalized Hermitian eigensolve of the projected pencil in FP64 on the
// device (the reference calls LAPACK zhegvd, src/pw_core.cpp:104-121).
void DavidsonSolver::rayleigh_ritz() {
  auto& ctx = op_.context();
  const cudaStream_t st = ctx.stream;
  // Traced runs drain the queue first so that the time is the Rayleigh-Ritz step's alone.
  static const bool trace = std::getenv("SDFT_B200_TRACE") != nullptr;
  if (trace) SDFT_CUDA(cudaStreamSynchronize(st));
  // Device time of the step, from events on the solver's stream (a host clock
  // would also count the work still queued ahead of it).
  if (!rr_events_[0]) {
    SDFT_CUDA(cudaEventCreate(&rr_events_[0]));
    SDFT_CUDA(cudaEventCreate(&rr_events_[1]));
  }
  SDFT_CUDA(cudaEventRecord(rr_events_[0], st));
  const int m = size_;
  auto* a = as<Cx<double>>(rr_a_, static_cast<std::size_t>(capacity_) * capacity_);
  auto* b = as<Cx<double>>(rr_b_, static_cast<std::size_t>(capacity_) * capacity_);
  hermitian_part(ch_, capacity_, a, m, m, st);
  hermitian_part(cs_, capacity_, b, m, m, st);
  // Only the lowest min(m, 2 roots) Ritz pairs are ever used (rotation and thick restart).
  // The search's projections carry FP32-accumulated products, so its pencil
  // drifts from S-orthonormal over a restart cycle (|E| up to ~1.3e-3 on
  // Si64); its Ritz pairs need no more than the first-order reduction's
  // O(|E|^2) <= 1e-8 below 1e-4 and the second-order O(|E|^3) <= 6e-8 up to
  // 4e-3. The FP64 phase stays tight.
  generalized_lowest(ctx.blas, ctx.solver, a, b, m, std::min(m, 2 * roots_), w_, a, eigen_, rr_mode(), st,
                     exact_mode_ ? 5e-5 : 4e-3, exact_mode_ ? 1e-8 : 1e-4);
  SDFT_CUDA(cudaEventRecord(rr_events_[1], st));
  values_ = download(w_, std::min(m, roots_));
  ++stats_.rayleigh_ritz;
  float ms = 0.0f;
  SDFT_CUDA(cudaEventElapsedTime(&ms, rr_events_[0], rr_events_[1]));
  stats_.rr_seconds += 1e-3 * ms;
}

DavidsonSolver::~DavidsonSolver() {
  for (cudaEvent_t& e : rr_events_)
    if (e) cudaEventDestroy(e);
}

// Fresh FP64 certificate of the Ritz block (src/pw_core.cpp:1125-1149).
void DavidsonSolver::certify() {
  const cudaStream_t st = op_.context().stream;
  ++stats_.certifications;
  apply_s(x_, roots_, sx_, true);
  metric_norms(x_, sx_, n_, n_, roots_, dsmall_, st);
  const auto metric = download(dsmall_, roots_);
  for (double m : metric)
    if (!std::isfinite(m) || !(m > 0)) throw std::runtime_error("invalid Davidson Ritz S norm");
  scale_columns(x_, n_, n_, roots_, dsmall_, true, st);
  apply_pair(x_, roots_, hx_, sx_, true);
  double* values = dsmall_ + roots_;
  double* metrics = dsmall_ + 2 * roots_;
  double* norms = dsmall_ + 3 * roots_;
  rayleigh_certificate(x_, hx_, sx_, n_, n_, roots_, values, metrics, r_, norms, st);
  values_ = download(values, roots_);
  residual_norms_ = download(norms, roots_);
  SDFT_CUDA(cudaMemcpyAsync(w_, values, sizeof(double) * roots_, cudaMemcpyDeviceToDevice, st));
}

double DavidsonSolver::max_residual() const {
  return residual_norms_.empty() ? 0.0 : *std::max_element(residual_norms_.begin(), residual_norms_.end());
}

// Normalises `trial` in the S metric with a fresh FP64 pair, re-applies the
// pair to the normalised block, certifies it, and keeps it in place of X only
// when it is S-orthonormal within 1e-12 (and S-orthogonal to completed bands)
// and its fresh maximum residual meets the tolerance or is below 0.999 of
// old_max (src/strict_residual_polish.hpp:97-115, 169-195).
bool DavidsonSolver::commit_trial(Cx<double>* trial, Cx<double>* th, Cx<double>* ts, Cx<double>* errors,
                                  double old_max) {
  auto& ctx = op_.context();
  const cudaStream_t st = ctx.stream;
  apply_pair(trial, roots_, th, ts, true);
  metric_norms(trial, ts, n_, n_, roots_, dsmall_, st);
  for (double m : download(dsmall_, roots_))
    if (!std::isfinite(m) || !(m > 0)) return false;
  scale_columns(trial, n_, n_, roots_, dsmall_, true, st);
  apply_pair(trial, roots_, th, ts, true);
  double* values = dsmall_ + roots_;
  double* metrics = dsmall_ + 2 * roots_;
  double* norms = dsmall_ + 3 * roots_;
  rayleigh_certificate(trial, th, ts, n_, n_, roots_, values, metrics, errors, norms, st);
  const auto energies = download(values, roots_);
  const auto fresh = download(norms, roots_);
  double new_max = 0.0;
  for (std::size_t i = 0; i < fresh.size(); ++i) {
    if (!std::isfinite(fresh[i]) || !std::isfinite(energies[i])) return false;
    new_max = std::max(new_max, fresh[i]);
  }
  Cx<double>* gram = as<Cx<double>>(gram_, static_cast<std::size_t>(kmax_) * kmax_ * 4);
  zgemm(ctx.blas, Op::C, Op::N, roots_, roots_, n_, trial, n_, ts, n_, gram, roots_, false);
  const double deviation = identity_deviation(gram, roots_, eigen_, st);
  if (!std::isfinite(deviation) || deviation > 1e-12) return false;
  if (excluded_count_) {
    std::vector<Cx<double>> overlap(static_cast<std::size_t>(excluded_count_) * roots_);
    zgemm(ctx.blas, Op::C, Op::N, excluded_count_, roots_, n_, excluded_s_, n_, trial, n_, gram, excluded_count_,
          false);
    SDFT_CUDA(cudaMemcpyAsync(overlap.data(), gram, sizeof(Cx<double>) * overlap.size(), cudaMemcpyDeviceToHost, st));
    ctx.synchronize();
    for (const auto& v : overlap)
      if (!(std::hypot(v.re, v.im) <= 1e-12)) return false;
  }
  if (!(new_max <= tolerance_ || new_max < 0.999 * old_max)) return false;
  const std::size_t block = static_cast<std::size_t>(n_) * roots_;
  SDFT_CUDA(cudaMemcpyAsync(x_, trial, sizeof(Cx<double>) * block, cudaMemcpyDeviceToDevice, st));
  SDFT_CUDA(cudaMemcpyAsync(sx_, ts, sizeof(Cx<double>) * block, cudaMemcpyDeviceToDevice, st));
  SDFT_CUDA(cudaMemcpyAsync(hx_, th, sizeof(Cx<double>) * block, cudaMemcpyDeviceToDevice, st));
  SDFT_CUDA(cudaMemcpyAsync(r_, errors, sizeof(Cx<double>) * block, cudaMemcpyDeviceToDevice, st));
  SDFT_CUDA(cudaMemcpyAsync(w_, values, sizeof(double) * roots_, cudaMemcpyDeviceToDevice, st));
  values_ = energies;
  residual_norms_ = fresh;
  return true;
}

// src/strict_residual_polish.hpp:70-116: the generalized Ritz problem of the
// original pair inside span(X) (compensated inner products), solved by the
// device Rayleigh-Ritz; it repairs rotations among the requested roots that a
// tangent step, orthogonal to all of them, cannot.
bool DavidsonSolver::root_manifold_step() {
  const double old_max = max_residual();
  if (old_max <= tolerance_) return false;
  ++stats_.manifold_steps;
  auto& ctx = op_.context();
  const cudaStream_t st = ctx.stream;
  const std::size_t block = static_cast<std::size_t>(n_) * roots_;
  Cx<double>* base = as<Cx<double>>(b_.polish, 6 * block);
  Cx<double>* trial = base;
  Cx<double>* th = base + block;
  Cx<double>* ts = base + 2 * block;
  Cx<double>* hx = base + 3 * block;
  Cx<double>* sx = base + 4 * block;
  apply_pair(x_, roots_, hx, sx, true);
  const std::size_t rr = static_cast<std::size_t>(roots_) * roots_;
  Cx<double>* small = as<Cx<double>>(b_.polish_small, 4 * rr);
  compensated_inner_matrix(x_, hx, n_, n_, roots_, roots_, small, roots_, st);
  compensated_inner_matrix(x_, sx, n_, n_, roots_, roots_, small + rr, roots_, st);
  hermitian_part(small, roots_, small + 2 * rr, roots_, roots_, st);
  hermitian_part(small + rr, roots_, small + 3 * rr, roots_, roots_, st);
  double* values = as<double>(b_.polish_values, roots_);
  generalized_lowest(ctx.blas, ctx.solver, small + 2 * rr, small + 3 * rr, roots_, roots_, values, small + 2 * rr,
                     eigen_, rr_mode(), st);
  zgemm(ctx.blas, Op::N, Op::N, n_, roots_, roots_, x_, n_, small + 2 * rr, roots_, trial, n_, false);
  const bool accepted = commit_trial(trial, th, ts, hx, old_max);
  if (accepted) ++stats_.manifold_accepted;
  return accepted;
}

// src/strict_residual_polish.hpp:118-197: per root, the step alpha = -g/c
// along the preconditioned residual d (S-orthogonalised twice against the
// completed bands and X), g = Re<d, r>, c = Re<d, H d> - e Re<d, S d>, taken
// only when alpha > 0 and alpha |d| <= 1e-4, with x + alpha d formed by fma.
bool DavidsonSolver::tangent_polish_step() {
  const double old_max = max_residual();
  if (old_max <= tolerance_) return false;
  ++stats_.polish_steps;
  auto& ctx = op_.context();
  const cudaStream_t st = ctx.stream;
  const std::size_t block = static_cast<std::size_t>(n_) * roots_;
  Cx<double>* base = as<Cx<double>>(b_.polish, 6 * block);
  Cx<double>* trial = base;
  Cx<double>* th = base + block;
  Cx<double>* ts = base + 2 * block;
  Cx<double>* d = base + 3 * block;
  Cx<double>* dh = base + 4 * block;
  Cx<double>* ds = base + 5 * block;
  kinetic_precondition(r_, x_, n_, n_, roots_, op_.device_kinetic(), d, n_, st);  // -P r
  Cx<double>* coef = as<Cx<double>>(b_.polish_small, 4 * static_cast<std::size_t>(roots_) * roots_);
  for (int pass = 0; pass < 2; ++pass) {
    if (excluded_count_) remove_excluded(d, roots_);
    zgemm(ctx.blas, Op::C, Op::N, roots_, roots_, n_, sx_, n_, d, n_, coef, roots_, false);
    zgemm(ctx.blas, Op::N, Op::N, n_, roots_, roots_, x_, n_, coef, roots_, d, n_, true, -1.0);
  }
  apply_pair(d, roots_, dh, ds, true);
  metric_norms(d, r_, n_, n_, roots_, dsmall_, st);
  metric_norms(d, dh, n_, n_, roots_, dsmall_ + roots_, st);
  metric_norms(d, ds, n_, n_, roots_, dsmall_ + 2 * roots_, st);
  column_norms(d, n_, n_, roots_, dsmall_ + 3 * roots_, st);
  const auto scalars = download(dsmall_, 4 * roots_);
  std::vector<double> alpha(roots_, 0.0);
  bool moved = false;
  for (int root = 0; root < roots_; ++root) {
    if (residual_norms_[root] <= 0.5 * tolerance_) continue;
    const double gradient = scalars[root];
    const double curvature = scalars[roots_ + root] - values_[root] * scalars[2 * roots_ + root];
    if (!(curvature > 0.0) || !std::isfinite(curvature) || !std::isfinite(gradient)) continue;
    const double a = -gradient / curvature;
    if (!(a > 0.0) || !std::isfinite(a) || a * scalars[3 * roots_ + root] > 1e-4) continue;
    alpha[root] = a;
    moved = true;
  }
  if (!moved) return false;
  double* dalpha = as<double>(b_.polish_values, roots_);
  SDFT_CUDA(cudaMemcpyAsync(dalpha, alpha.data(), sizeof(double) * roots_, cudaMemcpyHostToDevice, st));
  fma_columns(dalpha, d, x_, n_, n_, roots_, trial, st);
  const bool accepted = commit_trial(trial, th, ts, d, old_max);
  if (accepted) ++stats_.polish_accepted;
  return accepted;
}

void DavidsonSolver::preserve_search_subspace() {
  auto& ctx = op_.context();
  const cudaStream_t st = ctx.stream;
  const bool at_capacity = size_ + roots_ > capacity_;
  const int keep = at_capacity ? std::min(size_, 2 * roots_) : size_;
  Cx<double>* retained = hv_;  // the images are recomputed for the new basis
  copy_block(x_, n_, retained, n_, n_, roots_, st);
  if (keep > roots_) {
    Cx<double>* rest = retained + static_cast<long long>(roots_) * n_;
    if (at_capacity) {
      const Cx<double>* rotation = static_cast<const Cx<double>*>(rr_a_.ptr);
      gemm(Op::N, n_, keep - roots_, size_, v_, n_, rotation + static_cast<long long>(roots_) * size_, size_, rest,
           n_, false, 1.0, true);
    } else {
      // Complement of X in the basis: V Q2, Q2 the columns of the full Q of
      // the QR factorisation of V^H S X beyond the first roots.
      auto* q = as<Cx<double>>(rr_b_, static_cast<std::size_t>(size_) * size_);
      gemm(Op::C, size_, roots_, n_, v_, n_, sx_, n_, q, size_, false, 1.0, true);
      auto* tau = as<cuDoubleComplex>(small_, static_cast<std::size_t>(std::max(kmax_, roots_)) * 2);
      int lwork = 0, lwork2 = 0;
      auto* qz = reinterpret_cast<cuDoubleComplex*>(q);
      check_solver(cusolverDnZgeqrf_bufferSize(ctx.solver, size_, roots_, qz, size_, &lwork), "zgeqrf_bufferSize");
      check_solver(cusolverDnZungqr_bufferSize(ctx.solver, size_, size_, roots_, qz, size_, tau, &lwork2),
                   "zungqr_bufferSize");
      const int work_size = std::max({1, lwork, lwork2});
      auto* work = as<cuDoubleComplex>(rr_work_, static_cast<std::size_t>(work_size));
      int* info = as<int>(info_, 4);
      check_solver(cusolverDnZgeqrf(ctx.solver, size_, roots_, qz, size_, tau, work, work_size, info), "zgeqrf");
      check_solver(cusolverDnZungqr(ctx.solver, size_, size_, roots_, qz, size_, tau, work, work_size, info),
                   "zungqr");
      int host_info = 0;
      SDFT_CUDA(cudaMemcpyAsync(&host_info, info, sizeof(int), cudaMemcpyDeviceToHost, st));
      ctx.synchronize();
      if (host_info) throw std::runtime_error("corrected Davidson search subspace factorisation failed");
      gemm(Op::N, n_, size_ - roots_, size_, v_, n_, q + static_cast<long long>(roots_) * size_, size_, rest, n_,
           false, 1.0, true);
    }
  }
  size_ = computed_h_ = projected_size_ = 0;
  for (int first = 0; first < keep; first += kmax_)
    append_block(retained + static_cast<long long>(first) * n_, std::min(kmax_, keep - first));
}

void DavidsonSolver::refresh_images() {
  apply_pair(v_, size_, hv_, sv_, true);
  computed_h_ = size_;
  projected_size_ = 0;
}

void DavidsonSolver::solve(const DavidsonOptions& o, const Cx<double>* initial) {
  auto& ctx = op_.context();
  SDFT_CUDA(cudaSetDevice(ctx.device));
  const cudaStream_t st = ctx.stream;
  const double start = now();
  const bool trace = std::getenv("SDFT_B200_TRACE") != nullptr;
  stats_ = DavidsonStats{};
  n_ = op_.npw();
  roots_ = o.roots;
  if (roots_ < 1 || roots_ > n_ || o.max_iterations < 1 || !std::isfinite(o.tolerance) || o.tolerance <= 0)
    throw InvalidArgument("invalid matrix-free Davidson problem");
  if (o.subspace_factor < 4 || o.subspace_factor > 16)
    throw InvalidArgument("SDFT_DAVIDSON_SUBSPACE_FACTOR must be in [4,16]");
  for (std::size_t i = 0; i < op_.s_diagonal().size(); ++i)
    if (!std::isfinite(op_.h_diagonal()[i]) || !std::isfinite(op_.s_diagonal()[i]) || op_.s_diagonal()[i] <= 0)
      throw InvalidArgument("invalid Davidson operator diagonal");
  tolerance_ = o.tolerance;
  capacity_ = o.capacity > 0 ? std::min(n_, o.capacity) : std::min(n_, std::max(o.subspace_factor * roots_, 64));
  if (o.excluded_count < 0 || (o.excluded_count && !o.excluded) || o.excluded_count + roots_ > n_ ||
      capacity_ < roots_)
    throw InvalidArgument("invalid matrix-free Davidson problem");
  const bool warm = initial != nullptr && 2 * roots_ < n_;
  const int guard_count = std::min(n_, 2 * roots_);
  kmax_ = std::min(capacity_, std::max(3 * roots_, 2));
  exact_mode_ = o.precision == Precision::FP64;
  packs_ = !exact_mode_;
  if (o.correction_steps < 0 || (exact_mode_ && o.correction_steps > 0))
    throw InvalidArgument("Jacobi-Davidson correction steps apply to the mixed form only");
  correction_steps_ = exact_mode_ ? 0 : o.correction_steps;
  if (packs_) {
    split_ = search_split();
    ld_rows_ = expanded_k(n_, split_);
    ld_cols_ = expanded_k(capacity_, split_);
  }
  incremental_ = o.tolerance >= 1e-12;
  strict_projection_ = false;
  // The reference's strict-refinement switches (src/pw_core.cpp:611-612),
  // off for band-group local solves with an explicit capacity (:1273).
  polish_enabled_ = boolean_control("SDFT_FRESH_RESIDUAL_POLISH", true) && o.capacity <= 0;
  manifold_enabled_ = boolean_control("SDFT_STRICT_ROOT_MANIFOLD", true);
  polish_attempts_ = manifold_attempts_ = 0;
  strict_entry_ = std::numeric_limits<double>::infinity();
  size_ = computed_h_ = projected_size_ = 0;
  residual_history_.clear();
  const std::size_t nc = static_cast<std::size_t>(n_) * capacity_;
  v_ = as<Cx<double>>(basis_, nc);
  hv_ = as<Cx<double>>(hbasis_, nc);
  sv_ = as<Cx<double>>(sbasis_, nc);
  ch_ = as<Cx<double>>(cached_h_, static_cast<std::size_t>(capacity_) * capacity_);
  cs_ = as<Cx<double>>(cached_s_, static_cast<std::size_t>(capacity_) * capacity_);
  w_ = as<double>(rr_w_, capacity_);
  x_ = as<Cx<double>>(xs_, static_cast<std::size_t>(n_) * roots_);
  sx_ = as<Cx<double>>(sxs_, static_cast<std::size_t>(n_) * roots_);
  hx_ = as<Cx<double>>(hxs_, static_cast<std::size_t>(n_) * roots_);
  r_ = as<Cx<double>>(res_, static_cast<std::size_t>(n_) * roots_);
  dsmall_ = as<double>(order_, static_cast<std::size_t>(std::max(capacity_, 4 * roots_)) * 4);
  Cx<double>* block = as<Cx<double>>(block_, static_cast<std::size_t>(n_) * kmax_);
  if (packs_) {
    const std::size_t rows_bytes = sizeof(std::uint16_t) * static_cast<std::size_t>(ld_rows_) * capacity_;
    const std::size_t cols_bytes = sizeof(std::uint16_t) * static_cast<std::size_t>(ld_cols_) * n_;
    pack_vc_.reserve(rows_bytes);
    pack_hb_.reserve(2 * rows_bytes);
    pack_sb_.reserve(2 * rows_bytes);
    // The left factors are read over whole 64-wide K blocks; the entries past
    // the current size meet zero padding on the other side and must be finite.
    for (Scratch* s : {&pack_vn_, &pack_hn_, &pack_sn_}) SDFT_CUDA(cudaMemsetAsync(s->reserve(cols_bytes), 0, cols_bytes, st));
  }
  int* dselect = as<int>(select_, static_cast<std::size_t>(std::max(n_, roots_)));
  // Completed bands of a band-group local solve: their S images (FP64) and
  // the S-orthonormality the reference requires (src/pw_core.cpp:675-700).
  excluded_count_ = o.excluded_count;
  excluded_ = o.excluded;
  if (excluded_count_) {
    const std::size_t ne = static_cast<std::size_t>(n_) * excluded_count_;
    excluded_s_ = as<Cx<double>>(b_.excluded, ne + static_cast<std::size_t>(excluded_count_) *
                                                       std::max(excluded_count_, kmax_));
    op_.apply_overlap(excluded_, excluded_count_, excluded_s_, Precision::FP64);
    Cx<double>* gram = excluded_s_ + ne;
    zgemm(ctx.blas, Op::C, Op::N, excluded_count_, excluded_count_, n_, excluded_, n_, excluded_s_, n_, gram,
          excluded_count_, false);
    if (identity_deviation(gram, excluded_count_, eigen_, st) > 1e-10)
      throw InvalidArgument("completed bands must be S orthonormal");
  }

  // Seeds (src/pw_core.cpp:1016-1112): warm vectors (perturbed) + 2*roots
  // canonical guards on the lowest H/S diagonal ratios, each with full support.
  std::vector<int> order(n_);
  std::iota(order.begin(), order.end(), 0);
  const auto& hd = op_.h_diagonal();
  const auto& sd = op_.s_diagonal();
  std::stable_sort(order.begin(), order.end(), [&](int i, int j) { return hd[i] / sd[i] < hd[j] / sd[j]; });
  int seeds = 0;
  unsigned long long draw = 0;
  if (warm) {
    copy_block(initial, n_, block, n_, n_, roots_, st);
    seeds = roots_;
  }
  {
    const int guards = std::min(guard_count, kmax_ - seeds);
    SDFT_CUDA(cudaMemcpyAsync(dselect, order.data(), sizeof(int) * guards, cudaMemcpyHostToDevice, st));
    broad_seed_block(n_, guards, draw, dselect, block + static_cast<long long>(seeds) * n_, n_, st);
    draw += 2ULL * n_ * guards;
    seeds += guards;
  }
  append_block(block, seeds);

  values_.assign(roots_, 0.0);
  residual_norms_.assign(roots_, 0.0);
  bool certified = false;
  int iteration = 0;
  // SDFT_B200_TRACE: per-iteration phase times (the stream is drained at each mark).
  std::string phases;
  double phase_start = now();
  auto phase = [&](const char* name) {
    if (!trace) return;
    SDFT_CUDA(cudaStreamSynchronize(st));
    const double t = now();
    char item[64];
    std::snprintf(item, sizeof(item), " %s=%.2f", name, 1e3 * (t - phase_start));
    phases += item;
    phase_start = t;
  };
  for (; iteration < o.max_iterations; ++iteration) {
    if (trace && !phases.empty()) {
      std::fprintf(stderr, "sdft_b200 davidson phases ms:%s\n", phases.c_str());
      phases.clear();
    }
    phase("tail");
    // flush_h (src/pw_core.cpp:786-795)
    if (computed_h_ < size_) {
      apply_h(v_ + static_cast<long long>(computed_h_) * n_, size_ - computed_h_,
              hv_ + static_cast<long long>(computed_h_) * n_, exact_mode_);
      if (searching()) pack_images(computed_h_, size_ - computed_h_);
      computed_h_ = size_;
    }
    phase("apply_h");
    update_projected(hv_, ch_, static_cast<std::uint16_t*>(pack_hb_.ptr));
    update_projected(sv_, cs_, static_cast<std::uint16_t*>(pack_sb_.ptr));
    projected_size_ = size_;
    phase("projections");
    rayleigh_ritz();
    phase("rayleigh_ritz");
    const Cx<double>* rotation = static_cast<const Cx<double>*>(rr_a_.ptr);  // size x size, ld size
    // Ritz block, its S image and search residual (src/pw_core.cpp:1178-1181)
    if (searching()) {
      gemm_left(static_cast<std::uint16_t*>(pack_vn_.ptr), roots_, size_, rotation, size_, x_, n_, false, 1.0);
      gemm_left(static_cast<std::uint16_t*>(pack_sn_.ptr), roots_, size_, rotation, size_, sx_, n_, false, 1.0);
      gemm_left(static_cast<std::uint16_t*>(pack_hn_.ptr), roots_, size_, rotation, size_, r_, n_, false, 1.0);
    } else {
      gemm(Op::N, n_, roots_, size_, v_, n_, rotation, size_, x_, n_, false, 1.0, exact_mode_);
      gemm(Op::N, n_, roots_, size_, sv_, n_, rotation, size_, sx_, n_, false, 1.0, exact_mode_);
      gemm(Op::N, n_, roots_, size_, hv_, n_, rotation, size_, r_, n_, false, 1.0, exact_mode_);
    }
    search_residual(r_, sx_, n_, n_, roots_, w_, r_, st);
    column_norms(r_, n_, n_, roots_, dsmall_, st);
    residual_norms_ = download(dsmall_, roots_);
    phase("ritz_residual");
    stats_.iterations = iteration + 1;
    double max_res = *std::max_element(residual_norms_.begin(), residual_norms_.end());
    bool converged = std::all_of(residual_norms_.begin(), residual_norms_.end(),
                                 [&](double r) { return r <= tolerance_; });
    residual_history_.push_back(max_res);
    if (trace)
      std::fprintf(stderr, "sdft_b200 davidson iteration=%d size=%d mode=%s max_search_residual=%.3e t=%.1fms rr=%.1fms\n",
                   iteration, size_, exact_mode_ ? "fp64" : "mixed", max_res, 1e3 * (now() - start),
                   1e3 * stats_.rr_seconds);
    // Approximate search hands over to FP64 (src/pw_core.cpp:1184-1196). FP32
    // arithmetic cannot reach 1e-8, so a stalled search hands over as well.
    if (!exact_mode_) {
      bool stalled = false;
      const std::size_t h = residual_history_.size();
      if (h >= 6 && max_res < 1e-3) {
        const double recent = std::min({residual_history_[h - 1], residual_history_[h - 2], residual_history_[h - 3]});
        const double earlier = *std::min_element(residual_history_.begin(), residual_history_.end() - 3);
        stalled = recent > 0.5 * earlier;
      }
      if (max_res < o.handoff || stalled || iteration + 1 == o.max_iterations) {
        // The Jacobi-Davidson-steered form hands over its 2*roots lowest Ritz
        // vectors only (they carry the search), so the FP64 re-application
        // covers that block rather than the whole basis.
        const bool compact = correction_steps_ > 0 && size_ > 2 * roots_;
        if (compact) gemm_left(static_cast<std::uint16_t*>(pack_vn_.ptr), 2 * roots_, size_, rotation, size_, block,
                               n_, false, 1.0);
        exact_mode_ = true;
        ++stats_.fp64_refreshes;
        stats_.handoff_iteration = iteration;
        if (compact) {
          size_ = computed_h_ = projected_size_ = 0;
          ++stats_.restarts;
          append_block(block, 2 * roots_);
        }
        refresh_images();
        continue;
      }
    }
    bool fresh = false;
    if (exact_mode_ && max_res <= 8 * tolerance_) {
      certify();
      fresh = true;
      converged = std::all_of(residual_norms_.begin(), residual_norms_.end(), [&](double r) { return r <= tolerance_; });
      max_res = *std::max_element(residual_norms_.begin(), residual_norms_.end());
    }
    if (converged && !fresh) {
      certify();
      fresh = true;
      converged = std::all_of(residual_norms_.begin(), residual_norms_.end(), [&](double r) { return r <= tolerance_; });
      max_res = *std::max_element(residual_norms_.begin(), residual_norms_.end());
      if (!converged && !exact_mode_) {
        exact_mode_ = true;
        ++stats_.fp64_refreshes;
        refresh_images();
        continue;
      }
    }
    // Rebuild the whole projected pencil at the FP64 floor (src/pw_core.cpp:1247-1267).
    if (exact_mode_ && !converged && tolerance_ <= 1e-12 && !strict_projection_ && max_res <= 1e-10) {
      if (!fresh) {
        certify();
        fresh = true;
        converged = std::all_of(residual_norms_.begin(), residual_norms_.end(), [&](double r) { return r <= tolerance_; });
      }
      if (!converged) {
        refresh_images();
        incremental_ = false;
        strict_projection_ = true;
        continue;
      }
    }
    // Strict FP64 refinements once Davidson stalls at the FP64 floor
    // (src/pw_core.cpp:1273-1336); every step counts against the iteration budget.
    // The Jacobi-Davidson-steered mixed form converges faster through its own
    // corrections than through tangent steps, so it refines only once two
    // successive FP64 iterations fail to halve the residual.
    bool strict_polished = false;
    const std::size_t hist = residual_history_.size();
    const bool fp64_stalled = hist >= 3 && residual_history_[hist - 1] > 0.5 * residual_history_[hist - 2] &&
                              residual_history_[hist - 2] > 0.5 * residual_history_[hist - 3];
    if (polish_enabled_ && exact_mode_ && !converged && tolerance_ <= 1e-12 && max_res <= 1e-10 &&
        (correction_steps_ == 0 || fp64_stalled) && max_res < 0.5 * strict_entry_ &&
        (polish_attempts_ < 16 || (manifold_enabled_ && manifold_attempts_ < 4))) {
      auto all_converged = [&]() {
        return std::all_of(residual_norms_.begin(), residual_norms_.end(), [&](double r) { return r <= tolerance_; });
      };
      if (!fresh) {
        certify();
        fresh = true;
        converged = all_converged();
      }
      strict_entry_ = max_residual();
      if (manifold_enabled_ && !converged && manifold_attempts_ < 4 && iteration + 1 < o.max_iterations) {
        ++manifold_attempts_;
        ++iteration;
        stats_.iterations = iteration + 1;
        strict_polished |= root_manifold_step();
        converged = all_converged();
      }
      for (; !converged && polish_attempts_ < 16 && iteration + 1 < o.max_iterations; ++polish_attempts_) {
        ++iteration;
        stats_.iterations = iteration + 1;
        const bool improved = tangent_polish_step();
        strict_polished |= improved;
        if (!improved) {
          ++polish_attempts_;
          break;
        }
        converged = all_converged();
      }
      max_res = max_residual();
      phase("strict_refinement");
    }
    if (converged) {
      certified = fresh;
      if (certified) break;
    }
    if (strict_polished && iteration + 1 < o.max_iterations) {
      preserve_search_subspace();
      phase("preserve");
    }
    // Thick restart (src/pw_core.cpp:1357-1383).
    if (size_ + roots_ > capacity_) {
      const int keep = std::min(size_, 2 * roots_);
      if (searching())
        gemm_left(static_cast<std::uint16_t*>(pack_vn_.ptr), keep, size_, rotation, size_, block, n_, false, 1.0);
      else
        gemm(Op::N, n_, keep, size_, v_, n_, rotation, size_, block, n_, false, 1.0, exact_mode_);
      size_ = computed_h_ = projected_size_ = 0;
      ++stats_.restarts;
      append_block(block, keep);
      phase("restart");
    }
    // Preconditioned corrections for unconverged roots (src/pw_core.cpp:1384-1401).
    const int previous = size_;
    std::vector<int> selected;
    for (int r = 0; r < roots_ && size_ + static_cast<int>(selected.size()) < capacity_; ++r)
      if (residual_norms_[r] > 0.5 * tolerance_) selected.push_back(r);
    if (!selected.empty()) {
      const int count = static_cast<int>(selected.size());
      if (correction_steps_ > 0) {
        jacobi_davidson_corrections(op_, b_.corrections, x_, sx_, r_, w_, roots_, selected.data(), count,
                                    correction_steps_, block);
        stats_.correction_columns += static_cast<long long>(count) * correction_steps_;
        stats_.h_columns_search += static_cast<long long>(count) * correction_steps_;
        stats_.s_columns_search += static_cast<long long>(count) * correction_steps_;
      } else {
        Cx<double>* corrections = static_cast<Cx<double>*>(res_.ptr);  // precondition in place into r_
        kinetic_precondition(r_, x_, n_, n_, roots_, op_.device_kinetic(), corrections, n_, st);
        SDFT_CUDA(cudaMemcpyAsync(dselect, selected.data(), sizeof(int) * selected.size(), cudaMemcpyHostToDevice, st));
        gather_columns(corrections, n_, n_, dselect, count, block, n_, st);
      }
      phase("corrections");
      append_block(block, count);
      phase("append");
    }
    if (size_ == previous) {
      bool added = false;
      for (int j = 0; j < n_ && !added; ++j) {
        zero_block(block, n_, n_, 1, st);
        const Cx<double> one{1.0, 0.0};
        SDFT_CUDA(cudaMemcpyAsync(block + order[j], &one, sizeof(one), cudaMemcpyHostToDevice, st));
        added = append_single(block);
      }
      if (!added) break;
    }
  }
  if (!certified) certify();
  stats_.converged = std::all_of(residual_norms_.begin(), residual_norms_.end(), [&](double r) { return r <= tolerance_; });
  stats_.max_residual = *std::max_element(residual_norms_.begin(), residual_norms_.end());
  ctx.synchronize();
  stats_.seconds = now() - start;
}

}  // namespace sdft_b200
