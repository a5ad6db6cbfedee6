// Device-resident plane-wave PAW operator and its execution context.
#pragma once
#include <cublas_v2.h>
#include <cusolverDn.h>

#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "eigensolver.cuh"
#include "gemm.cuh"
#include "local_hamiltonian.cuh"
#include "umma_gemm.cuh"

namespace sdft_b200 {

enum class Precision : int { FP64 = 0, Mixed = 1 };

// Device copies kept across Accelerator-style calls, keyed by the caller's
// immutable identity tokens (src/compute_backend.hpp:32-41).
struct AcceleratorCache {
  std::uint64_t local_identity = 0;
  int shape[3] = {0, 0, 0};
  SpherePlan plan;
  Scratch v64, v32, kinetic;
  std::uint64_t projector_identity = 0, onsite_identity = 0;
  int npw = 0, projectors = 0;
  Scratch b, d, q;
  PackedA b_packed, bh_packed;
  ~AcceleratorCache() {
    plan.release();
    release(b_packed);
    release(bh_packed);
  }
};

// Left operands the caller promises immutable for an identity token
// (src/compute_backend.hpp:32-41): the FP64 matrix and, once a mixed
// product needs it, its tensor-core packing stay on the device; dynamic
// right operands are uploaded anew on every call. Four entries, least
// recently used replaced.
struct ImmutableLeft {
  std::uint64_t identity = 0;
  int aop = 0;
  std::size_t rows = 0, cols = 0;  // stored A (rows x cols, leading dimension rows)
  Scratch fp64;
  PackedA packed;
  unsigned long long used = 0;
  ~ImmutableLeft() { release(packed); }
};
struct ImmutableCache {
  ImmutableLeft entries[4];
  unsigned long long clock = 0;
};

// Density-side device state: the sphere plan of the last band-density call
// (reused while the density grid and the plane-wave keys repeat) and its slabs.
struct DensityCache {
  int shape[3] = {0, 0, 0};
  std::vector<std::uint64_t> indices;
  SpherePlan plan;
  Scratch rows, planes, grid, meta;
  ~DensityCache() { plan.release(); }
};

// One CUDA stream with its library handles and grow-only scratch. A context is
// used by one host thread at a time (the reference keeps one Accelerator per
// host thread, src/compute_backend.cpp:62-73).
// Device state of a Davidson solve (basis and images, projected pencil,
// Rayleigh-Ritz and eigensolver workspace, correction blocks, packed search
// operands). Owned by the context, so solves of successive operators on one
// context reuse the allocations.
// Device state of the Jacobi-Davidson corrections (correction.cu).
struct CorrectionBuffers {
  Scratch res, z, p, hp;       // n x count blocks (the corrections themselves go to the caller's block)
  Scratch xh, sxh, xl, sxl;    // packed X^H, (SX)^H (rows) and X, SX (left factors)
  Scratch coefficients;        // roots x count projections
  Scratch scalars;             // per column: theta, kinetic energy, two (res, z) slots, (p, q)
  Scratch index;               // selected roots
};

struct DavidsonBuffers {
  Scratch basis, hbasis, sbasis, cached_h, cached_s, rr_a, rr_b, rr_w, rr_work, info;
  EigenWorkspace eigen;
  Scratch xs, sxs, hxs, res, block, metric, original, projections, gram, small, order, select;
  Scratch pack_vc, pack_vn, pack_hn, pack_sn, pack_hb, pack_sb;
  Scratch excluded;  // S images and projections of a band-group solve's completed bands
  CorrectionBuffers corrections;
  Scratch polish;         // strict refinements: direction, trial and their images (n x roots each)
  Scratch polish_small;   // their roots x roots matrices
  Scratch polish_values;  // their per-root scalars
};

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool owns_stream = false;
  cublasHandle_t blas = nullptr;
  cusolverDnHandle_t solver = nullptr;
  Scratch slab32, slab64, staging_in, staging_out, staging_aux, projections, onsite;
  TensorCoreWorkspace tc;
  AcceleratorCache accel;
  ImmutableCache immutable;
  DensityCache density;
  EigenWorkspace eigen;
  DavidsonBuffers davidson;
  explicit Context(int device, cudaStream_t stream);
  ~Context();
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  void synchronize() const;
  // The grow-only working buffers (slabs, staging, Davidson and eigensolver
  // state) and the identity-keyed caches; every one is stream-ordered pool
  // memory on this context's stream.
  std::vector<Scratch*> working_buffers();
  std::vector<Scratch*> cache_buffers();
  // Returns every working buffer to the library's pool, which keeps the
  // memory for the next allocation (no device-wide synchronisation).
  void recycle_scratch();
  // recycle_scratch, then hands the pool's unused memory back to the device.
  void release_scratch();
};

// Accelerator-style calls on caller host arrays (accelerator.cu).
void accelerator_local_hamiltonian(Context& ctx, const int shape[3], const std::uint64_t* indices, std::size_t npw,
                                   const double* kinetic, const double* potential, const double* input,
                                   std::size_t columns, double* output, Precision precision, std::uint64_t identity);
void accelerator_paw_pair(Context& ctx, std::uint64_t identity, std::size_t npw, std::size_t np,
                          std::size_t columns, const double* b, const double* d, const double* q, const double* input,
                          double* h, double* s, Precision precision, std::uint64_t projector_identity);

class DeviceOperator;
// Local part of H~ on device arrays with all scratch in a static device array
// (local_noalloc.cu); allocates nothing.
void apply_local_noalloc(DeviceOperator& op, const Cx<double>* x, int columns, Cx<double>* y, Precision precision);

// PBE per point on device arrays (pbe.cu): out holds 7 values per point.
void pbe_points(Context& ctx, const double* density, const double* gradient, std::size_t count, double* out);

struct GVectorList {
  std::vector<int> hkl;         // 3 per vector
  std::vector<double> cartesian;
  std::vector<double> kinetic_ev;
};

// Plane-wave sphere enumeration, same arithmetic/order as src/pw_core.cpp:140-171.
GVectorList enumerate_g_vectors(const double reciprocal[9], double cutoff_ev, const double kpoint[3],
                                double hartree_to_ev);

struct OperatorInput {
  std::size_t npw = 0;
  const int* hkl = nullptr;          // npw x 3
  const double* kinetic_ev = nullptr;
  std::size_t potential_count = 0;
  const int* potential_hkl = nullptr;  // x3
  const double* potential = nullptr;   // interleaved complex
  std::size_t atoms = 0;
  const std::uint64_t* projectors = nullptr;  // per atom
  const double* amplitudes = nullptr;  // per atom row-major np_a x npw, interleaved complex
  const double* d = nullptr;           // per atom row-major np_a x np_a
  const double* q = nullptr;
  double hartree_to_ev = 27.211386245988;
  double regularization = 1e-12;
};

// A solver snapshot in the reference's SDFTPWO3 format (per-atom D/Q
// blocks): the operator's internal arrays and the solve settings. Little-
// endian uint64 header; FP64 arrays; complex arrays interleaved, column-major.
struct OperatorSnapshot {
  int shape[3] = {0, 0, 0};
  std::size_t npw = 0, count = 0, projectors = 0, roots = 0, iterations = 0, initial_values = 0;
  double regularization = 0, tolerance = 0;
  std::vector<std::uint64_t> channels;  // projectors per atom
  std::vector<std::uint64_t> indices;   // wrapped row-major grid index per plane wave
  std::vector<double> kinetic, h_diagonal, s_diagonal, local_real;
  std::vector<Cx<double>> all_b;        // projectors x npw, column-major
  std::vector<Cx<double>> d, q;         // per atom channels^2, column-major, concatenated
  std::vector<Cx<double>> initial;      // roots x npw band-major warm vectors, or empty
};

// Reads and validates a snapshot (the reference's load_solver_snapshot
// checks: dimensions, exact file length, unique in-range indices, finite
// arrays, positive overlap diagonal, Hermitian blocks). header_only skips
// the arrays after the atom boundaries.
OperatorSnapshot read_operator_snapshot(const std::string& path, bool header_only = false);

// Signature of S~ from its nontrivial projector block, as the reference's
// overlap() determines it (src/plane_wave_operator.cpp:702-717): with
// R = (B B^H)^(1/2) (eigenvalues clamped at 0), S~ restricted to span(B^H)
// is similar to (1+reg) I + R Q R, and every other direction has the norm
// 1+reg.
struct MetricSignature {
  double minimum = 1.0;     // min(1+reg, lowest eigenvalue of (1+reg) I + R Q R)
  bool indefinite = false;  // minimum < -1e-10
  bool singular = false;    // |minimum| <= 1e-10
};

class DeviceOperator {
 public:
  DeviceOperator(Context& ctx, const OperatorInput& input);
  // From a solver snapshot's internal arrays (no rebuild from G components).
  DeviceOperator(Context& ctx, const OperatorSnapshot& snapshot);
  ~DeviceOperator();
  DeviceOperator(const DeviceOperator&) = delete;
  DeviceOperator& operator=(const DeviceOperator&) = delete;

  Context& context() const { return ctx_; }
  int npw() const { return npw_; }
  int projectors() const { return np_; }
  int atoms() const { return atoms_; }
  const SpherePlan& plan() const { return plan_; }
  double regularization() const { return regularization_; }
  const std::vector<double>& kinetic() const { return h_kinetic_; }
  const std::vector<double>& h_diagonal() const { return h_diag_; }
  const std::vector<double>& s_diagonal() const { return s_diag_; }
  const std::vector<std::uint64_t>& indices() const { return h_indices_; }
  const std::vector<double>& local_real() const { return h_local_real_; }
  const double* device_kinetic() const { return kinetic_; }
  const double* device_potential64() const { return v64_; }
  const float* device_potential32() const { return v32_; }

  // Device-pointer applies on ctx.stream; x, y are npw x columns (ld npw).
  void apply_hamiltonian(const Cx<double>* x, int columns, Cx<double>* y, Precision precision);
  void apply_overlap(const Cx<double>* x, int columns, Cx<double>* y, Precision precision);
  void apply_pair(const Cx<double>* x, int columns, Cx<double>* hy, Cx<double>* sy, Precision precision);
  // y(:, c) = (H~ - shift[c] S~) x(:, c), shift on the device: the local part,
  // minus shift (1+reg) x, plus B^H (D - shift Q) B x -- one projection and one
  // back-projection for both operators.
  void apply_shifted(const Cx<double>* x, int columns, const double* shift, Cx<double>* y, Precision precision);
  // Local part only: y = T x + V(r) term.
  void apply_local(const Cx<double>* x, int columns, Cx<double>* y, Precision precision) {
    local_part(x, columns, y, precision);
  }
  // P = B x (np x columns, ld np)
  void project(const Cx<double>* x, int columns, Cx<double>* p, Precision precision);
  // SCF refresh: replaces V(G) and the per-atom D/Q (the constructor's input
  // layouts) and recomputes V(r) and the diagonals; the basis maps, FFT plan,
  // B and its tensor-core packing stay resident. The result equals a new
  // operator built from the same basis, B and the new V(G), D, Q (the grid
  // depends on the basis extent alone: only keys inside it are retained).
  // Rejected (operator unchanged) when a check fails, when SDFT_FFT_GRID
  // changed so that the grid would differ, or for a snapshot operator.
  void update(std::size_t potential_count, const int* potential_hkl, const double* potential, const double* d,
              const double* q);

  std::size_t device_bytes() const;

  // FP64 on the device, computed at the first call and kept until update().
  const MetricSignature& metric_signature();
  // The checks a Davidson solve of this pencil makes first: a numerically
  // singular S~ is the reference's runtime_error; an indefinite one, which
  // the reference hands to its indefinite-pencil solver
  // (src/pw_core.cpp:556-557), throws Unsupported.
  void require_positive_metric();

 private:
  // Device arrays from the host state (plan, kinetic, V(r), D/Q blocks and
  // boundaries); B and the diagonals are the caller's.
  void upload_common(const int shape[3], const std::vector<Cx<double>>& d_blocks,
                     const std::vector<Cx<double>>& q_blocks, const std::vector<int>& offsets,
                     const std::vector<long long>& storage);
  void local_part(const Cx<double>* x, int columns, Cx<double>* y, Precision precision);
  void paw_add(const Cx<double>* p, int columns, bool overlap, Cx<double>* y, Precision precision);
  void backproject(const Cx<double>* dp, int columns, Cx<double>* y, Precision precision);

  Context& ctx_;
  int npw_ = 0, np_ = 0, atoms_ = 0, max_block_ = 0;
  double regularization_ = 0;
  SpherePlan plan_;
  std::vector<double> h_kinetic_, h_diag_, h_local_real_;
  std::vector<double> s_diag_;
  std::vector<std::uint64_t> h_indices_;
  std::vector<std::uint64_t> h_channels_;  // projectors per atom
  int span_[3] = {-1, -1, -1};             // basis extent high - low per axis; -1 for a snapshot operator
  double* kinetic_ = nullptr;
  double* v64_ = nullptr;
  float* v32_ = nullptr;
  Cx<double>* b_ = nullptr;      // np x npw column-major (ld np)
  PackedA b_packed_;             // B (np x npw) for P = B x on the tensor cores
  PackedA bh_packed_;            // B^H (npw x np) for y += B^H P
  Cx<double>* d_ = nullptr;      // per-atom column-major blocks
  Cx<double>* q_ = nullptr;
  int* block_offsets_ = nullptr;         // [atoms+1]
  long long* block_storage_ = nullptr;   // [atoms]
  MetricSignature signature_;
  bool signature_ready_ = false;
};

}  // namespace sdft_b200
