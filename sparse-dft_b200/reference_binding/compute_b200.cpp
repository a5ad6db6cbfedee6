// B200 accelerator for the Sparse-DFT compute backend.
//
// A maintainer compiles this file into the reference build in place of
// src/compute_cuda.cu: it defines make_cuda_accelerator()
// (src/compute_backend.hpp:91) and implements the Accelerator interface
// (src/compute_backend.hpp:64-89) by forwarding to libsdft_b200's C ABI, so
// SDFT_COMPUTE_BACKEND=cuda, SDFT_GPU_FFT=1 and SDFT_GPU_PAW_CHAIN=1 route the
// reference's exact=false work to the hand-written sm_100a kernels. Statuses
// map back to the reference's exception classes. The device-resident solver
// (sdft_b200_davidson) is reached through the same library.
//
// SDFT_B200_ACCELERATOR_PRECISION=fp64 (default, the arithmetic the
// reference's CUDA accelerator promises) or mixed (FP32 FFT, BF16-split
// tensor-core products) selects the search arithmetic; SDFT_B200_DEVICE
// selects the device (default 0).
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "b200_solver.hpp"
#include "compute_backend.hpp"
#include "sdft_b200.h"

namespace sdft {
namespace {

void check(sdft_b200_status status) { b200::throw_on_error(status); }

int search_precision() {
  const char* value = std::getenv("SDFT_B200_ACCELERATOR_PRECISION");
  if (!value || std::string(value) == "fp64") return SDFT_B200_PRECISION_FP64;
  if (std::string(value) == "mixed") return SDFT_B200_PRECISION_MIXED;
  throw std::invalid_argument("SDFT_B200_ACCELERATOR_PRECISION must be fp64 or mixed");
}

int op(MatrixOp o) { return o == MatrixOp::Adjoint ? SDFT_B200_OP_ADJOINT : SDFT_B200_OP_NORMAL; }

class B200Accelerator final : public Accelerator {
 public:
  B200Accelerator() : precision_(search_precision()) {
    const char* device = std::getenv("SDFT_B200_DEVICE");
    check(sdft_b200_context_create(device ? std::atoi(device) : 0, nullptr, &context_));
  }
  ~B200Accelerator() override { sdft_b200_context_destroy(context_); }

  std::string device() const override { return std::string("NVIDIA B200 (") + sdft_b200_version() + ")"; }

  void gemm(MatrixOp ao, MatrixOp bo, std::size_t m, std::size_t n, std::size_t k, const Complex64* a,
            std::size_t lda, const Complex64* b, std::size_t ldb, Complex64* c, std::size_t ldc, bool add) override {
    check(sdft_b200_complex_gemm(context_, op(ao), op(bo), m, n, k, reinterpret_cast<const double*>(a), lda,
                                 reinterpret_cast<const double*>(b), ldb, reinterpret_cast<double*>(c), ldc,
                                 precision_, add ? 1 : 0, SDFT_B200_MEMORY_HOST));
  }

  // The left operand stays on the device for its identity (and, in the mixed
  // form, its tensor-core packing); only B and C cross the bus.
  void gemm_immutable_left(std::uint64_t identity, MatrixOp ao, std::size_t m, std::size_t n, std::size_t k,
                           const Complex64* a, std::size_t lda, const Complex64* b, std::size_t ldb, Complex64* c,
                           std::size_t ldc, bool add) override {
    check(sdft_b200_complex_gemm_immutable_left(context_, identity, op(ao), m, n, k, reinterpret_cast<const double*>(a),
                                                lda, reinterpret_cast<const double*>(b), ldb,
                                                reinterpret_cast<double*>(c), ldc, precision_, add ? 1 : 0,
                                                SDFT_B200_MEMORY_HOST));
  }

  // One upload of the shared right operand for the three products.
  void gemm_triple_right(std::size_t m, std::size_t n, std::size_t k, const std::array<const Complex64*, 3>& a,
                         std::size_t lda, const Complex64* b, std::size_t ldb, const std::array<Complex64*, 3>& c,
                         std::size_t ldc) override {
    const double* left[3] = {reinterpret_cast<const double*>(a[0]), reinterpret_cast<const double*>(a[1]),
                             reinterpret_cast<const double*>(a[2])};
    double* out[3] = {reinterpret_cast<double*>(c[0]), reinterpret_cast<double*>(c[1]), reinterpret_cast<double*>(c[2])};
    check(sdft_b200_complex_gemm_triple_right(context_, m, n, k, left, lda, reinterpret_cast<const double*>(b), ldb,
                                              out, ldc, precision_, SDFT_B200_MEMORY_HOST));
  }

  void local_hamiltonian(const std::array<int, 3>& shape, const std::vector<std::size_t>& indices,
                         const std::vector<double>& kinetic, const std::vector<double>& potential,
                         const Complex64* input, std::size_t columns, Complex64* output,
                         std::uint64_t operator_identity) override {
    static_assert(sizeof(std::size_t) == sizeof(std::uint64_t), "LP64 index map expected");
    const std::int32_t s[3] = {shape[0], shape[1], shape[2]};
    check(sdft_b200_local_hamiltonian(context_, s, reinterpret_cast<const std::uint64_t*>(indices.data()),
                                      indices.size(), kinetic.data(), potential.data(),
                                      reinterpret_cast<const double*>(input), columns,
                                      reinterpret_cast<double*>(output), precision_, operator_identity));
  }

  void pbe_points(const double* density, const double* gradient, std::size_t count, PbeXcPoint* output) override {
    static_assert(sizeof(PbeXcPoint) == 7 * sizeof(double), "PbeXcPoint is seven doubles");
    check(sdft_b200_pbe_points(context_, density, gradient, count, reinterpret_cast<double*>(output),
                               SDFT_B200_MEMORY_HOST));
  }

  bool paw_pair(std::uint64_t identity, std::size_t npw, std::size_t projectors, std::size_t columns,
                const Complex64* b, const Complex64* d, const Complex64* q, const Complex64* input, Complex64* h,
                Complex64* s, std::uint64_t projector_identity) override {
    check(sdft_b200_paw_pair(context_, identity, npw, projectors, columns, reinterpret_cast<const double*>(b),
                             reinterpret_cast<const double*>(d), reinterpret_cast<const double*>(q),
                             reinterpret_cast<const double*>(input), reinterpret_cast<double*>(h),
                             reinterpret_cast<double*>(s), precision_, projector_identity));
    return true;
  }

 private:
  sdft_b200_context* context_ = nullptr;
  int precision_;
};

}  // namespace

std::unique_ptr<Accelerator> make_cuda_accelerator() {
  PerformanceTimer timer("gpu_initialization");
  return std::make_unique<B200Accelerator>();
}

}  // namespace sdft
