// Complex GEMMs for the PAW projector chain and the Davidson subspace work.
#pragma once
#include <cublas_v2.h>

#include "common.cuh"

namespace sdft_b200 {

enum class Op { N, C };  // C = conjugate transpose (the reference's MatrixOp::Adjoint)

// Grow-only device scratch owned by a context.
// Grow-only device buffer. With `stream` set (by the owning context) its
// memory is stream-ordered pool memory on that stream (stream_alloc), so
// growing or releasing it never synchronises the device; without, plain
// cudaMalloc / cudaFree.
struct Scratch {
  void* ptr = nullptr;
  std::size_t bytes = 0;
  cudaStream_t stream = nullptr;
  void* reserve(std::size_t need);
  void release();
  ~Scratch() { release(); }
};

// C(m x n, ldc) = alpha op(A) B (+ C if add), all complex FP64 column-major,
// FP64 arithmetic through cuBLAS ZGEMM (plain library GEMM).
void zgemm(cublasHandle_t handle, Op aop, Op bop, int m, int n, int k, const Cx<double>* a, long long lda,
           const Cx<double>* b, long long ldb, Cx<double>* c, long long ldc, bool add, double alpha = 1.0);

// Per-atom block-diagonal product out[off_a + i, c] = sum_j M_a(i,j) P[off_a + j, c]
// with error-free FP64 products and compensated sums (TwoSum + FMA), the
// reference's compensated_paw_product order (src/paw_compensated_product.hpp:41-56).
// blocks: column-major per atom, block a at storage[a]; offsets[a] = first row.
void block_product(int atoms, const int* offsets, const long long* storage, int max_block, const Cx<double>* blocks,
                   const Cx<double>* p, long long ldp, int columns, Cx<double>* out, long long ldo,
                   cudaStream_t stream);

// out(:, c) = (M_a - shift[c] N_a) P(:, c) per atom block (shift on the
// device), both products compensated as in block_product.
void shifted_block_product(int atoms, const int* offsets, const long long* storage, int max_block,
                           const Cx<double>* m_blocks, const Cx<double>* n_blocks, const double* shift,
                           const Cx<double>* p, long long ldp, int columns, Cx<double>* out, long long ldo,
                           cudaStream_t stream);

// y(:, c) -= shift[c] * scale * x(:, c) (shift on the device).
void shifted_axpy(const Cx<double>* x, long long ldx, Cx<double>* y, long long ldy, int n, int columns,
                  const double* shift, double scale, cudaStream_t stream);

// y = alpha * x (columns of length n, leading dims ldx/ldy).
void scale_copy(const Cx<double>* x, long long ldx, Cx<double>* y, long long ldy, int n, int columns, double alpha,
                cudaStream_t stream);

// FP64 -> FP32 copy of n complex values.
void demote(const Cx<double>* src, Cx<float>* dst, std::size_t n, cudaStream_t stream);

}  // namespace sdft_b200
