// Tensor-core (tcgen05 / TMEM / TMA) complex GEMM with BF16 split products.
//
// A complex product C = op(A) B is evaluated as one real BF16 GEMM over an
// expanded K axis. Every complex k contributes P split-product terms
// (x ~ x0 + x1 + x2 in BF16, products a_i b_j for the pairs of the chosen
// pattern) and, for each term, the pair (re, im):
//   Ahat[i, (k*P+p)*2 + 0] = A_{ia(p)}(Re A[i,k]),  Ahat[i, (k*P+p)*2 + 1] = A_{ia(p)}(Im A[i,k])
//   Bhat[2j,   (k*P+p)*2 + {0,1}] = ( B_{ib(p)}(Re B[k,j]), -B_{ib(p)}(Im B[k,j]) )
//   Bhat[2j+1, (k*P+p)*2 + {0,1}] = ( B_{ib(p)}(Im B[k,j]),  B_{ib(p)}(Re B[k,j]) )
// so that (Ahat Bhat^T)[i, 2j] = Re C[i,j] and [i, 2j+1] = Im C[i,j], with the
// FP32 accumulator held in tensor memory. Both operands are K-major BF16 rows.
#pragma once
#include <cstdint>

#include "common.cuh"
#include "gemm.cuh"

namespace sdft_b200 {

// Split-product patterns: BF16x3 keeps (0,0),(0,1),(1,0) (~16 significant
// bits); BF16x6 adds (0,2),(1,1),(2,0) (~24 bits, FP32-class).
enum class Split : int { BF16x3 = 3, BF16x6 = 6 };

inline int split_terms(Split s) { return static_cast<int>(s); }

// Expanded-K length (bf16 elements) of a K-long complex contraction, padded to
// the 64-element tensor-core K block.
inline long long expanded_k(int k, Split s) {
  const long long raw = 2LL * split_terms(s) * k;
  return (raw + 63) / 64 * 64;
}

// A side: out[i][kexp] for i < rows (row stride ldo bf16 elements), from the
// complex FP64 matrix op(src): aop N -> A[i,k] = src[i + k*lds],
// aop C -> A[i,k] = conj(src[k + i*lds]). Padding columns are zeroed.
void pack_a(Op aop, const Cx<double>* src, long long lds, int rows, int k, Split split, std::uint16_t* out,
            long long ldo, cudaStream_t stream);

// B side for C = A B with B (k x n, ld ldb) normal: out rows 2j, 2j+1.
void pack_b(const Cx<double>* src, long long ldb, int k, int n, Split split, std::uint16_t* out, long long ldo,
            cudaStream_t stream);

// Same, but writes the A-side layout for `count` new K entries of an
// existing packed row block: columns [first, first+count) of the complex
// source (ld lds, rows rows) become expanded-K entries first*2P.. of each row
// (used to extend a packed transposed basis without repacking it).
void pack_a_columns(const Cx<double>* src, long long lds, int rows, int first, int count, Split split,
                    std::uint16_t* out, long long ldo, cudaStream_t stream);

// C (m x n complex, ld ldc, FP64) = alpha * Ahat Bhat^T (+ C if add), where
// Ahat is m x kexp and Bhat is 2n x kexp (BF16, K-major, leading dims lda/ldb
// in elements, 16-byte multiples). kexp = expanded_k(k, split).
void umma_complex_gemm(const std::uint16_t* a, long long lda, const std::uint16_t* b, long long ldb, int m, int n,
                       long long kexp, Cx<double>* c, long long ldc, bool add, double alpha, Scratch& workspace,
                       cudaStream_t stream);

// The tile autotuner's table so far: per shape class (rows rounded up to
// 128, real columns rounded up to 32, K blocks of 64 rounded up to a geometric
// grid of ratio 2^(1/8)) the chosen column tile
// width and split-K count, five ints per class into rows[0..5*capacity).
// Returns the number of classes.
std::size_t gemm_tuned_classes(std::size_t capacity, int* rows);

// True when the running device supports the tcgen05 path (sm_100).
bool umma_available();

// A packed A-side operand kept across calls (e.g. the projector matrix).
struct PackedA {
  std::uint16_t* data = nullptr;
  long long ld = 0;
  int rows = 0;
  int k = 0;
  Split split = Split::BF16x3;
  cudaStream_t stream = nullptr;  // data is stream-ordered pool memory on this stream
};

struct TensorCoreWorkspace {
  Scratch a, b, partial;
  Scratch adjoint;  // a right operand formed as B^H for the tensor-core path
};

// Search-precision split (SDFT_B200_SPLIT=x3|x6, default x3: on the Si64
// pencil its mixed-apply error is that of the FP32 FFTs, 5e-7), read once.
Split search_split();

// Packs op(A) (rows x k) into a new device buffer owned by `out`.
void pack_persistent(Op aop, const Cx<double>* a, long long lda, int rows, int k, Split split, PackedA& out,
                     cudaStream_t stream);
void release(PackedA& packed);

// C(m x n) = alpha op(A) B (+ C if add) on the tensor cores. `packed` (may be
// null) replaces op(A) when given; otherwise op(A) is packed into ws.a.
void gemm_tc(Op aop, int m, int n, int k, const Cx<double>* a, long long lda, const PackedA* packed,
             const Cx<double>* b, long long ldb, Cx<double>* c, long long ldc, bool add, double alpha, Split split,
             TensorCoreWorkspace& ws, cudaStream_t stream);

// Reads the device word set when a tensor-core kernel's bounded wait ran out
// (0 = no failure). The word is never cleared: concurrent solvers share it,
// and after a failure every later tensor-core product winds down and reports
// it too. Synchronous.
unsigned int umma_error_flag();

}  // namespace sdft_b200
