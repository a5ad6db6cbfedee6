// Complex GEMMs and small PAW block products (see gemm.cuh).
#include <algorithm>

#include "gemm.cuh"

namespace sdft_b200 {

void* Scratch::reserve(std::size_t need) {
  if (need <= bytes) return ptr;
  release();
  const std::size_t grown = std::max(need, bytes + bytes / 4);
  SDFT_CUDA(cudaMalloc(&ptr, grown));
  bytes = grown;
  return ptr;
}

void Scratch::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  bytes = 0;
}

namespace {

void check_blas(cublasStatus_t status, const char* what) {
  if (status != CUBLAS_STATUS_SUCCESS)
    throw CudaError(std::string("cuBLAS error ") + std::to_string(static_cast<int>(status)) + " in " + what);
}

constexpr int BM = 64, BN = 64, BK = 16, kGemmThreads = 256;

// Split-K SIMT complex GEMM, FP32 accumulation. Partial sums go to
// partial[split][col][row] (ld m); the reduction kernel adds them in fixed
// split order so the result is deterministic.
template <Op AOP, typename TA>
__global__ void __launch_bounds__(kGemmThreads) cgemm_simt_kernel(int m, int n, int k, int k_per_split,
                                                                  const Cx<TA>* __restrict__ a, long long lda,
                                                                  const Cx<double>* __restrict__ b, long long ldb,
                                                                  Cx<float>* __restrict__ partial) {
  __shared__ float Ar[BK][BM], Ai[BK][BM], Br[BK][BN], Bi[BK][BN];
  const int tid = threadIdx.x;
  const int tx = tid % 16, ty = tid / 16;
  const int tile_m = blockIdx.x * BM, tile_n = blockIdx.y * BN, split = blockIdx.z;
  const int k_begin = split * k_per_split;
  const int k_end = min(k, k_begin + k_per_split);
  float cr[4][4] = {}, ci[4][4] = {};
  for (int k0 = k_begin; k0 < k_end; k0 += BK) {
#pragma unroll
    for (int r = 0; r < (BM * BK) / kGemmThreads; ++r) {
      const int idx = tid + r * kGemmThreads;
      int i, kk;
      if (AOP == Op::N) {
        i = idx % BM;
        kk = idx / BM;
      } else {
        kk = idx % BK;
        i = idx / BK;
      }
      const int gi = tile_m + i, gk = k0 + kk;
      float re = 0.f, im = 0.f;
      if (gi < m && gk < k_end) {
        const Cx<TA> v = AOP == Op::N ? a[gi + static_cast<long long>(gk) * lda]
                                      : a[gk + static_cast<long long>(gi) * lda];
        re = static_cast<float>(v.re);
        im = AOP == Op::N ? static_cast<float>(v.im) : -static_cast<float>(v.im);
      }
      Ar[kk][i] = re;
      Ai[kk][i] = im;
    }
#pragma unroll
    for (int r = 0; r < (BN * BK) / kGemmThreads; ++r) {
      const int idx = tid + r * kGemmThreads;
      const int kk = idx % BK, j = idx / BK;
      const int gj = tile_n + j, gk = k0 + kk;
      float re = 0.f, im = 0.f;
      if (gj < n && gk < k_end) {
        const Cx<double> v = b[gk + static_cast<long long>(gj) * ldb];
        re = static_cast<float>(v.re);
        im = static_cast<float>(v.im);
      }
      Br[kk][j] = re;
      Bi[kk][j] = im;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      float ar[4], ai[4], br[4], bi[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        ar[q] = Ar[kk][tx + 16 * q];
        ai[q] = Ai[kk][tx + 16 * q];
        br[q] = Br[kk][ty + 16 * q];
        bi[q] = Bi[kk][ty + 16 * q];
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          cr[p][q] += ar[p] * br[q] - ai[p] * bi[q];
          ci[p][q] += ar[p] * bi[q] + ai[p] * br[q];
        }
    }
    __syncthreads();
  }
  Cx<float>* out = partial + static_cast<long long>(split) * m * n;
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int gi = tile_m + tx + 16 * p, gj = tile_n + ty + 16 * q;
      if (gi < m && gj < n) out[gi + static_cast<long long>(gj) * m] = Cx<float>{cr[p][q], ci[p][q]};
    }
}

__global__ void reduce_partials_kernel(int m, int n, int splits, const Cx<float>* __restrict__ partial,
                                       Cx<double>* __restrict__ c, long long ldc, bool add, double alpha) {
  const long long total = static_cast<long long>(m) * n;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    double re = 0.0, im = 0.0;
    for (int s = 0; s < splits; ++s) {
      const Cx<float> v = partial[s * total + idx];
      re += v.re;
      im += v.im;
    }
    const long long i = idx % m, j = idx / m;
    Cx<double>& out = c[i + j * ldc];
    re *= alpha;
    im *= alpha;
    if (add) {
      re += out.re;
      im += out.im;
    }
    out = Cx<double>{re, im};
  }
}

struct CompensatedSum {
  double sum = 0.0, correction = 0.0;
  __device__ __forceinline__ void add(double value) {
    const double next = __dadd_rn(sum, value);
    const double back = __dsub_rn(next, sum);
    correction = __dadd_rn(correction, __dadd_rn(__dsub_rn(sum, __dsub_rn(next, back)), __dsub_rn(value, back)));
    sum = next;
  }
  __device__ __forceinline__ void product(double a, double b) {
    const double rounded = __dmul_rn(a, b);
    add(rounded);
    add(__fma_rn(a, b, -rounded));
  }
  __device__ __forceinline__ double value() const { return __dadd_rn(sum, correction); }
};

__global__ void block_product_kernel(const int* __restrict__ offsets, const long long* __restrict__ storage,
                                     const Cx<double>* __restrict__ blocks, const Cx<double>* __restrict__ p,
                                     long long ldp, int columns, Cx<double>* __restrict__ out, long long ldo) {
  const int atom = blockIdx.x;
  const int first = offsets[atom], rows = offsets[atom + 1] - first;
  const Cx<double>* m = blocks + storage[atom];
  const int per_block = blockDim.x / rows;
  if (per_block == 0) return;
  const int local = threadIdx.x % rows;
  const int column = blockIdx.y * per_block + threadIdx.x / rows;
  if (threadIdx.x >= per_block * rows || column >= columns) return;
  CompensatedSum re, im;
  const Cx<double>* pc = p + static_cast<long long>(column) * ldp + first;
  for (int j = 0; j < rows; ++j) {
    const Cx<double> left = m[local + static_cast<long long>(j) * rows];
    const Cx<double> right = pc[j];
    re.product(left.re, right.re);
    re.product(-left.im, right.im);
    im.product(left.re, right.im);
    im.product(left.im, right.re);
  }
  out[static_cast<long long>(column) * ldo + first + local] = Cx<double>{re.value(), im.value()};
}

__global__ void scale_copy_kernel(const Cx<double>* __restrict__ x, long long ldx, Cx<double>* __restrict__ y,
                                  long long ldy, int n, int columns, double alpha) {
  const long long total = static_cast<long long>(n) * columns;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long i = idx % n, c = idx / n;
    const Cx<double> v = x[i + c * ldx];
    y[i + c * ldy] = Cx<double>{v.re * alpha, v.im * alpha};
  }
}

__global__ void demote_kernel(const Cx<double>* __restrict__ src, Cx<float>* __restrict__ dst, std::size_t n) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x)
    dst[i] = cconvert<float>(src[i]);
}

unsigned grid_for(long long total, int threads) {
  return static_cast<unsigned>(std::min<long long>(std::max<long long>(1, (total + threads - 1) / threads), 148LL * 32));
}

}  // namespace

void zgemm(cublasHandle_t handle, Op aop, Op bop, int m, int n, int k, const Cx<double>* a, long long lda,
           const Cx<double>* b, long long ldb, Cx<double>* c, long long ldc, bool add, double alpha) {
  if (m <= 0 || n <= 0 || k <= 0) return;
  const cuDoubleComplex one = make_cuDoubleComplex(alpha, 0.0);
  const cuDoubleComplex beta = make_cuDoubleComplex(add ? 1.0 : 0.0, 0.0);
  check_blas(cublasZgemm(handle, aop == Op::N ? CUBLAS_OP_N : CUBLAS_OP_C, bop == Op::N ? CUBLAS_OP_N : CUBLAS_OP_C,
                         m, n, k, &one, reinterpret_cast<const cuDoubleComplex*>(a), static_cast<int>(lda),
                         reinterpret_cast<const cuDoubleComplex*>(b), static_cast<int>(ldb), &beta,
                         reinterpret_cast<cuDoubleComplex*>(c), static_cast<int>(ldc)),
             "cublasZgemm");
}

void gemm_mixed(Op aop, int m, int n, int k, const Cx<double>* a, const Cx<float>* a32, long long lda,
                const Cx<double>* b, long long ldb, Cx<double>* c, long long ldc, bool add, Scratch& workspace,
                cudaStream_t stream, double alpha) {
  if (m <= 0 || n <= 0 || k <= 0) return;
  const long long tiles = static_cast<long long>(ceil_div(m, BM)) * static_cast<long long>(ceil_div(n, BN));
  int splits = static_cast<int>(std::min<long long>(std::max<long long>(1, (2 * 148 + tiles - 1) / tiles),
                                                    std::max(1, k / 512)));
  splits = std::min(splits, 64);
  const int k_per_split = static_cast<int>(ceil_div(ceil_div(k, splits), BK) * BK);
  splits = static_cast<int>(ceil_div(k, k_per_split));
  auto* partial = static_cast<Cx<float>*>(
      workspace.reserve(sizeof(Cx<float>) * static_cast<std::size_t>(m) * n * splits));
  const dim3 grid(static_cast<unsigned>(ceil_div(m, BM)), static_cast<unsigned>(ceil_div(n, BN)), splits);
  if (aop == Op::N) {
    if (a32) cgemm_simt_kernel<Op::N, float><<<grid, kGemmThreads, 0, stream>>>(m, n, k, k_per_split, a32, lda, b, ldb, partial);
    else cgemm_simt_kernel<Op::N, double><<<grid, kGemmThreads, 0, stream>>>(m, n, k, k_per_split, a, lda, b, ldb, partial);
  } else {
    if (a32) cgemm_simt_kernel<Op::C, float><<<grid, kGemmThreads, 0, stream>>>(m, n, k, k_per_split, a32, lda, b, ldb, partial);
    else cgemm_simt_kernel<Op::C, double><<<grid, kGemmThreads, 0, stream>>>(m, n, k, k_per_split, a, lda, b, ldb, partial);
  }
  SDFT_LAUNCH("cgemm_simt_kernel");
  const long long total = static_cast<long long>(m) * n;
  reduce_partials_kernel<<<grid_for(total, 256), 256, 0, stream>>>(m, n, splits, partial, c, ldc, add, alpha);
  SDFT_LAUNCH("reduce_partials_kernel");
}

void block_product(int atoms, const int* offsets, const long long* storage, int max_block, const Cx<double>* blocks,
                   const Cx<double>* p, long long ldp, int columns, Cx<double>* out, long long ldo,
                   cudaStream_t stream) {
  if (atoms <= 0 || columns <= 0) return;
  if (max_block < 1 || max_block > 256) throw InvalidArgument("PAW block size out of range");
  const int threads = 256;
  const int per_block = threads / max_block;
  const dim3 grid(atoms, static_cast<unsigned>(ceil_div(columns, per_block)));
  // Blocks smaller than max_block still map per_block(their size) >= per_block(max) columns per CTA.
  block_product_kernel<<<grid, threads, 0, stream>>>(offsets, storage, blocks, p, ldp, columns, out, ldo);
  SDFT_LAUNCH("block_product_kernel");
}

void scale_copy(const Cx<double>* x, long long ldx, Cx<double>* y, long long ldy, int n, int columns, double alpha,
                cudaStream_t stream) {
  const long long total = static_cast<long long>(n) * columns;
  scale_copy_kernel<<<grid_for(total, 256), 256, 0, stream>>>(x, ldx, y, ldy, n, columns, alpha);
  SDFT_LAUNCH("scale_copy_kernel");
}

void demote(const Cx<double>* src, Cx<float>* dst, std::size_t n, cudaStream_t stream) {
  demote_kernel<<<grid_for(static_cast<long long>(n), 256), 256, 0, stream>>>(src, dst, n);
  SDFT_LAUNCH("demote_kernel");
}

}  // namespace sdft_b200
