// Complex GEMMs and small PAW block products (see gemm.cuh).
#include <algorithm>

#include "gemm.cuh"

namespace sdft_b200 {

void* Scratch::reserve(std::size_t need) {
  if (need <= bytes) return ptr;
  const std::size_t grown = std::max(need, bytes + bytes / 4);
  release();
  if (stream) ptr = stream_alloc(grown, stream);
  else SDFT_CUDA(cudaMalloc(&ptr, grown));
  bytes = grown;
  return ptr;
}

void Scratch::release() {
  if (ptr) {
    if (stream) stream_free(ptr, stream);
    else cudaFree(ptr);
  }
  ptr = nullptr;
  bytes = 0;
}

namespace {

void check_blas(cublasStatus_t status, const char* what) {
  if (status != CUBLAS_STATUS_SUCCESS)
    throw CudaError(std::string("cuBLAS error ") + std::to_string(static_cast<int>(status)) + " in " + what);
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

// out(:, c) = (M_a - shift[c] N_a) P(:, c) per atom block: both products with
// the compensated sums of block_product_kernel, combined once.
__global__ void shifted_block_product_kernel(const int* __restrict__ offsets, const long long* __restrict__ storage,
                                             const Cx<double>* __restrict__ m_blocks,
                                             const Cx<double>* __restrict__ n_blocks, const double* __restrict__ shift,
                                             const Cx<double>* __restrict__ p, long long ldp, int columns,
                                             Cx<double>* __restrict__ out, long long ldo) {
  const int atom = blockIdx.x;
  const int first = offsets[atom], rows = offsets[atom + 1] - first;
  const Cx<double>* m = m_blocks + storage[atom];
  const Cx<double>* nb = n_blocks + storage[atom];
  const int per_block = blockDim.x / rows;
  if (per_block == 0) return;
  const int local = threadIdx.x % rows;
  const int column = blockIdx.y * per_block + threadIdx.x / rows;
  if (threadIdx.x >= per_block * rows || column >= columns) return;
  CompensatedSum mre, mim, nre, nim;
  const Cx<double>* pc = p + static_cast<long long>(column) * ldp + first;
  for (int j = 0; j < rows; ++j) {
    const Cx<double> a = m[local + static_cast<long long>(j) * rows], b = nb[local + static_cast<long long>(j) * rows];
    const Cx<double> right = pc[j];
    mre.product(a.re, right.re);
    mre.product(-a.im, right.im);
    mim.product(a.re, right.im);
    mim.product(a.im, right.re);
    nre.product(b.re, right.re);
    nre.product(-b.im, right.im);
    nim.product(b.re, right.im);
    nim.product(b.im, right.re);
  }
  const double s = shift[column];
  out[static_cast<long long>(column) * ldo + first + local] =
      Cx<double>{__fma_rn(-s, nre.value(), mre.value()), __fma_rn(-s, nim.value(), mim.value())};
}

// y(:, c) -= shift[c] * scale * x(:, c).
__global__ void shifted_axpy_kernel(const Cx<double>* __restrict__ x, long long ldx, Cx<double>* __restrict__ y,
                                    long long ldy, int n, const double* __restrict__ shift, double scale) {
  const int c = blockIdx.y;
  const double a = shift[c] * scale;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const Cx<double> v = x[i + c * ldx], w = y[i + c * ldy];
    y[i + c * ldy] = Cx<double>{__fma_rn(-a, v.re, w.re), __fma_rn(-a, v.im, w.im)};
  }
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

void shifted_block_product(int atoms, const int* offsets, const long long* storage, int max_block,
                           const Cx<double>* m_blocks, const Cx<double>* n_blocks, const double* shift,
                           const Cx<double>* p, long long ldp, int columns, Cx<double>* out, long long ldo,
                           cudaStream_t stream) {
  if (atoms <= 0 || columns <= 0) return;
  if (max_block < 1 || max_block > 256) throw InvalidArgument("PAW block size out of range");
  const int threads = 256;
  const int per_block = threads / max_block;
  const dim3 grid(atoms, static_cast<unsigned>(ceil_div(columns, per_block)));
  shifted_block_product_kernel<<<grid, threads, 0, stream>>>(offsets, storage, m_blocks, n_blocks, shift, p, ldp,
                                                            columns, out, ldo);
  SDFT_LAUNCH("shifted_block_product_kernel");
}

void shifted_axpy(const Cx<double>* x, long long ldx, Cx<double>* y, long long ldy, int n, int columns,
                  const double* shift, double scale, cudaStream_t stream) {
  if (n <= 0 || columns <= 0) return;
  const dim3 grid(static_cast<unsigned>(std::min<long long>(ceil_div(n, 256), 64)), static_cast<unsigned>(columns));
  shifted_axpy_kernel<<<grid, 256, 0, stream>>>(x, ldx, y, ldy, n, shift, scale);
  SDFT_LAUNCH("shifted_axpy_kernel");
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
