// Column reductions and small dense helpers for the device Davidson solver.
#include <algorithm>

#include "dense.cuh"
#include "preconditioner.cuh"

namespace sdft_b200 {

namespace {

constexpr int kReduceThreads = 256;

// Error-free sum of two compensated partials (TwoSum on the leading parts).
struct Neumaier {
  double sum = 0.0, correction = 0.0;
  __device__ __forceinline__ void add(double v) {
    const double next = __dadd_rn(sum, v);
    correction = __dadd_rn(correction, fabs(sum) >= fabs(v) ? __dadd_rn(__dsub_rn(sum, next), v)
                                                            : __dadd_rn(__dsub_rn(v, next), sum));
    sum = next;
  }
  __device__ __forceinline__ void merge(const Neumaier& o) {
    add(o.sum);
    correction = __dadd_rn(correction, o.correction);
  }
  __device__ __forceinline__ double value() const { return __dadd_rn(sum, correction); }
};

template <typename R>
__device__ R block_reduce(R value, R* shared) {
  // shared: kReduceThreads entries; deterministic pairwise tree.
  const int tid = threadIdx.x;
  shared[tid] = value;
  __syncthreads();
  for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
    if (tid < stride) shared[tid] = shared[tid] + shared[tid + stride];
    __syncthreads();
  }
  R result = shared[0];
  __syncthreads();
  return result;
}

__device__ Neumaier block_reduce_compensated(Neumaier value, Neumaier* shared) {
  const int tid = threadIdx.x;
  shared[tid] = value;
  __syncthreads();
  for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
    if (tid < stride) {
      Neumaier a = shared[tid];
      a.merge(shared[tid + stride]);
      shared[tid] = a;
    }
    __syncthreads();
  }
  Neumaier result = shared[0];
  __syncthreads();
  return result;
}

__global__ void hermitian_part_kernel(const Cx<double>* __restrict__ src, long long lds, Cx<double>* __restrict__ dst,
                                      long long ldd, int m) {
  const long long total = static_cast<long long>(m) * m;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(idx % m), j = static_cast<int>(idx / m);
    const Cx<double> a = src[i + j * lds], b = src[j + i * lds];
    dst[i + j * ldd] = Cx<double>{0.5 * (a.re + b.re), 0.5 * (a.im - b.im)};
  }
}

__global__ void hermitian_from_lower_kernel(const Cx<double>* __restrict__ src, long long lds,
                                            Cx<double>* __restrict__ dst, long long ldd, int m) {
  const long long total = static_cast<long long>(m) * m;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(idx % m), j = static_cast<int>(idx / m);
    Cx<double> v;
    if (i > j) v = src[i + j * lds];
    else if (i < j) v = Cx<double>{src[j + i * lds].re, -src[j + i * lds].im};
    else v = Cx<double>{src[i + j * lds].re, 0.0};
    dst[i + j * ldd] = v;
  }
}

__global__ void column_norms_kernel(const Cx<double>* __restrict__ a, long long lda, int rows, double* __restrict__ out) {
  __shared__ double shared[kReduceThreads];
  const Cx<double>* col = a + blockIdx.x * lda;
  double s = 0.0;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) s += col[i].re * col[i].re + col[i].im * col[i].im;
  s = block_reduce(s, shared);
  if (threadIdx.x == 0) out[blockIdx.x] = sqrt(s);
}

__global__ void search_residual_kernel(const Cx<double>* __restrict__ hx, const Cx<double>* __restrict__ sx, long long ld,
                                       int rows, const double* __restrict__ values, Cx<double>* __restrict__ r) {
  const double v = values[blockIdx.y];
  const long long base = blockIdx.y * ld;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const Cx<double> h = hx[base + i], s = sx[base + i];
    r[base + i] = Cx<double>{h.re - s.re * v, h.im - s.im * v};
  }
}

__global__ void rayleigh_certificate_kernel(const Cx<double>* __restrict__ x, const Cx<double>* __restrict__ hx,
                                            const Cx<double>* __restrict__ sx, long long ld, int rows,
                                            double* __restrict__ values, double* __restrict__ metric,
                                            Cx<double>* __restrict__ r, double* __restrict__ norms) {
  __shared__ Neumaier shared[kReduceThreads];
  __shared__ double shared_d[kReduceThreads];
  const long long base = blockIdx.x * ld;
  Neumaier m, h;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    const Cx<double> a = x[base + i], s = sx[base + i], hv = hx[base + i];
    m.add(__dmul_rn(a.re, s.re));
    m.add(__dmul_rn(a.im, s.im));
    h.add(__dmul_rn(a.re, hv.re));
    h.add(__dmul_rn(a.im, hv.im));
  }
  const double mv = block_reduce_compensated(m, shared).value();
  const double hv_sum = block_reduce_compensated(h, shared).value();
  const double value = hv_sum / mv;
  double s2 = 0.0;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    const Cx<double> s = sx[base + i], hv = hx[base + i];
    const Cx<double> e{__fma_rn(-value, s.re, hv.re), __fma_rn(-value, s.im, hv.im)};
    r[base + i] = e;
    s2 += e.re * e.re + e.im * e.im;
  }
  s2 = block_reduce(s2, shared_d);
  if (threadIdx.x == 0) {
    values[blockIdx.x] = value;
    metric[blockIdx.x] = mv;
    norms[blockIdx.x] = sqrt(s2);
  }
}

__global__ void metric_norms_kernel(const Cx<double>* __restrict__ x, const Cx<double>* __restrict__ sx, long long ld,
                                    int rows, double* __restrict__ out) {
  __shared__ Neumaier shared[kReduceThreads];
  const long long base = blockIdx.x * ld;
  Neumaier m;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    const Cx<double> a = x[base + i], s = sx[base + i];
    m.add(__dmul_rn(a.re, s.re));
    m.add(__dmul_rn(a.im, s.im));
  }
  const double v = block_reduce_compensated(m, shared).value();
  if (threadIdx.x == 0) out[blockIdx.x] = v;
}

// out(i, j) = sum_k conj(a(k, i)) b(k, j) with compensated sums of the
// reference's terms (re: a.re b.re + a.im b.im; im: a.re b.im - a.im b.re).
__global__ void compensated_inner_matrix_kernel(const Cx<double>* __restrict__ a, const Cx<double>* __restrict__ b,
                                                long long ld, int rows, Cx<double>* __restrict__ out, long long ldo) {
  __shared__ Neumaier shared[kReduceThreads];
  const long long ia = blockIdx.x * ld, jb = blockIdx.y * ld;
  Neumaier re, im;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    const Cx<double> u = a[ia + i], v = b[jb + i];
    re.add(__dmul_rn(u.re, v.re));
    re.add(__dmul_rn(u.im, v.im));
    im.add(__dmul_rn(u.re, v.im));
    im.add(-__dmul_rn(u.im, v.re));
  }
  const double r = block_reduce_compensated(re, shared).value();
  const double m = block_reduce_compensated(im, shared).value();
  if (threadIdx.x == 0) out[blockIdx.x + blockIdx.y * ldo] = Cx<double>{r, m};
}

// out(:, c) = fma(alpha[c], d(:, c), x(:, c)) componentwise.
__global__ void fma_columns_kernel(const double* __restrict__ alpha, const Cx<double>* __restrict__ d,
                                   const Cx<double>* __restrict__ x, long long ld, int rows, Cx<double>* __restrict__ out) {
  const double a = alpha[blockIdx.y];
  const long long base = blockIdx.y * ld;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const Cx<double> dv = d[base + i], xv = x[base + i];
    out[base + i] = Cx<double>{__fma_rn(a, dv.re, xv.re), __fma_rn(a, dv.im, xv.im)};
  }
}

__global__ void scale_columns_kernel(Cx<double>* __restrict__ x, long long ld, int rows, const double* __restrict__ scale,
                                     bool reciprocal_sqrt) {
  const double s = reciprocal_sqrt ? 1.0 / sqrt(scale[blockIdx.y]) : scale[blockIdx.y];
  const long long base = blockIdx.y * ld;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const Cx<double> v = x[base + i];
    x[base + i] = Cx<double>{v.re * s, v.im * s};
  }
}

__global__ void unit_columns_kernel(Cx<double>* __restrict__ x, long long ld, int rows, const double* __restrict__ norms) {
  const double n = norms[blockIdx.y];
  if (!(n > 0.0)) return;
  const long long base = blockIdx.y * ld;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const Cx<double> v = x[base + i];
    x[base + i] = Cx<double>{v.re / n, v.im / n};
  }
}


__global__ void kinetic_precondition_kernel(const Cx<double>* __restrict__ r, const Cx<double>* __restrict__ x,
                                            long long ld, int rows, const double* __restrict__ kinetic,
                                            Cx<double>* out, long long ldo) {
  __shared__ double shared[kReduceThreads];
  const long long base = blockIdx.x * ld;
  double wk = 0.0;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    const Cx<double> v = x[base + i];
    wk += (v.re * v.re + v.im * v.im) * kinetic[i];
  }
  wk = block_reduce(wk, shared);
  const long long obase = blockIdx.x * ldo;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    const double p = -kinetic_preconditioner(kinetic[i], wk);
    const Cx<double> v = r[base + i];
    out[obase + i] = Cx<double>{v.re * p, v.im * p};
  }
}

__device__ __forceinline__ double splitmix_uniform(unsigned long long draw) {
  unsigned long long z = 0x6a09e667f3bcc909ULL + (draw + 1ULL) * 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return static_cast<double>(z >> 11) * 0x1.0p-53 - 0.5;
}

__global__ void broad_seed_kernel(int rows, unsigned long long first_draw, const int* __restrict__ order,
                                  Cx<double>* __restrict__ out, long long ld) {
  __shared__ double shared[kReduceThreads];
  const int j = blockIdx.x;
  const unsigned long long start = first_draw + 2ULL * rows * j;
  Cx<double>* col = out + j * ld;
  double s = 0.0;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    const double re = splitmix_uniform(start + 2ULL * i), im = splitmix_uniform(start + 2ULL * i + 1);
    col[i] = Cx<double>{re, im};
    s += re * re + im * im;
  }
  s = block_reduce(s, shared);
  const double scale = 0.05 / sqrt(s);
  for (int i = threadIdx.x; i < rows; i += blockDim.x) {
    const Cx<double> v = col[i];
    col[i] = Cx<double>{v.re * scale + (i == order[j] ? 1.0 : 0.0), v.im * scale};
  }
}

__global__ void copy_block_kernel(const Cx<double>* __restrict__ src, long long lds, Cx<double>* __restrict__ dst,
                                  long long ldd, int rows) {
  const long long s = blockIdx.y * lds, d = blockIdx.y * ldd;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) dst[d + i] = src[s + i];
}

__global__ void add_block_kernel(const Cx<double>* __restrict__ src, long long lds, Cx<double>* __restrict__ dst,
                                 long long ldd, int rows) {
  const long long s = blockIdx.y * lds, d = blockIdx.y * ldd;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const Cx<double> x = src[s + i], y = dst[d + i];
    dst[d + i] = Cx<double>{y.re + x.re, y.im + x.im};
  }
}

__global__ void gather_columns_kernel(const Cx<double>* __restrict__ src, long long lds, int rows,
                                      const int* __restrict__ index, Cx<double>* __restrict__ dst, long long ldd) {
  const long long s = index[blockIdx.y] * lds, d = blockIdx.y * ldd;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) dst[d + i] = src[s + i];
}

__global__ void zero_block_kernel(Cx<double>* __restrict__ a, long long lda, int rows) {
  const long long base = blockIdx.y * lda;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) a[base + i] = Cx<double>{0, 0};
}

dim3 column_grid(int rows, int cols) {
  return dim3(static_cast<unsigned>(std::min<std::size_t>(ceil_div(rows, 256), 64)), static_cast<unsigned>(cols));
}

}  // namespace

void hermitian_part(const Cx<double>* src, long long lds, Cx<double>* dst, long long ldd, int m, cudaStream_t stream) {
  if (m <= 0) return;
  const long long total = static_cast<long long>(m) * m;
  hermitian_part_kernel<<<static_cast<unsigned>(std::min<long long>(ceil_div(total, 256), 4096)), 256, 0, stream>>>(
      src, lds, dst, ldd, m);
  SDFT_LAUNCH("hermitian_part_kernel");
}

void hermitian_from_lower(const Cx<double>* src, long long lds, Cx<double>* dst, long long ldd, int m,
                          cudaStream_t stream) {
  const long long total = static_cast<long long>(m) * m;
  hermitian_from_lower_kernel<<<static_cast<unsigned>(std::min<long long>(ceil_div(total, 256), 4096)), 256, 0,
                                stream>>>(src, lds, dst, ldd, m);
  SDFT_LAUNCH("hermitian_from_lower_kernel");
}

void column_norms(const Cx<double>* a, long long lda, int rows, int cols, double* out, cudaStream_t stream) {
  if (cols <= 0) return;
  column_norms_kernel<<<cols, kReduceThreads, 0, stream>>>(a, lda, rows, out);
  SDFT_LAUNCH("column_norms_kernel");
}

void search_residual(const Cx<double>* hx, const Cx<double>* sx, long long ld, int rows, int cols,
                     const double* values, Cx<double>* r, cudaStream_t stream) {
  if (cols <= 0) return;
  search_residual_kernel<<<column_grid(rows, cols), 256, 0, stream>>>(hx, sx, ld, rows, values, r);
  SDFT_LAUNCH("search_residual_kernel");
}

void rayleigh_certificate(const Cx<double>* x, const Cx<double>* hx, const Cx<double>* sx, long long ld, int rows,
                          int cols, double* values, double* metric, Cx<double>* r, double* norms, cudaStream_t stream) {
  if (cols <= 0) return;
  rayleigh_certificate_kernel<<<cols, kReduceThreads, 0, stream>>>(x, hx, sx, ld, rows, values, metric, r, norms);
  SDFT_LAUNCH("rayleigh_certificate_kernel");
}

void metric_norms(const Cx<double>* x, const Cx<double>* sx, long long ld, int rows, int cols, double* out,
                  cudaStream_t stream) {
  if (cols <= 0) return;
  metric_norms_kernel<<<cols, kReduceThreads, 0, stream>>>(x, sx, ld, rows, out);
  SDFT_LAUNCH("metric_norms_kernel");
}

__global__ void adjoint_block_kernel(const Cx<double>* __restrict__ src, long long lds, int rows, int cols,
                                     Cx<double>* __restrict__ dst, long long ldd) {
  __shared__ Cx<double> tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + dy;
    if (i < rows && j < cols) tile[dy][threadIdx.x] = src[i + static_cast<long long>(j) * lds];
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int j = j0 + threadIdx.x, i = i0 + dy;
    if (i < rows && j < cols) {
      const Cx<double> v = tile[threadIdx.x][dy];
      dst[j + static_cast<long long>(i) * ldd] = Cx<double>{v.re, -v.im};
    }
  }
}

void adjoint_block(const Cx<double>* src, long long lds, int rows, int cols, Cx<double>* dst, long long ldd,
                   cudaStream_t stream) {
  if (rows <= 0 || cols <= 0) return;
  const dim3 grid(static_cast<unsigned>(ceil_div(rows, 32)), static_cast<unsigned>(ceil_div(cols, 32)));
  adjoint_block_kernel<<<grid, dim3(32, 8), 0, stream>>>(src, lds, rows, cols, dst, ldd);
  SDFT_LAUNCH("adjoint_block_kernel");
}

void compensated_inner_matrix(const Cx<double>* a, const Cx<double>* b, long long ld, int rows, int cols_a,
                              int cols_b, Cx<double>* out, long long ldo, cudaStream_t stream) {
  if (cols_a <= 0 || cols_b <= 0) return;
  compensated_inner_matrix_kernel<<<dim3(cols_a, cols_b), kReduceThreads, 0, stream>>>(a, b, ld, rows, out, ldo);
  SDFT_LAUNCH("compensated_inner_matrix_kernel");
}

void fma_columns(const double* alpha, const Cx<double>* d, const Cx<double>* x, long long ld, int rows, int cols,
                 Cx<double>* out, cudaStream_t stream) {
  if (cols <= 0 || rows <= 0) return;
  fma_columns_kernel<<<column_grid(rows, cols), 256, 0, stream>>>(alpha, d, x, ld, rows, out);
  SDFT_LAUNCH("fma_columns_kernel");
}

void scale_columns(Cx<double>* x, long long ld, int rows, int cols, const double* scale, bool reciprocal_sqrt,
                   cudaStream_t stream) {
  if (cols <= 0) return;
  scale_columns_kernel<<<column_grid(rows, cols), 256, 0, stream>>>(x, ld, rows, scale, reciprocal_sqrt);
  SDFT_LAUNCH("scale_columns_kernel");
}

void kinetic_precondition(const Cx<double>* r, const Cx<double>* x, long long ld, int rows, int cols,
                          const double* kinetic, Cx<double>* out, long long ldo, cudaStream_t stream) {
  if (cols <= 0) return;
  kinetic_precondition_kernel<<<cols, kReduceThreads, 0, stream>>>(r, x, ld, rows, kinetic, out, ldo);
  SDFT_LAUNCH("kinetic_precondition_kernel");
}

void broad_seed_block(int rows, int cols, unsigned long long first_draw, const int* order, Cx<double>* out,
                      long long ld, cudaStream_t stream) {
  if (cols <= 0) return;
  broad_seed_kernel<<<cols, kReduceThreads, 0, stream>>>(rows, first_draw, order, out, ld);
  SDFT_LAUNCH("broad_seed_kernel");
}

void copy_block(const Cx<double>* src, long long lds, Cx<double>* dst, long long ldd, int rows, int cols,
                cudaStream_t stream) {
  if (cols <= 0 || rows <= 0) return;
  copy_block_kernel<<<column_grid(rows, cols), 256, 0, stream>>>(src, lds, dst, ldd, rows);
  SDFT_LAUNCH("copy_block_kernel");
}

void add_block(const Cx<double>* src, long long lds, Cx<double>* dst, long long ldd, int rows, int cols,
               cudaStream_t stream) {
  if (cols <= 0 || rows <= 0) return;
  add_block_kernel<<<column_grid(rows, cols), 256, 0, stream>>>(src, lds, dst, ldd, rows);
  SDFT_LAUNCH("add_block_kernel");
}

void gather_columns(const Cx<double>* src, long long lds, int rows, const int* index, int count, Cx<double>* dst,
                    long long ldd, cudaStream_t stream) {
  if (count <= 0 || rows <= 0) return;
  gather_columns_kernel<<<column_grid(rows, count), 256, 0, stream>>>(src, lds, rows, index, dst, ldd);
  SDFT_LAUNCH("gather_columns_kernel");
}

void zero_block(Cx<double>* a, long long lda, int rows, int cols, cudaStream_t stream) {
  if (cols <= 0 || rows <= 0) return;
  zero_block_kernel<<<column_grid(rows, cols), 256, 0, stream>>>(a, lda, rows);
  SDFT_LAUNCH("zero_block_kernel");
}

void unit_columns(Cx<double>* x, long long ld, int rows, int cols, const double* norms, cudaStream_t stream) {
  if (cols <= 0) return;
  unit_columns_kernel<<<column_grid(rows, cols), 256, 0, stream>>>(x, ld, rows, norms);
  SDFT_LAUNCH("unit_columns_kernel");
}

}  // namespace sdft_b200
