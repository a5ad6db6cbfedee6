// Jacobi-Davidson corrections with preconditioned CG (the mixed form's
// expansion step; see correction.cuh).
//
// Per CG step, for all selected columns at once: the mixed-form shifted
// product q = (H - theta S) p (one projection and back-projection), the left projection
// q <- q - S X (X^H q), the step length alpha = (res, z) / (p, q) per column,
// t += alpha p, res -= alpha q, then z = P res, the right projection
// z <- z - X ((S X)^H z) and the next direction p = z + beta p. Every scalar
// stays on the device (no host round trip inside the loop); a column whose
// curvature (p, q) is not positive stops moving (alpha = 0).
#include <algorithm>

#include "correction.cuh"
#include "dense.cuh"
#include "preconditioner.cuh"

namespace sdft_b200 {

namespace {

constexpr int kThreads = 256;
constexpr int kDotThreads = 1024;  // one CTA per column: the column's NPW terms over 1024 threads

__device__ double block_sum(double value, double* shared) {
  const int tid = threadIdx.x;
  shared[tid] = value;
  __syncthreads();
  for (int stride = blockDim.x / 2; stride > 0; stride >>= 1) {
    if (tid < stride) shared[tid] += shared[tid + stride];
    __syncthreads();
  }
  const double result = shared[0];
  __syncthreads();
  return result;
}

// theta[j] = theta_all[selected[j]]; kinetic energy of Ritz vector selected[j].
__global__ void setup_kernel(const Cx<double>* __restrict__ x, long long ld, int rows, const double* __restrict__ kinetic,
                             const double* __restrict__ theta_all, const int* __restrict__ selected,
                             double* __restrict__ theta, double* __restrict__ energy) {
  __shared__ double shared[kThreads];
  const int j = blockIdx.x, column = selected[j];
  const Cx<double>* v = x + static_cast<long long>(column) * ld;
  double s = 0.0;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) s += (v[i].re * v[i].re + v[i].im * v[i].im) * kinetic[i];
  s = block_sum(s, shared);
  if (threadIdx.x == 0) {
    theta[j] = theta_all[column];
    energy[j] = s;
  }
}

// out(:, j) = -r(:, selected[j]).
__global__ void gather_negated_kernel(const Cx<double>* __restrict__ r, long long ld, int rows,
                                      const int* __restrict__ selected, Cx<double>* __restrict__ out) {
  const int j = blockIdx.y;
  const Cx<double>* src = r + static_cast<long long>(selected[j]) * ld;
  Cx<double>* dst = out + static_cast<long long>(j) * rows;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x)
    dst[i] = Cx<double>{-src[i].re, -src[i].im};
}

// z(:, j) = P(T, energy[j]) res(:, j).
__global__ void precondition_kernel(const Cx<double>* __restrict__ res, int rows, const double* __restrict__ kinetic,
                                    const double* __restrict__ energy, Cx<double>* __restrict__ z) {
  const int j = blockIdx.y;
  const double e = energy[j];
  const long long base = static_cast<long long>(j) * rows;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const double p = kinetic_preconditioner(kinetic[i], e);
    const Cx<double> v = res[base + i];
    z[base + i] = Cx<double>{v.re * p, v.im * p};
  }
}

// out[j] = Re sum_i conj(a(i, j)) b(i, j).
__global__ void __launch_bounds__(kDotThreads) column_dots_kernel(const Cx<double>* __restrict__ a,
                                                                  const Cx<double>* __restrict__ b, int rows,
                                                                  double* __restrict__ out) {
  __shared__ double shared[kDotThreads];
  const long long base = static_cast<long long>(blockIdx.x) * rows;
  double s = 0.0;
  for (int i = threadIdx.x; i < rows; i += blockDim.x) s += a[base + i].re * b[base + i].re + a[base + i].im * b[base + i].im;
  s = block_sum(s, shared);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

__device__ __forceinline__ double step_length(double rz, double pq) {
  return (pq > 0.0 && isfinite(pq) && isfinite(rz)) ? rz / pq : 0.0;
}

// t += alpha p, res -= alpha q with alpha = rz / pq per column; with z given,
// also z = P(T, energy[j]) res for the next direction (one pass over res).
__global__ void cg_step_kernel(Cx<double>* __restrict__ t, Cx<double>* __restrict__ res, const Cx<double>* __restrict__ p,
                               const Cx<double>* __restrict__ q, int rows, const double* __restrict__ rz,
                               const double* __restrict__ pq, const double* __restrict__ kinetic,
                               const double* __restrict__ energy, Cx<double>* __restrict__ z) {
  const int j = blockIdx.y;
  const double alpha = step_length(rz[j], pq[j]);
  const double e = z ? energy[j] : 0.0;
  const long long base = static_cast<long long>(j) * rows;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    Cx<double> rv = res[base + i];
    if (alpha != 0.0) {
      const Cx<double> pv = p[base + i], qv = q[base + i], tv = t[base + i];
      t[base + i] = Cx<double>{tv.re + alpha * pv.re, tv.im + alpha * pv.im};
      rv = Cx<double>{rv.re - alpha * qv.re, rv.im - alpha * qv.im};
      res[base + i] = rv;
    }
    if (z) {
      const double scale = kinetic_preconditioner(kinetic[i], e);
      z[base + i] = Cx<double>{rv.re * scale, rv.im * scale};
    }
  }
}

// p = z + beta p with beta = rz_new / rz_old per column (0 when rz_old <= 0).
__global__ void cg_direction_kernel(Cx<double>* __restrict__ p, const Cx<double>* __restrict__ z, int rows,
                                    const double* __restrict__ rz_new, const double* __restrict__ rz_old) {
  const int j = blockIdx.y;
  const double beta = (rz_old[j] > 0.0 && isfinite(rz_new[j])) ? rz_new[j] / rz_old[j] : 0.0;
  const long long base = static_cast<long long>(j) * rows;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    const Cx<double> zv = z[base + i], pv = p[base + i];
    p[base + i] = Cx<double>{zv.re + beta * pv.re, zv.im + beta * pv.im};
  }
}

dim3 column_grid(int rows, int cols) {
  return dim3(static_cast<unsigned>(std::min<std::size_t>(ceil_div(rows, kThreads), 64)), static_cast<unsigned>(cols));
}

template <typename T>
T* as(Scratch& s, std::size_t count) {
  return static_cast<T*>(s.reserve(sizeof(T) * std::max<std::size_t>(count, 1)));
}

}  // namespace

void jacobi_davidson_corrections(DeviceOperator& op, CorrectionBuffers& buf, const Cx<double>* x,
                                 const Cx<double>* sx, const Cx<double>* r, const double* theta_all, int roots,
                                 const int* selected, int count, int steps, Cx<double>* out) {
  if (count <= 0) return;
  if (count > roots || steps < 1) throw InvalidArgument("invalid Jacobi-Davidson correction block");
  Context& ctx = op.context();
  const cudaStream_t st = ctx.stream;
  const int n = op.npw();
  const std::size_t block = static_cast<std::size_t>(n) * count;
  // Projections: BF16x3 products are ample for a search direction.
  const Split split = Split::BF16x3;
  const long long ld_rows = expanded_k(n, split), ld_cols = expanded_k(roots, split);
  PackedA xh{as<std::uint16_t>(buf.xh, static_cast<std::size_t>(ld_rows) * roots), ld_rows, roots, n, split};
  PackedA sxh{as<std::uint16_t>(buf.sxh, static_cast<std::size_t>(ld_rows) * roots), ld_rows, roots, n, split};
  PackedA xl{as<std::uint16_t>(buf.xl, static_cast<std::size_t>(ld_cols) * n), ld_cols, n, roots, split};
  PackedA sxl{as<std::uint16_t>(buf.sxl, static_cast<std::size_t>(ld_cols) * n), ld_cols, n, roots, split};
  pack_a(Op::C, x, n, roots, n, split, xh.data, ld_rows, st);
  pack_a(Op::C, sx, n, roots, n, split, sxh.data, ld_rows, st);
  pack_a(Op::N, x, n, n, roots, split, xl.data, ld_cols, st);
  pack_a(Op::N, sx, n, n, roots, split, sxl.data, ld_cols, st);

  Cx<double>* t = out;
  Cx<double>* res = as<Cx<double>>(buf.res, block);
  Cx<double>* z = as<Cx<double>>(buf.z, block);
  Cx<double>* p = as<Cx<double>>(buf.p, block);
  Cx<double>* hp = as<Cx<double>>(buf.hp, block);
  Cx<double>* coef = as<Cx<double>>(buf.coefficients, static_cast<std::size_t>(roots) * count);
  double* scalars = as<double>(buf.scalars, 5 * static_cast<std::size_t>(count));
  double* theta = scalars;
  double* energy = scalars + count;
  double* rz[2] = {scalars + 2 * count, scalars + 3 * count};
  double* pq = scalars + 4 * count;
  int* index = as<int>(buf.index, count);
  SDFT_CUDA(cudaMemcpyAsync(index, selected, sizeof(int) * count, cudaMemcpyHostToDevice, st));

  // v <- v - S X (X^H v) and v <- v - X ((S X)^H v).
  auto project_left = [&](Cx<double>* v) {
    gemm_tc(Op::C, roots, count, n, nullptr, 0, &xh, v, n, coef, roots, false, 1.0, split, ctx.tc, st);
    gemm_tc(Op::N, n, count, roots, nullptr, 0, &sxl, coef, roots, v, n, true, -1.0, split, ctx.tc, st);
  };
  auto project_right = [&](Cx<double>* v) {
    gemm_tc(Op::C, roots, count, n, nullptr, 0, &sxh, v, n, coef, roots, false, 1.0, split, ctx.tc, st);
    gemm_tc(Op::N, n, count, roots, nullptr, 0, &xl, coef, roots, v, n, true, -1.0, split, ctx.tc, st);
  };
  const dim3 grid = column_grid(n, count);
  auto precondition = [&]() {
    precondition_kernel<<<grid, kThreads, 0, st>>>(res, n, op.device_kinetic(), energy, z);
    SDFT_LAUNCH("precondition_kernel");
    project_right(z);
  };
  auto dots = [&](const Cx<double>* a, const Cx<double>* b, double* dst) {
    column_dots_kernel<<<count, kDotThreads, 0, st>>>(a, b, n, dst);
    SDFT_LAUNCH("column_dots_kernel");
  };

  setup_kernel<<<count, kThreads, 0, st>>>(x, n, n, op.device_kinetic(), theta_all, index, theta, energy);
  SDFT_LAUNCH("setup_kernel");
  gather_negated_kernel<<<grid, kThreads, 0, st>>>(r, n, n, index, res);
  SDFT_LAUNCH("gather_negated_kernel");
  project_left(res);
  zero_block(t, n, n, count, st);
  precondition();
  dots(res, z, rz[0]);
  copy_block(z, n, p, n, n, count, st);
  for (int step = 0; step < steps; ++step) {
    double* rz_old = rz[step & 1];
    double* rz_new = rz[(step + 1) & 1];
    op.apply_shifted(p, count, theta, hp, Precision::Mixed);  // (H - theta S) p
    project_left(hp);
    dots(p, hp, pq);
    const bool last = step + 1 == steps;
    cg_step_kernel<<<grid, kThreads, 0, st>>>(t, res, p, hp, n, rz_old, pq, op.device_kinetic(), energy,
                                              last ? nullptr : z);
    SDFT_LAUNCH("cg_step_kernel");
    if (last) break;
    project_right(z);
    dots(res, z, rz_new);
    cg_direction_kernel<<<grid, kThreads, 0, st>>>(p, z, n, rz_new, rz_old);
    SDFT_LAUNCH("cg_direction_kernel");
  }
}

}  // namespace sdft_b200
