// Residual-minimisation trial for SCF warm solves on the device: the
// reference's solve_generalized_hermitian_rmm_trial (src/rmm_trial.cpp:128-206,
// selected by SDFT_SCF_RMM_TRIAL=1 for SCF warm requests,
// src/pw_core.cpp:558-563). At most min(16, max_iterations/2) steps, each:
//   roots x roots generalized rotation of the block and of the previous
//   directions (src/rmm_trial.cpp:57-80, :153-156);
//   Rayleigh quotients and residuals (:99-117); at residual <= tolerance a
//   fresh FP64 application and S-orthonormality within 1e-10 end the trial
//   as a residual-checked, explicitly not converged manifold (:158-170);
//   kinetically preconditioned directions, applied in FP64 for tolerances
//   below 1e-6 and in the mixed form otherwise (:171-176);
//   two projections of the directions and of the previous directions out of
//   the block, S-normalisation (:82-97, :176-178);
//   per band the 2 x 2 least-squares combination of the two directions that
//   minimises ||r - e_j (S d) + (H d)||, skipped when singular or large
//   (:179-199); S-normalisation and a rank check of the new block (:200-201).
// Any failed step, or the step limit, hands the current block (or the
// initial one) to the Davidson solver with the remaining iterations (:136-146).
#include <algorithm>
#include <cmath>

#include "dense.cuh"
#include "eigensolver.cuh"
#include "rmm_trial.cuh"

namespace sdft_b200 {

namespace {

constexpr int kThreads = 256;

// v(:, j) *= 1/sqrt(metric[j]) for x, h, s when metric[j] > 1e-28 and
// finite, else the three columns are zeroed (src/rmm_trial.cpp:91-97).
__global__ void normalize_images_kernel(Cx<double>* x, Cx<double>* h, Cx<double>* s, int rows,
                                        const double* __restrict__ metric) {
  const int j = blockIdx.y;
  const double m = metric[j];
  const bool keep = m > 1e-28 && isfinite(m);
  const double scale = keep ? 1.0 / sqrt(m) : 0.0;
  const std::size_t base = static_cast<std::size_t>(j) * rows;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    for (Cx<double>* v : {x, h, s}) {
      const Cx<double> a = v[base + i];
      v[base + i] = keep ? Cx<double>{a.re * scale, a.im * scale} : Cx<double>{0.0, 0.0};
    }
  }
}

struct Sum {
  double hi, lo;
};

__device__ __forceinline__ Sum sum_add(Sum a, double b) {
  const double s = a.hi + b;
  const double bb = s - a.hi;
  const double e = (a.hi - (s - bb)) + (b - bb);
  return {s, a.lo + e};
}

// Per band j (one CTA): corrections c0 = Hd - e_j Sd and c1 = Hp - e_j Sp
// (zero without previous directions), the Gram matrix C^H C and C^H r
// (compensated sums), then the scaled, regularised 2 x 2 solve
// (src/rmm_trial.cpp:179-193): coefficients and an ok flag per band.
__global__ void __launch_bounds__(kThreads) band_minimize_kernel(const Cx<double>* dh, const Cx<double>* ds,
                                                                 const Cx<double>* ph, const Cx<double>* ps,
                                                                 const Cx<double>* r, int rows,
                                                                 const double* values, bool previous,
                                                                 Cx<double>* coeff, int* ok) {
  const int j = blockIdx.x;
  const double e = values[j];
  const std::size_t base = static_cast<std::size_t>(j) * rows;
  // g00, Re g01, Im g01, g11, Re b0, Im b0, Re b1, Im b1
  Sum acc[8];
  for (auto& a : acc) a = Sum{0.0, 0.0};
  for (int i = threadIdx.x; i < rows; i += kThreads) {
    const Cx<double> a = dh[base + i], b = ds[base + i], res = r[base + i];
    const Cx<double> c0{a.re - e * b.re, a.im - e * b.im};
    Cx<double> c1{0.0, 0.0};
    if (previous) {
      const Cx<double> pa = ph[base + i], pb = ps[base + i];
      c1 = Cx<double>{pa.re - e * pb.re, pa.im - e * pb.im};
    }
    acc[0] = sum_add(acc[0], c0.re * c0.re + c0.im * c0.im);
    acc[1] = sum_add(acc[1], c0.re * c1.re + c0.im * c1.im);  // conj(c0) c1
    acc[2] = sum_add(acc[2], c0.re * c1.im - c0.im * c1.re);
    acc[3] = sum_add(acc[3], c1.re * c1.re + c1.im * c1.im);
    acc[4] = sum_add(acc[4], c0.re * res.re + c0.im * res.im);  // conj(c0) r
    acc[5] = sum_add(acc[5], c0.re * res.im - c0.im * res.re);
    acc[6] = sum_add(acc[6], c1.re * res.re + c1.im * res.im);  // conj(c1) r
    acc[7] = sum_add(acc[7], c1.re * res.im - c1.im * res.re);
  }
  __shared__ double shared[8][kThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < 8; ++k) {
    double v = acc[k].hi + acc[k].lo;
    for (int offset = 16; offset > 0; offset /= 2) v += __shfl_down_sync(0xffffffffu, v, offset);
    if (lane == 0) shared[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double t[8];
  for (int k = 0; k < 8; ++k) {
    double v = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) v += shared[k][w];
    t[k] = v;
  }
  double g00 = t[0], g11 = t[3];
  Cx<double> g01{t[1], t[2]};
  const double scale = fmax(g00, g11);
  ok[j] = 0;
  coeff[2 * j] = Cx<double>{0.0, 0.0};
  coeff[2 * j + 1] = Cx<double>{0.0, 0.0};
  if (!(scale > 0) || !isfinite(scale)) return;
  g00 = g00 / scale + 1e-14;
  g11 = g11 / scale + 1e-14;
  g01 = Cx<double>{g01.re / scale, g01.im / scale};
  const Cx<double> b0{-t[4] / scale, -t[5] / scale}, b1{-t[6] / scale, -t[7] / scale};
  // LDL^H of [[g00, g01], [conj g01, g11]] with the larger diagonal first.
  Cx<double> x0, x1;
  if (g00 >= g11) {
    const Cx<double> l{g01.re / g00, -g01.im / g00};  // conj(g01) / g00
    const double d1 = g11 - (g01.re * g01.re + g01.im * g01.im) / g00;
    const Cx<double> y1{b1.re - (l.re * b0.re - l.im * b0.im), b1.im - (l.re * b0.im + l.im * b0.re)};
    x1 = Cx<double>{y1.re / d1, y1.im / d1};
    // x0 = b0 / g00 - conj(l) x1
    x0 = Cx<double>{b0.re / g00 - (l.re * x1.re + l.im * x1.im), b0.im / g00 - (l.re * x1.im - l.im * x1.re)};
  } else {
    const Cx<double> l{g01.re / g11, g01.im / g11};  // g01 / g11
    const double d0 = g00 - (g01.re * g01.re + g01.im * g01.im) / g11;
    const Cx<double> y0{b0.re - (l.re * b1.re - l.im * b1.im), b0.im - (l.re * b1.im + l.im * b1.re)};
    x0 = Cx<double>{y0.re / d0, y0.im / d0};
    // x1 = b1 / g11 - conj(l) x0
    x1 = Cx<double>{b1.re / g11 - (l.re * x0.re + l.im * x0.im), b1.im / g11 - (l.re * x0.im - l.im * x0.re)};
  }
  const double largest = fmax(fmax(fabs(x0.re), fabs(x0.im)), fmax(fabs(x1.re), fabs(x1.im)));
  if (!isfinite(largest) || hypot(x0.re, x0.im) > 1e6 || hypot(x1.re, x1.im) > 1e6) return;
  coeff[2 * j] = x0;
  coeff[2 * j + 1] = x1;
  ok[j] = 1;
}

// next = x + c0 d + c1 p per band with an ok flag, else next = x (x, h, s).
__global__ void band_update_kernel(const Cx<double>* x, const Cx<double>* xh, const Cx<double>* xs,
                                   const Cx<double>* d, const Cx<double>* dh, const Cx<double>* ds,
                                   const Cx<double>* p, const Cx<double>* ph, const Cx<double>* ps, bool previous,
                                   int rows, const Cx<double>* coeff, const int* ok, Cx<double>* nx, Cx<double>* nh,
                                   Cx<double>* ns) {
  const int j = blockIdx.y;
  const bool use = ok[j] != 0;
  const Cx<double> c0 = coeff[2 * j], c1 = coeff[2 * j + 1];
  const std::size_t base = static_cast<std::size_t>(j) * rows;
  const Cx<double>* src[3] = {x, xh, xs};
  const Cx<double>* dir[3] = {d, dh, ds};
  const Cx<double>* prev[3] = {p, ph, ps};
  Cx<double>* dst[3] = {nx, nh, ns};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += gridDim.x * blockDim.x) {
    for (int b = 0; b < 3; ++b) {
      Cx<double> v = src[b][base + i];
      if (use) {
        const Cx<double> a = dir[b][base + i];
        v = Cx<double>{v.re + (c0.re * a.re - c0.im * a.im), v.im + (c0.re * a.im + c0.im * a.re)};
        if (previous) {
          const Cx<double> q = prev[b][base + i];
          v = Cx<double>{v.re + (c1.re * q.re - c1.im * q.im), v.im + (c1.re * q.im + c1.im * q.re)};
        }
      }
      dst[b][base + i] = v;
    }
  }
}

__global__ void nonfinite_kernel(const Cx<double>* a, std::size_t count, int* flag) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x)
    if (!isfinite(a[i].re) || !isfinite(a[i].im)) *flag = 1;
}

}  // namespace

void RmmTrial::apply(Images& v, bool exact) {
  auto& ctx = op_.context();
  op_.apply_pair(v.x, k_, v.h, v.s, exact ? Precision::FP64 : Precision::Mixed);
  SDFT_CUDA(cudaMemsetAsync(flags_ + k_, 0, sizeof(int), ctx.stream));
  const std::size_t count = static_cast<std::size_t>(n_) * k_;
  const unsigned grid = static_cast<unsigned>(std::min<std::size_t>(ceil_div(count, kThreads), 148 * 8));
  for (const Cx<double>* a : {v.x, v.h, v.s}) {
    nonfinite_kernel<<<grid, kThreads, 0, ctx.stream>>>(a, count, flags_ + k_);
    SDFT_LAUNCH("nonfinite_kernel");
  }
  int bad = 0;
  SDFT_CUDA(cudaMemcpyAsync(&bad, flags_ + k_, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.synchronize();
  if (bad) throw std::runtime_error("nonfinite RMM original operator output");
}

// Gram X^H S X of the block: finite eigenvalues with the smallest above
// 1e-13 max(1, largest) (src/rmm_trial.cpp:76-81).
bool RmmTrial::full_rank(const Images& v) {
  auto& ctx = op_.context();
  zgemm(ctx.blas, Op::C, Op::N, k_, k_, n_, v.x, n_, v.s, n_, ss_, k_, false);
  hermitian_part(ss_, k_, hs_, k_, k_, ctx.stream);
  hermitian_lowest(ctx.blas, hs_, k_, k_, values_, hs_, eigen_, ctx.stream);
  std::vector<double> values(k_);
  SDFT_CUDA(cudaMemcpyAsync(values.data(), values_, sizeof(double) * k_, cudaMemcpyDeviceToHost, ctx.stream));
  ctx.synchronize();
  for (double e : values)
    if (!std::isfinite(e)) return false;
  return values.front() > 1e-13 * std::max(1.0, values.back());
}

void RmmTrial::rotate(Images& v, const Cx<double>* u, Images& spare) {
  auto& ctx = op_.context();
  zgemm(ctx.blas, Op::N, Op::N, n_, k_, k_, v.x, n_, u, k_, spare.x, n_, false);
  zgemm(ctx.blas, Op::N, Op::N, n_, k_, k_, v.h, n_, u, k_, spare.h, n_, false);
  zgemm(ctx.blas, Op::N, Op::N, n_, k_, k_, v.s, n_, u, k_, spare.s, n_, false);
  std::swap(v, spare);
}

void RmmTrial::project(Images& d, const Images& x) {
  auto& ctx = op_.context();
  for (int pass = 0; pass < 2; ++pass) {
    zgemm(ctx.blas, Op::C, Op::N, k_, k_, n_, x.x, n_, d.s, n_, u_, k_, false);
    zgemm(ctx.blas, Op::N, Op::N, n_, k_, k_, x.x, n_, u_, k_, d.x, n_, true, -1.0);
    zgemm(ctx.blas, Op::N, Op::N, n_, k_, k_, x.h, n_, u_, k_, d.h, n_, true, -1.0);
    zgemm(ctx.blas, Op::N, Op::N, n_, k_, k_, x.s, n_, u_, k_, d.s, n_, true, -1.0);
  }
}

void RmmTrial::normalize(Images& v) {
  auto& ctx = op_.context();
  metric_norms(v.x, v.s, n_, n_, k_, metric_, ctx.stream);
  const dim3 grid(static_cast<unsigned>(std::min<long long>(ceil_div(n_, kThreads), 64)), static_cast<unsigned>(k_));
  normalize_images_kernel<<<grid, kThreads, 0, ctx.stream>>>(v.x, v.h, v.s, n_, metric_);
  SDFT_LAUNCH("normalize_images_kernel");
}

double RmmTrial::residual(const Images& v) {
  auto& ctx = op_.context();
  rayleigh_certificate(v.x, v.h, v.s, n_, n_, k_, values_, metric_, r_, norms_, ctx.stream);
  host_values_.resize(k_);
  host_norms_.resize(k_);
  std::vector<double> metric(k_);
  SDFT_CUDA(cudaMemcpyAsync(host_values_.data(), values_, sizeof(double) * k_, cudaMemcpyDeviceToHost, ctx.stream));
  SDFT_CUDA(cudaMemcpyAsync(host_norms_.data(), norms_, sizeof(double) * k_, cudaMemcpyDeviceToHost, ctx.stream));
  SDFT_CUDA(cudaMemcpyAsync(metric.data(), metric_, sizeof(double) * k_, cudaMemcpyDeviceToHost, ctx.stream));
  ctx.synchronize();
  double maximum = 0;
  for (int j = 0; j < k_; ++j) {
    if (!(metric[j] > 0)) throw std::runtime_error("RMM nonpositive wavefunction metric");
    maximum = std::max(maximum, host_norms_[j]);
  }
  return maximum;
}

RmmResult RmmTrial::solve(const DavidsonOptions& options, const Cx<double>* initial) {
  const int n = op_.npw(), k = options.roots;
  const double tolerance = options.tolerance;
  if (!initial || !(tolerance > 1e-9) || !std::isfinite(tolerance) || k < 1 || k > n || options.max_iterations < 1)
    throw InvalidArgument("RMM trial requires a coarse explicit SCF warm request with physical kinetic energies");
  for (double t : op_.kinetic())
    if (!std::isfinite(t) || t < 0) throw InvalidArgument("invalid RMM kinetic diagonal");
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(op_.h_diagonal()[i]) || !std::isfinite(op_.s_diagonal()[i]) || op_.s_diagonal()[i] <= 0)
      throw InvalidArgument("invalid RMM H/S diagonals");
  auto& ctx = op_.context();
  SDFT_CUDA(cudaSetDevice(ctx.device));
  n_ = n;
  k_ = k;
  const std::size_t block = static_cast<std::size_t>(n) * k;
  auto* base = static_cast<Cx<double>*>(blocks_.reserve(sizeof(Cx<double>) * block * 13));
  auto take = [&](int i) { return base + block * i; };
  Images x{take(0), take(1), take(2)}, d{take(3), take(4), take(5)}, p{take(6), take(7), take(8)},
      spare{take(9), take(10), take(11)};
  r_ = take(12);
  const std::size_t kk = static_cast<std::size_t>(k) * k;
  auto* small = static_cast<Cx<double>*>(small_.reserve(sizeof(Cx<double>) * (3 * kk + 2 * k)));
  hs_ = small;
  ss_ = small + kk;
  u_ = small + 2 * kk;
  coeff_ = small + 3 * kk;
  auto* sc = static_cast<double*>(scalars_.reserve(sizeof(double) * 3 * k + sizeof(int) * (k + 2)));
  values_ = sc;
  metric_ = sc + k;
  norms_ = sc + 2 * k;
  flags_ = reinterpret_cast<int*>(sc + 3 * k);

  RmmResult result;
  int used = 0;
  bool have_vectors = false;  // x.x holds a completed step's block
  auto fallback = [&](const Cx<double>* guess) {
    DavidsonOptions rest = options;
    rest.max_iterations = options.max_iterations - used;
    fallback_.solve(rest, guess);
    RmmResult out;
    out.eigenvalues = fallback_.eigenvalues();
    out.residuals = fallback_.residuals();
    out.fallback_stats = fallback_.stats();
    out.iterations = fallback_.stats().iterations + used;
    out.trial_steps = used;
    out.converged = fallback_.stats().converged;
    out.fell_back = true;
    vectors_ = fallback_.vectors();
    return out;
  };
  const int limit = std::min(16, options.max_iterations / 2);
  if (!limit) return fallback(initial);
  copy_block(initial, n, x.x, n, n, k, ctx.stream);
  apply(x, true);
  if (!full_rank(x)) return fallback(initial);
  bool previous = false;
  for (int step = 0; step < limit; ++step) {
    ++used;
    // Global rotation of the block (and of the previous directions).
    zgemm(ctx.blas, Op::C, Op::N, k, k, n, x.x, n, x.h, n, u_, k, false);
    hermitian_part(u_, k, hs_, k, k, ctx.stream);
    zgemm(ctx.blas, Op::C, Op::N, k, k, n, x.x, n, x.s, n, u_, k, false);
    hermitian_part(u_, k, ss_, k, k, ctx.stream);
    generalized_lowest(ctx.blas, ctx.solver, hs_, ss_, k, k, values_, u_, eigen_, rr_mode(), ctx.stream);
    rotate(x, u_, spare);
    if (previous) rotate(p, u_, spare);
    double maximum = residual(x);
    if (maximum <= tolerance) {
      // Fresh FP64 original operators, independent of all reused images.
      apply(x, true);
      const double fresh = residual(x);
      zgemm(ctx.blas, Op::C, Op::N, k, k, n, x.x, n, x.s, n, hs_, k, false);
      const double gram_error = identity_deviation(hs_, k, eigen_, ctx.stream);
      if (fresh <= tolerance && gram_error <= 1e-10) {
        result.eigenvalues = host_values_;
        result.residuals = host_norms_;
        result.iterations = used;
        result.trial_steps = used;
        result.trial_manifold = true;
        vectors_ = x.x;
        return result;
      }
    }
    kinetic_precondition(r_, x.x, n, n, k, op_.device_kinetic(), d.x, n, ctx.stream);
    apply(d, tolerance < 1e-6);
    project(d, x);
    normalize(d);
    if (previous) {
      project(p, x);
      normalize(p);
    }
    band_minimize_kernel<<<k, kThreads, 0, ctx.stream>>>(d.h, d.s, p.h, p.s, r_, n, values_, previous, coeff_,
                                                         flags_);
    SDFT_LAUNCH("band_minimize_kernel");
    const dim3 grid(static_cast<unsigned>(std::min<long long>(ceil_div(n, kThreads), 64)), static_cast<unsigned>(k));
    band_update_kernel<<<grid, kThreads, 0, ctx.stream>>>(x.x, x.h, x.s, d.x, d.h, d.s, p.x, p.h, p.s, previous, n,
                                                          coeff_, flags_, spare.x, spare.h, spare.s);
    SDFT_LAUNCH("band_update_kernel");
    normalize(spare);
    if (!full_rank(spare)) break;
    std::swap(x, spare);  // x = next
    std::swap(p, d);      // previous = d
    previous = true;
    have_vectors = true;
  }
  return fallback(have_vectors ? x.x : initial);
}

}  // namespace sdft_b200
