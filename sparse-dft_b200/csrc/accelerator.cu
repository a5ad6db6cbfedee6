// Accelerator-style entry points on caller-owned host arrays (the reference's
// plugin boundary, src/compute_backend.hpp:64-89): the local Hamiltonian on a
// caller grid and the PAW chain with dense D/Q. Device copies of the immutable
// operands are cached by the caller's identity tokens.
#include <algorithm>
#include <cstring>
#include <limits>
#include <vector>

#include "operator.cuh"

namespace sdft_b200 {

namespace {
template <typename T>
T* as(Scratch& s, std::size_t count) {
  return static_cast<T*>(s.reserve(sizeof(T) * std::max<std::size_t>(count, 1)));
}

__global__ void demote_real_kernel(const double* __restrict__ src, float* __restrict__ dst, std::size_t n) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x)
    dst[i] = static_cast<float>(src[i]);
}
}  // namespace

void accelerator_local_hamiltonian(Context& ctx, const int shape[3], const std::uint64_t* indices, std::size_t npw,
                                   const double* kinetic, const double* potential, const double* input,
                                   std::size_t columns, double* output, Precision precision,
                                   std::uint64_t identity) {
  if (!columns || !npw || !indices || !kinetic || !potential || !input || !output)
    throw InvalidArgument("invalid accelerated FFT dimensions");
  for (int a = 0; a < 3; ++a)
    if (shape[a] <= 0) throw InvalidArgument("invalid accelerated FFT dimensions");
  const std::size_t count = static_cast<std::size_t>(shape[0]) * shape[1] * shape[2];
  if (columns > static_cast<std::size_t>(std::numeric_limits<int>::max()) || npw > count)
    throw Overflow("accelerated FFT dimensions exceed limits");
  auto& cache = ctx.accel;
  const cudaStream_t st = ctx.stream;
  const bool reuse = identity && cache.local_identity == identity && cache.shape[0] == shape[0] &&
                     cache.shape[1] == shape[1] && cache.shape[2] == shape[2] && cache.plan.npw == static_cast<int>(npw);
  if (!reuse) {
    cache.local_identity = 0;
    std::vector<std::uint64_t> idx(indices, indices + npw);
    for (auto i : idx)
      if (i >= count) throw InvalidArgument("accelerated FFT plane-wave index out of range");
    cache.plan.build(shape, idx, st);
    double* v64 = as<double>(cache.v64, count);
    float* v32 = as<float>(cache.v32, count);
    SDFT_CUDA(cudaMemcpyAsync(v64, potential, sizeof(double) * count, cudaMemcpyHostToDevice, st));
    demote_real_kernel<<<static_cast<unsigned>(std::min<std::size_t>(ceil_div(count, 256), 148 * 16)), 256, 0, st>>>(
        v64, v32, count);
    SDFT_LAUNCH("demote_real_kernel");
    for (int a = 0; a < 3; ++a) cache.shape[a] = shape[a];
    cache.local_identity = identity;
  }
  double* dkin = as<double>(cache.kinetic, npw);
  SDFT_CUDA(cudaMemcpyAsync(dkin, kinetic, sizeof(double) * npw, cudaMemcpyHostToDevice, st));
  const std::size_t n = npw * columns;
  auto* x = static_cast<Cx<double>*>(ctx.staging_in.reserve(sizeof(Cx<double>) * n));
  auto* y = static_cast<Cx<double>*>(ctx.staging_out.reserve(sizeof(Cx<double>) * n));
  SDFT_CUDA(cudaMemcpyAsync(x, input, sizeof(Cx<double>) * n, cudaMemcpyHostToDevice, st));
  if (precision == Precision::FP64) {
    auto* slab = static_cast<Cx<double>*>(ctx.slab64.reserve(sizeof(Cx<double>) * cache.plan.slab_elements(columns)));
    local_hamiltonian<double>(cache.plan, x, static_cast<long long>(npw), static_cast<int>(columns),
                              static_cast<const double*>(cache.v64.ptr), dkin, y, static_cast<long long>(npw), slab, st);
  } else {
    auto* slab = static_cast<Cx<float>*>(ctx.slab32.reserve(sizeof(Cx<float>) * cache.plan.slab_elements(columns)));
    local_hamiltonian<float>(cache.plan, x, static_cast<long long>(npw), static_cast<int>(columns),
                             static_cast<const float*>(cache.v32.ptr), dkin, y, static_cast<long long>(npw), slab, st);
  }
  SDFT_CUDA(cudaMemcpyAsync(output, y, sizeof(Cx<double>) * n, cudaMemcpyDeviceToHost, st));
  ctx.synchronize();
}

void accelerator_paw_pair(Context& ctx, std::uint64_t identity, std::size_t npw, std::size_t np,
                          std::size_t columns, const double* b, const double* d, const double* q, const double* input,
                          double* h, double* s, Precision precision, std::uint64_t projector_identity) {
  if (!identity || !npw || !np || !columns || !b || !d || !q || !input || !h || !s)
    throw InvalidArgument("invalid CUDA PAW chain shape");
  if (std::max({npw, np, columns}) > static_cast<std::size_t>(std::numeric_limits<int>::max()))
    throw InvalidArgument("invalid CUDA PAW chain shape");
  auto& c = ctx.accel;
  const cudaStream_t st = ctx.stream;
  const int inpw = static_cast<int>(npw), inp = static_cast<int>(np), icols = static_cast<int>(columns);
  const bool reuse_b = projector_identity && c.projector_identity == projector_identity && c.npw == inpw &&
                       c.projectors == inp;
  const bool reuse_d = reuse_b && c.onsite_identity == identity;
  auto* db = static_cast<Cx<double>*>(c.b.reserve(sizeof(Cx<double>) * npw * np));
  if (!reuse_b) {
    c.projector_identity = 0;
    SDFT_CUDA(cudaMemcpyAsync(db, b, sizeof(Cx<double>) * npw * np, cudaMemcpyHostToDevice, st));
    release(c.b_packed);
    release(c.bh_packed);
    c.npw = inpw;
    c.projectors = inp;
  }
  if (precision == Precision::Mixed && !c.b_packed.data) {
    const Split split = search_split();
    pack_persistent(Op::N, db, inp, inp, inpw, split, c.b_packed, st);
    pack_persistent(Op::C, db, inp, inpw, inp, split, c.bh_packed, st);
  }
  auto* dd = static_cast<Cx<double>*>(c.d.reserve(sizeof(Cx<double>) * np * np));
  auto* dq = static_cast<Cx<double>*>(c.q.reserve(sizeof(Cx<double>) * np * np));
  if (!reuse_d) {
    SDFT_CUDA(cudaMemcpyAsync(dd, d, sizeof(Cx<double>) * np * np, cudaMemcpyHostToDevice, st));
    SDFT_CUDA(cudaMemcpyAsync(dq, q, sizeof(Cx<double>) * np * np, cudaMemcpyHostToDevice, st));
  }
  const std::size_t n = npw * columns;
  auto* x = static_cast<Cx<double>*>(ctx.staging_in.reserve(sizeof(Cx<double>) * n));
  auto* hy = static_cast<Cx<double>*>(ctx.staging_out.reserve(sizeof(Cx<double>) * n));
  auto* sy = static_cast<Cx<double>*>(ctx.staging_aux.reserve(sizeof(Cx<double>) * n));
  auto* p = static_cast<Cx<double>*>(ctx.projections.reserve(sizeof(Cx<double>) * 3 * np * columns));
  Cx<double>* dp = p + np * columns;
  Cx<double>* qp = dp + np * columns;
  SDFT_CUDA(cudaMemcpyAsync(x, input, sizeof(Cx<double>) * n, cudaMemcpyHostToDevice, st));
  const bool mixed = precision == Precision::Mixed;
  if (mixed)
    gemm_tc(Op::N, inp, icols, inpw, db, inp, &c.b_packed, x, inpw, p, inp, false, 1.0, c.b_packed.split, ctx.tc, st);
  else
    zgemm(ctx.blas, Op::N, Op::N, inp, icols, inpw, db, inp, x, inpw, p, inp, false);
  zgemm(ctx.blas, Op::N, Op::N, inp, icols, inp, dd, inp, p, inp, dp, inp, false);
  zgemm(ctx.blas, Op::N, Op::N, inp, icols, inp, dq, inp, p, inp, qp, inp, false);
  if (mixed) {
    gemm_tc(Op::C, inpw, icols, inp, db, inp, &c.bh_packed, dp, inp, hy, inpw, false, 1.0, c.bh_packed.split, ctx.tc, st);
    gemm_tc(Op::C, inpw, icols, inp, db, inp, &c.bh_packed, qp, inp, sy, inpw, false, 1.0, c.bh_packed.split, ctx.tc, st);
  } else {
    zgemm(ctx.blas, Op::C, Op::N, inpw, icols, inp, db, inp, dp, inp, hy, inpw, false);
    zgemm(ctx.blas, Op::C, Op::N, inpw, icols, inp, db, inp, qp, inp, sy, inpw, false);
  }
  SDFT_CUDA(cudaMemcpyAsync(h, hy, sizeof(Cx<double>) * n, cudaMemcpyDeviceToHost, st));
  SDFT_CUDA(cudaMemcpyAsync(s, sy, sizeof(Cx<double>) * n, cudaMemcpyDeviceToHost, st));
  ctx.synchronize();
  c.projector_identity = projector_identity;
  c.onsite_identity = identity;
  if (umma_error_flag()) throw CudaError("tensor-core GEMM wait limit exceeded");
}

}  // namespace sdft_b200
