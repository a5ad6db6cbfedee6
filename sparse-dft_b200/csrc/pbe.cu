// Spin-unpolarised PBE exchange-correlation per grid point in FP64 on
// caller arrays (the reference's accelerated_pbe_points,
// src/compute_backend.hpp:46-47); the point arithmetic is pbe.cuh.
#include <algorithm>

#include "operator.cuh"
#include "pbe.cuh"

namespace sdft_b200 {

namespace {

using pbe::Point;
using pbe::pbe_point;

__global__ void pbe_points_kernel(const double* __restrict__ density, const double* __restrict__ gradient,
                                  std::size_t count, double* __restrict__ out, unsigned int* __restrict__ flags) {
  for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const double n = density[i], g = gradient[i];
    double* o = out + 7 * i;
    if (!(n > 0.0) || !isfinite(n) || g < 0.0 || !isfinite(g)) {
      atomicOr(flags, 1u);
      for (int q = 0; q < 7; ++q) o[q] = 0.0;
      continue;
    }
    const Point p = pbe_point(n, g);
    o[0] = p.energy;
    o[1] = p.energy / n;
    o[2] = p.exchange_energy;
    o[3] = p.correlation_energy;
    o[4] = p.vx;
    o[5] = p.vc;
    o[6] = p.sigma;
    if (!isfinite(p.energy) || !isfinite(p.vx) || !isfinite(p.vc) || !isfinite(p.sigma)) atomicOr(flags, 2u);
  }
}

}  // namespace

void pbe_points(Context& ctx, const double* density, const double* gradient, std::size_t count, double* out) {
  if (!count) throw InvalidArgument("invalid GPU PBE dimensions");
  auto* flags = static_cast<unsigned int*>(ctx.onsite.reserve(sizeof(unsigned int)));
  SDFT_CUDA(cudaMemsetAsync(flags, 0, sizeof(unsigned int), ctx.stream));
  const unsigned grid = static_cast<unsigned>(std::min<std::size_t>(ceil_div(count, 256), 148ULL * 32));
  pbe_points_kernel<<<grid, 256, 0, ctx.stream>>>(density, gradient, count, out, flags);
  SDFT_LAUNCH("pbe_points_kernel");
  unsigned int host = 0;
  SDFT_CUDA(cudaMemcpyAsync(&host, flags, sizeof(host), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.synchronize();
  if (host & 1u) throw InvalidArgument("invalid GPU PBE point");
  if (host & 2u) throw NonFinite("nonfinite CUDA PBE output");
}

}  // namespace sdft_b200
