// Band density Sum_b f_b/Omega |psi_b(r)|^2 and its Fourier coefficients on a
// support (src/density_functionals.cpp:407-460), as three pruned FP64 passes
// over all occupied bands followed by one forward 3D FFT:
//
//   rows     (per active i0 row, block of active i1 rows, band): scatter the
//            sphere points into shared memory, backward FFT along i2, store
//            only the active (i0, i1) rows.
//   columns  (per active i0 row, 32 i2 columns, band): zero-pad the active i1
//            entries to n1, backward FFT along i1, store the i0 plane.
//   pencils  (per 32 (i1, i2) lines, looping over the bands): zero-pad the
//            active i0 entries to n0, backward FFT along i0 and accumulate
//            f_b/Omega |.|^2 in shared memory in band order; the density
//            line is written once.
//
// The density grid is then transformed forward in place (unnormalised) and
// the support keys gathered and divided by N (src/density_functionals.cpp:269-284).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <unordered_set>

#include "band_density.cuh"
#include "operator.cuh"

namespace sdft_b200 {

namespace {

constexpr int kThreads = 256;
constexpr std::size_t kSmemLimit = 220 * 1024;
// Slab bytes (both intermediate passes) held at once; bands beyond it are
// processed in further chunks that accumulate into the same density grid.
// SDFT_B200_DENSITY_SLAB_BYTES lowers it (tests use it to force chunking).
std::size_t slab_budget() {
  std::size_t budget = std::size_t(4) << 30;
  if (const char* text = std::getenv("SDFT_B200_DENSITY_SLAB_BYTES")) {
    char* end = nullptr;
    const unsigned long long value = std::strtoull(text, &end, 10);
    if (!*text || *end || value == 0) throw InvalidArgument("SDFT_B200_DENSITY_SLAB_BYTES must be a positive integer");
    budget = std::min<std::size_t>(budget, value);
  }
  return budget;
}

struct DensityArgs {
  int n0, n1, n2, slots, krows;
  long long n12;
  const int* slot_row;
  const int* point_offset;
  const int* point_g;
  const int* point_compact;
  const int* krow;
  const int* band;       // occupied band index per slab band
  const double* weight;  // f_b / Omega per slab band
  LinePlan p0, p1, p2;
  const Cx<double>* tw0;
  const Cx<double>* tw1;
  const Cx<double>* tw2;
};

__global__ void __launch_bounds__(kThreads) density_rows_kernel(const Cx<double>* __restrict__ psi, long long npw,
                                                                DensityArgs a, int rows_per_cta,
                                                                Cx<double>* __restrict__ rows_out,
                                                                unsigned int* __restrict__ flags) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int n2 = a.n2, n2p = n2 | 1;
  Cx<double>* tw = reinterpret_cast<Cx<double>*>(smem_raw);
  Cx<double>* buf_a = tw + n2;
  const int s = blockIdx.x, r0 = blockIdx.y * rows_per_cta, b = blockIdx.z;
  const int rows = min(rows_per_cta, a.krows - r0);
  Cx<double>* buf_b = buf_a + rows_per_cta * n2p;
  const int tid = threadIdx.x;
  for (int i = tid; i < n2; i += blockDim.x) tw[i] = a.tw2[i];
  for (int i = tid; i < rows * n2p; i += blockDim.x) buf_a[i] = Cx<double>{0.0, 0.0};
  __syncthreads();
  const Cx<double>* column = psi + static_cast<long long>(a.band[b]) * npw;
  const int p_end = a.point_offset[s + 1];
  bool finite = true;
  for (int p = a.point_offset[s] + tid; p < p_end; p += blockDim.x) {
    const int pc = a.point_compact[p];
    const int k = pc / n2;
    if (k < r0 || k >= r0 + rows) continue;
    const Cx<double> v = column[a.point_g[p]];
    finite = finite && isfinite(v.re) && isfinite(v.im);
    buf_a[(k - r0) * n2p + (pc - k * n2)] = v;
  }
  if (!finite) atomicOr(flags, 1u);
  __syncthreads();
  const Cx<double>* done = fft_lines_pp<double, true>(buf_a, buf_b, rows, n2p, 1, nullptr, a.p2, tw);
  Cx<double>* out = rows_out + ((static_cast<long long>(b) * a.slots + s) * a.krows + r0) * n2;
  for (int i = tid; i < rows * n2; i += blockDim.x) {
    const int r = i / n2, e = i - r * n2;
    out[i] = done[r * n2p + e];
  }
}

template <int TL>
__global__ void __launch_bounds__(kThreads) density_columns_kernel(const Cx<double>* __restrict__ rows_in,
                                                                   DensityArgs a, Cx<double>* __restrict__ planes) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int STRIDE = TL + 1;
  Cx<double>* tw = reinterpret_cast<Cx<double>*>(smem_raw);
  Cx<double>* tile_a = tw + a.n1;
  Cx<double>* tile_b = tile_a + a.n1 * STRIDE;
  const int i20 = blockIdx.x * TL, s = blockIdx.y, b = blockIdx.z;
  const int lines = min(TL, a.n2 - i20);
  const int tid = threadIdx.x;
  for (int i = tid; i < a.n1; i += blockDim.x) tw[i] = a.tw1[i];
  for (int i = tid; i < a.n1 * STRIDE; i += blockDim.x) tile_a[i] = Cx<double>{0.0, 0.0};
  __syncthreads();
  const long long sb = static_cast<long long>(b) * a.slots + s;
  const Cx<double>* in = rows_in + sb * a.krows * a.n2 + i20;
  for (int idx = tid; idx < a.krows * TL; idx += blockDim.x) {
    const int k = idx / TL, t = idx - k * TL;
    if (t < lines) tile_a[a.krow[k] * STRIDE + t] = in[static_cast<long long>(k) * a.n2 + t];
  }
  __syncthreads();
  const Cx<double>* done = fft_lines_pp<double, true>(tile_a, tile_b, lines, 1, STRIDE, nullptr, a.p1, tw);
  Cx<double>* out = planes + sb * a.n12 + i20;
  for (int idx = tid; idx < a.n1 * TL; idx += blockDim.x) {
    const int i = idx / TL, t = idx - i * TL;
    if (t < lines) out[static_cast<long long>(i) * a.n2 + t] = done[i * STRIDE + t];
  }
}

template <int TL>
__global__ void __launch_bounds__(kThreads) density_pencils_kernel(const Cx<double>* __restrict__ planes,
                                                                   DensityArgs a, int bands, bool accumulate,
                                                                   Cx<double>* __restrict__ grid) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int STRIDE = TL + 1;
  Cx<double>* tw = reinterpret_cast<Cx<double>*>(smem_raw);
  Cx<double>* tile_a = tw + a.n0;
  Cx<double>* tile_b = tile_a + a.n0 * STRIDE;
  double* acc = reinterpret_cast<double*>(tile_b + a.n0 * STRIDE);
  const long long kl0 = static_cast<long long>(blockIdx.x) * TL;
  const int lines = static_cast<int>(min(static_cast<long long>(TL), a.n12 - kl0));
  const int tid = threadIdx.x;
  for (int i = tid; i < a.n0; i += blockDim.x) tw[i] = a.tw0[i];
  for (int idx = tid; idx < a.n0 * TL; idx += blockDim.x) {
    const int i = idx / TL, t = idx - i * TL;
    acc[idx] = accumulate && t < lines ? grid[static_cast<long long>(i) * a.n12 + kl0 + t].re : 0.0;
  }
  for (int b = 0; b < bands; ++b) {
    const double w = a.weight[b];
    for (int i = tid; i < a.n0 * STRIDE; i += blockDim.x) tile_a[i] = Cx<double>{0.0, 0.0};
    __syncthreads();
    const Cx<double>* base = planes + static_cast<long long>(b) * a.slots * a.n12 + kl0;
    for (int idx = tid; idx < a.slots * TL; idx += blockDim.x) {
      const int s = idx / TL, t = idx - s * TL;
      if (t < lines) tile_a[a.slot_row[s] * STRIDE + t] = base[static_cast<long long>(s) * a.n12 + t];
    }
    __syncthreads();
    const Cx<double>* field = fft_lines_pp<double, true>(tile_a, tile_b, lines, 1, STRIDE, nullptr, a.p0, tw);
    for (int idx = tid; idx < a.n0 * TL; idx += blockDim.x) {
      const int i = idx / TL, t = idx - i * TL;
      if (t < lines) {
        const Cx<double> v = field[i * STRIDE + t];
        acc[idx] += w * (v.re * v.re + v.im * v.im);
      }
    }
    __syncthreads();
  }
  for (int idx = tid; idx < a.n0 * TL; idx += blockDim.x) {
    const int i = idx / TL, t = idx - i * TL;
    if (t < lines) grid[static_cast<long long>(i) * a.n12 + kl0 + t] = Cx<double>{acc[idx], 0.0};
  }
}

__global__ void gather_support_kernel(const Cx<double>* __restrict__ grid, int n0, int n1, int n2,
                                      const std::int32_t* __restrict__ keys, std::size_t count, double points,
                                      Cx<double>* __restrict__ out) {
  for (std::size_t j = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; j < count;
       j += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    int h = keys[3 * j] % n0, k = keys[3 * j + 1] % n1, l = keys[3 * j + 2] % n2;
    h += h < 0 ? n0 : 0;
    k += k < 0 ? n1 : 0;
    l += l < 0 ? n2 : 0;
    const Cx<double> v = grid[(static_cast<long long>(h) * n1 + k) * n2 + l];
    out[j] = Cx<double>{v.re / points, v.im / points};
  }
}

template <typename Kernel>
void allow(Kernel kernel, std::size_t bytes) {
  if (bytes > kMaxDynamicSmem) throw InvalidArgument("density FFT tile does not fit in shared memory");
  allow_dynamic_smem(kernel, bytes);
}

std::size_t pencil_smem(int n0, int tl) {
  return sizeof(Cx<double>) * (n0 + 2 * static_cast<std::size_t>(n0) * (tl + 1)) + sizeof(double) * n0 * tl;
}

std::size_t column_smem(int n1, int tl) {
  return sizeof(Cx<double>) * (n1 + 2 * static_cast<std::size_t>(n1) * (tl + 1));
}

int wrap(int p, int n) {
  const int v = p % n;
  return v < 0 ? v + n : v;
}

template <int TL>
void launch_passes(const DensityArgs& a, const Cx<double>* psi, long long npw, int bands, int rows_per_cta,
                   Cx<double>* rows, Cx<double>* planes, bool accumulate, Cx<double>* grid, unsigned int* flags,
                   cudaStream_t stream) {
  const std::size_t rows_smem =
      sizeof(Cx<double>) * (a.n2 + 2 * static_cast<std::size_t>(rows_per_cta) * (a.n2 | 1));
  allow(density_rows_kernel, rows_smem);
  const dim3 g1(a.slots, static_cast<unsigned>(ceil_div(a.krows, rows_per_cta)), bands);
  density_rows_kernel<<<g1, kThreads, rows_smem, stream>>>(psi, npw, a, rows_per_cta, rows, flags);
  SDFT_LAUNCH("density_rows_kernel");
  const std::size_t c_smem = column_smem(a.n1, TL);
  allow(density_columns_kernel<TL>, c_smem);
  const dim3 g2(static_cast<unsigned>(ceil_div(a.n2, TL)), a.slots, bands);
  density_columns_kernel<TL><<<g2, kThreads, c_smem, stream>>>(rows, a, planes);
  SDFT_LAUNCH("density_columns_kernel");
  const std::size_t p_smem = pencil_smem(a.n0, TL);
  allow(density_pencils_kernel<TL>, p_smem);
  const unsigned g3 = static_cast<unsigned>(ceil_div(static_cast<std::size_t>(a.n12), TL));
  density_pencils_kernel<TL><<<g3, kThreads, p_smem, stream>>>(planes, a, bands, accumulate, grid);
  SDFT_LAUNCH("density_pencils_kernel");
}

}  // namespace

void density_grid_shape(const std::int32_t* hkl, std::size_t npw, const std::int32_t* support, std::size_t count,
                        int shape[3]) {
  long long m[3] = {0, 0, 0}, lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  for (std::size_t j = 0; j < count; ++j)
    for (int a = 0; a < 3; ++a) m[a] = std::max<long long>(m[a], std::llabs(support[3 * j + a]));
  for (std::size_t g = 0; g < npw; ++g)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min<long long>(lo[a], hkl[3 * g + a]);
      hi[a] = std::max<long long>(hi[a], hkl[3 * g + a]);
    }
  for (int a = 0; a < 3; ++a) {
    m[a] = std::max(m[a], hi[a] - lo[a]);
    if (m[a] > 255) throw InvalidArgument("density grid axis above 512 points is not supported");
    shape[a] = fast_fft_length(std::max<int>(3, static_cast<int>(2 * m[a] + 1)));
    if (!fft_length_supported(shape[a])) throw InvalidArgument("density grid axis above 512 points is not supported");
  }
}

void band_density(Context& ctx, const std::int32_t* hkl, std::size_t npw, const Cx<double>* psi,
                  const double* occupations, std::size_t bands, double volume, const std::int32_t* support,
                  std::size_t count, Cx<double>* out) {
  if (!npw || !count || !std::isfinite(volume) || volume <= 0 || !bands)
    throw InvalidArgument("invalid plane-wave FFT density dimensions");
  if (npw > static_cast<std::size_t>(std::numeric_limits<int>::max()) ||
      bands > static_cast<std::size_t>(std::numeric_limits<int>::max()))
    throw Overflow("plane-wave density dimensions overflow");
  std::vector<int> occupied;
  std::vector<double> weight;
  for (std::size_t b = 0; b < bands; ++b) {
    const double f = occupations[b];
    if (!std::isfinite(f) || f < 0 || f > 2) throw InvalidArgument("invalid FFT spin-summed occupation");
    if (f == 0) continue;
    occupied.push_back(static_cast<int>(b));
    weight.push_back(f / volume);
  }
  int shape[3];
  density_grid_shape(hkl, npw, support, count, shape);
  const long long n12 = static_cast<long long>(shape[1]) * shape[2];
  const std::size_t points = static_cast<std::size_t>(n12) * shape[0];

  DensityCache& cache = ctx.density;
  std::vector<std::uint64_t> indices(npw);
  for (std::size_t g = 0; g < npw; ++g)
    indices[g] = (static_cast<std::uint64_t>(wrap(hkl[3 * g], shape[0])) * shape[1] + wrap(hkl[3 * g + 1], shape[1])) *
                     shape[2] +
                 wrap(hkl[3 * g + 2], shape[2]);
  if (std::memcmp(cache.shape, shape, sizeof(shape)) != 0 || cache.indices != indices) {
    std::unordered_set<std::uint64_t> seen(indices.begin(), indices.end());
    if (seen.size() != indices.size()) throw InvalidArgument("duplicate plane-wave key in density basis");
    cache.plan.build(shape, indices, ctx.stream);
    std::memcpy(cache.shape, shape, sizeof(shape));
    cache.indices = std::move(indices);
  }
  const SpherePlan& plan = cache.plan;

  auto* grid = static_cast<Cx<double>*>(cache.grid.reserve(sizeof(Cx<double>) * points));
  const std::size_t meta_bytes = sizeof(unsigned int) * 4 + sizeof(double) * std::max<std::size_t>(1, occupied.size()) +
                                 sizeof(int) * std::max<std::size_t>(1, occupied.size()) +
                                 sizeof(std::int32_t) * 3 * count + 256;
  auto* meta = static_cast<unsigned char*>(cache.meta.reserve(meta_bytes));
  auto* flags = reinterpret_cast<unsigned int*>(meta);
  auto* d_weight = reinterpret_cast<double*>(meta + 16);
  auto* d_band = reinterpret_cast<int*>(d_weight + std::max<std::size_t>(1, occupied.size()));
  auto* d_keys = reinterpret_cast<std::int32_t*>(
      (reinterpret_cast<std::uintptr_t>(d_band + std::max<std::size_t>(1, occupied.size())) + 15) & ~std::uintptr_t(15));
  SDFT_CUDA(cudaMemsetAsync(flags, 0, sizeof(unsigned int), ctx.stream));
  if (!occupied.empty()) {
    SDFT_CUDA(cudaMemcpyAsync(d_weight, weight.data(), sizeof(double) * weight.size(), cudaMemcpyHostToDevice,
                              ctx.stream));
    SDFT_CUDA(cudaMemcpyAsync(d_band, occupied.data(), sizeof(int) * occupied.size(), cudaMemcpyHostToDevice,
                              ctx.stream));
  }
  SDFT_CUDA(cudaMemcpyAsync(d_keys, support, sizeof(std::int32_t) * 3 * count, cudaMemcpyHostToDevice, ctx.stream));

  DensityArgs a{};
  a.n0 = shape[0];
  a.n1 = shape[1];
  a.n2 = shape[2];
  a.slots = plan.slots;
  a.krows = plan.krows;
  a.n12 = n12;
  a.slot_row = plan.slot_row;
  a.point_offset = plan.point_offset;
  a.point_g = plan.point_g;
  a.point_compact = plan.point_compact;
  a.krow = plan.krow;
  a.p0 = plan.line[0];
  a.p1 = plan.line[1];
  a.p2 = plan.line[2];
  a.tw0 = device_twiddles<double>(shape[0]);
  a.tw1 = device_twiddles<double>(shape[1]);
  a.tw2 = device_twiddles<double>(shape[2]);

  const int nmax = std::max({shape[0], shape[1], shape[2]});
  const int tl = pencil_smem(nmax, 32) <= kSmemLimit ? 32 : pencil_smem(nmax, 16) <= kSmemLimit ? 16 : 8;
  const int n2p = shape[2] | 1;
  const int rows_per_cta = std::max(
      1, std::min<int>(plan.krows, static_cast<int>((kSmemLimit - sizeof(Cx<double>) * shape[2]) /
                                                    (2 * sizeof(Cx<double>) * n2p))));
  const std::size_t rows_band = static_cast<std::size_t>(plan.slots) * plan.krows * shape[2];
  const std::size_t planes_band = static_cast<std::size_t>(plan.slots) * n12;
  const std::size_t per_band = sizeof(Cx<double>) * (rows_band + planes_band);
  const std::size_t chunk = std::max<std::size_t>(
      1, std::min<std::size_t>({occupied.size(), slab_budget() / per_band, std::size_t(65535)}));
  if (occupied.empty()) {
    SDFT_CUDA(cudaMemsetAsync(grid, 0, sizeof(Cx<double>) * points, ctx.stream));
  } else {
    auto* rows = static_cast<Cx<double>*>(cache.rows.reserve(sizeof(Cx<double>) * rows_band * chunk));
    auto* planes = static_cast<Cx<double>*>(cache.planes.reserve(sizeof(Cx<double>) * planes_band * chunk));
    for (std::size_t first = 0; first < occupied.size(); first += chunk) {
      const int width = static_cast<int>(std::min(chunk, occupied.size() - first));
      DensityArgs c = a;
      c.band = d_band + first;
      c.weight = d_weight + first;
      const bool accumulate = first > 0;
      if (tl == 32)
        launch_passes<32>(c, psi, static_cast<long long>(npw), width, rows_per_cta, rows, planes, accumulate, grid,
                          flags, ctx.stream);
      else if (tl == 16)
        launch_passes<16>(c, psi, static_cast<long long>(npw), width, rows_per_cta, rows, planes, accumulate, grid,
                          flags, ctx.stream);
      else
        launch_passes<8>(c, psi, static_cast<long long>(npw), width, rows_per_cta, rows, planes, accumulate, grid,
                         flags, ctx.stream);
    }
  }
  fft3d<double>(grid, shape, 1, false, ctx.stream);
  const unsigned blocks = static_cast<unsigned>(std::min<std::size_t>(ceil_div(count, 256), 148ULL * 16));
  gather_support_kernel<<<blocks, 256, 0, ctx.stream>>>(grid, shape[0], shape[1], shape[2], d_keys, count,
                                                        static_cast<double>(points), out);
  SDFT_LAUNCH("gather_support_kernel");
  unsigned int host = 0;
  SDFT_CUDA(cudaMemcpyAsync(&host, flags, sizeof(host), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.synchronize();
  if (host & 1u) throw InvalidArgument("nonfinite wavefunction coefficient");
}

}  // namespace sdft_b200
