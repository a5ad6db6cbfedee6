// One-centre occupations and the compensation charge on the device.
//
// Set-up (CompensationCharge constructor, src/paw_compensation.cpp:185-342):
// the host forms the reciprocal vectors of the keys and the distinct |G|
// shells (exact double radii, as the reference's radius cache), the device
// integrates int g_L(r) r^2 j_L(|G| r) dr on the radial mesh once per shell
// and L (Simpson weights of src/paw_compensation.cpp:51-74, spherical Bessel
// functions by the series / upward / Miller-downward recurrences of :76-114)
// and fills the compact form table F_LM(G) = 4 pi (-i)^L Y_LM(G^) I_L(|G|)
// with the real harmonics of :116-139.
//
// Per call: the (L,M) moments M_a = transform . rho_a (one thread per atom and
// LM), then one thread per G sums exp(-i G.tau_a) (F(G) . M_a) / Omega over the
// atoms in order (src/paw_compensation.cpp:508-520). Products and sums use
// explicitly rounded operations so the device arithmetic follows the
// reference's unfused order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <unordered_map>

#include "operator.cuh"
#include "paw_density.cuh"

namespace sdft_b200 {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kBohrPerAngstrom = 1.8897261254578281;  // CODATA convention of the reference

__device__ __forceinline__ double dot3(double ax, double ay, double az, double bx, double by, double bz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(ax, bx), __dmul_rn(ay, by)), __dmul_rn(az, bz));
}

__device__ __forceinline__ Cx<double> mul_rn(Cx<double> a, Cx<double> b) {
  return {__dsub_rn(__dmul_rn(a.re, b.re), __dmul_rn(a.im, b.im)),
          __dadd_rn(__dmul_rn(a.re, b.im), __dmul_rn(a.im, b.re))};
}

// Spherical Bessel j_l(x) for 0 <= l <= 6.
__device__ double spherical_bessel(int l, double x) {
  if (fabs(x) < 0.5) {
    double term = 1.0;
    for (int k = 1; k <= l; ++k) term *= x / (2.0 * k + 1.0);
    double value = term;
    for (int k = 1; k < 30; ++k) {
      term *= -x * x / (2.0 * k * (2.0 * l + 2.0 * k + 1.0));
      value += term;
      if (fabs(term) < 1e-17 * fmax(1.0, fabs(value))) break;
    }
    return value;
  }
  if (x > l + 1.0) {
    double previous = sin(x) / x;
    if (l == 0) return previous;
    double current = sin(x) / (x * x) - cos(x) / x;
    for (int n = 1; n < l; ++n) {
      const double next = (2.0 * n + 1.0) * current / x - previous;
      previous = current;
      current = next;
    }
    return current;
  }
  constexpr int kExtra = 32;
  double j[6 + kExtra + 2];
  const int top = l + kExtra;
  for (int i = 0; i <= top + 1; ++i) j[i] = 0.0;
  j[top] = 1.0;
  for (int n = top; n >= 1; --n) {
    j[n - 1] = (2.0 * n + 1.0) * j[n] / x - j[n + 1];
    if (fabs(j[n - 1]) > 1e100)
      for (int k = n - 1; k <= top + 1; ++k) j[k] *= 1e-100;
  }
  return j[l] * ((sin(x) / x) / j[0]);
}

// Real harmonic Y_lm (m<0: sin(|m| phi), m>0: cos(m phi), no Condon-Shortley phase).
__device__ double real_harmonic(int l, int m, double qx, double qy, double qz) {
  const double radius = sqrt(dot3(qx, qy, qz, qx, qy, qz));
  if (radius < 1e-14) return l == 0 ? 1.0 / sqrt(4.0 * kPi) : 0.0;
  const double z = fmin(fmax(qz / radius, -1.0), 1.0);
  const double s = sqrt(fmax(0.0, 1.0 - z * z));
  const int order = abs(m);
  double pmm = 1.0;
  for (int k = 1; k <= order; ++k) pmm *= (2.0 * k - 1.0) * s;
  double previous = 0.0, value = pmm;
  if (l > order) {
    previous = pmm;
    value = (2.0 * order + 1.0) * z * pmm;
    for (int degree = order + 2; degree <= l; ++degree) {
      const double next = ((2.0 * degree - 1.0) * z * value - (degree + order - 1.0) * previous) / (degree - order);
      previous = value;
      value = next;
    }
  }
  const double factor = sqrt((2.0 * l + 1.0) / (4.0 * kPi) * exp(lgamma(l - order + 1.0) - lgamma(l + order + 1.0))) *
                        (order ? sqrt(2.0) : 1.0);
  const double angle = order * atan2(qy, qx);
  return factor * value * (m < 0 ? sin(angle) : cos(angle));
}

__global__ void radial_integrals_kernel(const double* __restrict__ shells, int count, int max_l,
                                        const double* __restrict__ r, const double* __restrict__ weights,
                                        const double* __restrict__ r2, int radial, double* __restrict__ integrals) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= count * (max_l + 1)) return;
  const int shell = id / (max_l + 1), L = id - shell * (max_l + 1);
  const double q = shells[shell];
  double sum = 0.0;
  for (int i = 0; i < radial; ++i)
    sum = __dadd_rn(sum, __dmul_rn(__dmul_rn(weights[i], r2[L * radial + i]), spherical_bessel(L, __dmul_rn(q, r[i]))));
  if (q < 1e-14 && L == 0) sum = 1.0;
  integrals[id] = sum;
}

__global__ void form_factor_kernel(const double* __restrict__ q, const int* __restrict__ shell, std::size_t count,
                                   int max_l, const double* __restrict__ integrals, double* __restrict__ form) {
  for (std::size_t g = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; g < count;
       g += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const double qx = q[3 * g], qy = q[3 * g + 1], qz = q[3 * g + 2];
    const double* in = integrals + static_cast<std::size_t>(shell[g]) * (max_l + 1);
    for (int L = 0; L <= max_l; ++L) {
      // 4 pi (-i)^L: the nonzero component of the exact quarter-turn phase.
      const double sign = (L % 4 == 0 || L % 4 == 3) ? 1.0 : -1.0;
      const double factor = sign * (4.0 * kPi);
      for (int M = -L; M <= L; ++M) {
        const double h = real_harmonic(L, M, qx, qy, qz);
        form[static_cast<std::size_t>(L * L + M + L) * count + g] = __dmul_rn(__dmul_rn(factor, h), in[L]);
      }
    }
  }
}

__global__ void check_onsite_kernel(const Cx<double>* __restrict__ rho, int atoms, int dim,
                                    unsigned int* __restrict__ flags) {
  const int entries = dim * dim;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= atoms * entries) return;
  const int a = id / entries, e = id - a * entries, i = e / dim, j = e - i * dim;
  const Cx<double> p = rho[id], t = rho[a * entries + j * dim + i];
  if (!isfinite(p.re) || !isfinite(p.im) || hypot(p.re - t.re, p.im + t.im) > 1e-9) atomicOr(flags, 1u);
}

__global__ void multipoles_kernel(const Cx<double>* __restrict__ rho, const Cx<double>* __restrict__ transform,
                                  int atoms, int dim, int lms, Cx<double>* __restrict__ moments) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= atoms * lms) return;
  const int a = id / lms, lm = id - a * lms;
  const int entries = dim * dim;
  Cx<double> sum{0.0, 0.0};
  for (int e = 0; e < entries; ++e) {
    const Cx<double> term = mul_rn(transform[static_cast<std::size_t>(lm) * entries + e], rho[a * entries + e]);
    sum = {__dadd_rn(sum.re, term.re), __dadd_rn(sum.im, term.im)};
  }
  moments[id] = sum;
}

// e^{-i G.tau_a} for the integer key (h, k, l): G.tau = 2 pi (h f1 + k f2 +
// l f3) for G on the reciprocal lattice and fractional coordinates f, so the
// phase is sincospi of -2 (h f1 + k f2 + l f3), an argument formed without
// the 2 pi scaling and reduced exactly by sincospi.
__device__ __forceinline__ Cx<double> atom_phase(const double* __restrict__ fractional, int a, int h, int k, int l) {
  const double x = __dadd_rn(__dadd_rn(__dmul_rn(static_cast<double>(h), __ldg(fractional + 3 * a)),
                                       __dmul_rn(static_cast<double>(k), __ldg(fractional + 3 * a + 1))),
                             __dmul_rn(static_cast<double>(l), __ldg(fractional + 3 * a + 2)));
  double s, c;
  sincospi(-2.0 * x, &s, &c);
  return Cx<double>{c, s};
}

template <int LMS>
__global__ void compensation_kernel(const int* __restrict__ keys, const double* __restrict__ form, std::size_t count,
                                    const double* __restrict__ fractional, const Cx<double>* __restrict__ moments,
                                    int atoms, int lms_runtime, double volume, Cx<double>* __restrict__ out) {
  const int lms = LMS > 0 ? LMS : lms_runtime;
  for (std::size_t g = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; g < count;
       g += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
    const int h = keys[3 * g], k = keys[3 * g + 1], l = keys[3 * g + 2];
    double f[LMS > 0 ? LMS : 1];
    if (LMS > 0) {
#pragma unroll
      for (int lm = 0; lm < (LMS > 0 ? LMS : 1); ++lm) f[lm] = form[static_cast<std::size_t>(lm) * count + g];
    }
    // Atoms in order; F.M_a by fused multiply-adds, one division by the
    // volume per G (within the 1e-12 relative bar of the reference's
    // per-atom division).
    Cx<double> sum{0.0, 0.0};
    for (int a = 0; a < atoms; ++a) {
      Cx<double> value{0.0, 0.0};
      const Cx<double>* m = moments + static_cast<std::size_t>(a) * lms;
      int lm = 0;
      for (int L = 0; lm < lms; ++L) {
        const bool imaginary = L & 1;
        for (int M = 0; M <= 2 * L; ++M, ++lm) {
          const double fv = LMS > 0 ? f[lm] : form[static_cast<std::size_t>(lm) * count + g];
          const Cx<double> mv = m[lm];
          // (fv, 0) or (0, fv) times the moment.
          if (imaginary) value = {fma(-fv, mv.im, value.re), fma(fv, mv.re, value.im)};
          else value = {fma(fv, mv.re, value.re), fma(fv, mv.im, value.im)};
        }
      }
      const Cx<double> p = atom_phase(fractional, a, h, k, l);
      sum = {fma(p.re, value.re, fma(-p.im, value.im, sum.re)), fma(p.re, value.im, fma(p.im, value.re, sum.im))};
    }
    out[g] = Cx<double>{sum.re / volume, sum.im / volume};
  }
}

// Adjoint partial sums: CTA b adds, for every atom in order, V(-G)
// e^{-iG.tau_a} F_LM(G) over its grid-stride share of G (F imaginary for odd
// L), reduced over the CTA in a fixed order into partials[(b * atoms + a) * LMS + lm].
constexpr int kProjectThreads = 256;

template <int LMS>
__global__ void __launch_bounds__(kProjectThreads) project_partials_kernel(
    const int* __restrict__ keys, const double* __restrict__ form, std::size_t count,
    const double* __restrict__ fractional,
    int atoms, const int* __restrict__ opposite, const Cx<double>* __restrict__ potential,
    Cx<double>* __restrict__ partials) {
  __shared__ Cx<double> red[kProjectThreads / 32][LMS];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int a = 0; a < atoms; ++a) {
    Cx<double> acc[LMS];
#pragma unroll
    for (int lm = 0; lm < LMS; ++lm) acc[lm] = Cx<double>{0.0, 0.0};
    for (std::size_t g = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; g < count;
         g += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
      const int o = opposite[g];
      if (o < 0) continue;
      const Cx<double> w = mul_rn(potential[o], atom_phase(fractional, a, keys[3 * g], keys[3 * g + 1], keys[3 * g + 2]));
      int lm = 0;
#pragma unroll
      for (int L = 0; L * L < LMS; ++L) {
#pragma unroll
        for (int M = 0; M <= 2 * L; ++M, ++lm) {
          const double fv = form[static_cast<std::size_t>(lm) * count + g];
          if (L & 1) acc[lm] = {acc[lm].re - w.im * fv, acc[lm].im + w.re * fv};
          else acc[lm] = {acc[lm].re + w.re * fv, acc[lm].im + w.im * fv};
        }
      }
    }
#pragma unroll
    for (int lm = 0; lm < LMS; ++lm) {
      double re = acc[lm].re, im = acc[lm].im;
#pragma unroll
      for (int s = 16; s > 0; s >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, s);
        im += __shfl_xor_sync(0xffffffffu, im, s);
      }
      if (lane == 0) red[warp][lm] = Cx<double>{re, im};
    }
    __syncthreads();
    if (threadIdx.x < LMS) {
      Cx<double> sum{0.0, 0.0};
      for (int w = 0; w < kProjectThreads / 32; ++w) sum = {sum.re + red[w][threadIdx.x].re, sum.im + red[w][threadIdx.x].im};
      partials[(static_cast<std::size_t>(blockIdx.x) * atoms + a) * LMS + threadIdx.x] = sum;
    }
    __syncthreads();
  }
}

// responses[a][lm] = sum over CTAs in order; then out[a][e] = sum_lm responses * transform.
__global__ void project_responses_kernel(const Cx<double>* __restrict__ partials, int blocks, int atoms, int lms,
                                         Cx<double>* __restrict__ responses) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= atoms * lms) return;
  Cx<double> sum{0.0, 0.0};
  for (int b = 0; b < blocks; ++b) {
    const Cx<double> v = partials[static_cast<std::size_t>(b) * atoms * lms + id];
    sum = {sum.re + v.re, sum.im + v.im};
  }
  responses[id] = sum;
}

__global__ void project_contract_kernel(const Cx<double>* __restrict__ responses,
                                        const Cx<double>* __restrict__ transform, int atoms, int lms, int entries,
                                        Cx<double>* __restrict__ out) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= atoms * entries) return;
  const int a = id / entries, e = id - a * entries;
  Cx<double> sum{0.0, 0.0};
  for (int lm = 0; lm < lms; ++lm) {
    const Cx<double> t = mul_rn(responses[a * lms + lm], transform[static_cast<std::size_t>(lm) * entries + e]);
    sum = {__dadd_rn(sum.re, t.re), __dadd_rn(sum.im, t.im)};
  }
  out[id] = sum;
}

__global__ void onsite_kernel(const Cx<double>* __restrict__ p, long long stride, int rows, int atoms, int bands,
                              const double* __restrict__ occupations, Cx<double>* __restrict__ out,
                              unsigned int* __restrict__ flags) {
  const int entries = rows * rows;
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= atoms * entries) return;
  const int a = id / entries, e = id - a * entries, i = e / rows, j = e - i * rows;
  const Cx<double>* pi = p + static_cast<long long>(a) * rows + i;
  const Cx<double>* pj = p + static_cast<long long>(a) * rows + j;
  Cx<double> sum{0.0, 0.0};
  bool finite = true;
  for (int n = 0; n < bands; ++n) {
    const double f = occupations[n];
    const Cx<double> u = pi[n * stride], v = pj[n * stride];
    finite = finite && isfinite(u.re) && isfinite(u.im);
    const Cx<double> w{__dmul_rn(f, u.re), __dmul_rn(f, u.im)};
    const Cx<double> term = mul_rn(w, Cx<double>{v.re, -v.im});
    sum = {__dadd_rn(sum.re, term.re), __dadd_rn(sum.im, term.im)};
  }
  if (!finite) atomicOr(flags, 1u);
  out[id] = sum;
}

// Radial quadrature weights: Simpson panels from the outer end on a
// logarithmic mesh, trapezoids otherwise (src/paw_compensation.cpp:51-74).
std::vector<double> radial_weights(const double* r, std::size_t count) {
  if (count < 3 || !(r[0] > 0.0)) throw InvalidArgument("PAW compensation requires a positive radial mesh");
  const double h = std::log(r[1] / r[0]);
  bool logarithmic = std::isfinite(h) && h > 0.0;
  for (std::size_t i = 1; i < count; ++i) {
    if (!std::isfinite(r[i]) || r[i] <= r[i - 1]) throw InvalidArgument("PAW radial mesh must be finite and increasing");
    logarithmic = logarithmic && std::abs(std::log(r[i] / r[i - 1]) - h) < 2e-7;
  }
  std::vector<double> w(count, 0.0);
  if (logarithmic) {
    for (std::size_t k = count; k >= 3; k -= 2) {
      w[k - 1] += r[k - 1] * h / 3.0;
      w[k - 2] = 4.0 * r[k - 2] * h / 3.0;
      w[k - 3] = r[k - 3] * h / 3.0;
      if (k == 3) break;
    }
  } else {
    for (std::size_t i = 0; i + 1 < count; ++i) {
      w[i] += (r[i + 1] - r[i]) / 2.0;
      w[i + 1] += (r[i + 1] - r[i]) / 2.0;
    }
  }
  return w;
}

template <typename T>
T* upload(const T* host, std::size_t count) {
  T* dev = nullptr;
  SDFT_CUDA(cudaMalloc(&dev, sizeof(T) * std::max<std::size_t>(1, count)));
  if (count) SDFT_CUDA(cudaMemcpy(dev, host, sizeof(T) * count, cudaMemcpyHostToDevice));
  return dev;
}

struct V3 {
  double x, y, z;
};
V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 scaled(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
V3 combine(const V3 basis[3], double u, double v, double w) {
  return add(add(scaled(basis[0], u), scaled(basis[1], v)), scaled(basis[2], w));
}

}  // namespace

CompensationCharge::CompensationCharge(Context& ctx, const CompensationInput& in) : ctx_(ctx) {
  if (!in.lattice || !in.keys || !in.radial_grid || !in.compensation_r2 || !in.transform || !in.count ||
      !in.atoms || !in.fractional || !in.dimension)
    throw InvalidArgument("invalid PAW compensation dimensions");
  const V3 a[3] = {{in.lattice[0], in.lattice[1], in.lattice[2]},
                   {in.lattice[3], in.lattice[4], in.lattice[5]},
                   {in.lattice[6], in.lattice[7], in.lattice[8]}};
  const double signed_volume = dot(a[0], cross(a[1], a[2]));
  volume_ = std::abs(signed_volume);
  if (!std::isfinite(volume_) || volume_ < 1e-12) throw InvalidArgument("singular PAW compensation lattice");
  if (in.max_l < 0 || in.max_l > 6) throw InvalidArgument("incomplete PAW compensation multipoles");
  max_l_ = in.max_l;
  lms_ = (max_l_ + 1) * (max_l_ + 1);
  count_ = in.count;
  atoms_ = in.atoms;
  dim_ = in.dimension;
  if (count_ > static_cast<std::size_t>(std::numeric_limits<int>::max()) / 3 || atoms_ > 1000000 || dim_ > 1024)
    throw Overflow("PAW compensation dimensions overflow");
  const std::vector<double> weights = radial_weights(in.radial_grid, in.radial);
  for (std::size_t i = 0; i < (max_l_ + 1) * in.radial; ++i)
    if (!std::isfinite(in.compensation_r2[i])) throw InvalidArgument("PAW compensation radial shape mismatch");

  const double scale = 2.0 * kPi / signed_volume;
  const V3 b[3] = {scaled(cross(a[1], a[2]), scale), scaled(cross(a[2], a[0]), scale),
                   scaled(cross(a[0], a[1]), scale)};
  std::vector<double> q(3 * count_);
  std::vector<int> shell(count_);
  std::map<double, int> shells;
  std::vector<double> radii;
  for (std::size_t g = 0; g < count_; ++g) {
    const V3 v = combine(b, static_cast<double>(in.keys[3 * g]), static_cast<double>(in.keys[3 * g + 1]),
                         static_cast<double>(in.keys[3 * g + 2]));
    q[3 * g] = v.x;
    q[3 * g + 1] = v.y;
    q[3 * g + 2] = v.z;
    const double radius = std::sqrt(dot(v, v)) * kBohrPerAngstrom;
    auto found = shells.try_emplace(radius, static_cast<int>(radii.size()));
    if (found.second) radii.push_back(radius);
    shell[g] = found.first->second;
  }
  for (std::size_t i = 0; i < 3 * atoms_; ++i)
    if (!std::isfinite(in.fractional[i])) throw InvalidArgument("nonfinite PAW compensation position");
  q_ = upload(q.data(), q.size());
  keys_ = upload(in.keys, 3 * count_);
  fractional_ = upload(in.fractional, 3 * atoms_);
  transform_ = upload(reinterpret_cast<const Cx<double>*>(in.transform), static_cast<std::size_t>(lms_) * dim_ * dim_);
  SDFT_CUDA(cudaMalloc(&form_, sizeof(double) * lms_ * count_));
  SDFT_CUDA(cudaMalloc(&moments_, sizeof(Cx<double>) * lms_ * atoms_));
  SDFT_CUDA(cudaMalloc(&flags_, sizeof(unsigned int)));
  {
    // index of -G in the support (the adjoint samples V(-G)), -1 when absent
    std::unordered_map<std::uint64_t, int> where;
    where.reserve(count_ * 2);
    auto key = [](int h, int k, int l) {
      const auto b = [](int v) { return static_cast<std::uint64_t>(static_cast<std::int64_t>(v) + (1LL << 20)) & 0x1FFFFF; };
      return (b(h) << 42) | (b(k) << 21) | b(l);
    };
    for (std::size_t g = 0; g < count_; ++g)
      where[key(in.keys[3 * g], in.keys[3 * g + 1], in.keys[3 * g + 2])] = static_cast<int>(g);
    std::vector<int> opposite(count_);
    for (std::size_t g = 0; g < count_; ++g) {
      const auto found = where.find(key(-in.keys[3 * g], -in.keys[3 * g + 1], -in.keys[3 * g + 2]));
      opposite[g] = found == where.end() ? -1 : found->second;
    }
    opposite_ = upload(opposite.data(), opposite.size());
  }
  int* d_shell = upload(shell.data(), shell.size());
  double* d_radii = upload(radii.data(), radii.size());
  double* d_r = upload(in.radial_grid, in.radial);
  double* d_w = upload(weights.data(), weights.size());
  double* d_r2 = upload(in.compensation_r2, (max_l_ + 1) * in.radial);
  double* d_integrals = nullptr;
  SDFT_CUDA(cudaMalloc(&d_integrals, sizeof(double) * radii.size() * (max_l_ + 1)));
  const int jobs = static_cast<int>(radii.size()) * (max_l_ + 1);
  radial_integrals_kernel<<<static_cast<unsigned>(ceil_div(jobs, 128)), 128, 0, ctx.stream>>>(
      d_radii, static_cast<int>(radii.size()), max_l_, d_r, d_w, d_r2, static_cast<int>(in.radial), d_integrals);
  SDFT_LAUNCH("radial_integrals_kernel");
  const unsigned blocks = static_cast<unsigned>(std::min<std::size_t>(ceil_div(count_, 256), 148ULL * 16));
  form_factor_kernel<<<blocks, 256, 0, ctx.stream>>>(q_, d_shell, count_, max_l_, d_integrals, form_);
  SDFT_LAUNCH("form_factor_kernel");
  SDFT_CUDA(cudaStreamSynchronize(ctx.stream));
  for (void* p : {static_cast<void*>(d_shell), static_cast<void*>(d_radii), static_cast<void*>(d_r),
                  static_cast<void*>(d_w), static_cast<void*>(d_r2), static_cast<void*>(d_integrals)})
    cudaFree(p);
}

CompensationCharge::~CompensationCharge() {
  for (void* p : {static_cast<void*>(q_), static_cast<void*>(keys_), static_cast<void*>(fractional_),
                  static_cast<void*>(form_),
                  static_cast<void*>(transform_), static_cast<void*>(moments_), static_cast<void*>(flags_),
                  static_cast<void*>(opposite_), static_cast<void*>(partials_), static_cast<void*>(responses_)})
    if (p) cudaFree(p);
}

void CompensationCharge::project(const Cx<double>* potential, Cx<double>* out) {
  const int atoms = static_cast<int>(atoms_), entries = static_cast<int>(dim_ * dim_);
  const int blocks = static_cast<int>(std::min<std::size_t>(std::max<std::size_t>(1, ceil_div(count_, kProjectThreads)),
                                                            148ULL * 4));
  if (!partials_) {
    SDFT_CUDA(cudaMalloc(&partials_, sizeof(Cx<double>) * static_cast<std::size_t>(148 * 4) * atoms_ * lms_));
    SDFT_CUDA(cudaMalloc(&responses_, sizeof(Cx<double>) * atoms_ * lms_));
  }
#define SDFT_PROJECT_CASE(N)                                                                                     \
  case N:                                                                                                        \
    project_partials_kernel<N><<<blocks, kProjectThreads, 0, ctx_.stream>>>(keys_, form_, count_, fractional_, \
                                                                          atoms, opposite_, potential, partials_); \
    break;
  switch (lms_) {
    SDFT_PROJECT_CASE(1)
    SDFT_PROJECT_CASE(4)
    SDFT_PROJECT_CASE(9)
    SDFT_PROJECT_CASE(16)
    default:
      throw InvalidArgument("compensation potential projection supports L_max <= 3");
  }
#undef SDFT_PROJECT_CASE
  SDFT_LAUNCH("project_partials_kernel");
  project_responses_kernel<<<static_cast<unsigned>(ceil_div(atoms * lms_, 128)), 128, 0, ctx_.stream>>>(
      partials_, blocks, atoms, lms_, responses_);
  SDFT_LAUNCH("project_responses_kernel");
  project_contract_kernel<<<static_cast<unsigned>(ceil_div(atoms * entries, 128)), 128, 0, ctx_.stream>>>(
      responses_, transform_, atoms, lms_, entries, out);
  SDFT_LAUNCH("project_contract_kernel");
}

void CompensationCharge::density(const Cx<double>* onsite, Cx<double>* out) {
  const int dim = static_cast<int>(dim_), atoms = static_cast<int>(atoms_);
  SDFT_CUDA(cudaMemsetAsync(flags_, 0, sizeof(unsigned int), ctx_.stream));
  const int entries = atoms * dim * dim;
  check_onsite_kernel<<<static_cast<unsigned>(ceil_div(entries, 256)), 256, 0, ctx_.stream>>>(onsite, atoms, dim,
                                                                                               flags_);
  SDFT_LAUNCH("check_onsite_kernel");
  multipoles_kernel<<<static_cast<unsigned>(ceil_div(atoms * lms_, 128)), 128, 0, ctx_.stream>>>(
      onsite, transform_, atoms, dim, lms_, moments_);
  SDFT_LAUNCH("multipoles_kernel");
  const unsigned blocks = static_cast<unsigned>(std::min<std::size_t>(ceil_div(count_, 128), 148ULL * 32));
#define SDFT_COMPENSATION_CASE(N)                                                                                \
  case N:                                                                                                        \
    compensation_kernel<N><<<blocks, 128, 0, ctx_.stream>>>(keys_, form_, count_, fractional_, moments_, atoms, \
                                                            lms_, volume_, out);                                \
    break;
  switch (lms_) {
    SDFT_COMPENSATION_CASE(1)
    SDFT_COMPENSATION_CASE(4)
    SDFT_COMPENSATION_CASE(9)
    SDFT_COMPENSATION_CASE(16)
    default:
      compensation_kernel<0><<<blocks, 128, 0, ctx_.stream>>>(keys_, form_, count_, fractional_, moments_, atoms,
                                                              lms_, volume_, out);
  }
#undef SDFT_COMPENSATION_CASE
  SDFT_LAUNCH("compensation_kernel");
  unsigned int host = 0;
  SDFT_CUDA(cudaMemcpyAsync(&host, flags_, sizeof(host), cudaMemcpyDeviceToHost, ctx_.stream));
  SDFT_CUDA(cudaStreamSynchronize(ctx_.stream));
  if (host) throw InvalidArgument("PAW compensation density must be finite and Hermitian");
}

void onsite_density(Context& ctx, std::size_t rows, std::size_t atoms, std::size_t bands, const Cx<double>* amplitudes,
                    std::size_t stride, const double* occupations, Cx<double>* out) {
  if (!rows || !bands || !atoms || !amplitudes || !occupations || stride < rows * atoms ||
      rows > std::numeric_limits<std::size_t>::max() / std::max(rows, bands))
    throw InvalidArgument("invalid projected onsite density dimensions");
  if (rows * rows * atoms > static_cast<std::size_t>(std::numeric_limits<int>::max()) ||
      bands > static_cast<std::size_t>(std::numeric_limits<int>::max()))
    throw Overflow("projected onsite density dimensions overflow");
  for (std::size_t n = 0; n < bands; ++n)
    if (!std::isfinite(occupations[n]) || occupations[n] < 0 || occupations[n] > 2)
      throw InvalidArgument("invalid projected onsite occupation");
  auto* meta = static_cast<unsigned char*>(ctx.onsite.reserve(256 + sizeof(double) * bands));
  auto* flags = reinterpret_cast<unsigned int*>(meta);
  auto* d_occ = reinterpret_cast<double*>(meta + 256);
  SDFT_CUDA(cudaMemsetAsync(flags, 0, sizeof(unsigned int), ctx.stream));
  SDFT_CUDA(cudaMemcpyAsync(d_occ, occupations, sizeof(double) * bands, cudaMemcpyHostToDevice, ctx.stream));
  const int entries = static_cast<int>(rows * rows * atoms);
  onsite_kernel<<<static_cast<unsigned>(ceil_div(entries, 128)), 128, 0, ctx.stream>>>(
      amplitudes, static_cast<long long>(stride), static_cast<int>(rows), static_cast<int>(atoms),
      static_cast<int>(bands), d_occ, out, flags);
  SDFT_LAUNCH("onsite_kernel");
  unsigned int host = 0;
  SDFT_CUDA(cudaMemcpyAsync(&host, flags, sizeof(host), cudaMemcpyDeviceToHost, ctx.stream));
  SDFT_CUDA(cudaStreamSynchronize(ctx.stream));
  if (host) throw InvalidArgument("nonfinite onsite projection");
}

}  // namespace sdft_b200
