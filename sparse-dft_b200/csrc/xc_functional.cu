// Hartree + PBE exchange-correlation functional of a Fourier density on the
// device: the reference's evaluate_density_functionals
// (src/density_functionals.cpp:462-694 and the wrapper :696-729) with its
// default packing (paired real transforms, fused PBE tiles, fixed-tile
// ordered reductions, ordered Fourier accumulation).
//
// Pipeline (one context stream, every array device-resident):
//   1. host: keys sorted into the reference's map order (lexicographic h, k,
//      l), the union support of density and frozen core, wrapped grid
//      indices of +G and -G, G vectors with the reference's arithmetic;
//   2. scatter: two complex grids per density field set, n + i g_z and
//      g_x + i g_y (i q_a rho packed as the reference's real_components);
//      with a core, valence and core fields go to separate grids and are
//      added in real space, as the reference's frozen-core reuse does;
//   3. backward 3D FFTs (any axis length up to 512: the grid is
//      padding * max(3, 2m+1) per axis, usually not 2/3/5/7-smooth);
//   4. one pass over the grid in fixed tiles of 2048 points: PBE per point,
//      the tile's electrons, energy, stress, minimum and clipped count in
//      double-double, and the forward fields local + i d_x, d_y + i d_z
//      written over the inputs;
//   5. forward 3D FFTs, then per key the paired extraction, v_xc, the
//      Hartree potential, and per-block partial sums of the Hartree energy,
//      stress and <rho, v_xc>, merged in a fixed order.
// Sums are double-double where the reference sums long double or FP64; the
// results agree with the reference to rounding, not bit for bit.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <string>
#include <unordered_map>

#include "local_hamiltonian.cuh"
#include "pbe.cuh"
#include "xc_functional.cuh"

namespace sdft_b200 {

namespace {

constexpr double kPi = 3.1415926535897932384626433832795;
constexpr int kTile = 2048;       // points per reduction tile (the reference's width)
constexpr int kTileThreads = 256;
constexpr int kSums = 11;         // tile sums: electrons, energy, stress[9]
constexpr int kKeyThreads = 256;
constexpr int kKeySums = 11;      // key sums: Hartree energy, Hartree stress[9], <rho, v_xc>

struct DD {
  double hi, lo;
};

__device__ __forceinline__ DD dd_add(DD a, double b) {
  const double s = __dadd_rn(a.hi, b);
  const double bb = __dsub_rn(s, a.hi);
  const double e = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(s, bb)), __dsub_rn(b, bb));
  const double lo = __dadd_rn(a.lo, e);
  const double hi = __dadd_rn(s, lo);
  return {hi, __dsub_rn(lo, __dsub_rn(hi, s))};
}

__device__ __forceinline__ DD dd_add(DD a, DD b) {
  DD s = dd_add(a, b.hi);
  return dd_add(s, b.lo);
}

// Block reduction of `width` double-double sums per thread in a fixed order:
// a shuffle tree inside each warp, then warp 0 adds the warps' sums in
// order. The result is in thread 0's values.
template <int THREADS>
__device__ void block_reduce(DD* values, int width, DD* shared) {
  constexpr int kWarps = THREADS / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = 0; k < width; ++k) {
    DD v = values[k];
    for (int offset = 16; offset > 0; offset /= 2) {
      const DD other{__shfl_down_sync(0xffffffffu, v.hi, offset), __shfl_down_sync(0xffffffffu, v.lo, offset)};
      v = dd_add(v, other);
    }
    if (lane == 0) shared[k * kWarps + warp] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0)
    for (int k = 0; k < width; ++k) {
      DD v = shared[k * kWarps];
      for (int w = 1; w < kWarps; ++w) v = dd_add(v, shared[k * kWarps + w]);
      values[k] = v;
    }
  __syncthreads();
}

struct KeyData {
  const long long* index;     // wrapped grid index of +G
  const long long* opposite;  // wrapped grid index of -G
  const double* q;            // 3 per key, the reference's reciprocal_vector
  const Cx<double>* valence;  // density value (0 where absent)
  const Cx<double>* core;     // core value (0 where absent)
  const unsigned char* flags; // bit 0: in the density, bit 1: in the core
  const int* opposite_key;    // union position of -G, or -1
};

// i q rho as the reference packs it: (a + bi)(0 + qi) = (-b q, a q).
__device__ __forceinline__ Cx<double> times_iq(Cx<double> v, double q) { return {-(v.im * q), v.re * q}; }

// Fields of one coefficient into the grid pair (n + i g_z, g_x + i g_y):
// first + i * second with i * (x + iy) = (-y, x) and the reference's += order.
__device__ __forceinline__ void scatter_fields(Cx<double> v, const double* q, Cx<double>* nz, Cx<double>* xy,
                                               long long at) {
  const Cx<double> gz = times_iq(v, q[2]);
  nz[at] = Cx<double>{__dadd_rn(v.re, -gz.im), __dadd_rn(v.im, gz.re)};
  const Cx<double> gx = times_iq(v, q[0]), gy = times_iq(v, q[1]);
  xy[at] = Cx<double>{__dadd_rn(gx.re, -gy.im), __dadd_rn(gx.im, gy.re)};
}

// grids: [nz, xy] for the valence (or the whole density when there is no
// core), then [nz, xy] of the core. Without a core the density is the xc
// density itself.
__global__ void xc_scatter_kernel(KeyData keys, int count, Cx<double>* grids, long long points, bool with_core) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const long long at = keys.index[i];
    const double* q = keys.q + 3 * i;
    const unsigned char f = keys.flags[i];
    if (!with_core) {
      scatter_fields(keys.valence[i], q, grids, grids + points, at);
    } else {
      if (f & 1u) scatter_fields(keys.valence[i], q, grids, grids + points, at);
      if (f & 2u) scatter_fields(keys.core[i], q, grids + 2 * points, grids + 3 * points, at);
    }
  }
}

struct TileOut {
  double* sums;                 // [tiles][kSums][2]
  double* minimum;              // [tiles]
  unsigned long long* clipped;  // [tiles]
};

// PBE per point and the fixed-tile reductions (src/density_functionals.cpp
// :565-641, fused path); the forward fields overwrite the inputs.
__global__ void __launch_bounds__(kTileThreads) xc_points_kernel(Cx<double>* grids, long long points, bool with_core,
                                                                 long long tiles, TileOut out) {
  __shared__ DD shared[kSums * (kTileThreads / 32)];
  __shared__ double shared_min[kTileThreads];
  __shared__ unsigned long long shared_clip[kTileThreads];
  Cx<double>* nz = grids;
  Cx<double>* xy = grids + points;
  const Cx<double>* core_nz = grids + 2 * points;
  const Cx<double>* core_xy = grids + 3 * points;
  for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
    DD sums[kSums];
    for (int k = 0; k < kSums; ++k) sums[k] = DD{0.0, 0.0};
    double minimum = INFINITY;
    unsigned long long clipped = 0;
    const long long first = t * kTile;
    for (int p = threadIdx.x; p < kTile; p += kTileThreads) {
      const long long i = first + p;
      if (i >= points) break;
      const Cx<double> a = nz[i], b = xy[i];
      const double valence = a.re;
      double raw = a.re, gx = b.re, gy = b.im, gz = a.im;
      if (with_core) {
        const Cx<double> c = core_nz[i], d = core_xy[i];
        raw = __dadd_rn(a.re, c.re);
        gx = __dadd_rn(b.re, d.re);
        gy = __dadd_rn(b.im, d.im);
        gz = __dadd_rn(a.im, c.im);
      }
      const double n = 1e-10 < raw ? raw : 1e-10;
      const double grad =
          sqrt(__dadd_rn(__dadd_rn(__dmul_rn(gx, gx), __dmul_rn(gy, gy)), __dmul_rn(gz, gz)));
      const pbe::Point xc = pbe::pbe_point(n, grad);
      const double e = xc.energy;
      const double local = __dadd_rn(xc.vx, xc.vc);
      const double dx = __dmul_rn(xc.sigma, gx), dy = __dmul_rn(xc.sigma, gy), dz = __dmul_rn(xc.sigma, gz);
      nz[i] = Cx<double>{local, dx};
      xy[i] = Cx<double>{dy, dz};
      minimum = fmin(minimum, raw);
      clipped += raw < 1e-10;
      sums[0] = dd_add(sums[0], valence);
      sums[1] = dd_add(sums[1], e);
      const double g[3] = {gx, gy, gz}, v[3] = {dx, dy, dz};
      const double pressure = __dsub_rn(
          __dsub_rn(__dsub_rn(__dsub_rn(e, __dmul_rn(local, raw)), __dmul_rn(dx, gx)), __dmul_rn(dy, gy)),
          __dmul_rn(dz, gz));
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
          sums[2 + 3 * r + c] = dd_add(sums[2 + 3 * r + c], __dsub_rn(r == c ? pressure : 0.0, __dmul_rn(v[r], g[c])));
    }
    block_reduce<kTileThreads>(sums, kSums, shared);
    shared_min[threadIdx.x] = minimum;
    shared_clip[threadIdx.x] = clipped;
    __syncthreads();
    for (int stride = kTileThreads / 2; stride > 0; stride /= 2) {
      if (threadIdx.x < stride) {
        shared_min[threadIdx.x] = fmin(shared_min[threadIdx.x], shared_min[threadIdx.x + stride]);
        shared_clip[threadIdx.x] += shared_clip[threadIdx.x + stride];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      for (int k = 0; k < kSums; ++k) {
        out.sums[(t * kSums + k) * 2] = sums[k].hi;
        out.sums[(t * kSums + k) * 2 + 1] = sums[k].lo;
      }
      out.minimum[t] = shared_min[0];
      out.clipped[t] = shared_clip[0];
    }
    __syncthreads();
  }
}

// Paired forward extraction, v_xc and the potential per key, with the
// reference's complex arithmetic (src/density_functionals.cpp:296-314,
// :665-683): first = (D(G) + conj D(-G)) / 2N, second = -i (D(G) - conj D(-G)) / 2N,
// v_xc = l - i (q . d), potential = 4 pi rho / q^2 (q^2 > 1e-12, else 0) + v_xc.
__global__ void xc_gather_kernel(KeyData keys, int count, const Cx<double>* grids, long long points,
                                 Cx<double>* potential, Cx<double>* xc_potential) {
  const double twice = 2.0 * static_cast<double>(points);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const long long at = keys.index[i], op = keys.opposite[i];
    Cx<double> field[4];
    for (int g = 0; g < 2; ++g) {
      const Cx<double> direct = grids[g * points + at], o = grids[g * points + op];
      const Cx<double> opposite{o.re, -o.im};
      field[2 * g] = Cx<double>{__ddiv_rn(__dadd_rn(direct.re, opposite.re), twice),
                                __ddiv_rn(__dadd_rn(direct.im, opposite.im), twice)};
      const double dre = __dsub_rn(direct.re, opposite.re), dim = __dsub_rn(direct.im, opposite.im);
      field[2 * g + 1] = Cx<double>{__ddiv_rn(dim, twice), __ddiv_rn(-dre, twice)};
    }
    const double* q = keys.q + 3 * i;
    const double sre = __dadd_rn(__dadd_rn(__dmul_rn(q[0], field[1].re), __dmul_rn(q[1], field[2].re)),
                                 __dmul_rn(q[2], field[3].re));
    const double sim = __dadd_rn(__dadd_rn(__dmul_rn(q[0], field[1].im), __dmul_rn(q[1], field[2].im)),
                                 __dmul_rn(q[2], field[3].im));
    const Cx<double> vxc{__dadd_rn(field[0].re, sim), __dsub_rn(field[0].im, sre)};
    xc_potential[i] = vxc;
    Cx<double> total = vxc;
    if (keys.flags[i] & 1u) {
      const double q2 = __dadd_rn(__dadd_rn(__dmul_rn(q[0], q[0]), __dmul_rn(q[1], q[1])), __dmul_rn(q[2], q[2]));
      Cx<double> vh{0.0, 0.0};
      if (q2 > 1e-12) {
        const Cx<double> rho = keys.valence[i];
        vh = Cx<double>{__ddiv_rn(__dmul_rn(4.0 * kPi, rho.re), q2), __ddiv_rn(__dmul_rn(4.0 * kPi, rho.im), q2)};
      }
      total = Cx<double>{__dadd_rn(vh.re, vxc.re), __dadd_rn(vh.im, vxc.im)};
    }
    potential[i] = total;
  }
}

// Per-block partial sums over the density keys: Hartree energy
// 2 pi Omega |rho|^2 / q^2, stress 4 pi |rho|^2 q_a q_c / q^4 (:478-493) and
// <rho, v_xc> = Omega Re(rho(G) v_xc(-G)) (:685-691).
__global__ void __launch_bounds__(kKeyThreads) xc_key_sums_kernel(KeyData keys, int count,
                                                                  const Cx<double>* xc_potential, double volume,
                                                                  double* partials) {
  __shared__ DD shared[kKeySums * (kKeyThreads / 32)];
  DD sums[kKeySums];
  for (int k = 0; k < kKeySums; ++k) sums[k] = DD{0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    if (!(keys.flags[i] & 1u)) continue;
    const Cx<double> rho = keys.valence[i];
    const double* q = keys.q + 3 * i;
    const double q2 = __dadd_rn(__dadd_rn(__dmul_rn(q[0], q[0]), __dmul_rn(q[1], q[1])), __dmul_rn(q[2], q[2]));
    const double norm = __dadd_rn(__dmul_rn(rho.re, rho.re), __dmul_rn(rho.im, rho.im));
    if (q2 > 1e-12) {
      sums[0] = dd_add(sums[0], __ddiv_rn(__dmul_rn(__dmul_rn(2.0 * kPi, volume), norm), q2));
      const double q4 = __dmul_rn(q2, q2);
      for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c)
          sums[1 + 3 * a + c] =
              dd_add(sums[1 + 3 * a + c], __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(4.0 * kPi, norm), q[a]), q[c]), q4));
    }
    const int o = keys.opposite_key[i];
    if (o >= 0) {
      const Cx<double> v = xc_potential[o];
      sums[10] = dd_add(sums[10], __dmul_rn(volume, __dsub_rn(__dmul_rn(rho.re, v.re), __dmul_rn(rho.im, v.im))));
    }
  }
  block_reduce<kKeyThreads>(sums, kKeySums, shared);
  if (threadIdx.x == 0)
    for (int k = 0; k < kKeySums; ++k) {
      partials[(blockIdx.x * kKeySums + k) * 2] = sums[k].hi;
      partials[(blockIdx.x * kKeySums + k) * 2 + 1] = sums[k].lo;
    }
}

// Fixed-order merge of `records` double-double records of `width` sums (one
// CTA); minimum and clipped counts when given.
__global__ void __launch_bounds__(kTileThreads) xc_merge_kernel(const double* records, long long count, int width,
                                                                const double* minimum,
                                                                const unsigned long long* clipped, double* out) {
  __shared__ DD shared[kSums * (kTileThreads / 32)];
  __shared__ double shared_min[kTileThreads];
  __shared__ unsigned long long shared_clip[kTileThreads];
  DD sums[kSums];
  for (int k = 0; k < kSums; ++k) sums[k] = DD{0.0, 0.0};
  double lowest = INFINITY;
  unsigned long long clip = 0;
  for (long long r = threadIdx.x; r < count; r += kTileThreads) {
    for (int k = 0; k < width; ++k)
      sums[k] = dd_add(sums[k], DD{records[(r * width + k) * 2], records[(r * width + k) * 2 + 1]});
    if (minimum) lowest = fmin(lowest, minimum[r]);
    if (clipped) clip += clipped[r];
  }
  block_reduce<kTileThreads>(sums, width, shared);
  shared_min[threadIdx.x] = lowest;
  shared_clip[threadIdx.x] = clip;
  __syncthreads();
  for (int stride = kTileThreads / 2; stride > 0; stride /= 2) {
    if (threadIdx.x < stride) {
      shared_min[threadIdx.x] = fmin(shared_min[threadIdx.x], shared_min[threadIdx.x + stride]);
      shared_clip[threadIdx.x] += shared_clip[threadIdx.x + stride];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int k = 0; k < width; ++k) {
      out[2 * k] = sums[k].hi;
      out[2 * k + 1] = sums[k].lo;
    }
    out[2 * width] = shared_min[0];
    out[2 * width + 1] = static_cast<double>(shared_clip[0]);
  }
}

using Key = std::array<int, 3>;

struct SortedField {
  std::vector<Key> keys;
  std::vector<Cx<double>> values;
};

// Keys in the reference's std::map order; duplicates are rejected.
SortedField sorted_field(std::size_t count, const int* hkl, const double* values, const char* what) {
  std::vector<std::size_t> order(count);
  std::iota(order.begin(), order.end(), std::size_t(0));
  auto key = [&](std::size_t i) { return Key{hkl[3 * i], hkl[3 * i + 1], hkl[3 * i + 2]}; };
  std::sort(order.begin(), order.end(), [&](std::size_t a, std::size_t b) { return key(a) < key(b); });
  SortedField out;
  out.keys.reserve(count);
  out.values.reserve(count);
  for (std::size_t i : order) {
    if (!out.keys.empty() && out.keys.back() == key(i)) throw InvalidArgument(std::string("duplicate ") + what + " Fourier key");
    out.keys.push_back(key(i));
    out.values.push_back(Cx<double>{values[2 * i], values[2 * i + 1]});
  }
  return out;
}

int env_padding() {
  int padding = 2;
  if (const char* env = std::getenv("SDFT_FFT_OVERSAMPLING")) {
    char* end = nullptr;
    const long parsed = std::strtol(env, &end, 10);
    if (!end || *end != '\0' || parsed < 1 || parsed > 8)
      throw InvalidArgument("SDFT_FFT_OVERSAMPLING must be an integer in [1,8]");
    padding = static_cast<int>(parsed);
  }
  return padding;
}

bool env_fast_grid() {
  const char* setting = std::getenv("SDFT_FAST_DENSITY_GRID");
  if (!setting) return false;
  if (std::string(setting) != "0" && std::string(setting) != "1")
    throw InvalidArgument("SDFT_FAST_DENSITY_GRID must be 0 or 1");
  return std::string(setting) == "1";
}

struct V3 {
  double x, y, z;
};

}  // namespace

FunctionalSupport functional_support(const double lattice[9], std::size_t count, const int* hkl,
                                     const double* density, std::size_t core_count, const int* core_hkl,
                                     const double* core, int quadrature_padding) {
  const V3 a0{lattice[0], lattice[1], lattice[2]}, a1{lattice[3], lattice[4], lattice[5]},
      a2{lattice[6], lattice[7], lattice[8]};
  auto cross = [](V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; };
  auto dot = [](V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; };
  const double det = dot(a0, cross(a1, a2));
  const double volume = std::abs(det);
  if (volume < 1e-12 || !std::isfinite(volume)) throw InvalidArgument("singular density-grid lattice");
  if (!count) throw InvalidArgument("density Fourier support is empty");
  FunctionalSupport s;
  s.volume = volume;
  auto scale = [](V3 v, double t) { return V3{v.x * t, v.y * t, v.z * t}; };
  const V3 b[3] = {scale(cross(a1, a2), 2.0 * kPi / det), scale(cross(a2, a0), 2.0 * kPi / det),
                   scale(cross(a0, a1), 2.0 * kPi / det)};
  SortedField valence = sorted_field(count, hkl, density, "density");
  for (const auto& v : valence.values)
    if (!std::isfinite(v.re) || !std::isfinite(v.im))
      throw InvalidArgument("non-finite valence density Fourier coefficient");
  SortedField frozen;
  if (core_count) frozen = sorted_field(core_count, core_hkl, core, "core");
  s.with_core = core_count != 0;
  // Union in map order (the xc density's support).
  std::size_t i = 0, j = 0;
  while (i < valence.keys.size() || j < frozen.keys.size()) {
    Cx<double> v{0, 0}, c{0, 0};
    unsigned char f = 0;
    Key k;
    if (j == frozen.keys.size() || (i < valence.keys.size() && valence.keys[i] < frozen.keys[j])) {
      k = valence.keys[i];
      v = valence.values[i++];
      f = 1;
    } else if (i == valence.keys.size() || frozen.keys[j] < valence.keys[i]) {
      k = frozen.keys[j];
      c = frozen.values[j++];
      f = 2;
    } else {
      k = valence.keys[i];
      v = valence.values[i++];
      c = frozen.values[j++];
      f = 3;
    }
    const double xr = (f & 1 ? v.re : 0.0) + (f & 2 ? c.re : 0.0), xi = (f & 1 ? v.im : 0.0) + (f & 2 ? c.im : 0.0);
    if (!std::isfinite(xr) || !std::isfinite(xi))
      throw InvalidArgument("non-finite valence plus pseudo-core Fourier coefficient");
    s.keys.push_back(k);
    s.valence.push_back(v);
    s.core.push_back(c);
    s.flags.push_back(f);
  }
  int m[3] = {0, 0, 0};
  for (const auto& k : s.keys)
    for (int a = 0; a < 3; ++a) m[a] = std::max(m[a], std::abs(k[a]));
  int padding = env_padding();
  if (quadrature_padding) {
    if (quadrature_padding < 1 || quadrature_padding > 8) throw InvalidArgument("invalid XC quadrature override");
    padding = quadrature_padding;
  }
  const bool fast = env_fast_grid();
  for (int a = 0; a < 3; ++a) {
    const long long n = static_cast<long long>(padding) * std::max(3, 2 * m[a] + 1);
    const long long length = fast ? fast_fft_length(static_cast<int>(std::min<long long>(n, 1 << 20))) : n;
    if (length > kMaxLine) throw InvalidArgument("XC grid axis above 512 points is not supported");
    s.shape[a] = static_cast<int>(length);
  }
  s.points = static_cast<long long>(s.shape[0]) * s.shape[1] * s.shape[2];
  auto wrap = [](int p, int dim) {
    const int value = p % dim;
    return value < 0 ? value + dim : value;
  };
  auto index = [&](const Key& k) {
    return (static_cast<long long>(wrap(k[0], s.shape[0])) * s.shape[1] + wrap(k[1], s.shape[1])) * s.shape[2] +
           wrap(k[2], s.shape[2]);
  };
  std::unordered_map<long long, int> position;
  position.reserve(s.keys.size() * 2);
  for (std::size_t u = 0; u < s.keys.size(); ++u) position[index(s.keys[u])] = static_cast<int>(u);
  s.index.resize(s.keys.size());
  s.opposite.resize(s.keys.size());
  s.opposite_key.resize(s.keys.size());
  s.q.resize(3 * s.keys.size());
  for (std::size_t u = 0; u < s.keys.size(); ++u) {
    const Key& k = s.keys[u];
    const Key o{-k[0], -k[1], -k[2]};
    s.index[u] = index(k);
    s.opposite[u] = index(o);
    const auto found = position.find(s.opposite[u]);
    s.opposite_key[u] = found == position.end() ? -1 : found->second;
    // reciprocal_vector (src/density_functionals.cpp:34-39): h b0 + k b1 + l b2 per component.
    s.q[3 * u] = k[0] * b[0].x + k[1] * b[1].x + k[2] * b[2].x;
    s.q[3 * u + 1] = k[0] * b[0].y + k[1] * b[1].y + k[2] * b[2].y;
    s.q[3 * u + 2] = k[0] * b[0].z + k[1] * b[1].z + k[2] * b[2].z;
  }
  return s;
}

void density_functionals(Context& ctx, const FunctionalSupport& s, Cx<double>* potential, Cx<double>* xc_potential,
                         FunctionalResult& result) {
  SDFT_CUDA(cudaSetDevice(ctx.device));
  const int count = static_cast<int>(s.keys.size());
  const long long points = s.points;
  const int grids_used = s.with_core ? 4 : 2;
  // Key arrays, packed into one upload.
  const std::size_t n = s.keys.size();
  std::size_t offset = 0;
  auto take = [&](std::size_t bytes) {
    const std::size_t at = offset;
    offset += (bytes + 255) / 256 * 256;
    return at;
  };
  const std::size_t o_index = take(8 * n), o_opp = take(8 * n), o_q = take(24 * n), o_val = take(16 * n),
                    o_core = take(16 * n), o_flags = take(n), o_okey = take(4 * n);
  std::vector<unsigned char> host(offset);
  std::memcpy(host.data() + o_index, s.index.data(), 8 * n);
  std::memcpy(host.data() + o_opp, s.opposite.data(), 8 * n);
  std::memcpy(host.data() + o_q, s.q.data(), 24 * n);
  std::memcpy(host.data() + o_val, s.valence.data(), 16 * n);
  std::memcpy(host.data() + o_core, s.core.data(), 16 * n);
  std::memcpy(host.data() + o_flags, s.flags.data(), n);
  std::memcpy(host.data() + o_okey, s.opposite_key.data(), 4 * n);
  auto* dkeys = static_cast<unsigned char*>(ctx.staging_in.reserve(offset));
  SDFT_CUDA(cudaMemcpyAsync(dkeys, host.data(), offset, cudaMemcpyHostToDevice, ctx.stream));
  KeyData keys;
  keys.index = reinterpret_cast<const long long*>(dkeys + o_index);
  keys.opposite = reinterpret_cast<const long long*>(dkeys + o_opp);
  keys.q = reinterpret_cast<const double*>(dkeys + o_q);
  keys.valence = reinterpret_cast<const Cx<double>*>(dkeys + o_val);
  keys.core = reinterpret_cast<const Cx<double>*>(dkeys + o_core);
  keys.flags = dkeys + o_flags;
  keys.opposite_key = reinterpret_cast<const int*>(dkeys + o_okey);

  auto* grids = static_cast<Cx<double>*>(ctx.slab64.reserve(sizeof(Cx<double>) * points * grids_used));
  SDFT_CUDA(cudaMemsetAsync(grids, 0, sizeof(Cx<double>) * points * grids_used, ctx.stream));
  const unsigned key_blocks = static_cast<unsigned>(std::min<long long>(ceil_div(count, kKeyThreads), 148LL * 8));
  xc_scatter_kernel<<<key_blocks, kKeyThreads, 0, ctx.stream>>>(keys, count, grids, points, s.with_core);
  SDFT_LAUNCH("xc_scatter_kernel");
  fft3d<double>(grids, s.shape, grids_used, true, ctx.stream, true);

  const long long tiles = ceil_div(points, static_cast<long long>(kTile));
  const std::size_t tile_bytes = sizeof(double) * tiles * (2 * kSums + 1) + sizeof(unsigned long long) * tiles;
  const std::size_t key_bytes = sizeof(double) * key_blocks * 2 * kKeySums;
  const std::size_t merged_bytes = sizeof(double) * (2 * (kSums + kKeySums) + 4);
  auto* work = static_cast<unsigned char*>(ctx.onsite.reserve(tile_bytes + key_bytes + merged_bytes + 512));
  TileOut tile_out;
  tile_out.sums = reinterpret_cast<double*>(work);
  tile_out.minimum = tile_out.sums + tiles * 2 * kSums;
  tile_out.clipped = reinterpret_cast<unsigned long long*>(tile_out.minimum + tiles);
  auto* key_partials = reinterpret_cast<double*>(work + (tile_bytes + 255) / 256 * 256);
  auto* merged = key_partials + key_blocks * 2 * kKeySums;
  const unsigned point_blocks = static_cast<unsigned>(std::min<long long>(tiles, 148LL * 4));
  xc_points_kernel<<<point_blocks, kTileThreads, 0, ctx.stream>>>(grids, points, s.with_core, tiles, tile_out);
  SDFT_LAUNCH("xc_points_kernel");
  fft3d<double>(grids, s.shape, 2, false, ctx.stream, true);

  auto* out = static_cast<Cx<double>*>(ctx.staging_out.reserve(sizeof(Cx<double>) * 2 * n));
  xc_gather_kernel<<<key_blocks, kKeyThreads, 0, ctx.stream>>>(keys, count, grids, points, out, out + n);
  SDFT_LAUNCH("xc_gather_kernel");
  xc_key_sums_kernel<<<key_blocks, kKeyThreads, 0, ctx.stream>>>(keys, count, out + n, s.volume, key_partials);
  SDFT_LAUNCH("xc_key_sums_kernel");
  xc_merge_kernel<<<1, kTileThreads, 0, ctx.stream>>>(tile_out.sums, tiles, kSums, tile_out.minimum,
                                                      tile_out.clipped, merged);
  SDFT_LAUNCH("xc_merge_kernel tiles");
  xc_merge_kernel<<<1, kTileThreads, 0, ctx.stream>>>(key_partials, key_blocks, kKeySums, nullptr, nullptr,
                                                      merged + 2 * kSums + 2);
  SDFT_LAUNCH("xc_merge_kernel keys");
  std::vector<double> scalars(2 * (kSums + kKeySums) + 4);
  SDFT_CUDA(cudaMemcpyAsync(scalars.data(), merged, sizeof(double) * scalars.size(), cudaMemcpyDeviceToHost,
                            ctx.stream));
  SDFT_CUDA(cudaMemcpyAsync(potential, out, sizeof(Cx<double>) * n, cudaMemcpyDeviceToHost, ctx.stream));
  SDFT_CUDA(cudaMemcpyAsync(xc_potential, out + n, sizeof(Cx<double>) * n, cudaMemcpyDeviceToHost, ctx.stream));
  ctx.synchronize();

  auto total = [&](int k) { return scalars[2 * k] + scalars[2 * k + 1]; };
  const double weight = s.volume / static_cast<double>(points);
  const double* keyed = scalars.data() + 2 * kSums + 2;
  auto key_total = [&](int k) { return keyed[2 * k] + keyed[2 * k + 1]; };
  // Scaled sums in double-double before the final rounding (the reference
  // scales its long double totals).
  auto scaled = [](double hi, double lo, double w) {
    const double p = hi * w;
    const double e = std::fma(hi, w, -p);
    return p + (e + lo * w);
  };
  result.sampled_electrons = scaled(scalars[0], scalars[1], weight);
  result.xc_energy = scaled(scalars[2], scalars[3], weight);
  for (int k = 0; k < 9; ++k) result.xc_stress[k] = total(2 + k) / static_cast<double>(points);
  result.minimum_density = scalars[2 * kSums];
  result.clipped_density_points = static_cast<std::uint64_t>(scalars[2 * kSums + 1]);
  result.hartree_energy = key_total(0);
  for (int k = 0; k < 9; ++k) result.hartree_stress[k] = key_total(1 + k);
  for (int a = 0; a < 3; ++a) result.hartree_stress[4 * a] -= result.hartree_energy / s.volume;
  result.vxc_density = key_total(10);
  result.grid_points = static_cast<std::uint64_t>(points);
  for (int a = 0; a < 3; ++a) result.grid[a] = s.shape[a];
}

}  // namespace sdft_b200
