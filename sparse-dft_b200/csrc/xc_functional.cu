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
#include <climits>
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
// CTA, width <= kMergeWidth); minimum and clipped counts when given.
constexpr int kMergeWidth = 12;
__global__ void __launch_bounds__(kTileThreads) xc_merge_kernel(const double* records, long long count, int width,
                                                                const double* minimum,
                                                                const unsigned long long* clipped, double* out) {
  __shared__ DD shared[kMergeWidth * (kTileThreads / 32)];
  __shared__ double shared_min[kTileThreads];
  __shared__ unsigned long long shared_clip[kTileThreads];
  DD sums[kMergeWidth];
  for (int k = 0; k < kMergeWidth; ++k) sums[k] = DD{0.0, 0.0};
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

// The XC grid padding * max(3, 2 m_a + 1) per axis (rounded to a smooth
// length under SDFT_FAST_DENSITY_GRID=1, the reference's cached_grid), the
// wrapped grid indices of +G and -G, the union position of -G and the G
// vectors of the support's keys.
void finish_support(FunctionalSupport& s, const V3 b[3], int padding) {
  int m[3] = {0, 0, 0};
  for (const auto& k : s.keys)
    for (int a = 0; a < 3; ++a) m[a] = std::max(m[a], std::abs(k[a]));
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
}

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
  int padding = env_padding();
  if (quadrature_padding) {
    if (quadrature_padding < 1 || quadrature_padding > 8) throw InvalidArgument("invalid XC quadrature override");
    padding = quadrature_padding;
  }
  finish_support(s, b, padding);
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

namespace {

constexpr int kSpinSums = 10;     // tile sums: energy, stress[9]
constexpr int kSpinKeySums = 12;  // key sums: Hartree energy, stress[9], <n_s, v_xc,s> for s = up, down
static_assert(kSums <= kMergeWidth && kKeySums <= kMergeWidth && kSpinSums <= kMergeWidth &&
                  kSpinKeySums <= kMergeWidth,
              "merge records wider than the merge kernel");

// xc density of channel s (density[s] + core / 2, src/density_functionals.cpp:767-768)
// of key i, and whether the key is in that xc density.
__device__ __forceinline__ bool spin_xc(const KeyData& keys, const Cx<double>* down, int i, int s, Cx<double>& v) {
  const unsigned char f = keys.flags[i];
  const bool has = s == 0 ? (f & 1u) : (f & 4u);
  const bool core = f & 2u;
  if (!has && !core) return false;
  v = has ? (s == 0 ? keys.valence[i] : down[i]) : Cx<double>{0.0, 0.0};
  if (core) {
    const Cx<double> c = keys.core[i];
    v = Cx<double>{__dadd_rn(v.re, 0.5 * c.re), __dadd_rn(v.im, 0.5 * c.im)};
  }
  return true;
}

// grids: [nz, xy] of the up channel's xc density, then of the down channel's.
__global__ void spin_scatter_kernel(KeyData keys, const Cx<double>* down, int count, Cx<double>* grids,
                                    long long points) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const long long at = keys.index[i];
    const double* q = keys.q + 3 * i;
    for (int s = 0; s < 2; ++s) {
      Cx<double> v;
      if (spin_xc(keys, down, i, s, v))
        scatter_fields(v, q, grids + 2 * s * points, grids + (2 * s + 1) * points, at);
    }
  }
}

struct SpinTileOut {
  double* sums;                  // [tiles][kSpinSums][2]
  double* minimum[2];            // [tiles] per channel
  unsigned long long* negative[2];
};

// Collinear PBE per point with the reference's density floors and fixed-tile
// sums (src/density_functionals.cpp:776-797); the four response fields
// v_s + i d_x,s and d_y,s + i d_z,s overwrite the inputs.
__global__ void __launch_bounds__(kTileThreads) spin_points_kernel(Cx<double>* grids, long long points,
                                                                   long long tiles, SpinTileOut out,
                                                                   unsigned int* nonfinite) {
  __shared__ DD shared[kSpinSums * (kTileThreads / 32)];
  __shared__ double shared_min[2][kTileThreads];
  __shared__ unsigned long long shared_neg[2][kTileThreads];
  for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
    DD sums[kSpinSums];
    for (int k = 0; k < kSpinSums; ++k) sums[k] = DD{0.0, 0.0};
    double minimum[2] = {INFINITY, INFINITY};
    unsigned long long negative[2] = {0, 0};
    bool bad = false;
    const long long first = t * kTile;
    for (int p = threadIdx.x; p < kTile; p += kTileThreads) {
      const long long i = first + p;
      if (i >= points) break;
      double raw[2], g[2][3];
      for (int s = 0; s < 2; ++s) {
        const Cx<double> a = grids[2 * s * points + i], b = grids[(2 * s + 1) * points + i];
        raw[s] = a.re;
        g[s][0] = b.re;
        g[s][1] = b.im;
        g[s][2] = a.im;
      }
      double n[2] = {raw[0], raw[1]};
      if (n[0] + n[1] < 1e-10) {
        n[0] = fmax(n[0], 5e-11);
        n[1] = fmax(n[1], 5e-11);
      }
      const pbe::SpinPoint xc = pbe::pbe_collinear(fmax(5e-11, n[0]), fmax(5e-11, n[1]), g[0], g[1]);
      bad |= !isfinite(xc.energy) || !isfinite(xc.density_potential[0]) || !isfinite(xc.density_potential[1]);
      sums[0] = dd_add(sums[0], xc.energy);
      double pressure = xc.energy;
      for (int s = 0; s < 2; ++s) {
        minimum[s] = fmin(minimum[s], raw[s]);
        negative[s] += raw[s] < 0;
        pressure = __dsub_rn(pressure, __dmul_rn(xc.density_potential[s], raw[s]));
        for (int a = 0; a < 3; ++a) {
          bad |= !isfinite(xc.gradient_response[s][a]);
          pressure = __dsub_rn(pressure, __dmul_rn(xc.gradient_response[s][a], g[s][a]));
        }
        grids[2 * s * points + i] = Cx<double>{xc.density_potential[s], xc.gradient_response[s][0]};
        grids[(2 * s + 1) * points + i] = Cx<double>{xc.gradient_response[s][1], xc.gradient_response[s][2]};
      }
      for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c) {
          double term = a == c ? pressure : 0.0;
          for (int s = 0; s < 2; ++s) term = __dsub_rn(term, __dmul_rn(xc.gradient_response[s][a], g[s][c]));
          sums[1 + 3 * a + c] = dd_add(sums[1 + 3 * a + c], term);
        }
    }
    if (bad) atomicOr(nonfinite, 1u);
    block_reduce<kTileThreads>(sums, kSpinSums, shared);
    for (int s = 0; s < 2; ++s) {
      shared_min[s][threadIdx.x] = minimum[s];
      shared_neg[s][threadIdx.x] = negative[s];
    }
    __syncthreads();
    for (int stride = kTileThreads / 2; stride > 0; stride /= 2) {
      if (threadIdx.x < stride)
        for (int s = 0; s < 2; ++s) {
          shared_min[s][threadIdx.x] = fmin(shared_min[s][threadIdx.x], shared_min[s][threadIdx.x + stride]);
          shared_neg[s][threadIdx.x] += shared_neg[s][threadIdx.x + stride];
        }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      for (int k = 0; k < kSpinSums; ++k) {
        out.sums[(t * kSpinSums + k) * 2] = sums[k].hi;
        out.sums[(t * kSpinSums + k) * 2 + 1] = sums[k].lo;
      }
      for (int s = 0; s < 2; ++s) {
        out.minimum[s][t] = shared_min[s][0];
        out.negative[s][t] = shared_neg[s][0];
      }
    }
    __syncthreads();
  }
}

// Per key and channel: paired extraction, v_xc,s, and the potential
// (Hartree of the total density where the key is a density key, :753-758,
// :800-803).
__global__ void spin_gather_kernel(KeyData keys, const Cx<double>* down, int count, const Cx<double>* grids,
                                   long long points, Cx<double>* potential, Cx<double>* xc_potential) {
  const double twice = 2.0 * static_cast<double>(points);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const long long at = keys.index[i], op = keys.opposite[i];
    const double* q = keys.q + 3 * i;
    const unsigned char f = keys.flags[i];
    const bool in_total = f & 5u;
    Cx<double> vh{0.0, 0.0};
    if (in_total) {
      const Cx<double> up = (f & 1u) ? keys.valence[i] : Cx<double>{0.0, 0.0};
      const Cx<double> dn = (f & 4u) ? down[i] : Cx<double>{0.0, 0.0};
      const Cx<double> total = (f & 1u) ? ((f & 4u) ? Cx<double>{__dadd_rn(up.re, dn.re), __dadd_rn(up.im, dn.im)} : up)
                                        : dn;
      const double q2 = __dadd_rn(__dadd_rn(__dmul_rn(q[0], q[0]), __dmul_rn(q[1], q[1])), __dmul_rn(q[2], q[2]));
      if (!(q2 < 1e-12))
        vh = Cx<double>{__ddiv_rn(__dmul_rn(4 * kPi, total.re), q2), __ddiv_rn(__dmul_rn(4 * kPi, total.im), q2)};
    }
    for (int s = 0; s < 2; ++s) {
      Cx<double> field[4];
      for (int g = 0; g < 2; ++g) {
        const long long base = (2 * s + g) * points;
        const Cx<double> direct = grids[base + at], o = grids[base + op];
        const Cx<double> opposite{o.re, -o.im};
        field[2 * g] = Cx<double>{__ddiv_rn(__dadd_rn(direct.re, opposite.re), twice),
                                  __ddiv_rn(__dadd_rn(direct.im, opposite.im), twice)};
        const double dre = __dsub_rn(direct.re, opposite.re), dim = __dsub_rn(direct.im, opposite.im);
        field[2 * g + 1] = Cx<double>{__ddiv_rn(dim, twice), __ddiv_rn(-dre, twice)};
      }
      const double sre = __dadd_rn(__dadd_rn(__dmul_rn(q[0], field[1].re), __dmul_rn(q[1], field[2].re)),
                                   __dmul_rn(q[2], field[3].re));
      const double sim = __dadd_rn(__dadd_rn(__dmul_rn(q[0], field[1].im), __dmul_rn(q[1], field[2].im)),
                                   __dmul_rn(q[2], field[3].im));
      const Cx<double> vxc{__dadd_rn(field[0].re, sim), __dsub_rn(field[0].im, sre)};
      xc_potential[static_cast<long long>(s) * count + i] = vxc;
      potential[static_cast<long long>(s) * count + i] = Cx<double>{__dadd_rn(vh.re, vxc.re), __dadd_rn(vh.im, vxc.im)};
    }
  }
}

// Per-block partial sums: Hartree energy and stress of the total density
// (:753-758) and <n_s, v_xc,s> over each channel's keys (:804).
__global__ void __launch_bounds__(kKeyThreads) spin_key_sums_kernel(KeyData keys, const Cx<double>* down, int count,
                                                                    const Cx<double>* xc_potential, double volume,
                                                                    double* partials) {
  __shared__ DD shared[kSpinKeySums * (kKeyThreads / 32)];
  DD sums[kSpinKeySums];
  for (int k = 0; k < kSpinKeySums; ++k) sums[k] = DD{0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const unsigned char f = keys.flags[i];
    if (!(f & 5u)) continue;
    const Cx<double> up = (f & 1u) ? keys.valence[i] : Cx<double>{0.0, 0.0};
    const Cx<double> dn = (f & 4u) ? down[i] : Cx<double>{0.0, 0.0};
    const Cx<double> total = (f & 1u) ? ((f & 4u) ? Cx<double>{__dadd_rn(up.re, dn.re), __dadd_rn(up.im, dn.im)} : up)
                                      : dn;
    const double* q = keys.q + 3 * i;
    const double q2 = __dadd_rn(__dadd_rn(__dmul_rn(q[0], q[0]), __dmul_rn(q[1], q[1])), __dmul_rn(q[2], q[2]));
    if (!(q2 < 1e-12)) {
      const double norm = __dadd_rn(__dmul_rn(total.re, total.re), __dmul_rn(total.im, total.im));
      sums[0] = dd_add(sums[0], __ddiv_rn(__dmul_rn(__dmul_rn(2 * kPi, volume), norm), q2));
      const double q4 = __dmul_rn(q2, q2);
      for (int a = 0; a < 3; ++a)
        for (int c = 0; c < 3; ++c)
          sums[1 + 3 * a + c] =
              dd_add(sums[1 + 3 * a + c], __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(4 * kPi, norm), q[a]), q[c]), q4));
    }
    const int o = keys.opposite_key[i];
    if (o >= 0)
      for (int s = 0; s < 2; ++s) {
        if (!(f & (s == 0 ? 1u : 4u))) continue;
        const Cx<double> rho = s == 0 ? up : dn;
        const Cx<double> v = xc_potential[static_cast<long long>(s) * count + o];
        sums[10 + s] =
            dd_add(sums[10 + s], __dmul_rn(volume, __dsub_rn(__dmul_rn(rho.re, v.re), __dmul_rn(rho.im, v.im))));
      }
  }
  block_reduce<kKeyThreads>(sums, kSpinKeySums, shared);
  if (threadIdx.x == 0)
    for (int k = 0; k < kSpinKeySums; ++k) {
      partials[(blockIdx.x * kSpinKeySums + k) * 2] = sums[k].hi;
      partials[(blockIdx.x * kSpinKeySums + k) * 2 + 1] = sums[k].lo;
    }
}

}  // namespace

FunctionalSupport collinear_support(const double lattice[9], const std::size_t count[2], const int* const hkl[2],
                                    const double* const density[2], std::size_t core_count, const int* core_hkl,
                                    const double* core, int padding) {
  const V3 a0{lattice[0], lattice[1], lattice[2]}, a1{lattice[3], lattice[4], lattice[5]},
      a2{lattice[6], lattice[7], lattice[8]};
  auto cross = [](V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; };
  auto dot = [](V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; };
  const double det = dot(a0, cross(a1, a2));
  const double volume = std::abs(det);
  if (!std::isfinite(volume) || volume < 1e-12 || !count[0] || !count[1])
    throw InvalidArgument("invalid collinear density/lattice");
  FunctionalSupport s;
  s.volume = volume;
  s.collinear = true;
  auto scale = [](V3 v, double t) { return V3{v.x * t, v.y * t, v.z * t}; };
  const V3 b[3] = {scale(cross(a1, a2), 2.0 * kPi / det), scale(cross(a2, a0), 2.0 * kPi / det),
                   scale(cross(a0, a1), 2.0 * kPi / det)};
  const SortedField up = sorted_field(count[0], hkl[0], density[0], "spin density");
  const SortedField dn = sorted_field(count[1], hkl[1], density[1], "spin density");
  SortedField frozen;
  if (core_count) frozen = sorted_field(core_count, core_hkl, core, "core");
  s.with_core = core_count != 0;
  // Three-way union in map order.
  std::size_t i = 0, j = 0, k = 0;
  while (i < up.keys.size() || j < dn.keys.size() || k < frozen.keys.size()) {
    Key least{INT32_MAX, INT32_MAX, INT32_MAX};
    if (i < up.keys.size()) least = std::min(least, up.keys[i]);
    if (j < dn.keys.size()) least = std::min(least, dn.keys[j]);
    if (k < frozen.keys.size()) least = std::min(least, frozen.keys[k]);
    Cx<double> u{0, 0}, d{0, 0}, c{0, 0};
    unsigned char f = 0;
    if (i < up.keys.size() && up.keys[i] == least) {
      u = up.values[i++];
      f |= 1;
    }
    if (j < dn.keys.size() && dn.keys[j] == least) {
      d = dn.values[j++];
      f |= 4;
    }
    if (k < frozen.keys.size() && frozen.keys[k] == least) {
      c = frozen.values[k++];
      f |= 2;
    }
    // The total density (:752-756) must be finite.
    if (f & 5) {
      const double tr = (f & 1 ? u.re : 0.0) + (f & 4 ? d.re : 0.0), ti = (f & 1 ? u.im : 0.0) + (f & 4 ? d.im : 0.0);
      if (!std::isfinite(tr) || !std::isfinite(ti)) throw InvalidArgument("nonfinite spin density");
    }
    s.keys.push_back(least);
    s.valence.push_back(u);
    s.down.push_back(d);
    s.core.push_back(c);
    s.flags.push_back(f);
  }
  if (!padding) {
    padding = 2;
    if (const char* v = std::getenv("SDFT_FFT_OVERSAMPLING")) {
      char* end = nullptr;
      const long n = std::strtol(v, &end, 10);
      if (!end || *end || n < 1 || n > 8) throw InvalidArgument("invalid FFT oversampling");
      padding = static_cast<int>(n);
    }
  }
  if (padding < 1 || padding > 8) throw InvalidArgument("invalid collinear XC padding");
  finish_support(s, b, padding);
  return s;
}

void collinear_functionals(Context& ctx, const FunctionalSupport& s, Cx<double>* const potential[2],
                           Cx<double>* const xc_potential[2], FunctionalResult result[2]) {
  if (!s.collinear) throw InvalidArgument("collinear functional needs a collinear support");
  SDFT_CUDA(cudaSetDevice(ctx.device));
  const int count = static_cast<int>(s.keys.size());
  const long long points = s.points;
  const std::size_t n = s.keys.size();
  std::size_t offset = 0;
  auto take = [&](std::size_t bytes) {
    const std::size_t at = offset;
    offset += (bytes + 255) / 256 * 256;
    return at;
  };
  const std::size_t o_index = take(8 * n), o_opp = take(8 * n), o_q = take(24 * n), o_val = take(16 * n),
                    o_core = take(16 * n), o_down = take(16 * n), o_flags = take(n), o_okey = take(4 * n);
  std::vector<unsigned char> host(offset);
  std::memcpy(host.data() + o_index, s.index.data(), 8 * n);
  std::memcpy(host.data() + o_opp, s.opposite.data(), 8 * n);
  std::memcpy(host.data() + o_q, s.q.data(), 24 * n);
  std::memcpy(host.data() + o_val, s.valence.data(), 16 * n);
  std::memcpy(host.data() + o_core, s.core.data(), 16 * n);
  std::memcpy(host.data() + o_down, s.down.data(), 16 * n);
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
  const auto* down = reinterpret_cast<const Cx<double>*>(dkeys + o_down);

  auto* grids = static_cast<Cx<double>*>(ctx.slab64.reserve(sizeof(Cx<double>) * points * 4));
  SDFT_CUDA(cudaMemsetAsync(grids, 0, sizeof(Cx<double>) * points * 4, ctx.stream));
  const unsigned key_blocks = static_cast<unsigned>(std::min<long long>(ceil_div(count, kKeyThreads), 148LL * 8));
  spin_scatter_kernel<<<key_blocks, kKeyThreads, 0, ctx.stream>>>(keys, down, count, grids, points);
  SDFT_LAUNCH("spin_scatter_kernel");
  fft3d<double>(grids, s.shape, 4, true, ctx.stream, true);

  const long long tiles = ceil_div(points, static_cast<long long>(kTile));
  const std::size_t tile_bytes = sizeof(double) * tiles * (2 * kSpinSums + 2) + sizeof(unsigned long long) * tiles * 2;
  const std::size_t key_bytes = sizeof(double) * key_blocks * 2 * kSpinKeySums;
  const std::size_t merged_doubles = 3 * (2 * kSpinKeySums + 2);
  auto* work = static_cast<unsigned char*>(ctx.onsite.reserve(tile_bytes + key_bytes + 8 * merged_doubles + 1024));
  SpinTileOut tile_out;
  tile_out.sums = reinterpret_cast<double*>(work);
  tile_out.minimum[0] = tile_out.sums + tiles * 2 * kSpinSums;
  tile_out.minimum[1] = tile_out.minimum[0] + tiles;
  tile_out.negative[0] = reinterpret_cast<unsigned long long*>(tile_out.minimum[1] + tiles);
  tile_out.negative[1] = tile_out.negative[0] + tiles;
  auto* key_partials = reinterpret_cast<double*>(work + (tile_bytes + 255) / 256 * 256);
  auto* flag_word = reinterpret_cast<unsigned int*>(key_partials + key_blocks * 2 * kSpinKeySums);
  auto* merged = reinterpret_cast<double*>(flag_word + 4);
  SDFT_CUDA(cudaMemsetAsync(flag_word, 0, sizeof(unsigned int), ctx.stream));
  const unsigned point_blocks = static_cast<unsigned>(std::min<long long>(tiles, 148LL * 4));
  spin_points_kernel<<<point_blocks, kTileThreads, 0, ctx.stream>>>(grids, points, tiles, tile_out, flag_word);
  SDFT_LAUNCH("spin_points_kernel");
  fft3d<double>(grids, s.shape, 4, false, ctx.stream, true);

  auto* out = static_cast<Cx<double>*>(ctx.staging_out.reserve(sizeof(Cx<double>) * 4 * n));
  spin_gather_kernel<<<key_blocks, kKeyThreads, 0, ctx.stream>>>(keys, down, count, grids, points, out, out + 2 * n);
  SDFT_LAUNCH("spin_gather_kernel");
  spin_key_sums_kernel<<<key_blocks, kKeyThreads, 0, ctx.stream>>>(keys, down, count, out + 2 * n, s.volume,
                                                                    key_partials);
  SDFT_LAUNCH("spin_key_sums_kernel");
  // Merged records: [tile sums, min up, negatives up], [min down, negatives down], [key sums].
  const int stride = 2 * kSpinKeySums + 2;
  xc_merge_kernel<<<1, kTileThreads, 0, ctx.stream>>>(tile_out.sums, tiles, kSpinSums, tile_out.minimum[0],
                                                      tile_out.negative[0], merged);
  SDFT_LAUNCH("xc_merge_kernel spin tiles");
  xc_merge_kernel<<<1, kTileThreads, 0, ctx.stream>>>(tile_out.sums, tiles, 0, tile_out.minimum[1],
                                                      tile_out.negative[1], merged + stride);
  SDFT_LAUNCH("xc_merge_kernel spin down");
  xc_merge_kernel<<<1, kTileThreads, 0, ctx.stream>>>(key_partials, key_blocks, kSpinKeySums, nullptr, nullptr,
                                                      merged + 2 * stride);
  SDFT_LAUNCH("xc_merge_kernel spin keys");
  std::vector<double> scalars(3 * stride);
  unsigned int bad = 0;
  SDFT_CUDA(cudaMemcpyAsync(scalars.data(), merged, sizeof(double) * scalars.size(), cudaMemcpyDeviceToHost,
                            ctx.stream));
  SDFT_CUDA(cudaMemcpyAsync(&bad, flag_word, sizeof(bad), cudaMemcpyDeviceToHost, ctx.stream));
  for (int c = 0; c < 2; ++c) {
    SDFT_CUDA(cudaMemcpyAsync(potential[c], out + c * n, sizeof(Cx<double>) * n, cudaMemcpyDeviceToHost, ctx.stream));
    SDFT_CUDA(cudaMemcpyAsync(xc_potential[c], out + (2 + c) * n, sizeof(Cx<double>) * n, cudaMemcpyDeviceToHost,
                              ctx.stream));
  }
  ctx.synchronize();
  if (bad) throw NonFinite("nonfinite spin PBE response");

  const double energy = scalars[0] + scalars[1];  // the reference rounds its long double total to double
  const double* keyed = scalars.data() + 2 * stride;
  auto key_total = [&](int k) { return keyed[2 * k] + keyed[2 * k + 1]; };
  const double eh = key_total(0);
  for (int c = 0; c < 2; ++c) {
    FunctionalResult& r = result[c];
    r.hartree_energy = .5 * eh;
    for (int k = 0; k < 9; ++k) {
      double h = key_total(1 + k);
      if (k % 4 == 0) h -= eh / s.volume;
      r.hartree_stress[k] = .5 * h;
      r.xc_stress[k] = .5 * (scalars[2 + 2 * k] + scalars[3 + 2 * k]) / static_cast<double>(points);
    }
    r.xc_energy = .5 * energy * s.volume / static_cast<double>(points);
    const double* channel = scalars.data() + c * stride;
    const int width = c == 0 ? kSpinSums : 0;
    r.minimum_density = channel[2 * width];
    r.clipped_density_points = static_cast<std::uint64_t>(channel[2 * width + 1]);
    r.vxc_density = key_total(10 + c);
    r.grid_points = static_cast<std::uint64_t>(points);
    for (int a = 0; a < 3; ++a) r.grid[a] = s.shape[a];
    r.sampled_electrons = 0.0;
    for (std::size_t u = 0; u < n; ++u)
      if (s.keys[u] == Key{0, 0, 0} && (s.flags[u] & (c == 0 ? 1 : 4)))
        r.sampled_electrons = s.volume * (c == 0 ? s.valence[u].re : s.down[u].re);
  }
}

}  // namespace sdft_b200
