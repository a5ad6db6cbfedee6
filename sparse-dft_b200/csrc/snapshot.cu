// Solver snapshot reader: the reference's SDFTPWO3 format
// (src/plane_wave_operator.cpp:542-569 writes it, :571-653 reads it), served
// directly into a device operator.
//
// Layout: 8-byte magic; nine little-endian uint64 (npw, grid points, three
// axis lengths, projector rows, roots, iterations, warm-vector entries); two
// FP64 (overlap regularisation, tolerance); uint64 atom count and per-atom
// projector counts; then npw uint64 grid indices, FP64 kinetic, H and S
// diagonals (npw each) and the real local potential (grid points), the
// projector matrix (complex, column-major projectors x npw), per atom its D
// then Q block (complex, column-major), and the warm vectors (complex).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <stdexcept>

#include "operator.cuh"

namespace sdft_b200 {

namespace {

constexpr std::uint64_t kLimit = std::uint64_t(1) << 40;  // bound on every array length

std::uint64_t product(std::uint64_t a, std::uint64_t b) {
  if (b && a > kLimit / b) throw std::runtime_error("solver snapshot dimension overflow");
  return a * b;
}

template <typename T>
void read_into(std::ifstream& f, T* values, std::uint64_t count) {
  if (count) f.read(reinterpret_cast<char*>(values), static_cast<std::streamsize>(count * sizeof(T)));
  if (!f) throw std::runtime_error("truncated solver snapshot");
}

void check_finite(const std::vector<double>& v, const char* what) {
  for (double x : v)
    if (!std::isfinite(x)) throw std::runtime_error(std::string("nonfinite solver snapshot ") + what);
}

void check_finite(const std::vector<Cx<double>>& v, const char* what) {
  for (const auto& z : v)
    if (!std::isfinite(z.re) || !std::isfinite(z.im)) throw std::runtime_error(std::string("nonfinite solver snapshot ") + what);
}

// Frobenius norms of M and of M - M^H for an n x n column-major block.
void hermitian_check(const Cx<double>* m, std::size_t n) {
  double norm = 0, skew = 0;
  for (std::size_t j = 0; j < n; ++j)
    for (std::size_t i = 0; i < n; ++i) {
      const Cx<double> a = m[i + j * n], b = m[j + i * n];
      norm += a.re * a.re + a.im * a.im;
      const double dr = a.re - b.re, di = a.im + b.im;
      skew += dr * dr + di * di;
    }
  if (std::sqrt(skew) > 1e-12 * std::max(1.0, std::sqrt(norm)))
    throw std::runtime_error("non-Hermitian solver snapshot onsite matrix");
}

}  // namespace

OperatorSnapshot read_operator_snapshot(const std::string& path, bool header_only) {
  static_assert(std::numeric_limits<double>::is_iec559, "IEEE754 doubles expected");
  const std::uint16_t probe = 1;
  unsigned char low;
  std::memcpy(&low, &probe, 1);
  if (low != 1) throw std::runtime_error("solver snapshot currently requires little-endian IEEE754 host");
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) throw std::runtime_error("cannot open solver snapshot: " + path);
  const auto length = static_cast<long long>(f.tellg());
  f.seekg(0);
  char magic[8];
  read_into(f, magic, 8);
  const std::string format(magic, 8);
  if (format == "SDFTPWO1" || format == "SDFTPWO2")
    throw std::runtime_error("solver snapshot " + format +
                             " (folded or full D/Q) is not served on the device; SDFTPWO3 (per-atom D/Q) is");
  if (format != "SDFTPWO3") throw std::runtime_error("unsupported solver snapshot format");
  std::uint64_t h[9];
  read_into(f, h, 9);
  const std::uint64_t n = h[0], count = h[1], s0 = h[2], s1 = h[3], s2 = h[4], projectors = h[5], roots = h[6],
                      iterations = h[7], warm = h[8];
  if (!n || !count || n > count || s0 < 3 || s1 < 3 || s2 < 3 || s0 > INT_MAX || s1 > INT_MAX || s2 > INT_MAX ||
      product(product(s0, s1), s2) != count || !roots || roots > n || !iterations || iterations > INT_MAX ||
      (warm && warm != product(n, roots)))
    throw std::runtime_error("invalid solver snapshot dimensions");
  double settings[2];
  read_into(f, settings, 2);
  OperatorSnapshot snap;
  snap.npw = n;
  snap.count = count;
  snap.shape[0] = static_cast<int>(s0);
  snap.shape[1] = static_cast<int>(s1);
  snap.shape[2] = static_cast<int>(s2);
  snap.projectors = projectors;
  snap.roots = roots;
  snap.iterations = iterations;
  snap.initial_values = warm;
  snap.regularization = settings[0];
  snap.tolerance = settings[1];
  if (!std::isfinite(snap.regularization) || snap.regularization < 0 || !std::isfinite(snap.tolerance) ||
      snap.tolerance <= 0)
    throw std::runtime_error("invalid solver snapshot scalars");
  std::uint64_t atoms = 0;
  read_into(f, &atoms, 1);
  if (!atoms || atoms > projectors || length < 0 || atoms > static_cast<std::uint64_t>(length) / 8)
    throw std::runtime_error("invalid solver snapshot atom count");
  snap.channels.resize(atoms);
  read_into(f, snap.channels.data(), atoms);
  std::uint64_t sum = 0, squares = 0;
  for (auto c : snap.channels) {
    if (!c || c > projectors - sum) throw std::runtime_error("invalid solver snapshot atom boundaries");
    sum += c;
    const std::uint64_t sq = product(c, c);
    if (sq > kLimit - squares) throw std::runtime_error("solver snapshot atom storage overflow");
    squares += sq;
  }
  if (sum != projectors) throw std::runtime_error("solver snapshot atom boundaries do not span projectors");
  const std::uint64_t doubles =
      product(4, n) + count + product(2, product(n, projectors)) + product(4, squares) + product(2, warm);
  if (doubles > kLimit / 8 || static_cast<std::uint64_t>(length) != 96 + 8 * (1 + atoms) + product(8, doubles))
    throw std::runtime_error("solver snapshot size mismatch");
  if (header_only) return snap;

  snap.indices.resize(n);
  read_into(f, snap.indices.data(), n);
  {
    std::vector<std::uint64_t> sorted = snap.indices;
    std::sort(sorted.begin(), sorted.end());
    if (sorted.back() >= count || std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
      throw std::runtime_error("invalid solver snapshot FFT indices");
  }
  for (auto* array : {&snap.kinetic, &snap.h_diagonal, &snap.s_diagonal}) {
    array->resize(n);
    read_into(f, array->data(), n);
    check_finite(*array, "array");
  }
  snap.local_real.resize(count);
  read_into(f, snap.local_real.data(), count);
  check_finite(snap.local_real, "array");
  for (double v : snap.s_diagonal)
    if (v <= 0) throw std::runtime_error("invalid solver snapshot overlap diagonal");
  snap.all_b.resize(product(n, projectors));
  read_into(f, snap.all_b.data(), snap.all_b.size());
  check_finite(snap.all_b, "projector array");
  snap.d.resize(squares);
  snap.q.resize(squares);
  std::uint64_t at = 0;
  for (auto c : snap.channels) {
    read_into(f, snap.d.data() + at, c * c);
    read_into(f, snap.q.data() + at, c * c);
    at += c * c;
  }
  check_finite(snap.d, "PAW array");
  check_finite(snap.q, "PAW array");
  at = 0;
  for (auto c : snap.channels) {
    hermitian_check(snap.d.data() + at, c);
    hermitian_check(snap.q.data() + at, c);
    at += c * c;
  }
  snap.initial.resize(warm);
  read_into(f, snap.initial.data(), warm);
  check_finite(snap.initial, "warm vector");
  return snap;
}

}  // namespace sdft_b200
