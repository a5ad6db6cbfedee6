// Project-written implementation of the FFTW3 entry points declared in fftw3.h.
// Test infrastructure only: it lets the reference's unmodified CPU sources
// (the oracle) run in an image without FFTW. It is never linked into the
// product library.
//
// Algorithm: iterative Stockham autosort mixed-radix DFT (radices 4, 2, 3, 5,
// 7 and a direct O(R^2) butterfly for any other prime factor), restated from
// the DFT definition. Multi-dimensional transforms run one axis at a time on
// batches of adjacent lines held as [element][line] so the inner loop runs over
// contiguous memory. Twiddles are evaluated in long double and rounded once.
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {
using cd = std::complex<double>;
constexpr int kLines = 8;  // lines transformed together
int g_plan_threads = 1;

struct Axis {
  int n = 1;
  int sign = -1;
  std::vector<int> radices;
  std::vector<cd> twiddle;  // exp(sign*2*pi*i*m/n), m in [0,n)
};

Axis make_axis(int n, int sign) {
  if (n < 1) throw std::invalid_argument("FFT length must be positive");
  Axis axis;
  axis.n = n;
  axis.sign = sign;
  int rest = n;
  while (rest % 4 == 0) { axis.radices.push_back(4); rest /= 4; }
  for (int p : {2, 3, 5, 7}) while (rest % p == 0) { axis.radices.push_back(p); rest /= p; }
  for (int p = 11; rest > 1; p += 2) while (rest % p == 0) { axis.radices.push_back(p); rest /= p; }
  axis.twiddle.resize(n);
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < n; ++m) {
    const long double angle = two_pi * static_cast<long double>(m) / static_cast<long double>(n);
    axis.twiddle[m] = cd(static_cast<double>(std::cos(angle)),
                         static_cast<double>(sign * std::sin(angle)));
  }
  return axis;
}

// One Stockham stage of radix R on `lines` interleaved lines: element e of
// line b lives at index e*lines+b.
template <int R>
void stage_fixed(const Axis& axis, int ns, const cd* in, cd* out, int lines) {
  const int n = axis.n, m = n / R, stride = n / (ns * R), unit = n / R;
  cd omega[R];
  for (int q = 0; q < R; ++q) omega[q] = axis.twiddle[static_cast<std::size_t>(q) * unit];
  for (int j = 0; j < m; ++j) {
    const int k = j % ns;
    const int out_base = (j / ns) * ns * R + k;
    cd w[R];
    for (int r = 0; r < R; ++r) w[r] = axis.twiddle[(static_cast<std::int64_t>(r) * k * stride) % n];
    for (int b = 0; b < lines; ++b) {
      cd v[R];
      for (int r = 0; r < R; ++r) v[r] = in[static_cast<std::size_t>(j + r * m) * lines + b] * w[r];
      cd y[R];
      if constexpr (R == 2) {
        y[0] = v[0] + v[1];
        y[1] = v[0] - v[1];
      } else if constexpr (R == 4) {
        const cd a = v[0] + v[2], c = v[0] - v[2], d = v[1] + v[3];
        const cd e = (v[1] - v[3]) * omega[1];  // omega[1] = sign*i
        y[0] = a + d;
        y[2] = a - d;
        y[1] = c + e;
        y[3] = c - e;
      } else {
        for (int q = 0; q < R; ++q) {
          cd s = v[0];
          for (int r = 1; r < R; ++r) s += v[r] * omega[(r * q) % R];
          y[q] = s;
        }
      }
      for (int r = 0; r < R; ++r) out[static_cast<std::size_t>(out_base + r * ns) * lines + b] = y[r];
    }
  }
}

void stage_generic(const Axis& axis, int radix, int ns, const cd* in, cd* out, int lines) {
  const int n = axis.n, m = n / radix, stride = n / (ns * radix), unit = n / radix;
  std::vector<cd> v(radix), w(radix), omega(radix);
  for (int q = 0; q < radix; ++q) omega[q] = axis.twiddle[static_cast<std::size_t>(q) * unit];
  for (int j = 0; j < m; ++j) {
    const int k = j % ns;
    const int out_base = (j / ns) * ns * radix + k;
    for (int r = 0; r < radix; ++r) w[r] = axis.twiddle[(static_cast<std::int64_t>(r) * k * stride) % n];
    for (int b = 0; b < lines; ++b) {
      for (int r = 0; r < radix; ++r) v[r] = in[static_cast<std::size_t>(j + r * m) * lines + b] * w[r];
      for (int q = 0; q < radix; ++q) {
        cd s = v[0];
        for (int r = 1; r < radix; ++r) s += v[r] * omega[(static_cast<std::int64_t>(r) * q) % radix];
        out[static_cast<std::size_t>(out_base + q * ns) * lines + b] = s;
      }
    }
  }
}

// Transforms `lines` interleaved lines in `a` (scratch `b` of equal size).
// Returns the buffer that holds the result.
cd* transform_lines(const Axis& axis, cd* a, cd* b, int lines) {
  int ns = 1;
  cd* src = a;
  cd* dst = b;
  for (int radix : axis.radices) {
    switch (radix) {
      case 2: stage_fixed<2>(axis, ns, src, dst, lines); break;
      case 3: stage_fixed<3>(axis, ns, src, dst, lines); break;
      case 4: stage_fixed<4>(axis, ns, src, dst, lines); break;
      case 5: stage_fixed<5>(axis, ns, src, dst, lines); break;
      case 7: stage_fixed<7>(axis, ns, src, dst, lines); break;
      default: stage_generic(axis, radix, ns, src, dst, lines); break;
    }
    ns *= radix;
    std::swap(src, dst);
  }
  return src;
}

struct Plan {
  int dims[3] = {1, 1, 1};
  int howmany = 1;
  std::ptrdiff_t idist = 0, odist = 0;
  fftw_complex* in = nullptr;
  fftw_complex* out = nullptr;
  int threads = 1;
  Axis axes[3];
};

// Axis `which` of a row-major d0 x d1 x d2 array, one transform in place.
void transform_axis(const Plan& plan, cd* data, int which) {
  const int d0 = plan.dims[0], d1 = plan.dims[1], d2 = plan.dims[2];
  const Axis& axis = plan.axes[which];
  const int n = axis.n;
  if (n == 1) return;
  // Groups: (base offset, element stride, line stride, lines).
  std::size_t groups_outer, groups_inner, element_stride, line_stride, inner_extent;
  if (which == 2) {
    // rows of length d2; adjacent rows share a group
    groups_outer = 1;
    inner_extent = static_cast<std::size_t>(d0) * d1;
    element_stride = 1;
    line_stride = d2;
  } else if (which == 1) {
    groups_outer = d0;
    inner_extent = d2;
    element_stride = d2;
    line_stride = 1;
  } else {
    groups_outer = 1;
    inner_extent = static_cast<std::size_t>(d1) * d2;
    element_stride = static_cast<std::size_t>(d1) * d2;
    line_stride = 1;
  }
  groups_inner = (inner_extent + kLines - 1) / kLines;
  const std::int64_t total = static_cast<std::int64_t>(groups_outer * groups_inner);
  const std::size_t outer_offset = static_cast<std::size_t>(d1) * d2;  // only used for axis 1
  bool parallel = plan.threads > 1 && total > 1;
#ifdef _OPENMP
  parallel = parallel && !omp_in_parallel();
#pragma omp parallel num_threads(plan.threads) if (parallel)
#endif
  {
    std::vector<cd> scratch_a(static_cast<std::size_t>(n) * kLines), scratch_b(scratch_a.size());
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (std::int64_t g = 0; g < total; ++g) {
      const std::size_t outer = static_cast<std::size_t>(g) / groups_inner;
      const std::size_t first = (static_cast<std::size_t>(g) % groups_inner) * kLines;
      const int lines = static_cast<int>(std::min<std::size_t>(kLines, inner_extent - first));
      const std::size_t base = outer * outer_offset + first * line_stride;
      for (int e = 0; e < n; ++e)
        for (int b = 0; b < lines; ++b)
          scratch_a[static_cast<std::size_t>(e) * lines + b] = data[base + e * element_stride + b * line_stride];
      const cd* result = transform_lines(axis, scratch_a.data(), scratch_b.data(), lines);
      for (int e = 0; e < n; ++e)
        for (int b = 0; b < lines; ++b)
          data[base + e * element_stride + b * line_stride] = result[static_cast<std::size_t>(e) * lines + b];
    }
  }
}

void execute(const Plan& plan, fftw_complex* in, fftw_complex* out) {
  const std::size_t count = static_cast<std::size_t>(plan.dims[0]) * plan.dims[1] * plan.dims[2];
  for (int t = 0; t < plan.howmany; ++t) {
    cd* target = reinterpret_cast<cd*>(out + t * plan.odist);
    const cd* source = reinterpret_cast<const cd*>(in + t * plan.idist);
    if (source != target) std::memmove(target, source, count * sizeof(cd));
    for (int a = 2; a >= 0; --a) transform_axis(plan, target, a);
  }
}

fftw_plan make_plan(int rank, const int* n, int howmany, fftw_complex* in, int idist,
                    fftw_complex* out, int odist, int sign) {
  if (rank < 1 || rank > 3 || howmany < 1 || (sign != -1 && sign != 1)) return nullptr;
  auto* plan = new (std::nothrow) Plan();
  if (!plan) return nullptr;
  for (int a = 0; a < rank; ++a) {
    if (n[a] < 1) { delete plan; return nullptr; }
    plan->dims[3 - rank + a] = n[a];
  }
  plan->howmany = howmany;
  plan->idist = idist;
  plan->odist = odist;
  plan->in = in;
  plan->out = out;
  plan->threads = g_plan_threads;
  for (int a = 0; a < 3; ++a) plan->axes[a] = make_axis(plan->dims[a], sign);
  return reinterpret_cast<fftw_plan>(plan);
}
}  // namespace

extern "C" {
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex* in, fftw_complex* out, int sign,
                           unsigned /*flags*/) {
  const int n[3] = {n0, n1, n2};
  return make_plan(3, n, 1, in, 0, out, 0, sign);
}
fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in,
                             const int* inembed, int istride, int idist, fftw_complex* out,
                             const int* onembed, int ostride, int odist, int sign,
                             unsigned /*flags*/) {
  if (inembed || onembed || istride != 1 || ostride != 1) return nullptr;  // unused layouts
  return make_plan(rank, n, howmany, in, idist, out, odist, sign);
}
void fftw_execute(const fftw_plan plan) {
  const auto* p = reinterpret_cast<const Plan*>(plan);
  execute(*p, p->in, p->out);
}
void fftw_execute_dft(const fftw_plan plan, fftw_complex* in, fftw_complex* out) {
  execute(*reinterpret_cast<const Plan*>(plan), in, out);
}
void fftw_destroy_plan(fftw_plan plan) { delete reinterpret_cast<Plan*>(plan); }
fftw_complex* fftw_alloc_complex(size_t n) {
  void* p = nullptr;
  if (posix_memalign(&p, 64, (n ? n : 1) * sizeof(fftw_complex)) != 0) return nullptr;
  return static_cast<fftw_complex*>(p);
}
void fftw_free(void* p) { std::free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { g_plan_threads = nthreads < 1 ? 1 : nthreads; }
}
