// Mixed-radix (2, 3, 4, 5, 7) line FFT on shared memory, one warp per line.
//
// Stockham autosort formulation (each stage reads x[j + r*n/R], applies the
// twiddle W^(r*(j mod Ns)*n/(Ns*R)), a radix-R DFT, and writes to
// (j/Ns)*Ns*R + (j mod Ns) + r*Ns), executed in place: every lane first loads
// all inputs of its butterflies into registers, the warp synchronises, then
// the lane writes its outputs. Lines may be strided in shared memory, so the
// same routine serves rows, columns and pencils of a staged tile.
//
// Sign convention (the reference's FFTW calls): forward X_k = sum x_j
// exp(-2 pi i jk/n), backward uses +i, both unnormalised. Twiddles come from a
// table w[m] = exp(-2 pi i m/n) evaluated on the host in long double.
#pragma once
#include "common.cuh"

namespace sdft_b200 {

constexpr int kMaxStages = 12;
constexpr int kMaxLine = 512;

struct LinePlan {
  int n = 1;
  int stages = 0;
  int radix[kMaxStages] = {};
};

// Host: factor n into supported radices (4 first, then 2, 3, 5, 7). With
// general = true the rest of n is factored into odd primes above 7, which
// only the general-length drivers (fft_lines_pp_general) execute.
LinePlan make_line_plan(int n, bool general = false);
bool fft_length_supported(int n);
// Smallest 2/3/5/7-smooth length >= minimum (the reference's fast_fft_length,
// src/fft_planning.hpp:16-23).
int fast_fft_length(int minimum);

template <typename T, bool INV>
__device__ __forceinline__ Cx<T> twiddle(const Cx<T>* tw, int index) {
  Cx<T> w = tw[index];
  if (INV) w.im = -w.im;
  return w;
}

// (a) * (+/- i)
template <typename T, bool INV>
__device__ __forceinline__ Cx<T> rotate_quarter(Cx<T> a) {
  // forward: multiply by -i -> (im, -re); backward: by +i -> (-im, re)
  return INV ? Cx<T>{-a.im, a.re} : Cx<T>{a.im, -a.re};
}

template <typename T, int R, bool INV>
__device__ __forceinline__ void radix_dft(Cx<T>* v, const Cx<T>* tw, int unit) {
  if constexpr (R == 2) {
    const Cx<T> a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
  } else if constexpr (R == 4) {
    const Cx<T> a = v[0] + v[2], c = v[0] - v[2], d = v[1] + v[3];
    const Cx<T> e = rotate_quarter<T, INV>(v[1] - v[3]);
    v[0] = a + d;
    v[2] = a - d;
    v[1] = c + e;
    v[3] = c - e;
  } else {
    // Odd R: pair r with R-r. omega^q = tw[q*unit] (forward sign).
    constexpr int H = (R - 1) / 2;
    Cx<T> a[H], b[H];
#pragma unroll
    for (int r = 1; r <= H; ++r) {
      a[r - 1] = v[r] + v[R - r];
      b[r - 1] = v[r] - v[R - r];
    }
    const Cx<T> x0 = v[0];
    Cx<T> sum = x0;
#pragma unroll
    for (int r = 0; r < H; ++r) sum = sum + a[r];
    v[0] = sum;
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      T cre = x0.re, cim = x0.im, sre = 0, sim = 0;
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        const Cx<T> w = tw[((r * q) % R) * unit];  // cos, -sin (forward)
        cre += a[r - 1].re * w.re;
        cim += a[r - 1].im * w.re;
        // i * S * b with S = w.im (forward) or -w.im (backward)
        const T s = INV ? -w.im : w.im;
        sre -= b[r - 1].im * s;
        sim += b[r - 1].re * s;
      }
      v[q] = Cx<T>{cre + sre, cim + sim};
      v[R - q] = Cx<T>{cre - sre, cim - sim};
    }
  }
}

template <typename T, int R, int NMAX, bool INV>
__device__ __forceinline__ void line_stage(Cx<T>* line, int stride, int n, int ns, const Cx<T>* tw, int lane) {
  constexpr int MAXB = (NMAX / R + kWarp - 1) / kWarp;
  const int m = n / R;
  const int twstride = n / (ns * R);
  const int unit = n / R;
  Cx<T> v[MAXB][R];
#pragma unroll
  for (int b = 0; b < MAXB; ++b) {
    const int j = lane + b * kWarp;
    if (j < m) {
      const int k = j % ns;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        Cx<T> x = line[(j + r * m) * stride];
        if (r > 0 && k > 0) x = cmul(x, twiddle<T, INV>(tw, r * k * twstride));
        v[b][r] = x;
      }
    }
  }
  __syncwarp();
#pragma unroll
  for (int b = 0; b < MAXB; ++b) {
    const int j = lane + b * kWarp;
    if (j < m) {
      radix_dft<T, R, INV>(v[b], tw, unit);
      const int k = j % ns;
      const int base = (j / ns) * ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) line[(base + r * ns) * stride] = v[b][r];
    }
  }
  __syncwarp();
}

// One warp transforms one line of plan.n elements at line[e*stride].
template <typename T, int NMAX, bool INV>
__device__ void fft_line(Cx<T>* line, int stride, const LinePlan& plan, const Cx<T>* tw, int lane) {
  int ns = 1;
  for (int s = 0; s < plan.stages; ++s) {
    const int r = plan.radix[s];
    switch (r) {
      case 2: line_stage<T, 2, NMAX, INV>(line, stride, plan.n, ns, tw, lane); break;
      case 3: line_stage<T, 3, NMAX, INV>(line, stride, plan.n, ns, tw, lane); break;
      case 4: line_stage<T, 4, NMAX, INV>(line, stride, plan.n, ns, tw, lane); break;
      case 5: line_stage<T, 5, NMAX, INV>(line, stride, plan.n, ns, tw, lane); break;
      case 7: line_stage<T, 7, NMAX, INV>(line, stride, plan.n, ns, tw, lane); break;
      default: break;  // rejected on the host
    }
    ns *= r;
  }
}

// Whole-CTA batched variant (blockDim.x == 256): lanes map to lines (32 per
// batch) and the 8 warps split each stage's butterflies, so index arithmetic
// and twiddle loads are warp-uniform and every lane works on its own line.
// Line t's element e lives at base[line_offset(t) * line_stride + e * elem_stride],
// line_offset(t) = rows ? rows[t] : t. Contains __syncthreads: call uniformly.
constexpr int kFftThreads = 256;
constexpr int kFftWarps = kFftThreads / kWarp;

template <typename T, int R, int NMAX, bool INV>
__device__ __forceinline__ void cta_stage(Cx<T>* line, int es, int n, int ns, const Cx<T>* tw, int warp,
                                          bool active) {
  constexpr int MAXB = ((NMAX + R - 1) / R + kFftWarps - 1) / kFftWarps;
  const int m = n / R;
  const int twstride = n / (ns * R);
  const int unit = n / R;
  Cx<T> v[MAXB][R];
#pragma unroll
  for (int b = 0; b < MAXB; ++b) {
    const int j = warp + b * kFftWarps;
    if (j < m && active) {
      const int k = j % ns;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        Cx<T> x = line[(j + r * m) * es];
        if (r > 0 && k > 0) x = cmul(x, twiddle<T, INV>(tw, r * k * twstride));
        v[b][r] = x;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int b = 0; b < MAXB; ++b) {
    const int j = warp + b * kFftWarps;
    if (j < m && active) {
      radix_dft<T, R, INV>(v[b], tw, unit);
      const int k = j % ns;
      const int base = (j / ns) * ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) line[(base + r * ns) * es] = v[b][r];
    }
  }
  __syncthreads();
}

template <typename T, int NMAX, bool INV>
__device__ void fft_lines(Cx<T>* base, int count, int line_stride, int elem_stride, const int* rows,
                          const LinePlan& plan, const Cx<T>* tw) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int b0 = 0; b0 < count; b0 += kWarp) {
    const int t = b0 + lane;
    const bool active = t < count;
    const int offset = active ? (rows ? rows[t] : t) : 0;
    Cx<T>* line = base + offset * line_stride;
    int ns = 1;
    for (int s = 0; s < plan.stages; ++s) {
      const int r = plan.radix[s];
      switch (r) {
        case 2: cta_stage<T, 2, NMAX, INV>(line, elem_stride, plan.n, ns, tw, warp, active); break;
        case 3: cta_stage<T, 3, NMAX, INV>(line, elem_stride, plan.n, ns, tw, warp, active); break;
        case 4: cta_stage<T, 4, NMAX, INV>(line, elem_stride, plan.n, ns, tw, warp, active); break;
        case 5: cta_stage<T, 5, NMAX, INV>(line, elem_stride, plan.n, ns, tw, warp, active); break;
        case 7: cta_stage<T, 7, NMAX, INV>(line, elem_stride, plan.n, ns, tw, warp, active); break;
        default: break;
      }
      ns *= r;
    }
  }
}

// Out-of-place (ping-pong) batched variant: every stage reads one buffer and
// writes the other, so only one butterfly is live per thread and any line
// length works. Lanes map to lines, warps split butterflies, one
// __syncthreads per stage. Returns the buffer that holds the result.
template <typename T, int R, bool INV>
__device__ __forceinline__ void pp_butterflies(const Cx<T>* src_line, Cx<T>* dst_line, int es, int n, int ns,
                                               const Cx<T>* tw, int warp) {
  const int m = n / R, twstride = n / (ns * R), unit = n / R;
  for (int j = warp; j < m; j += kFftWarps) {
    const int k = j % ns;
    Cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      Cx<T> x = src_line[(j + r * m) * es];
      if (r > 0 && k > 0) x = cmul(x, twiddle<T, INV>(tw, r * k * twstride));
      v[r] = x;
    }
    radix_dft<T, R, INV>(v, tw, unit);
    const int base = (j / ns) * ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst_line[(base + r * ns) * es] = v[r];
  }
}

// Radix-R DFT on v with the stage's roots held in registers:
// roots[p] = exp(-2 pi i p / R) for p = 1..R-1 (forward sign).
template <typename T, int R, bool INV>
__device__ __forceinline__ void radix_dft_roots(Cx<T>* v, const Cx<T>* roots) {
  if constexpr (R == 2 || R == 4) {
    radix_dft<T, R, INV>(v, nullptr, 0);
  } else {
    constexpr int H = (R - 1) / 2;
    Cx<T> a[H], b[H];
#pragma unroll
    for (int r = 1; r <= H; ++r) {
      a[r - 1] = v[r] + v[R - r];
      b[r - 1] = v[r] - v[R - r];
    }
    const Cx<T> x0 = v[0];
    Cx<T> sum = x0;
#pragma unroll
    for (int r = 0; r < H; ++r) sum = sum + a[r];
    v[0] = sum;
#pragma unroll
    for (int q = 1; q <= H; ++q) {
      T cre = x0.re, cim = x0.im, sre = 0, sim = 0;
#pragma unroll
      for (int r = 1; r <= H; ++r) {
        const Cx<T> w = roots[(r * q) % R];  // cos, -sin (forward)
        cre += a[r - 1].re * w.re;
        cim += a[r - 1].im * w.re;
        const T s = INV ? -w.im : w.im;
        sre -= b[r - 1].im * s;
        sim += b[r - 1].re * s;
      }
      v[q] = Cx<T>{cre + sre, cim + sim};
      v[R - q] = Cx<T>{cre - sre, cim - sim};
    }
  }
}

// One ping-pong stage over `count` lines (line offset rows[t] or t, times
// line_stride). Work items (butterfly j, line t) = divmod(item, count) with
// lines fastest; each thread walks items tid, tid + blockDim, ... and
// advances (j, t) and (j / ns, j mod ns) incrementally, so the loop carries
// no integer division. The stage's radix roots sit in registers.
template <typename T, int R, bool INV>
__device__ __forceinline__ void pp_stage_flat(const Cx<T>* src, Cx<T>* dst, int count, int line_stride, int es,
                                              const int* rows, int n, int ns, const Cx<T>* tw) {
  const int m = n / R;
  const int items = count * m;
  int item = threadIdx.x;
  if (item >= items) return;
  const int twstride = n / (ns * R);
  Cx<T> roots[R];
#pragma unroll
  for (int p = 1; p < R; ++p) roots[p] = tw[p * m];
  const int step = blockDim.x;
  const int dj = step / count, dt = step - dj * count;
  const int djq = dj / ns, djk = dj - djq * ns;
  int j = item / count, t = item - j * count;
  int jq = j / ns, jk = j - jq * ns;
  for (; item < items; item += step) {
    const int offset = (rows ? rows[t] : t) * line_stride;
    const Cx<T>* in = src + offset;
    Cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      Cx<T> x = in[(j + r * m) * es];
      if (r > 0 && jk > 0) x = cmul(x, twiddle<T, INV>(tw, r * jk * twstride));
      v[r] = x;
    }
    radix_dft_roots<T, R, INV>(v, roots);
    Cx<T>* out = dst + offset + (jq * ns * R + jk) * es;
#pragma unroll
    for (int r = 0; r < R; ++r) out[r * ns * es] = v[r];
    t += dt;
    j += dj;
    jk += djk;
    jq += djq;
    if (t >= count) {
      t -= count;
      ++j;
      ++jk;
    }
    if (jk >= ns) {
      jk -= ns;
      ++jq;
    }
  }
}

// ---- compile-time line length ------------------------------------------
// The same Stockham stages with N, the radix sequence (4 first, then 2, 3,
// 5, 7, as make_line_plan) and the line count known at compile time, so the
// stage loops unroll and all index arithmetic folds to constants.
__host__ __device__ constexpr int fixed_next_radix(int rest) {
  return rest % 4 == 0 ? 4 : rest % 2 == 0 ? 2 : rest % 3 == 0 ? 3 : rest % 5 == 0 ? 5 : rest % 7 == 0 ? 7 : 0;
}
__host__ __device__ constexpr int fixed_stage_count(int n) {
  int stages = 0;
  for (int rest = n; rest > 1; rest /= fixed_next_radix(rest)) {
    if (fixed_next_radix(rest) == 0) return -1;
    ++stages;
  }
  return stages;
}
// Radix of stage s and the product of the radices before it.
__host__ __device__ constexpr int fixed_radix(int n, int s) {
  int rest = n;
  for (int i = 0; i < s; ++i) rest /= fixed_next_radix(rest);
  return fixed_next_radix(rest);
}
__host__ __device__ constexpr int fixed_ns(int n, int s) {
  int ns = 1, rest = n;
  for (int i = 0; i < s; ++i) {
    const int r = fixed_next_radix(rest);
    ns *= r;
    rest /= r;
  }
  return ns;
}

template <typename T, int R, bool INV, int N, int NS, int COUNT, int THREADS>
__device__ __forceinline__ void pp_stage_fixed(const Cx<T>* src, Cx<T>* dst, int line_stride, int es,
                                               const Cx<T>* tw) {
  constexpr int M = N / R, ITEMS = COUNT * M, TWSTRIDE = N / (NS * R);
  Cx<T> roots[R];
#pragma unroll
  for (int p = 1; p < R; ++p) roots[p] = tw[p * M];
#pragma unroll
  for (int base = 0; base < ITEMS; base += THREADS) {
    const int item = base + static_cast<int>(threadIdx.x);
    if (ITEMS % THREADS != 0 && item >= ITEMS) break;
    const int j = item / COUNT, t = item - j * COUNT;
    const int jq = j / NS, jk = j - jq * NS;
    const int offset = t * line_stride;
    const Cx<T>* in = src + offset;
    Cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      Cx<T> x = in[(j + r * M) * es];
      if (r > 0 && jk > 0) x = cmul(x, twiddle<T, INV>(tw, r * jk * TWSTRIDE));
      v[r] = x;
    }
    radix_dft_roots<T, R, INV>(v, roots);
    Cx<T>* out = dst + offset + (jq * NS * R + jk) * es;
#pragma unroll
    for (int r = 0; r < R; ++r) out[r * NS * es] = v[r];
  }
}

// COUNT lines of length N (line t at t * line_stride, elements es apart),
// ping-pong between src and dst; returns the buffer holding the result.
template <typename T, bool INV, int N, int COUNT, int THREADS, int S = 0>
__device__ __forceinline__ Cx<T>* fft_lines_fixed(Cx<T>* src, Cx<T>* dst, int line_stride, int es, const Cx<T>* tw) {
  static_assert(fixed_stage_count(N) > 0, "line length must be 2/3/5/7-smooth");
  if constexpr (S == fixed_stage_count(N)) {
    return src;
  } else {
    pp_stage_fixed<T, fixed_radix(N, S), INV, N, fixed_ns(N, S), COUNT, THREADS>(src, dst, line_stride, es, tw);
    __syncthreads();
    return fft_lines_fixed<T, INV, N, COUNT, THREADS, S + 1>(dst, src, line_stride, es, tw);
  }
}

// One stage over `count` listed lines of compile-time length N with
// contiguous elements: line t starts at rows[t] * line_stride. Work items
// run butterfly-fastest, so neighbouring threads touch neighbouring words.
template <typename T, int R, bool INV, int N, int NS, int THREADS>
__device__ __forceinline__ void pp_stage_fixed_rows(const Cx<T>* src, Cx<T>* dst, int count, const int* rows,
                                                    int line_stride, const Cx<T>* tw) {
  constexpr int M = N / R, TWSTRIDE = N / (NS * R);
  Cx<T> roots[R];
#pragma unroll
  for (int p = 1; p < R; ++p) roots[p] = tw[p * M];
  const int items = count * M;
  for (int item = static_cast<int>(threadIdx.x); item < items; item += THREADS) {
    const int t = item / M, j = item - t * M;
    const int jq = j / NS, jk = j - jq * NS;
    const int offset = rows[t] * line_stride;
    const Cx<T>* in = src + offset;
    Cx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      Cx<T> x = in[j + r * M];
      if (r > 0 && jk > 0) x = cmul(x, twiddle<T, INV>(tw, r * jk * TWSTRIDE));
      v[r] = x;
    }
    radix_dft_roots<T, R, INV>(v, roots);
    Cx<T>* out = dst + offset + jq * NS * R + jk;
#pragma unroll
    for (int r = 0; r < R; ++r) out[r * NS] = v[r];
  }
}

// The listed lines of length N (contiguous elements), ping-pong between src
// and dst; returns the buffer holding the result. Lines not listed are not
// touched in either buffer.
template <typename T, bool INV, int N, int THREADS, int S = 0>
__device__ __forceinline__ Cx<T>* fft_rows_fixed(Cx<T>* src, Cx<T>* dst, int count, const int* rows, int line_stride,
                                                 const Cx<T>* tw) {
  static_assert(fixed_stage_count(N) > 0, "line length must be 2/3/5/7-smooth");
  if constexpr (S == fixed_stage_count(N)) {
    return src;
  } else {
    pp_stage_fixed_rows<T, fixed_radix(N, S), INV, N, fixed_ns(N, S), THREADS>(src, dst, count, rows, line_stride,
                                                                              tw);
    __syncthreads();
    return fft_rows_fixed<T, INV, N, THREADS, S + 1>(dst, src, count, rows, line_stride, tw);
  }
}

// In-place stage over lines of compile-time length N: every thread loads
// the inputs of all its butterflies into registers, the CTA synchronises,
// then every thread writes its outputs to the Stockham positions, so one
// buffer serves both sides of the stage. LISTED: `count` (<= N) lines at
// rows[t] * line_stride, butterfly index fastest (contiguous elements,
// es = 1); otherwise N lines at t * line_stride, line index fastest.
template <typename T, int R, bool INV, int N, int NS, bool LISTED, int THREADS>
__device__ __forceinline__ void ip_stage_fixed(Cx<T>* buf, int count, const int* rows, int line_stride, int es,
                                               const Cx<T>* tw) {
  constexpr int M = N / R, TWSTRIDE = N / (NS * R), MAX_ITEMS = N * M;
  constexpr int PER = (MAX_ITEMS + THREADS - 1) / THREADS;
  Cx<T> roots[R];
#pragma unroll
  for (int p = 1; p < R; ++p) roots[p] = tw[p * M];
  const int items = LISTED ? count * M : MAX_ITEMS;
  Cx<T> v[PER][R];
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int item = q * THREADS + static_cast<int>(threadIdx.x);
    if (item < items) {
      int t, j;
      if constexpr (LISTED) {
        t = item / M;
        j = item - t * M;
      } else {
        j = item / N;
        t = item - j * N;
      }
      const int jk = j % NS;
      const Cx<T>* in = buf + (LISTED ? rows[t] : t) * line_stride;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        Cx<T> x = in[(j + r * M) * es];
        if (r > 0 && jk > 0) x = cmul(x, twiddle<T, INV>(tw, r * jk * TWSTRIDE));
        v[q][r] = x;
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int item = q * THREADS + static_cast<int>(threadIdx.x);
    if (item < items) {
      int t, j;
      if constexpr (LISTED) {
        t = item / M;
        j = item - t * M;
      } else {
        j = item / N;
        t = item - j * N;
      }
      const int jq = j / NS, jk = j - jq * NS;
      radix_dft_roots<T, R, INV>(v[q], roots);
      Cx<T>* out = buf + (LISTED ? rows[t] : t) * line_stride + (jq * NS * R + jk) * es;
#pragma unroll
      for (int r = 0; r < R; ++r) out[r * NS * es] = v[q][r];
    }
  }
  __syncthreads();
}

// All stages of ip_stage_fixed (the buffer holds the result).
template <typename T, bool INV, int N, bool LISTED, int THREADS, int S = 0>
__device__ __forceinline__ void fft_inplace_fixed(Cx<T>* buf, int count, const int* rows, int line_stride, int es,
                                                  const Cx<T>* tw) {
  static_assert(fixed_stage_count(N) > 0, "line length must be 2/3/5/7-smooth");
  if constexpr (S < fixed_stage_count(N)) {
    ip_stage_fixed<T, fixed_radix(N, S), INV, N, fixed_ns(N, S), LISTED, THREADS>(buf, count, rows, line_stride, es,
                                                                                 tw);
    fft_inplace_fixed<T, INV, N, LISTED, THREADS, S + 1>(buf, count, rows, line_stride, es, tw);
  }
}

template <typename T, bool INV>
__device__ Cx<T>* fft_lines_pp(Cx<T>* src, Cx<T>* dst, int count, int line_stride, int elem_stride,
                               const int* rows, const LinePlan& plan, const Cx<T>* tw) {
  int ns = 1;
  for (int s = 0; s < plan.stages; ++s) {
    const int r = plan.radix[s];
    switch (r) {
      case 2: pp_stage_flat<T, 2, INV>(src, dst, count, line_stride, elem_stride, rows, plan.n, ns, tw); break;
      case 3: pp_stage_flat<T, 3, INV>(src, dst, count, line_stride, elem_stride, rows, plan.n, ns, tw); break;
      case 4: pp_stage_flat<T, 4, INV>(src, dst, count, line_stride, elem_stride, rows, plan.n, ns, tw); break;
      case 5: pp_stage_flat<T, 5, INV>(src, dst, count, line_stride, elem_stride, rows, plan.n, ns, tw); break;
      case 7: pp_stage_flat<T, 7, INV>(src, dst, count, line_stride, elem_stride, rows, plan.n, ns, tw); break;
      default: break;
    }
    __syncthreads();
    Cx<T>* swap = src;
    src = dst;
    dst = swap;
    ns *= r;
  }
  return src;
}

// Radix-R stage for a runtime odd prime R > 7 (a general length's large
// factors), in two passes so that no thread holds R values. Pass 1 (src ->
// dst), one butterfly (j, line) per item: applies the stage twiddles and
// stores x0, the pair sums a_r = x_r + x_{R-r} and differences
// b_r = x_r - x_{R-r} (r = 1..H, H = (R-1)/2) in the butterfly's R output
// slots. Pass 2 (dst -> src), one output q per item: y_0 = x0 + sum_r a_r and
// y_q = x0 + sum_r a_r cos(2 pi rq/R) -/+ i sum_r b_r sin(2 pi rq/R), the
// arithmetic of radix_dft for the compiled odd radices, with the roots read
// from the length-n table. The result is left in src.
template <typename T, bool INV>
__device__ void pp_stage_prime(Cx<T>* src, Cx<T>* dst, int count, int line_stride, int es, const int* rows, int n,
                               int ns, int R, const Cx<T>* tw) {
  const int m = n / R, twstride = n / (ns * R), unit = n / R, H = (R - 1) / 2;
  for (int item = threadIdx.x; item < count * m; item += blockDim.x) {
    const int j = item / count, t = item - j * count;
    const int k = j % ns;
    const int offset = (rows ? rows[t] : t) * line_stride;
    const Cx<T>* in = src + offset;
    Cx<T>* out = dst + offset + ((j / ns) * ns * R + k) * es;
    out[0] = in[j * es];
    for (int r = 1; r <= H; ++r) {
      Cx<T> x = in[(j + r * m) * es], y = in[(j + (R - r) * m) * es];
      if (k > 0) {
        x = cmul(x, twiddle<T, INV>(tw, r * k * twstride));
        y = cmul(y, twiddle<T, INV>(tw, (R - r) * k * twstride));
      }
      out[r * ns * es] = x + y;
      out[(H + r) * ns * es] = x - y;
    }
  }
  __syncthreads();
  for (int item = threadIdx.x; item < count * n; item += blockDim.x) {
    const int o = item / count, t = item - o * count;
    const int j = o / R, q = o - j * R;
    const int k = j % ns;
    const int offset = (rows ? rows[t] : t) * line_stride;
    const Cx<T>* packed = dst + offset + ((j / ns) * ns * R + k) * es;
    const Cx<T> x0 = packed[0];
    Cx<T> y;
    if (q == 0) {
      y = x0;
      for (int r = 1; r <= H; ++r) y = y + packed[r * ns * es];
    } else {
      const int qq = q <= H ? q : R - q;
      T cre = x0.re, cim = x0.im, sre = 0, sim = 0;
      int root = 0;
      for (int r = 1; r <= H; ++r) {
        root += qq;
        if (root >= R) root -= R;
        const Cx<T> w = tw[root * unit];  // cos, -sin (forward)
        const Cx<T> a = packed[r * ns * es], b = packed[(H + r) * ns * es];
        cre += a.re * w.re;
        cim += a.im * w.re;
        const T s = INV ? -w.im : w.im;
        sre -= b.im * s;
        sim += b.re * s;
      }
      y = q <= H ? Cx<T>{cre + sre, cim + sim} : Cx<T>{cre - sre, cim - sim};
    }
    src[offset + ((j / ns) * ns * R + k + q * ns) * es] = y;
  }
}

// fft_lines_pp for plans that may hold odd prime radices above 7 (general
// lengths); the compiled radices run the same ping-pong stages.
template <typename T, bool INV>
__device__ Cx<T>* fft_lines_pp_general(Cx<T>* src, Cx<T>* dst, int count, int line_stride, int elem_stride,
                                       const int* rows, const LinePlan& plan, const Cx<T>* tw) {
  int ns = 1;
  for (int s = 0; s < plan.stages; ++s) {
    const int r = plan.radix[s];
    bool swapped = true;
    switch (r) {
      case 2: pp_stage_flat<T, 2, INV>(src, dst, count, line_stride, elem_stride, rows, plan.n, ns, tw); break;
      case 3: pp_stage_flat<T, 3, INV>(src, dst, count, line_stride, elem_stride, rows, plan.n, ns, tw); break;
      case 4: pp_stage_flat<T, 4, INV>(src, dst, count, line_stride, elem_stride, rows, plan.n, ns, tw); break;
      case 5: pp_stage_flat<T, 5, INV>(src, dst, count, line_stride, elem_stride, rows, plan.n, ns, tw); break;
      case 7: pp_stage_flat<T, 7, INV>(src, dst, count, line_stride, elem_stride, rows, plan.n, ns, tw); break;
      default:
        pp_stage_prime<T, INV>(src, dst, count, line_stride, elem_stride, rows, plan.n, ns, r, tw);
        swapped = false;
        break;
    }
    __syncthreads();
    if (swapped) {
      Cx<T>* swap = src;
      src = dst;
      dst = swap;
    }
    ns *= r;
  }
  return src;
}

// ---- register-resident lines -----------------------------------------------
// One thread transforms one line of compile-time length N held in its
// registers: the Stockham stages of fft_lines_fixed unrolled over the whole
// line, so every element index and twiddle offset is a constant and the
// line never touches shared memory. The twiddles are read through `tw`,
// which callers point at a kernel-parameter table (RegTwiddles), so each
// twiddle is a constant-bank operand rather than a load.
template <typename T, int N>
struct RegTwiddles {
  Cx<T> w[N];  // w[m] = exp(-2 pi i m / N)
};

template <typename T, bool INV, int N, int S = 0>
__device__ __forceinline__ void fft_line_registers(Cx<T> (&v)[N], const Cx<T>* tw) {
  static_assert(fixed_stage_count(N) > 0, "line length must be 2/3/5/7-smooth");
  if constexpr (S < fixed_stage_count(N)) {
    constexpr int R = fixed_radix(N, S), NS = fixed_ns(N, S), M = N / R, TWSTRIDE = N / (NS * R);
    Cx<T> out[N];
#pragma unroll
    for (int j = 0; j < M; ++j) {
      const int jq = j / NS, jk = j - jq * NS;
      Cx<T> b[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        Cx<T> x = v[j + r * M];
        if (r > 0 && jk > 0) x = cmul(x, twiddle<T, INV>(tw, r * jk * TWSTRIDE));
        b[r] = x;
      }
      radix_dft<T, R, INV>(b, tw, M);
#pragma unroll
      for (int r = 0; r < R; ++r) out[jq * NS * R + jk + r * NS] = b[r];
    }
#pragma unroll
    for (int e = 0; e < N; ++e) v[e] = out[e];
    fft_line_registers<T, INV, N, S + 1>(v, tw);
  }
}

// ---- lines split over a lane pair --------------------------------------------
// A line of even length N held by lanes l and l ^ kPairXor of one warp, N/2
// values each. The radix-2 step of the transform is one exchange through
// warp shuffles; the halves then run independent length-N/2 transforms in
// registers (fft_line_registers). Lanes 0-15 hold the lower halves, 16-31
// the upper ones. Every lane of the warp must call these (shuffles).
//
//   fft_pair_dif: input in natural halves (lower x[j], upper x[j + N/2]),
//                 output interleaved (lower X[2m], upper X[2m + 1]);
//   fft_pair_dit: input interleaved, output in natural halves.
constexpr int kPairXor = 16;

// lower: v_j <- other_j + v_j; upper: v_j <- other_j - v_j.
template <typename T, int H>
__device__ __forceinline__ void pair_combine(Cx<T> (&v)[H], bool upper) {
  const T sign = upper ? T(-1) : T(1);
#pragma unroll
  for (int j = 0; j < H; ++j) {
    const T ore = __shfl_xor_sync(0xffffffffu, v[j].re, kPairXor);
    const T oim = __shfl_xor_sync(0xffffffffu, v[j].im, kPairXor);
    v[j] = Cx<T>{fma(sign, v[j].re, ore), fma(sign, v[j].im, oim)};
  }
}

// upper: v_j <- v_j W^j with W = exp(-+2 pi i / N) (sign of the transform); lower unchanged.
template <typename T, bool INV, int H>
__device__ __forceinline__ void pair_twiddle(Cx<T> (&v)[H], bool upper, const Cx<T>* tw_n) {
#pragma unroll
  for (int j = 1; j < H; ++j) {
    const Cx<T> w = twiddle<T, INV>(tw_n, j);
    v[j] = cmul(v[j], Cx<T>{upper ? w.re : T(1), upper ? w.im : T(0)});
  }
}

// tw_n: the length-N table; tw_half: the length-N/2 table (tw_half[m] = tw_n[2m]).
template <typename T, bool INV, int N>
__device__ __forceinline__ void fft_pair_dif(Cx<T> (&v)[N / 2], bool upper, const Cx<T>* tw_n,
                                             const Cx<T>* tw_half) {
  static_assert(N % 2 == 0, "pair-split lines have even length");
  pair_combine<T, N / 2>(v, upper);
  pair_twiddle<T, INV, N / 2>(v, upper, tw_n);
  fft_line_registers<T, INV, N / 2>(v, tw_half);
}

template <typename T, bool INV, int N>
__device__ __forceinline__ void fft_pair_dit(Cx<T> (&v)[N / 2], bool upper, const Cx<T>* tw_n,
                                             const Cx<T>* tw_half) {
  static_assert(N % 2 == 0, "pair-split lines have even length");
  fft_line_registers<T, INV, N / 2>(v, tw_half);
  pair_twiddle<T, INV, N / 2>(v, upper, tw_n);
  pair_combine<T, N / 2>(v, upper);
}

// Host-side twiddle tables, w[m] = exp(-2 pi i m / n), one per (n, precision).
template <typename T>
const Cx<T>* device_twiddles(int n);

// The same table values written into caller memory on the host (no device
// allocation, no cache).
template <typename T>
void host_twiddles(int n, Cx<T>* out);

}  // namespace sdft_b200
