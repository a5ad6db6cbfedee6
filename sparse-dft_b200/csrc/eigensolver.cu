// Device eigensolver for the Davidson Rayleigh-Ritz step (lowest `wanted`
// eigenpairs of an m x m Hermitian matrix, m up to ~1290).
//
// 1. tridiagonalize_kernel: one cooperative launch, one CTA per SM, columns
//    distributed cyclically and held in shared memory. Step j of the
//    Householder reduction (LAPACK zhetd2, lower, H_j = I - tau v v^H with
//    v[j+1] = 1) needs one grid-wide barrier: every CTA recomputes the
//    reflector from the published column j (plus the previous rank-2 update)
//    redundantly, computes p = tau A22 v for its own columns, publishes p and
//    its share of p^H v, and after the barrier forms w = p - tau/2 (p^H v) v
//    and updates its columns. Exchange buffers are double-buffered by step
//    parity. The barrier is a counting barrier with a time limit: on expiry
//    an error word is set and every CTA returns.
// 2. bisect_kernel: one warp per wanted eigenvalue, 32-point multisection on
//    Sturm counts of the tridiagonal matrix.
// 3. inverse_iteration_kernel: one thread per cluster of eigenvalues closer
//    than 1e-9 of the matrix scale; LU with partial pivoting of T - lambda I,
//    three solves, Gram-Schmidt against earlier members of the cluster.
// 4. backtransform_kernel: the reflectors applied to the tridiagonal
//    eigenvectors in reverse order, four columns per CTA in shared memory.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "dense.cuh"
#include "eigensolver.cuh"

namespace sdft_b200 {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxCpc = 12;
constexpr int kBackColumns = 4;
constexpr unsigned long long kWaitNs = 2000000000ULL;
constexpr double kClusterTolerance = 1e-9;

__device__ unsigned int g_eigen_error;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ Cx<double> cconj(Cx<double> a) { return {a.re, -a.im}; }
__device__ __forceinline__ Cx<double> cadd(Cx<double> a, Cx<double> b) { return {a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Cx<double> csub(Cx<double> a, Cx<double> b) { return {a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Cx<double> cmulz(Cx<double> a, Cx<double> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
// conj(a) * b
__device__ __forceinline__ Cx<double> cdot1(Cx<double> a, Cx<double> b) {
  return {a.re * b.re + a.im * b.im, a.re * b.im - a.im * b.re};
}

// Sum of N complex values over the CTA in a fixed order; result in out[0..N).
template <int N>
__device__ void block_sum(Cx<double> (&v)[N], int count, Cx<double>* scratch, Cx<double>* out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < N; ++q) {
    if (q < count) {
      double re = v[q].re, im = v[q].im;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        re += __shfl_xor_sync(0xffffffffu, re, o);
        im += __shfl_xor_sync(0xffffffffu, im, o);
      }
      if (lane == 0) scratch[warp * N + q] = Cx<double>{re, im};
    }
  }
  __syncthreads();
  if (threadIdx.x < count) {
    Cx<double> s{0.0, 0.0};
    for (int w = 0; w < kWarps; ++w) s = cadd(s, scratch[w * N + threadIdx.x]);
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

__device__ double block_sum_real(double v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < kWarps; ++w) s += scratch[w];
  __syncthreads();
  return s;
}

// Counting grid barrier with a time limit. Returns false (and every CTA
// should return) when the limit expired here or the error word is set.
__device__ bool grid_barrier(unsigned int* arrive, unsigned int target, int* ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(arrive, 1u);
    const unsigned long long start = global_ns();
    int good = 1;
    while (true) {
      if (*reinterpret_cast<volatile unsigned int*>(arrive) >= target) break;
      if (*reinterpret_cast<volatile unsigned int*>(&g_eigen_error) != 0u) {
        good = 0;
        break;
      }
      if (global_ns() - start > kWaitNs) {
        atomicOr(&g_eigen_error, 1u);
        good = 0;
        break;
      }
    }
    __threadfence();
    *ok = good;
  }
  __syncthreads();
  return *ok != 0;
}

struct TridiagArgs {
  const Cx<double>* a;
  int m, grid, cpc;
  double* d;
  double* e;
  Cx<double>* tau;
  Cx<double>* reflectors;  // m x m, column j holds v_j in rows j+1..m-1
  Cx<double>* colbuf;      // 2 x m
  Cx<double>* pbuf;        // 2 x m
  Cx<double>* dotbuf;      // 2 x grid
  unsigned int* arrive;
};

__global__ void __launch_bounds__(kThreads, 1) tridiagonalize_kernel(TridiagArgs t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int m = t.m, G = t.grid, cpc = t.cpc, cta = blockIdx.x, tid = threadIdx.x;
  Cx<double>* cols = reinterpret_cast<Cx<double>*>(smem_raw);
  Cx<double>* v = cols + static_cast<long long>(cpc) * m;
  Cx<double>* w = v + m;
  Cx<double>* red = w + m;             // kWarps * kMaxCpc
  Cx<double>* res = red + kWarps * kMaxCpc;  // kMaxCpc
  double* rred = reinterpret_cast<double*>(res + kMaxCpc);  // kWarps
  __shared__ int ok;
  __shared__ Cx<double> shared_tau, shared_scale;
  __shared__ double shared_beta;
  __shared__ int shared_trivial;

  for (int s = 0; s < cpc; ++s) {
    const int c = cta + s * G;
    if (c < m)
      for (int r = tid; r < m; r += kThreads) cols[static_cast<long long>(s) * m + r] = t.a[r + static_cast<long long>(c) * m];
  }
  __syncthreads();

  for (int j = 0; j < m - 1; ++j) {
    // P1: column j with updates 0..j-1 into w (rows j..m-1); reflector j.
    Cx<double> vj{0.0, 0.0}, wj{0.0, 0.0};
    if (j > 0) {
      vj = v[j];
      wj = w[j];
    }
    __syncthreads();
    double part = 0.0;
    const Cx<double>* src = t.colbuf + static_cast<long long>(j & 1) * m;
    for (int r = j + tid; r < m; r += kThreads) {
      Cx<double> c;
      if (j == 0) {
        c = t.a[r];
      } else {
        const double2 q = __ldcg(reinterpret_cast<const double2*>(src + r));
        c = Cx<double>{q.x, q.y};
        c = csub(c, cadd(cmulz(v[r], cconj(wj)), cmulz(w[r], cconj(vj))));
      }
      w[r] = c;
      if (r >= j + 2) part += c.re * c.re + c.im * c.im;
    }
    const double xnorm2 = block_sum_real(part, rred);
    if (tid == 0) {
      const Cx<double> alpha = w[j + 1];
      if (xnorm2 == 0.0 && alpha.im == 0.0) {
        shared_trivial = 1;
        shared_tau = Cx<double>{0.0, 0.0};
        shared_beta = alpha.re;
        shared_scale = Cx<double>{0.0, 0.0};
      } else {
        const double beta = -copysign(sqrt(alpha.re * alpha.re + alpha.im * alpha.im + xnorm2), alpha.re);
        shared_trivial = 0;
        shared_tau = Cx<double>{(beta - alpha.re) / beta, -alpha.im / beta};
        shared_beta = beta;
        // 1 / (alpha - beta)
        const double dr = alpha.re - beta, di = alpha.im, den = dr * dr + di * di;
        shared_scale = Cx<double>{dr / den, -di / den};
      }
      if (cta == 0) {
        t.d[j] = w[j].re;
        t.e[j] = shared_beta;
        t.tau[j] = shared_tau;
      }
    }
    __syncthreads();
    const Cx<double> tau = shared_tau, scale = shared_scale;
    const int trivial = shared_trivial;
    for (int r = j + 1 + tid; r < m; r += kThreads) {
      const Cx<double> vr = r == j + 1 ? Cx<double>{1.0, 0.0} : (trivial ? Cx<double>{0.0, 0.0} : cmulz(w[r], scale));
      v[r] = vr;
      if (cta == 0) t.reflectors[r + static_cast<long long>(j) * m] = vr;
    }
    __syncthreads();

    // P2: p[c] = tau sum_r conj(A[r,c]) v[r] for own columns c >= j+1.
    Cx<double> acc[kMaxCpc];
#pragma unroll
    for (int s = 0; s < kMaxCpc; ++s) acc[s] = Cx<double>{0.0, 0.0};
    if (!trivial) {
      for (int r = j + 1 + tid; r < m; r += kThreads) {
        const Cx<double> vr = v[r];
#pragma unroll
        for (int s = 0; s < kMaxCpc; ++s) {
          const int c = cta + s * G;
          if (s < cpc && c > j && c < m) acc[s] = cadd(acc[s], cdot1(cols[static_cast<long long>(s) * m + r], vr));
        }
      }
    }
    block_sum<kMaxCpc>(acc, cpc, red, res);
    if (tid == 0) {
      Cx<double> dot{0.0, 0.0};
      for (int s = 0; s < cpc; ++s) {
        const int c = cta + s * G;
        if (c > j && c < m) {
          const Cx<double> p = cmulz(tau, res[s]);
          t.pbuf[static_cast<long long>(j & 1) * m + c] = p;
          dot = cadd(dot, cdot1(p, v[c]));
        }
      }
      t.dotbuf[static_cast<long long>(j & 1) * G + cta] = dot;
    }
    // Publish column j+1 (updates 0..j-1) for the next step.
    if ((j + 1) % G == cta) {
      const int s1 = (j + 1) / G;
      Cx<double>* dst = t.colbuf + static_cast<long long>((j + 1) & 1) * m;
      for (int r = j + 1 + tid; r < m; r += kThreads) dst[r] = cols[static_cast<long long>(s1) * m + r];
    }
    __threadfence();
    if (!grid_barrier(t.arrive, static_cast<unsigned int>(G) * static_cast<unsigned int>(j + 1), &ok)) return;

    // P3: w = p - tau/2 (p^H v) v.
    if (tid < 32) {
      Cx<double> s{0.0, 0.0};
      const double* db = reinterpret_cast<const double*>(t.dotbuf + static_cast<long long>(j & 1) * G);
      for (int g = tid; g < G; g += 32) s = cadd(s, Cx<double>{__ldcg(db + 2 * g), __ldcg(db + 2 * g + 1)});
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        s.re += __shfl_xor_sync(0xffffffffu, s.re, o);
        s.im += __shfl_xor_sync(0xffffffffu, s.im, o);
      }
      if (tid == 0) res[0] = cmulz(Cx<double>{-0.5 * tau.re, -0.5 * tau.im}, s);
    }
    __syncthreads();
    const Cx<double> alpha = res[0];
    const double* pb = reinterpret_cast<const double*>(t.pbuf + static_cast<long long>(j & 1) * m);
    for (int r = j + 1 + tid; r < m; r += kThreads) {
      const Cx<double> p = trivial ? Cx<double>{0.0, 0.0} : Cx<double>{__ldcg(pb + 2 * r), __ldcg(pb + 2 * r + 1)};
      w[r] = cadd(p, cmulz(alpha, v[r]));
    }
    __syncthreads();

    // P4: own columns -= v w^H + w v^H.
    if (!trivial) {
      for (int s = 0; s < cpc; ++s) {
        const int c = cta + s * G;
        if (c <= j || c >= m) continue;
        const Cx<double> wc = cconj(w[c]), vc = cconj(v[c]);
        Cx<double>* col = cols + static_cast<long long>(s) * m;
        for (int r = j + 1 + tid; r < m; r += kThreads) col[r] = csub(col[r], cadd(cmulz(v[r], wc), cmulz(w[r], vc)));
      }
    }
    __syncthreads();
  }
  if ((m - 1) % G == cta && tid == 0) t.d[m - 1] = cols[static_cast<long long>((m - 1) / G) * m + m - 1].re;
}

__device__ int sturm_count(const double* d, const double* e2, int m, double x, double pivmin) {
  double q = d[0] - x;
  if (fabs(q) <= pivmin) q = -pivmin;
  int count = q < 0.0;
  for (int i = 1; i < m; ++i) {
    q = (d[i] - x) - e2[i - 1] / q;
    if (fabs(q) <= pivmin) q = -pivmin;
    count += q < 0.0;
  }
  return count;
}

__global__ void bisect_kernel(const double* __restrict__ d, const double* __restrict__ e, int m, int wanted,
                              double* __restrict__ values) {
  extern __shared__ double sm[];
  double* sd = sm;
  double* se2 = sm + m;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    sd[i] = d[i];
    if (i + 1 < m) se2[i] = e[i] * e[i];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int k = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  if (k >= wanted) return;
  // Gershgorin bounds and pivot guard (the same in every warp).
  double lo = DBL_MAX, hi = -DBL_MAX, emax = 0.0;
  for (int i = lane; i < m; i += 32) {
    const double left = i > 0 ? fabs(e[i - 1]) : 0.0, right = i + 1 < m ? fabs(e[i]) : 0.0;
    lo = fmin(lo, sd[i] - left - right);
    hi = fmax(hi, sd[i] + left + right);
    if (i + 1 < m) emax = fmax(emax, se2[i]);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    emax = fmax(emax, __shfl_xor_sync(0xffffffffu, emax, o));
  }
  const double pivmin = DBL_MIN * fmax(1.0, emax);
  const double pad = 4.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + pivmin;
  lo -= pad;
  hi += pad;
  for (int round = 0; round < 64; ++round) {
    const double width = hi - lo;
    if (width <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) || width <= pivmin) break;
    const double x = lo + (lane + 1) * (width / 33.0);
    const int count = sturm_count(sd, se2, m, x, pivmin);
    const unsigned above = __ballot_sync(0xffffffffu, count > k);
    const int first = above ? __ffs(above) - 1 : 32;
    const double x_prev = __shfl_sync(0xffffffffu, x, first > 0 ? first - 1 : 0);
    const double x_first = __shfl_sync(0xffffffffu, x, first < 32 ? first : 31);
    const double new_lo = first == 0 ? lo : x_prev;
    const double new_hi = first == 32 ? hi : x_first;
    if (new_lo == lo && new_hi == hi) break;
    lo = new_lo;
    hi = new_hi;
  }
  if (lane == 0) values[k] = 0.5 * (lo + hi);
}

__device__ __forceinline__ double start_entry(int k, int i) {
  unsigned long long z = (static_cast<unsigned long long>(k) << 32) ^ static_cast<unsigned long long>(i) ^
                         0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  z ^= z >> 31;
  return static_cast<double>(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// Work layout: field f, row i, vector q at ((f * m + i) * wanted + q).
__global__ void inverse_iteration_kernel(const double* __restrict__ d, const double* __restrict__ e, int m, int wanted,
                                         const double* __restrict__ values, double* __restrict__ work,
                                         double* __restrict__ zt) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= wanted) return;
  double norm = 0.0;
  for (int i = 0; i < m; ++i) norm = fmax(norm, fabs(d[i]) + (i + 1 < m ? fabs(e[i]) : 0.0));
  const double cluster = kClusterTolerance * fmax(norm, DBL_MIN);
  if (k > 0 && values[k] - values[k - 1] <= cluster) return;
  int end = k;
  while (end + 1 < wanted && values[end + 1] - values[end] <= cluster) ++end;
  const double tiny = DBL_EPSILON * fmax(norm, DBL_MIN);
  const long long W = wanted;
  for (int q = k; q <= end; ++q) {
    const double lam = values[q];
    double* u0 = work + (0LL * m) * W + q;
    double* u1 = work + (1LL * m) * W + q;
    double* u2 = work + (2LL * m) * W + q;
    double* mult = work + (3LL * m) * W + q;
    double* piv = work + (4LL * m) * W + q;
    // LU of T - lam I with partial pivoting (rows i, i+1 swapped when |sub| wins).
    double cur_d = d[0] - lam, cur_u = m > 1 ? e[0] : 0.0;
    for (int i = 0; i + 1 < m; ++i) {
      const double nd = d[i + 1] - lam, nu = i + 2 < m ? e[i + 1] : 0.0, l = e[i];
      if (fabs(cur_d) >= fabs(l)) {
        if (fabs(cur_d) < tiny) cur_d = copysign(tiny, cur_d == 0.0 ? 1.0 : cur_d);
        const double mu = l / cur_d;
        u0[i * W] = cur_d;
        u1[i * W] = cur_u;
        u2[i * W] = 0.0;
        mult[i * W] = mu;
        piv[i * W] = 0.0;
        cur_d = nd - mu * cur_u;
        cur_u = nu;
      } else {
        const double mu = cur_d / l;
        u0[i * W] = l;
        u1[i * W] = nd;
        u2[i * W] = nu;
        mult[i * W] = mu;
        piv[i * W] = 1.0;
        cur_d = cur_u - mu * nd;
        cur_u = -mu * nu;
      }
    }
    if (fabs(cur_d) < tiny) cur_d = copysign(tiny, cur_d == 0.0 ? 1.0 : cur_d);
    u0[(m - 1) * W] = cur_d;
    double* z = zt + q;
    for (int i = 0; i < m; ++i) z[i * W] = start_entry(q, i);
    for (int it = 0; it < 3; ++it) {
      for (int i = 0; i + 1 < m; ++i) {
        if (piv[i * W] != 0.0) {
          const double tmp = z[i * W];
          z[i * W] = z[(i + 1) * W];
          z[(i + 1) * W] = tmp;
        }
        z[(i + 1) * W] -= mult[i * W] * z[i * W];
      }
      z[(m - 1) * W] /= u0[(m - 1) * W];
      if (m > 1) z[(m - 2) * W] = (z[(m - 2) * W] - u1[(m - 2) * W] * z[(m - 1) * W]) / u0[(m - 2) * W];
      for (int i = m - 3; i >= 0; --i)
        z[i * W] = (z[i * W] - u1[i * W] * z[(i + 1) * W] - u2[i * W] * z[(i + 2) * W]) / u0[i * W];
      for (int p = k; p < q; ++p) {
        double dot = 0.0;
        for (int i = 0; i < m; ++i) dot += zt[i * W + p] * z[i * W];
        for (int i = 0; i < m; ++i) z[i * W] -= dot * zt[i * W + p];
      }
      double nrm = 0.0;
      for (int i = 0; i < m; ++i) nrm += z[i * W] * z[i * W];
      const double inv = 1.0 / sqrt(nrm);
      for (int i = 0; i < m; ++i) z[i * W] *= inv;
    }
  }
}

__global__ void __launch_bounds__(kThreads) backtransform_kernel(const Cx<double>* __restrict__ reflectors,
                                                                 const Cx<double>* __restrict__ tau, int m, int wanted,
                                                                 const double* __restrict__ zt,
                                                                 Cx<double>* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int NB = kBackColumns;
  Cx<double>* z = reinterpret_cast<Cx<double>*>(smem_raw);  // m x NB, row-major
  Cx<double>* red = z + static_cast<long long>(m) * NB;     // kWarps * NB
  Cx<double>* res = red + kWarps * NB;                       // NB
  const int q0 = blockIdx.x * NB;
  const int count = min(NB, wanted - q0);
  for (int idx = threadIdx.x; idx < m * NB; idx += kThreads) {
    const int i = idx / NB, c = idx - i * NB;
    z[idx] = Cx<double>{c < count ? zt[static_cast<long long>(i) * wanted + q0 + c] : 0.0, 0.0};
  }
  __syncthreads();
  for (int j = m - 2; j >= 0; --j) {
    const Cx<double> t = tau[j];
    if (t.re == 0.0 && t.im == 0.0) continue;
    const Cx<double>* v = reflectors + static_cast<long long>(j) * m;
    Cx<double> acc[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) acc[c] = Cx<double>{0.0, 0.0};
    for (int r = j + 1 + threadIdx.x; r < m; r += kThreads) {
      const Cx<double> vr = v[r];
#pragma unroll
      for (int c = 0; c < NB; ++c) acc[c] = cadd(acc[c], cdot1(vr, z[r * NB + c]));
    }
    block_sum<NB>(acc, NB, red, res);
    Cx<double> coef[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) coef[c] = cmulz(t, res[c]);
    for (int r = j + 1 + threadIdx.x; r < m; r += kThreads) {
      const Cx<double> vr = v[r];
#pragma unroll
      for (int c = 0; c < NB; ++c) z[r * NB + c] = csub(z[r * NB + c], cmulz(vr, coef[c]));
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < m * NB; idx += kThreads) {
    const int i = idx / NB, c = idx - i * NB;
    if (c < count) out[i + static_cast<long long>(q0 + c) * m] = z[idx];
  }
}

__global__ void identity_deviation_kernel(Cx<double>* __restrict__ b, int m, unsigned long long* __restrict__ max_bits) {
  const long long total = static_cast<long long>(m) * m;
  double local = 0.0;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long i = idx % m, j = idx / m;
    Cx<double> v = b[idx];
    if (i == j) v.re -= 1.0;
    b[idx] = v;
    local = fmax(local, fmax(fabs(v.re), fabs(v.im)));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) local = fmax(local, __shfl_xor_sync(0xffffffffu, local, o));
  if ((threadIdx.x & 31) == 0) atomicMax(max_bits, static_cast<unsigned long long>(__double_as_longlong(local)));
}

__global__ void add_identity_kernel(Cx<double>* __restrict__ b, int m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) b[i + static_cast<long long>(i) * m].re += 1.0;
}

// a <- a - (f + f^H) / 2
__global__ void lowdin_combine_kernel(Cx<double>* __restrict__ a, const Cx<double>* __restrict__ f, int m) {
  const long long total = static_cast<long long>(m) * m;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long i = idx % m, j = idx / m;
    const Cx<double> x = f[idx], y = f[j + i * m];
    a[idx] = Cx<double>{a[idx].re - 0.5 * (x.re + y.re), a[idx].im - 0.5 * (x.im - y.im)};
  }
}

int sm_count() {
  static int count = [] {
    int device = 0, value = 0;
    SDFT_CUDA(cudaGetDevice(&device));
    SDFT_CUDA(cudaDeviceGetAttribute(&value, cudaDevAttrMultiProcessorCount, device));
    return value;
  }();
  return count;
}

std::size_t tridiag_smem(int m, int cpc) {
  return sizeof(Cx<double>) * (static_cast<std::size_t>(cpc + 2) * m + kWarps * kMaxCpc + kMaxCpc) +
         sizeof(double) * kWarps;
}

constexpr std::size_t kSmemLimit = 227 * 1024;

}  // namespace

int hermitian_eigen_max_order() {
  const int g = sm_count();
  int best = 0;
  for (int m = 2; m <= 4096; ++m) {
    const int grid = std::min(g, m);
    const int cpc = (m + grid - 1) / grid;
    if (cpc > kMaxCpc || tridiag_smem(m, cpc) > kSmemLimit) break;
    best = m;
  }
  return best;
}

void hermitian_lowest(Cx<double>* a, int m, int wanted, double* values, Cx<double>* vectors, EigenWorkspace& ws,
                      cudaStream_t stream) {
  if (m < 2 || wanted < 1 || wanted > m) throw InvalidArgument("invalid Hermitian eigenproblem size");
  const int grid = std::min(sm_count(), m);
  const int cpc = (m + grid - 1) / grid;
  const std::size_t smem = tridiag_smem(m, cpc);
  if (cpc > kMaxCpc || smem > kSmemLimit) throw InvalidArgument("Hermitian eigenproblem too large for the device solver");

  // Layout of the tridiagonal workspace.
  const std::size_t mm = static_cast<std::size_t>(m);
  const std::size_t bytes = sizeof(double) * 2 * mm + sizeof(Cx<double>) * (mm + mm * mm + 4 * mm + 2 * grid) + 256;
  auto* base = static_cast<unsigned char*>(ws.tridiagonal.reserve(bytes));
  auto* arrive = reinterpret_cast<unsigned int*>(base);
  auto* d = reinterpret_cast<double*>(base + 256);
  double* e = d + mm;
  auto* tau = reinterpret_cast<Cx<double>*>(e + mm);
  Cx<double>* reflectors = tau + mm;
  Cx<double>* colbuf = reflectors + mm * mm;
  Cx<double>* pbuf = colbuf + 2 * mm;
  Cx<double>* dotbuf = pbuf + 2 * mm;
  SDFT_CUDA(cudaMemsetAsync(arrive, 0, sizeof(unsigned int), stream));
  const unsigned int zero = 0;
  SDFT_CUDA(cudaMemcpyToSymbolAsync(g_eigen_error, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, stream));

  SDFT_CUDA(cudaFuncSetAttribute(tridiagonalize_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem)));
  int per_sm = 0;
  SDFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tridiagonalize_kernel, kThreads, smem));
  if (per_sm < 1) throw InvalidArgument("tridiagonalization kernel cannot be resident");
  TridiagArgs t{a, m, grid, cpc, d, e, tau, reflectors, colbuf, pbuf, dotbuf, arrive};
  void* args[] = {&t};
  SDFT_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(tridiagonalize_kernel), dim3(grid), dim3(kThreads),
                                        args, smem, stream));
  SDFT_LAUNCH("tridiagonalize_kernel");

  const int warps_per_block = 4;
  const std::size_t bisect_smem = sizeof(double) * 2 * mm;
  if (bisect_smem > 48 * 1024)
    SDFT_CUDA(cudaFuncSetAttribute(bisect_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(bisect_smem)));
  bisect_kernel<<<static_cast<unsigned>(ceil_div(wanted, warps_per_block)), 32 * warps_per_block, bisect_smem,
                  stream>>>(d, e, m, wanted, values);
  SDFT_LAUNCH("bisect_kernel");

  const std::size_t vbytes = sizeof(double) * static_cast<std::size_t>(wanted) * mm * 6;
  auto* vbase = static_cast<double*>(ws.vectors.reserve(vbytes));
  double* work = vbase;
  double* zt = vbase + static_cast<std::size_t>(wanted) * mm * 5;
  inverse_iteration_kernel<<<static_cast<unsigned>(ceil_div(wanted, 64)), 64, 0, stream>>>(d, e, m, wanted, values,
                                                                                          work, zt);
  SDFT_LAUNCH("inverse_iteration_kernel");

  const std::size_t back_smem = sizeof(Cx<double>) * (mm * kBackColumns + kWarps * kBackColumns + kBackColumns);
  SDFT_CUDA(cudaFuncSetAttribute(backtransform_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(back_smem)));
  backtransform_kernel<<<static_cast<unsigned>(ceil_div(wanted, kBackColumns)), kThreads, back_smem, stream>>>(
      reflectors, tau, m, wanted, zt, vectors);
  SDFT_LAUNCH("backtransform_kernel");

  unsigned int error = 0;
  SDFT_CUDA(cudaMemcpyFromSymbolAsync(&error, g_eigen_error, sizeof(error), 0, cudaMemcpyDeviceToHost, stream));
  SDFT_CUDA(cudaStreamSynchronize(stream));
  if (error) throw CudaError("tridiagonalization barrier wait limit exceeded");
}

double identity_deviation(Cx<double>* b, int m, EigenWorkspace& ws, cudaStream_t stream) {
  auto* bits = static_cast<unsigned long long*>(ws.scalar.reserve(sizeof(unsigned long long)));
  SDFT_CUDA(cudaMemsetAsync(bits, 0, sizeof(unsigned long long), stream));
  const long long total = static_cast<long long>(m) * m;
  identity_deviation_kernel<<<static_cast<unsigned>(std::min<long long>(ceil_div(total, 256), 148 * 8)), 256, 0,
                              stream>>>(b, m, bits);
  SDFT_LAUNCH("identity_deviation_kernel");
  unsigned long long host = 0;
  SDFT_CUDA(cudaMemcpyAsync(&host, bits, sizeof(host), cudaMemcpyDeviceToHost, stream));
  SDFT_CUDA(cudaStreamSynchronize(stream));
  double value;
  std::memcpy(&value, &host, sizeof(value));
  return value;
}

void add_identity(Cx<double>* b, int m, cudaStream_t stream) {
  add_identity_kernel<<<static_cast<unsigned>(ceil_div(m, 256)), 256, 0, stream>>>(b, m);
  SDFT_LAUNCH("add_identity_kernel");
}

RitzSolver rr_mode() {
  static const RitzSolver mode = [] {
    const char* v = std::getenv("SDFT_B200_RR");
    if (!v || std::string(v) == "device") return RitzSolver::Device;
    if (std::string(v) == "subset") return RitzSolver::Subset;
    if (std::string(v) == "full") return RitzSolver::Full;
    throw InvalidArgument("SDFT_B200_RR must be device, subset or full");
  }();
  return mode;
}

namespace {
void check_solver(cusolverStatus_t status, const char* what) {
  if (status != CUSOLVER_STATUS_SUCCESS)
    throw CudaError(std::string("cuSOLVER error ") + std::to_string(static_cast<int>(status)) + " in " + what);
}
}  // namespace

void generalized_lowest(cublasHandle_t blas, cusolverDnHandle_t solver, Cx<double>* h, Cx<double>* s, int m,
                        int wanted, double* values, Cx<double>* vectors, EigenWorkspace& ws, RitzSolver mode,
                        cudaStream_t st) {
  if (m < 1 || wanted < 1 || wanted > m) throw InvalidArgument("invalid Rayleigh-Ritz dimensions");
  const std::size_t mm = static_cast<std::size_t>(m);
  if (mode == RitzSolver::Device && m >= 2 && m <= hermitian_eigen_max_order()) {
    const double deviation = identity_deviation(s, m, ws, st);
    if (!std::isfinite(deviation)) throw NonFinite("Rayleigh-Ritz overlap is not finite");
    if (deviation <= 1e-6) {
      const bool correct = deviation > 1e-14;
      Cx<double>* f = nullptr;
      if (correct) {
        f = static_cast<Cx<double>*>(ws.product.reserve(sizeof(Cx<double>) * mm * mm));
        zgemm(blas, Op::N, Op::N, m, m, m, s, m, h, m, f, m, false);
        lowdin_combine(h, f, m, st);
      }
      hermitian_lowest(h, m, wanted, values, vectors, ws, st);
      if (correct) {
        // y -> y - E y / 2
        zgemm(blas, Op::N, Op::N, m, wanted, m, s, m, vectors, m, f, m, false, -0.5);
        add_block(f, m, vectors, m, m, wanted, st);
      }
      return;
    }
    // Far from S-orthonormal: restore S and solve the pencil with cuSOLVER.
    add_identity(s, m, st);
  }
  auto* info = static_cast<int*>(ws.scalar.reserve(sizeof(unsigned long long) + sizeof(int))) + 2;
  int lwork = 0;
  auto* hz = reinterpret_cast<cuDoubleComplex*>(h);
  auto* sz = reinterpret_cast<cuDoubleComplex*>(s);
  const bool full = mode == RitzSolver::Full || wanted == m;
  if (full) {
    check_solver(cusolverDnZhegvd_bufferSize(solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                             CUBLAS_FILL_MODE_LOWER, m, hz, m, sz, m, values, &lwork),
                 "zhegvd_bufferSize");
    auto* work = static_cast<cuDoubleComplex*>(ws.solver_work.reserve(sizeof(cuDoubleComplex) * std::max(1, lwork)));
    check_solver(cusolverDnZhegvd(solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m,
                                  hz, m, sz, m, values, work, lwork, info),
                 "zhegvd");
  } else {
    int found = 0;
    check_solver(cusolverDnZhegvdx_bufferSize(solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                              CUSOLVER_EIG_RANGE_I, CUBLAS_FILL_MODE_LOWER, m, hz, m, sz, m, 0.0,
                                              0.0, 1, wanted, &found, values, &lwork),
                 "zhegvdx_bufferSize");
    auto* work = static_cast<cuDoubleComplex*>(ws.solver_work.reserve(sizeof(cuDoubleComplex) * std::max(1, lwork)));
    check_solver(cusolverDnZhegvdx(solver, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUSOLVER_EIG_RANGE_I,
                                   CUBLAS_FILL_MODE_LOWER, m, hz, m, sz, m, 0.0, 0.0, 1, wanted, &found, values,
                                   work, lwork, info),
                 "zhegvdx");
    if (found != wanted) throw std::runtime_error("selected generalized Ritz failed: found " + std::to_string(found));
  }
  int host_info = 0;
  SDFT_CUDA(cudaMemcpyAsync(&host_info, info, sizeof(int), cudaMemcpyDeviceToHost, st));
  SDFT_CUDA(cudaStreamSynchronize(st));
  if (host_info) throw std::runtime_error("LAPACK generalized Rayleigh-Ritz failed: info=" + std::to_string(host_info));
  if (vectors != h) copy_block(h, m, vectors, m, m, full ? m : wanted, st);
}

void lowdin_combine(Cx<double>* a, const Cx<double>* f, int m, cudaStream_t stream) {
  const long long total = static_cast<long long>(m) * m;
  lowdin_combine_kernel<<<static_cast<unsigned>(std::min<long long>(ceil_div(total, 256), 148 * 8)), 256, 0,
                          stream>>>(a, f, m);
  SDFT_LAUNCH("lowdin_combine_kernel");
}

}  // namespace sdft_b200
