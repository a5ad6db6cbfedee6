// Device eigensolver for the Davidson Rayleigh-Ritz step (lowest `wanted`
// eigenpairs of an m x m Hermitian matrix, m up to ~1290).
//
// 1. tridiagonalize_kernel: one cooperative launch, one CTA per SM, columns
//    distributed cyclically and held in shared memory. Step j of the
//    Householder reduction (LAPACK zhetd2, lower, H_j = I - tau v v^H with
//    v[j+1] = 1) needs one grid-wide barrier: after it every CTA forms
//    w = p - tau/2 (p^H v) v from the published p and shares of p^H v,
//    recomputes the next reflector redundantly from the published next column
//    (plus this rank-2 update), then in one pass over its own columns applies
//    the update and accumulates p = tau A22 v for the next reflector, and
//    publishes p, its share of p^H v and the column after next. Exchange
//    buffers are double-buffered by step parity. The barrier is a counting
//    barrier with a time limit: on expiry an error word is set and every CTA
//    returns.
// 2. bisect_kernel: one warp per wanted eigenvalue, 64-point multisection on
//    division-free Sturm counts of the tridiagonal matrix.
// 3. inverse_iteration_kernel: one thread per wanted eigenvalue, factors in
//    shared memory; LU with partial pivoting of T - lambda I, two solves from
//    a start vector of its own; then cluster_orthonormalize_kernel, one CTA
//    per cluster of eigenvalues closer than 1e-9 of the matrix scale, runs
//    CGS2 over the cluster's vectors in eigenvalue order.
// 4. reflector_blocks_kernel: the reflectors in blocks of 64 as
//    I - V T V^H (compact WY); the blocks are applied to the tridiagonal
//    eigenvectors from the last to the first with three cuBLAS ZGEMMs each.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "dense.cuh"
#include "eigensolver.cuh"

namespace sdft_b200 {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxCpc = 10;
// The tridiagonalisation runs one CTA of kTridiagThreads per SM; each thread
// holds kRowsPerThread rows of the reflector and rank-2 vectors in registers
// (m <= kRowsPerThread * kTridiagThreads). 512 threads with 3 rows each
// measured slower than 256 with 5 (12.1 vs 9.9 ms at m = 1280): the step's
// CTA barriers and reductions grow with the warp count.
constexpr int kTridiagThreads = 256;
constexpr int kTridiagWarps = kTridiagThreads / 32;
constexpr int kRowsPerThread = 5;  // m <= 1280
constexpr int kReflectorBlock = 64;
constexpr int kInvitThreads = 4;
constexpr int kMaxShares = 5;  // CTA shares per lane: grid <= 160
constexpr unsigned long long kWaitNs = 2000000000ULL;
constexpr double kClusterTolerance = 1e-9;


void check_blas(cublasStatus_t status, const char* what) {
  if (status != CUBLAS_STATUS_SUCCESS)
    throw CudaError(std::string("cuBLAS error ") + std::to_string(static_cast<int>(status)) + " in " + what);
}

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

// Counting grid barrier with a time limit. Returns false (and every CTA
// should return) when the limit expired here or the error word is set. The
// CTA's writes (ordered before thread 0 by __syncthreads) are released by the
// arrival; the acquire fence after the wait orders the reads that follow.
__device__ bool grid_barrier(unsigned int* arrive, unsigned int* error, unsigned int target, int* ok) {
  __syncthreads();
  if (threadIdx.x == 0) {
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(arrive) : "memory");
    const unsigned long long start = global_ns();
    int good = 1;
    while (true) {
      unsigned int cur;
      asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(cur) : "l"(arrive) : "memory");
      if (cur >= target) break;
      if (*reinterpret_cast<volatile unsigned int*>(error) != 0u) {
        good = 0;
        break;
      }
      if (global_ns() - start > kWaitNs) {
        atomicOr(error, 1u);
        good = 0;
        break;
      }
    }
    asm volatile("fence.acq_rel.gpu;" ::: "memory");
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
  unsigned int* error;  // set when a barrier wait runs out; every CTA then returns
};

// Reflector scalars of one Householder step, formed redundantly by every
// thread from the same shared inputs (so every thread holds equal values).
struct Reflector {
  Cx<double> tau, scale;
  double beta;
  bool trivial;
};

__device__ __forceinline__ Reflector make_reflector(Cx<double> alpha, double xnorm2) {
  Reflector h;
  if (xnorm2 == 0.0 && alpha.im == 0.0) {
    h.trivial = true;
    h.tau = Cx<double>{0.0, 0.0};
    h.beta = alpha.re;
    h.scale = Cx<double>{0.0, 0.0};
  } else {
    const double beta = -copysign(sqrt(alpha.re * alpha.re + alpha.im * alpha.im + xnorm2), alpha.re);
    h.trivial = false;
    h.tau = Cx<double>{(beta - alpha.re) / beta, -alpha.im / beta};
    h.beta = beta;
    // 1 / (alpha - beta)
    const double dr = alpha.re - beta, di = alpha.im, den = dr * dr + di * di;
    h.scale = Cx<double>{dr / den, -di / den};
  }
  return h;
}

// Rows r = tid + kTridiagThreads k of the reflector and rank-2 vectors live in
// registers; own columns c = cta + G s in shared memory. Step j+1's reflector
// is formed before step j's rank-2 update, so the update of each own column
// and its product with the next reflector share one pass. Per step: one CTA
// barrier for the next column's norm, one for the column products, and the
// grid barrier.
__global__ void __launch_bounds__(kTridiagThreads, 1) tridiagonalize_kernel(TridiagArgs t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int R = kRowsPerThread;
  const int m = t.m, G = t.grid, cpc = t.cpc, cta = blockIdx.x, tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  Cx<double>* cols = reinterpret_cast<Cx<double>*>(smem_raw);
  Cx<double>* red = cols + static_cast<long long>(cpc) * m;  // kTridiagWarps x kMaxCpc column-product partials
  Cx<double>* colv = red + kTridiagWarps * kMaxCpc;                  // 2 x kMaxCpc: v at own columns, by step parity
  Cx<double>* colw = colv + 2 * kMaxCpc;                      // kMaxCpc: w at own columns
  Cx<double>* pick = colw + kMaxCpc;                          // alpha (row jc+1), diagonal (row jc)
  double* nrm = reinterpret_cast<double*>(pick + 2);          // kTridiagWarps norm partials
  __shared__ int ok;

  int slot_of_row[R];
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const int r = tid + k * kTridiagThreads;
    slot_of_row[k] = (r < m && r >= cta && (r - cta) % G == 0) ? (r - cta) / G : -1;
  }
  for (int s = 0; s < cpc; ++s) {
    const int c = cta + s * G;
    if (c < m)
      for (int r = tid; r < m; r += kTridiagThreads) cols[static_cast<long long>(s) * m + r] = t.a[r + static_cast<long long>(c) * m];
  }

  Cx<double> v[R], w[R], vn[R], col[R];
  Reflector cur, next;

  // Reflector of column jc from col[] (rows >= jc): vn[] for rows >= jc+1,
  // v at own columns into colv[jc & 1], and CTA 0's outputs. Contains the
  // step's first CTA barrier (after which colw, written before it, is visible).
  auto reflect = [&](int jc) -> Reflector {
    double part = 0.0;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int r = tid + k * kTridiagThreads;
      if (r < m && r >= jc + 2) part += col[k].re * col[k].re + col[k].im * col[k].im;
      if (r == jc + 1) pick[0] = col[k];
      if (r == jc) pick[1] = col[k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if (lane == 0) nrm[warp] = part;
    __syncthreads();
    double xnorm2 = 0.0;
#pragma unroll
    for (int q = 0; q < kTridiagWarps; ++q) xnorm2 += nrm[q];
    const Reflector h = make_reflector(pick[0], xnorm2);
    if (cta == 0 && tid == 0) {
      t.d[jc] = pick[1].re;
      t.e[jc] = h.beta;
      t.tau[jc] = h.tau;
    }
    Cx<double>* cv = colv + (jc & 1) * kMaxCpc;
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int r = tid + k * kTridiagThreads;
      Cx<double> vr{0.0, 0.0};
      if (r == jc + 1) vr = Cx<double>{1.0, 0.0};
      else if (r > jc + 1 && r < m && !h.trivial) vr = cmulz(col[k], h.scale);
      vn[k] = vr;
      if (cta == 0 && r > jc && r < m) t.reflectors[r + static_cast<long long>(jc) * m] = vr;
      if (slot_of_row[k] >= 0) cv[slot_of_row[k]] = vr;
    }
    return h;
  };

  // Column products conj(A(:,c)) . vn over the CTA (acc), then p = tau A v at
  // own columns c > jc, the CTA share of p^H v, and column jc+1 published.
  auto publish = [&](int jc, const Reflector& h, Cx<double> (&acc)[kMaxCpc]) {
#pragma unroll
    for (int q = 0; q < kMaxCpc; ++q) {
      if (q < cpc) {
        double re = acc[q].re, im = acc[q].im;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          re += __shfl_xor_sync(0xffffffffu, re, o);
          im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        if (lane == 0) red[warp * kMaxCpc + q] = Cx<double>{re, im};
      }
    }
    __syncthreads();
    if (warp == 0) {
      Cx<double> dot{0.0, 0.0};
      const int c = cta + lane * G;
      if (lane < cpc && c > jc && c < m) {
        Cx<double> s{0.0, 0.0};
        for (int q = 0; q < kTridiagWarps; ++q) s = cadd(s, red[q * kMaxCpc + lane]);
        const Cx<double> p = cmulz(h.tau, s);
        t.pbuf[static_cast<long long>(jc & 1) * m + c] = p;
        dot = cdot1(p, colv[(jc & 1) * kMaxCpc + lane]);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        dot.re += __shfl_xor_sync(0xffffffffu, dot.re, o);
        dot.im += __shfl_xor_sync(0xffffffffu, dot.im, o);
      }
      if (lane == 0) t.dotbuf[static_cast<long long>(jc & 1) * G + cta] = dot;
    }
    // Column jc+1 (updates 0..jc-1 applied) for step jc+1.
    if (jc + 1 < m && (jc + 1) % G == cta) {
      const long long slot = (jc + 1) / G;
      Cx<double>* dst = t.colbuf + static_cast<long long>((jc + 1) & 1) * m;
      for (int r = jc + 1 + tid; r < m; r += kTridiagThreads) dst[r] = cols[slot * m + r];
    }
  };

  // Step 0: reflector of column 0, p_0 over own columns, column 1 published.
#pragma unroll
  for (int k = 0; k < R; ++k) {
    const int r = tid + k * kTridiagThreads;
    col[k] = r < m ? t.a[r] : Cx<double>{0.0, 0.0};
  }
  __syncthreads();  // own columns in shared memory
  cur = reflect(0);
#pragma unroll
  for (int k = 0; k < R; ++k) v[k] = vn[k];
  {
    Cx<double> acc[kMaxCpc];
#pragma unroll
    for (int q = 0; q < kMaxCpc; ++q) {
      acc[q] = Cx<double>{0.0, 0.0};
      const int c = cta + q * G;
      if (q >= cpc || c < 1 || c >= m) continue;
      const Cx<double>* a = cols + static_cast<long long>(q) * m;
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const int r = tid + k * kTridiagThreads;
        if (r >= 1 && r < m) acc[q] = cadd(acc[q], cdot1(a[r], v[k]));
      }
    }
    publish(0, cur, acc);
  }
  if (!grid_barrier(t.arrive, t.error, static_cast<unsigned int>(G), &ok)) return;

  for (int j = 0; j < m - 1; ++j) {
    const bool last = j == m - 2;
    // All of this step's global reads first (one round of L2 latency): p on
    // own rows, column j+1, p at own columns and at row j+1, the CTA shares
    // of p^H v (every warp sums them in the same order).
    const double2* pb = reinterpret_cast<const double2*>(t.pbuf + static_cast<long long>(j & 1) * m);
    const double2* cb = reinterpret_cast<const double2*>(t.colbuf + static_cast<long long>((j + 1) & 1) * m);
    const double2* db = reinterpret_cast<const double2*>(t.dotbuf + static_cast<long long>(j & 1) * G);
    const double2 zero2 = make_double2(0.0, 0.0);
    double2 pq[R], cq[R], shares[kMaxShares];
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int r = tid + k * kTridiagThreads;
      const bool row = r > j && r < m;
      pq[k] = (row && !cur.trivial) ? __ldcg(pb + r) : zero2;
      cq[k] = (row && !last) ? __ldcg(cb + r) : zero2;
    }
    const int own_c = cta + tid * G;
    const bool own_w = !cur.trivial && tid < cpc && own_c > j && own_c < m;
    const double2 pc = own_w ? __ldcg(pb + own_c) : zero2;
    const double2 ph = cur.trivial ? zero2 : __ldcg(pb + j + 1);
#pragma unroll
    for (int i = 0; i < kMaxShares; ++i) {
      const int g = lane + 32 * i;
      shares[i] = (!cur.trivial && g < G) ? __ldcg(db + g) : zero2;
    }
    Cx<double> sum{0.0, 0.0};
#pragma unroll
    for (int i = 0; i < kMaxShares; ++i) sum = cadd(sum, Cx<double>{shares[i].x, shares[i].y});
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sum.re += __shfl_xor_sync(0xffffffffu, sum.re, o);
      sum.im += __shfl_xor_sync(0xffffffffu, sum.im, o);
    }
    const Cx<double> alpha = cmulz(Cx<double>{-0.5 * cur.tau.re, -0.5 * cur.tau.im}, sum);
    // w = p + alpha v on own rows; w at own columns for the update; w[j+1] (v[j+1] = 1).
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const int r = tid + k * kTridiagThreads;
      w[k] = (r > j && r < m && !cur.trivial) ? cadd(Cx<double>{pq[k].x, pq[k].y}, cmulz(alpha, v[k]))
                                               : Cx<double>{0.0, 0.0};
      col[k] = Cx<double>{cq[k].x, cq[k].y};
    }
    const Cx<double> head_w = cur.trivial ? Cx<double>{0.0, 0.0} : cadd(Cx<double>{ph.x, ph.y}, alpha);
    if (own_w) colw[tid] = cadd(Cx<double>{pc.x, pc.y}, cmulz(alpha, colv[(j & 1) * kMaxCpc + tid]));

    // Step j+1's reflector from column j+1 with update j applied.
    if (!last) {
      const Cx<double> hw = cconj(head_w);
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const int r = tid + k * kTridiagThreads;
        if (r > j && r < m) col[k] = csub(col[k], cadd(cmulz(v[k], hw), w[k]));
      }
      next = reflect(j + 1);
    } else {
      __syncthreads();  // colw visible
    }

    // Update j on own columns c > j; p_{j+1} partial sums over rows/columns > j+1.
    Cx<double> acc[kMaxCpc];
#pragma unroll
    for (int q = 0; q < kMaxCpc; ++q) {
      acc[q] = Cx<double>{0.0, 0.0};
      const int c = cta + q * G;
      if (q >= cpc || c <= j || c >= m) continue;
      const Cx<double> wc = cconj(colw[q]), vc = cconj(colv[(j & 1) * kMaxCpc + q]);
      Cx<double>* a = cols + static_cast<long long>(q) * m;
      const bool dot_column = !last && c > j + 1;
#pragma unroll
      for (int k = 0; k < R; ++k) {
        const int r = tid + k * kTridiagThreads;
        if (r > j && r < m) {
          Cx<double> x = a[r];
          if (!cur.trivial) {
            x = csub(x, cadd(cmulz(v[k], wc), cmulz(w[k], vc)));
            a[r] = x;
          }
          if (dot_column && r > j + 1) acc[q] = cadd(acc[q], cdot1(x, vn[k]));
        }
      }
    }
    if (last) break;
    publish(j + 1, next, acc);
    if (!grid_barrier(t.arrive, t.error, static_cast<unsigned int>(G) * static_cast<unsigned int>(j + 2), &ok))
      return;
    cur = next;
#pragma unroll
    for (int k = 0; k < R; ++k) v[k] = vn[k];
  }
  __syncthreads();
  if ((m - 1) % G == cta && tid == 0) t.d[m - 1] = cols[static_cast<long long>((m - 1) / G) * m + m - 1].re;
}

// Number of eigenvalues of the tridiagonal (d, e) below x: sign changes of
// the Sturm sequence p_0 = 1, p_1 = d_0 - x, p_i = (d_{i-1} - x) p_{i-1} -
// e_{i-2}^2 p_{i-2}, kept in range by exact power-of-two rescaling. A p_i
// below pivmin |p_{i-1}| counts as a sign change (the q = -pivmin convention
// of the quotient form q_i = p_i / p_{i-1}).
template <int P>
__device__ void sturm_counts(const double* d, const double* e2, int m, const double (&x)[P], double pivmin,
                             int (&count)[P]) {
  double p0[P], p1[P];
#pragma unroll
  for (int q = 0; q < P; ++q) {
    p0[q] = 1.0;
    p1[q] = d[0] - x[q];
    if (fabs(p1[q]) <= pivmin) p1[q] = -pivmin;
    count[q] = p1[q] < 0.0;
  }
  for (int i = 1; i < m; ++i) {
    const double di = d[i], ei = e2[i - 1];
#pragma unroll
    for (int q = 0; q < P; ++q) {
      double p2 = fma(di - x[q], p1[q], -ei * p0[q]);
      if (fabs(p2) <= pivmin * fabs(p1[q])) p2 = -pivmin * p1[q];
      count[q] += (p2 < 0.0) != (p1[q] < 0.0);
      p0[q] = p1[q];
      p1[q] = p2;
    }
    // Exact rescaling by 2^-400 / 2^400 every fourth step: a step grows the
    // sequence by far less than 2^100 here, so nothing leaves the exponent
    // range in between, and power-of-two scaling changes no sign or ratio.
    if ((i & 3) == 0) {
#pragma unroll
      for (int q = 0; q < P; ++q) {
        const double mag = fabs(p1[q]);
        const double f = mag > 0x1p+400 ? 0x1p-400 : (mag < 0x1p-400 ? 0x1p+400 : 1.0);
        p0[q] *= f;
        p1[q] *= f;
      }
    }
  }
}

// One warp per wanted eigenvalue; 32 x P points per round (P per lane).
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
  const double tnorm = fmax(fabs(lo), fabs(hi));  // Gershgorin bound of the spectrum
  const double pad = 4.0 * DBL_EPSILON * tnorm + pivmin;
  lo -= pad;
  hi += pad;
  // Absolute tolerance of the matrix scale (LAPACK dstebz's default abstol,
  // eps * max(|gl|, |gu|)), beside the relative one: eigenvalues near zero
  // stop at eps * |T| instead of running every round.
  const double atol = DBL_EPSILON * tnorm;
  constexpr int P = 4;
  for (int round = 0; round < 64; ++round) {
    const double width = hi - lo;
    if (width <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) || width <= atol || width <= pivmin) break;
    const double step = width / (32 * P + 1);
    // point q of lane l is lo + (q * 32 + l + 1) step: increasing over (q, l);
    // the lane's P Sturm sequences run interleaved.
    double x[P];
    int counts[P];
#pragma unroll
    for (int q = 0; q < P; ++q) x[q] = lo + (q * 32 + lane + 1) * step;
    sturm_counts<P>(sd, se2, m, x, pivmin, counts);
    unsigned masks[P];
#pragma unroll
    for (int q = 0; q < P; ++q) masks[q] = __ballot_sync(0xffffffffu, counts[q] > k);
    int above = -1;  // first point index with count > k
#pragma unroll
    for (int q = P - 1; q >= 0; --q)
      if (masks[q]) above = q * 32 + __ffs(masks[q]) - 1;
    double new_lo = lo, new_hi = hi;
    if (above >= 0) new_hi = lo + (above + 1) * step;
    if (above != 0) new_lo = lo + (above < 0 ? 32 * P : above) * step;
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

// One thread per wanted eigenvalue, kInvitThreads threads per CTA, each with
// its LU factors and vector in shared memory: reciprocal pivots, the two U
// superdiagonals, multipliers, z and pivot flags (bytes); two solves from a
// start vector of its own. Clusters are orthonormalised afterwards
// (cluster_orthonormalize_kernel).
__global__ void inverse_iteration_kernel(const double* __restrict__ d, const double* __restrict__ e, int m, int wanted,
                                         const double* __restrict__ values, double* __restrict__ zt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  double* base = reinterpret_cast<double*>(smem_raw) + static_cast<long long>(threadIdx.x) * 5 * m;
  double* rinv = base;
  double* u1 = base + m;
  double* u2 = base + 2 * m;
  double* mult = base + 3 * m;
  double* z = base + 4 * m;
  unsigned char* piv =
      reinterpret_cast<unsigned char*>(reinterpret_cast<double*>(smem_raw) + static_cast<long long>(blockDim.x) * 5 * m) +
      static_cast<long long>(threadIdx.x) * m;
  if (k >= wanted) return;
  double norm = 0.0;
  for (int i = 0; i < m; ++i) norm = fmax(norm, fabs(d[i]) + (i + 1 < m ? fabs(e[i]) : 0.0));
  const double tiny = DBL_EPSILON * fmax(norm, DBL_MIN);
  const long long W = wanted;
  {
    const int q = k;
    const double lam = values[q];
    // LU of T - lam I with partial pivoting (rows i, i+1 swapped when |sub| wins).
    double cur_d = d[0] - lam, cur_u = m > 1 ? e[0] : 0.0;
    for (int i = 0; i + 1 < m; ++i) {
      const double nd = d[i + 1] - lam, nu = i + 2 < m ? e[i + 1] : 0.0, l = e[i];
      if (fabs(cur_d) >= fabs(l)) {
        if (fabs(cur_d) < tiny) cur_d = copysign(tiny, cur_d == 0.0 ? 1.0 : cur_d);
        const double r = 1.0 / cur_d;
        rinv[i] = r;
        u1[i] = cur_u;
        u2[i] = 0.0;
        mult[i] = l * r;
        piv[i] = 0;
        cur_d = nd - mult[i] * cur_u;
        cur_u = nu;
      } else {
        const double mu = cur_d / l;
        rinv[i] = 1.0 / l;
        u1[i] = nd;
        u2[i] = nu;
        mult[i] = mu;
        piv[i] = 1;
        cur_d = cur_u - mu * nd;
        cur_u = -mu * nu;
      }
    }
    if (fabs(cur_d) < tiny) cur_d = copysign(tiny, cur_d == 0.0 ? 1.0 : cur_d);
    rinv[m - 1] = 1.0 / cur_d;
    for (int i = 0; i < m; ++i) z[i] = start_entry(q, i);
    for (int it = 0; it < 2; ++it) {
      for (int i = 0; i + 1 < m; ++i) {
        double a = z[i], b = z[i + 1];
        if (piv[i]) {
          const double tmp = a;
          a = b;
          b = tmp;
        }
        z[i] = a;
        z[i + 1] = b - mult[i] * a;
      }
      double z2 = z[m - 1] * rinv[m - 1];
      z[m - 1] = z2;
      double z1 = 0.0;
      if (m > 1) {
        z1 = (z[m - 2] - u1[m - 2] * z2) * rinv[m - 2];
        z[m - 2] = z1;
      }
      for (int i = m - 3; i >= 0; --i) {
        const double zi = (z[i] - u1[i] * z1 - u2[i] * z2) * rinv[i];
        z[i] = zi;
        z2 = z1;
        z1 = zi;
      }
      double nrm = 0.0;
      for (int i = 0; i < m; ++i) nrm += z[i] * z[i];
      const double inv = 1.0 / sqrt(nrm);
      for (int i = 0; i < m; ++i) z[i] *= inv;
    }
    for (int i = 0; i < m; ++i) zt[i * W + q] = z[i];
  }
}

// Orthonormalises the inverse-iteration vectors of each cluster of
// eigenvalues closer than kClusterTolerance of the matrix scale (chains of
// such gaps), in eigenvalue order: classical Gram-Schmidt against the earlier
// members, twice, then normalisation. One CTA per cluster (CTAs whose index
// does not start a cluster of two or more return at once); the vectors,
// found independently from distinct start vectors, span the cluster's
// invariant subspace.
__global__ void __launch_bounds__(kThreads) cluster_orthonormalize_kernel(const double* __restrict__ d,
                                                                          const double* __restrict__ e, int m,
                                                                          int wanted, const double* __restrict__ values,
                                                                          double* __restrict__ zt) {
  extern __shared__ double dots[];  // one per earlier cluster member
  __shared__ double partial[kWarps];
  const int k = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double norm = 0.0;
  for (int i = tid; i < m; i += kThreads) norm = fmax(norm, fabs(d[i]) + (i + 1 < m ? fabs(e[i]) : 0.0));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) norm = fmax(norm, __shfl_xor_sync(0xffffffffu, norm, o));
  if (lane == 0) partial[warp] = norm;
  __syncthreads();
  norm = 0.0;
  for (int w = 0; w < kWarps; ++w) norm = fmax(norm, partial[w]);
  const double cluster = kClusterTolerance * fmax(norm, DBL_MIN);
  if (k > 0 && values[k] - values[k - 1] <= cluster) return;
  int end = k;
  while (end + 1 < wanted && values[end + 1] - values[end] <= cluster) ++end;
  if (end == k) return;
  const long long W = wanted;
  for (int q = k + 1; q <= end; ++q) {
    for (int pass = 0; pass < 2; ++pass) {
      __syncthreads();
      // dots with the earlier members: warp w takes members k + w, k + w + kWarps, ...
      for (int p = k + warp; p < q; p += kWarps) {
        double s = 0.0;
        for (int i = lane; i < m; i += 32) s += zt[i * W + p] * zt[i * W + q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) dots[p - k] = s;
      }
      __syncthreads();
      for (int i = tid; i < m; i += kThreads) {
        double v = zt[i * W + q];
        for (int p = k; p < q; ++p) v -= dots[p - k] * zt[i * W + p];
        zt[i * W + q] = v;
      }
    }
    __syncthreads();
    double s = 0.0;
    for (int i = tid; i < m; i += kThreads) s += zt[i * W + q] * zt[i * W + q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) partial[warp] = s;
    __syncthreads();
    double total = 0.0;
    for (int w = 0; w < kWarps; ++w) total += partial[w];
    const double inv = 1.0 / sqrt(total);
    for (int i = tid; i < m; i += kThreads) zt[i * W + q] *= inv;
  }
}

// Compact WY factor of each block of kReflectorBlock reflectors:
// H_j0 ... H_j0+nb-1 = I - V T V^H (LAPACK zlarft, forward, columnwise),
// T upper triangular (column-major, leading dimension kReflectorBlock), from
// the block's Gram matrix V^H V. One CTA per block.
__global__ void __launch_bounds__(kThreads) reflector_blocks_kernel(const Cx<double>* __restrict__ grams,
                                                                    const Cx<double>* __restrict__ tau, int m,
                                                                    Cx<double>* __restrict__ tfac) {
  // One CTA per block of NB reflectors: T of I - V T V^H (zlarft) from the
  // block's Gram matrix G = V^H V (column-major NB x NB, computed by cuBLAS).
  constexpr int NB = kReflectorBlock, LD = NB + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<double>* gram = reinterpret_cast<Cx<double>*>(smem_raw);  // NB x LD, gram[a * LD + b] = G(a, b)
  Cx<double>* tmat = gram + NB * LD;                            // NB x LD
  const int j0 = blockIdx.x * NB;
  const int nb = min(NB, m - 1 - j0);
  const int tid = threadIdx.x;
  const Cx<double>* g = grams + static_cast<long long>(blockIdx.x) * NB * NB;
  for (int idx = tid; idx < NB * NB; idx += kThreads) {
    const int col = idx / NB, row = idx % NB;
    gram[row * LD + col] = g[idx];
    tmat[(idx / NB) * LD + idx % NB] = Cx<double>{0.0, 0.0};
  }
  __syncthreads();
  // T(i,i) = tau_i; T(0:i, i) = -tau_i T(0:i, 0:i) G(0:i, i).
  for (int i = 0; i < nb; ++i) {
    const Cx<double> ti = tau[j0 + i];
    if (tid < i) {
      Cx<double> sum{0.0, 0.0};
      for (int c = tid; c < i; ++c) sum = cadd(sum, cmulz(tmat[tid * LD + c], gram[c * LD + i]));
      tmat[tid * LD + i] = cmulz(Cx<double>{-ti.re, -ti.im}, sum);
    }
    if (tid == 0) tmat[i * LD + i] = ti;
    __syncthreads();
  }
  for (int idx = tid; idx < NB * NB; idx += kThreads) {
    const int col = idx / NB, row = idx % NB;
    tfac[static_cast<long long>(blockIdx.x) * NB * NB + idx] = tmat[row * LD + col];
  }
}

// X (complex, column-major, leading dimension m) from the row-major real
// tridiagonal eigenvectors zt (m x wanted).
__global__ void complex_columns_kernel(const double* __restrict__ zt, int m, int wanted, Cx<double>* __restrict__ x) {
  const long long total = static_cast<long long>(m) * wanted;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long i = idx % m, q = idx / m;
    x[idx] = Cx<double>{zt[i * wanted + q], 0.0};
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

// c <- I - e/2 + 3/8 c (c holds E^2 on entry)
__global__ void lowdin_second_order_kernel(const Cx<double>* __restrict__ e, Cx<double>* __restrict__ c, int m) {
  const long long total = static_cast<long long>(m) * m;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long i = idx % m, j = idx / m;
    const Cx<double> x = e[idx], y = c[idx];
    c[idx] = Cx<double>{(i == j ? 1.0 : 0.0) - 0.5 * x.re + 0.375 * y.re, -0.5 * x.im + 0.375 * y.im};
  }
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
  return sizeof(Cx<double>) * (static_cast<std::size_t>(cpc) * m + kTridiagWarps * kMaxCpc + 3 * kMaxCpc + 2) +
         sizeof(double) * kTridiagWarps;
}

constexpr std::size_t kSmemLimit = 227 * 1024;

std::size_t invit_smem(int m) { return static_cast<std::size_t>(kInvitThreads) * (5 * sizeof(double) + 1) * m; }

constexpr std::size_t kBlockSmem = sizeof(Cx<double>) * 2 * kReflectorBlock * (kReflectorBlock + 1);

}  // namespace

namespace {
// Cooperative kernels that fill every SM must not run at the same time (two
// of them could each hold part of the SMs and wait on each other's missing
// CTAs), so every solver on a device, whatever its stream, launches them in
// order on one shared stream: the caller's stream hands over with an event
// and waits for the kernel's completion event.
struct CooperativeLane {
  std::mutex mutex;
  cudaStream_t stream = nullptr;
};

CooperativeLane& cooperative_lane(int device) {
  static CooperativeLane lanes[64];
  if (device < 0 || device >= 64) throw InvalidArgument("device ordinal out of range");
  return lanes[device];
}

void cooperative_launch(void* kernel, int grid, int threads, TridiagArgs& args, std::size_t smem, cudaStream_t stream) {
  int device = 0;
  SDFT_CUDA(cudaGetDevice(&device));
  CooperativeLane& lane = cooperative_lane(device);
  cudaEvent_t ready = nullptr, done = nullptr;
  SDFT_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  SDFT_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
  try {
    std::lock_guard<std::mutex> lock(lane.mutex);
    if (!lane.stream) SDFT_CUDA(cudaStreamCreateWithFlags(&lane.stream, cudaStreamNonBlocking));
    SDFT_CUDA(cudaEventRecord(ready, stream));
    SDFT_CUDA(cudaStreamWaitEvent(lane.stream, ready, 0));
    void* params[] = {&args};
    SDFT_CUDA(cudaLaunchCooperativeKernel(kernel, dim3(grid), dim3(threads), params, smem, lane.stream));
    SDFT_LAUNCH("tridiagonalize_kernel");
    SDFT_CUDA(cudaEventRecord(done, lane.stream));
    SDFT_CUDA(cudaStreamWaitEvent(stream, done, 0));
  } catch (...) {
    cudaEventDestroy(ready);
    cudaEventDestroy(done);
    throw;
  }
  cudaEventDestroy(ready);  // released once the recorded work completes
  cudaEventDestroy(done);
}
}  // namespace

int hermitian_eigen_max_order() {
  const int g = sm_count();
  int best = 0;
  for (int m = 2; m <= 4096; ++m) {
    const int grid = std::min({g, m, 32 * kMaxShares});
    const int cpc = (m + grid - 1) / grid;
    if (cpc > kMaxCpc || tridiag_smem(m, cpc) > kSmemLimit || m > kRowsPerThread * kTridiagThreads ||
        invit_smem(m) > kSmemLimit)
      break;
    best = m;
  }
  return best;
}

void hermitian_lowest(cublasHandle_t blas, Cx<double>* a, int m, int wanted, double* values, Cx<double>* vectors,
                      EigenWorkspace& ws, cudaStream_t stream) {
  if (m < 2 || wanted < 1 || wanted > m) throw InvalidArgument("invalid Hermitian eigenproblem size");
  const int grid = std::min({sm_count(), m, 32 * kMaxShares});
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
  unsigned int* error_word = arrive + 1;
  SDFT_CUDA(cudaMemsetAsync(arrive, 0, 2 * sizeof(unsigned int), stream));
  // Entries above each reflector's unit element stay zero for the block products.
  SDFT_CUDA(cudaMemsetAsync(reflectors, 0, sizeof(Cx<double>) * mm * mm, stream));

  allow_dynamic_smem(tridiagonalize_kernel, smem);
  int per_sm = 0;
  SDFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tridiagonalize_kernel, kTridiagThreads, smem));
  if (per_sm < 1) throw InvalidArgument("tridiagonalization kernel cannot be resident");
  // SDFT_B200_TRACE: device times of the stages, printed after the final synchronisation.
  static const bool trace = std::getenv("SDFT_B200_TRACE") != nullptr;
  cudaEvent_t marks[6] = {};
  if (trace)
    for (auto& ev : marks) SDFT_CUDA(cudaEventCreate(&ev));
  auto mark = [&](int i) {
    if (trace) SDFT_CUDA(cudaEventRecord(marks[i], stream));
  };
  mark(0);
  TridiagArgs t{a, m, grid, cpc, d, e, tau, reflectors, colbuf, pbuf, dotbuf, arrive, error_word};
  cooperative_launch(reinterpret_cast<void*>(tridiagonalize_kernel), grid, kTridiagThreads, t, smem, stream);
  mark(1);

  const int warps_per_block = 4;
  const std::size_t bisect_smem = sizeof(double) * 2 * mm;
  allow_dynamic_smem(bisect_kernel, bisect_smem);
  bisect_kernel<<<static_cast<unsigned>(ceil_div(wanted, warps_per_block)), 32 * warps_per_block, bisect_smem,
                  stream>>>(d, e, m, wanted, values);
  SDFT_LAUNCH("bisect_kernel");
  mark(2);

  const int blocks = static_cast<int>(ceil_div(m - 1, kReflectorBlock));
  // The complex arrays after the real eigenvectors start on a 16-byte
  // boundary: wanted * m doubles are rounded up to an even count (an odd
  // product left them 8-byte aligned, which cuBLAS refuses for complex data).
  const std::size_t zt_doubles = (static_cast<std::size_t>(wanted) * mm + 1) & ~static_cast<std::size_t>(1);
  const std::size_t vbytes =
      sizeof(double) * zt_doubles +
      sizeof(Cx<double>) * (2 * static_cast<std::size_t>(blocks) + 2 * static_cast<std::size_t>(wanted)) *
          kReflectorBlock * kReflectorBlock;
  auto* zt = static_cast<double*>(ws.vectors.reserve(vbytes));
  auto* tfac = reinterpret_cast<Cx<double>*>(zt + zt_doubles);
  Cx<double>* grams = tfac + static_cast<std::size_t>(blocks) * kReflectorBlock * kReflectorBlock;
  Cx<double>* wtmp = grams + static_cast<std::size_t>(blocks) * kReflectorBlock * kReflectorBlock;
  Cx<double>* utmp = wtmp + static_cast<std::size_t>(wanted) * kReflectorBlock;
  const std::size_t inv_smem = invit_smem(m);
  allow_dynamic_smem(inverse_iteration_kernel, inv_smem);
  inverse_iteration_kernel<<<static_cast<unsigned>(ceil_div(wanted, kInvitThreads)), kInvitThreads, inv_smem,
                             stream>>>(d, e, m, wanted, values, zt);
  SDFT_LAUNCH("inverse_iteration_kernel");
  const std::size_t dots_smem = sizeof(double) * static_cast<std::size_t>(wanted);
  allow_dynamic_smem(cluster_orthonormalize_kernel, dots_smem);
  cluster_orthonormalize_kernel<<<static_cast<unsigned>(wanted), kThreads, dots_smem, stream>>>(d, e, m, wanted,
                                                                                                values, zt);
  SDFT_LAUNCH("cluster_orthonormalize_kernel");
  mark(3);

  // Gram blocks V_b^H V_b of the reflector blocks (zeros above each unit
  // element): one strided-batched ZGEMM over the full blocks, one for the rest.
  {
    const cuDoubleComplex one{1.0, 0.0}, zero{0.0, 0.0};
    const int full = (m - 1) / kReflectorBlock, rest = (m - 1) % kReflectorBlock;
    const long long block_stride = static_cast<long long>(kReflectorBlock) * m;
    const long long gram_stride = static_cast<long long>(kReflectorBlock) * kReflectorBlock;
    auto* v = reinterpret_cast<const cuDoubleComplex*>(reflectors);
    auto* gz = reinterpret_cast<cuDoubleComplex*>(grams);
    if (full > 0)
      check_blas(cublasZgemmStridedBatched(blas, CUBLAS_OP_C, CUBLAS_OP_N, kReflectorBlock, kReflectorBlock, m, &one,
                                           v, m, block_stride, v, m, block_stride, &zero, gz, kReflectorBlock,
                                           gram_stride, full),
                 "zgemmStridedBatched");
    if (rest > 0)
      check_blas(cublasZgemm(blas, CUBLAS_OP_C, CUBLAS_OP_N, rest, rest, m, &one, v + full * block_stride, m,
                             v + full * block_stride, m, &zero, gz + full * gram_stride, kReflectorBlock),
                 "zgemm");
  }
  allow_dynamic_smem(reflector_blocks_kernel, kBlockSmem);
  reflector_blocks_kernel<<<static_cast<unsigned>(blocks), kThreads, kBlockSmem, stream>>>(grams, tau, m, tfac);
  SDFT_LAUNCH("reflector_blocks_kernel");
  mark(4);

  // X = Q Z: blocks from the last to the first, X <- X - V (T (V^H X)) on rows > j0.
  const long long total = static_cast<long long>(m) * wanted;
  complex_columns_kernel<<<static_cast<unsigned>(std::min<long long>(ceil_div(total, 256), 148 * 8)), 256, 0,
                           stream>>>(zt, m, wanted, vectors);
  SDFT_LAUNCH("complex_columns_kernel");
  for (int b = blocks - 1; b >= 0; --b) {
    const int j0 = b * kReflectorBlock;
    const int nb = std::min(kReflectorBlock, m - 1 - j0);
    const int rows = m - 1 - j0;
    const Cx<double>* vb = reflectors + (j0 + 1) + static_cast<long long>(j0) * m;
    Cx<double>* xs = vectors + (j0 + 1);
    const Cx<double>* tb = tfac + static_cast<long long>(b) * kReflectorBlock * kReflectorBlock;
    zgemm(blas, Op::C, Op::N, nb, wanted, rows, vb, m, xs, m, wtmp, kReflectorBlock, false);
    zgemm(blas, Op::N, Op::N, nb, wanted, nb, tb, kReflectorBlock, wtmp, kReflectorBlock, utmp, kReflectorBlock, false);
    zgemm(blas, Op::N, Op::N, rows, wanted, nb, vb, m, utmp, kReflectorBlock, xs, m, true, -1.0);
  }
  mark(5);

  unsigned int error = 0;
  SDFT_CUDA(cudaMemcpyAsync(&error, error_word, sizeof(error), cudaMemcpyDeviceToHost, stream));
  SDFT_CUDA(cudaStreamSynchronize(stream));
  if (trace) {
    float ms[5];
    for (int i = 0; i < 5; ++i) SDFT_CUDA(cudaEventElapsedTime(&ms[i], marks[i], marks[i + 1]));
    std::fprintf(stderr,
                 "hermitian-lowest m=%d wanted=%d tridiagonalize=%.3fms bisect=%.3fms inverse_iteration=%.3fms "
                 "reflector_blocks=%.3fms back_transform=%.3fms\n",
                 m, wanted, ms[0], ms[1], ms[2], ms[3], ms[4]);
    for (auto& ev : marks) cudaEventDestroy(ev);
  }
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

void lowdin_second_order(const Cx<double>* e, Cx<double>* c, int m, cudaStream_t stream) {
  const long long total = static_cast<long long>(m) * m;
  lowdin_second_order_kernel<<<static_cast<unsigned>(std::min<long long>(ceil_div(total, 256), 148 * 8)), 256, 0,
                               stream>>>(e, c, m);
  SDFT_LAUNCH("lowdin_second_order_kernel");
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
                        cudaStream_t st, double max_deviation, double first_order_limit) {
  if (m < 1 || wanted < 1 || wanted > m) throw InvalidArgument("invalid Rayleigh-Ritz dimensions");
  const std::size_t mm = static_cast<std::size_t>(m);
  if (mode == RitzSolver::Device && m >= 2 && m <= hermitian_eigen_max_order()) {
    const double deviation = identity_deviation(s, m, ws, st);
    if (!std::isfinite(deviation)) throw NonFinite("Rayleigh-Ritz overlap is not finite");
    static const bool trace = std::getenv("SDFT_B200_TRACE") != nullptr;
    if (trace)
      std::fprintf(stderr, "rayleigh-ritz m=%d |S-I|max=%.3e path=%s\n", m, deviation,
                   deviation <= first_order_limit ? "device" : deviation <= max_deviation ? "device-loewdin2" : "cusolver");
    if (deviation <= first_order_limit) {
      // First order: H' = H - (E H + H E)/2, y -> y - E y / 2 (error O(|E|^2)).
      const bool correct = deviation > 1e-14;
      Cx<double>* f = nullptr;
      if (correct) {
        f = static_cast<Cx<double>*>(ws.product.reserve(sizeof(Cx<double>) * mm * mm));
        zgemm(blas, Op::N, Op::N, m, m, m, s, m, h, m, f, m, false);
        lowdin_combine(h, f, m, st);
      }
      hermitian_lowest(blas, h, m, wanted, values, vectors, ws, st);
      if (correct) {
        zgemm(blas, Op::N, Op::N, m, wanted, m, s, m, vectors, m, f, m, false, -0.5);
        add_block(f, m, vectors, m, m, wanted, st);
      }
      return;
    }
    if (deviation <= max_deviation) {
      // Second order: C = I - E/2 + 3/8 E^2 = S^(-1/2) + O(|E|^3); H' = C H C, y -> C y.
      auto* f = static_cast<Cx<double>*>(ws.product.reserve(sizeof(Cx<double>) * mm * mm));
      auto* c = static_cast<Cx<double>*>(ws.product2.reserve(sizeof(Cx<double>) * mm * mm));
      zgemm(blas, Op::N, Op::N, m, m, m, s, m, s, m, c, m, false);
      lowdin_second_order(s, c, m, st);
      zgemm(blas, Op::N, Op::N, m, m, m, c, m, h, m, f, m, false);
      zgemm(blas, Op::N, Op::N, m, m, m, f, m, c, m, h, m, false);
      hermitian_lowest(blas, h, m, wanted, values, vectors, ws, st);
      zgemm(blas, Op::N, Op::N, m, wanted, m, c, m, vectors, m, f, m, false);
      copy_block(f, m, vectors, m, m, wanted, st);
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
