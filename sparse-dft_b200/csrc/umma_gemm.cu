// tcgen05 / TMEM / TMA BF16 GEMM for the mixed-precision complex products.
//
// One CTA computes a 128 x BN FP32 tile of Ahat Bhat^T over a range of 64-wide
// K blocks (split-K across CTAs). Warp 0 lane 0 streams A and B tiles with TMA
// (128-byte swizzle, no multicast) into a STAGES-deep shared-memory ring;
// warp 1 lane 0 issues tcgen05.mma (M=128, N=BN, K=16 per instruction) into a
// tensor-memory accumulator and releases ring slots with tcgen05.commit; then
// all four warps drain the accumulator with tcgen05.ld (warp w owns TMEM lanes
// 32w..32w+31) and write either FP32 split-K partials or the final FP64
// complex result. Every mbarrier wait is bounded; a wait that runs out sets a
// device error word and the CTA winds down (the host turns it into an error).
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <string>

#include <map>
#include <tuple>
#include <vector>
#include "umma_gemm.cuh"

namespace sdft_b200 {

namespace {

constexpr int BM = 128, BK = 64, kThreads = 128;
constexpr unsigned long long kWaitLimitNs = 2000000000ULL;  // 2 s per wait

__device__ unsigned int g_umma_error = 0;

__device__ __forceinline__ std::uint32_t smem_u32(const void* p) {
  return static_cast<std::uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(std::uint64_t* bar, std::uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(std::uint64_t* bar, std::uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(std::uint64_t* bar, std::uint32_t parity) {
  std::uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false (and the error word set) when the phase does not
// complete within the limit or another thread already gave up.
__device__ bool mbar_wait(std::uint64_t* bar, std::uint32_t parity) {
  const unsigned long long start = globaltimer();
  for (std::uint32_t spin = 0;; ++spin) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((spin & 255u) == 255u) {
      if (*reinterpret_cast<volatile unsigned int*>(&g_umma_error) != 0u) return false;
      if (globaltimer() - start > kWaitLimitNs) {
        atomicExch(&g_umma_error, 1u);
        return false;
      }
    }
  }
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, std::uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<std::uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void umma_bf16(std::uint32_t d_tmem, std::uint64_t adesc, std::uint64_t bdesc,
                                          std::uint32_t idesc, std::uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\ttcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(
          d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void umma_commit(std::uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// K-major, 128-byte swizzle shared-memory matrix descriptor (rows of 128 B,
// 8-row atoms 1024 B apart): start>>4, LBO 1, SBO 64 (x16 B), version 1, SWIZZLE_128B.
__device__ __forceinline__ std::uint64_t smem_desc(std::uint32_t addr) {
  return (static_cast<std::uint64_t>((addr >> 4) & 0x3FFFu)) | (1ULL << 16) | (64ULL << 32) | (1ULL << 46) |
         (2ULL << 61);
}

template <int BN>
__host__ __device__ constexpr std::uint32_t instr_desc() {
  // D=F32 (bits 4-5 = 1), A=B=BF16 (bits 7-9 = 1, 10-12 = 1), K-major both, N>>3 at 17, M>>4 at 24.
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<std::uint32_t>(BN >> 3) << 17) |
         (static_cast<std::uint32_t>(BM >> 4) << 24);
}

template <int BN>
__host__ __device__ constexpr int stages() {
  return BN >= 256 ? 4 : 6;
}

struct EpilogueArgs {
  int m, n2;                   // rows, real columns (2 x complex columns)
  Cx<float>* partial;          // split-K output [split][n2/2][m] or null
  Cx<double>* c;               // direct output (when partial is null)
  long long ldc;
  double alpha;
  int add;
};

template <int BN>
__global__ void __launch_bounds__(kThreads, 1)
    umma_gemm_kernel(const __grid_constant__ CUtensorMap map_a, const __grid_constant__ CUtensorMap map_b,
                     int k_blocks_total, int k_blocks_per_split, EpilogueArgs ep) {
  constexpr int S = stages<BN>();
  constexpr int A_BYTES = BM * BK * 2, B_BYTES = BN * BK * 2, STAGE = A_BYTES + B_BYTES;
  constexpr std::uint32_t TMEM_COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* smem = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<std::uintptr_t>(smem_raw) + 1023) & ~static_cast<std::uintptr_t>(1023));
  std::uint64_t* full = reinterpret_cast<std::uint64_t*>(smem + S * STAGE);
  std::uint64_t* empty = full + S;
  std::uint64_t* accum = empty + S;
  std::uint32_t* tmem_holder = reinterpret_cast<std::uint32_t*>(accum + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Column tiles run fastest, so the CTAs sharing an A tile are resident
  // together and all but the first read it from L2.
  const int tile_n = blockIdx.x * BN, tile_m = blockIdx.y * BM;
  const int kb0 = blockIdx.z * k_blocks_per_split;
  const int nkb = max(0, min(k_blocks_total, kb0 + k_blocks_per_split) - kb0);

  if (threadIdx.x == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accum, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_holder)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const std::uint32_t tmem = *tmem_holder;

  int issued = 0;
  if (warp == 0 && lane == 0) {
    // TMA producer
    for (int i = 0; i < nkb; ++i) {
      const int s = i % S;
      if (i >= S && !mbar_wait(&empty[s], ((i / S) - 1) & 1)) break;
      mbar_arrive_expect_tx(&full[s], STAGE);
      const int kc = (kb0 + i) * BK;
      tma_load_2d(smem + s * STAGE, &map_a, kc, tile_m, &full[s]);
      tma_load_2d(smem + s * STAGE + A_BYTES, &map_b, kc, tile_n, &full[s]);
      issued = i + 1;
    }
  } else if (warp == 1 && lane == 0) {
    // tcgen05.mma issuer
    constexpr std::uint32_t idesc = instr_desc<BN>();
    for (int i = 0; i < nkb; ++i) {
      const int s = i % S;
      if (!mbar_wait(&full[s], (i / S) & 1)) break;
      tc_fence_after();
      const std::uint32_t a_addr = smem_u32(smem + s * STAGE), b_addr = a_addr + A_BYTES;
#pragma unroll
      for (int kk = 0; kk < BK / 16; ++kk)
        umma_bf16(tmem, smem_desc(a_addr + kk * 32), smem_desc(b_addr + kk * 32), idesc, (i | kk) != 0);
      umma_commit(&empty[s]);
    }
    umma_commit(accum);
  }
  __syncwarp();
  // Epilogue: warp w reads TMEM lanes 32w..32w+31 (tile rows).
  const bool have = __all_sync(0xffffffffu, nkb > 0 && mbar_wait(accum, 0));
  tc_fence_after();
  const int row = tile_m + warp * 32 + lane;
  const int n_complex_total = ep.n2 / 2;
  for (int c0 = 0; c0 < BN; c0 += 16) {
    // The chunk's earlier C values (accumulating products) are requested
    // before the accumulator read, all eight at once.
    Cx<double> prior[8];
    const bool accumulate = !ep.partial && ep.add && row < ep.m;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int j = (tile_n + c0) / 2 + q;
      prior[q] = (accumulate && j < n_complex_total) ? ep.c[row + static_cast<long long>(j) * ep.ldc]
                                                     : Cx<double>{0.0, 0.0};
    }
    std::uint32_t r[16];
    if (have) {
      const std::uint32_t taddr = tmem + (static_cast<std::uint32_t>(warp * 32) << 16) + static_cast<std::uint32_t>(c0);
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
            "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    } else {
#pragma unroll
      for (int q = 0; q < 16; ++q) r[q] = 0u;
    }
    if (row < ep.m) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int j = (tile_n + c0) / 2 + q;
        if (j >= n_complex_total) break;
        const float re = __uint_as_float(r[2 * q]), im = __uint_as_float(r[2 * q + 1]);
        if (ep.partial) {
          ep.partial[(static_cast<long long>(blockIdx.z) * n_complex_total + j) * ep.m + row] = Cx<float>{re, im};
        } else {
          double vr = ep.alpha * static_cast<double>(re), vi = ep.alpha * static_cast<double>(im);
          if (ep.add) {
            vr += prior[q].re;
            vi += prior[q].im;
          }
          ep.c[row + static_cast<long long>(j) * ep.ldc] = Cx<double>{vr, vi};
        }
      }
    }
  }
  // Wind-down: drain TMA copies still in flight on the error path, free TMEM.
  if (warp == 0 && lane == 0 && *reinterpret_cast<volatile unsigned int*>(&g_umma_error) != 0u) {
    for (int i = max(0, issued - S); i < issued; ++i) mbar_wait(&full[i % S], (i / S) & 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

// C = alpha * sum_s partial[s] (+ C): one thread per (row i = x, column j = y),
// the splits summed in order with two interleaved accumulators.
__global__ void reduce_splits_kernel(int m, int n, int splits, const Cx<float>* __restrict__ partial,
                                     Cx<double>* __restrict__ c, long long ldc, bool add, double alpha) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const long long total = static_cast<long long>(m) * n;
  for (int j = blockIdx.y; j < n; j += gridDim.y) {
    const Cx<float>* p = partial + static_cast<long long>(j) * m + i;
    double re0 = 0.0, im0 = 0.0, re1 = 0.0, im1 = 0.0;
    int s = 0;
    for (; s + 1 < splits; s += 2) {
      const Cx<float> a = p[s * total], b = p[(s + 1) * total];
      re0 += a.re;
      im0 += a.im;
      re1 += b.re;
      im1 += b.im;
    }
    if (s < splits) {
      const Cx<float> a = p[s * total];
      re0 += a.re;
      im0 += a.im;
    }
    double re = (re0 + re1) * alpha, im = (im0 + im1) * alpha;
    Cx<double>& out = c[i + static_cast<long long>(j) * ldc];
    if (add) {
      re += out.re;
      im += out.im;
    }
    out = Cx<double>{re, im};
  }
}

// ---- packing (FP64 complex -> BF16 split terms) ---------------------------

// Split-term index of product p on the A and B side: BF16x3 pairs (0,0) (0,1)
// (1,0); BF16x6 adds (0,2) (1,1) (2,0).
__host__ __device__ constexpr int term_a(int p) { return p == 2 || p == 4 ? 1 : p == 5 ? 2 : 0; }
__host__ __device__ constexpr int term_b(int p) { return p == 1 || p == 4 ? 1 : p == 3 ? 2 : 0; }

__device__ __forceinline__ void split3(double x, std::uint16_t t[3]) {
  const __nv_bfloat16 h0 = __double2bfloat16(x);
  const double r1 = x - static_cast<double>(__bfloat162float(h0));
  const __nv_bfloat16 h1 = __double2bfloat16(r1);
  const double r2 = r1 - static_cast<double>(__bfloat162float(h1));
  const __nv_bfloat16 h2 = __double2bfloat16(r2);
  t[0] = __bfloat16_as_ushort(h0);
  t[1] = __bfloat16_as_ushort(h1);
  t[2] = __bfloat16_as_ushort(h2);
}

// Stores P (lo, hi) uint16 pairs at dst with 8-byte stores when P is even
// (dst is then 8-byte aligned: rows are 128-byte aligned and each value
// takes 4P bytes), else 4-byte stores.
template <int P>
__device__ __forceinline__ void store_pairs(std::uint16_t* dst, const std::uint32_t (&pairs)[P]) {
  if constexpr (P % 2 == 0) {
    auto* d = reinterpret_cast<uint2*>(dst);
#pragma unroll
    for (int q = 0; q < P / 2; ++q) d[q] = make_uint2(pairs[2 * q], pairs[2 * q + 1]);
  } else {
    auto* d = reinterpret_cast<std::uint32_t*>(dst);
#pragma unroll
    for (int q = 0; q < P; ++q) d[q] = pairs[q];
  }
}

__device__ __forceinline__ std::uint32_t pair(std::uint16_t lo, std::uint16_t hi) {
  return static_cast<std::uint32_t>(lo) | (static_cast<std::uint32_t>(hi) << 16);
}

// Writes the 2P A-side entries of one complex value.
template <int P>
__device__ __forceinline__ void write_a(std::uint16_t* dst, Cx<double> v) {
  std::uint16_t re[3], im[3];
  split3(v.re, re);
  split3(v.im, im);
  std::uint32_t pairs[P];
#pragma unroll
  for (int p = 0; p < P; ++p) pairs[p] = pair(re[term_a(p)], im[term_a(p)]);
  store_pairs<P>(dst, pairs);
}

// One row i of A per blockIdx.y; threads stride over k.
template <int P, bool CONJ_T>
__global__ void pack_a_direct_kernel(const Cx<double>* __restrict__ src, long long lds, int rows, int k,
                                     std::uint16_t* __restrict__ out, long long ldo, long long kexp) {
  // CONJ_T: A[i,k] = conj(src[k + i*lds]) (k contiguous in the source).
  // Rows i = blockIdx.y, blockIdx.y + gridDim.y, ... (any row count).
  for (int i = blockIdx.y; i < rows; i += gridDim.y) {
    const Cx<double>* in = src + static_cast<long long>(i) * lds;
    std::uint16_t* row = out + static_cast<long long>(i) * ldo;
    for (int kk = blockIdx.x * blockDim.x + threadIdx.x; kk < k; kk += gridDim.x * blockDim.x) {
      Cx<double> v = in[kk];
      if (CONJ_T) v.im = -v.im;
      write_a<P>(row + static_cast<long long>(kk) * 2 * P, v);
    }
    // zero padding [2Pk, kexp) of the row
    for (long long q = 2LL * P * k + blockIdx.x * blockDim.x + threadIdx.x; q < kexp;
         q += static_cast<long long>(gridDim.x) * blockDim.x)
      row[q] = 0;
  }
}

// A[i,k] = src[i + k*lds] (rows contiguous): 32x32 shared-memory transpose.
template <int P>
__global__ void pack_a_transpose_kernel(const Cx<double>* __restrict__ src, long long lds, int rows, int k,
                                        std::uint16_t* __restrict__ out, long long ldo, long long out_k_offset) {
  __shared__ Cx<double> tile[32][33];
  const int i0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    const int i = i0 + tx, kk = k0 + r;
    tile[r][tx] = (i < rows && kk < k) ? src[i + static_cast<long long>(kk) * lds] : Cx<double>{0, 0};
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    const int i = i0 + r, kk = k0 + tx;
    if (i < rows && kk < k) write_a<P>(out + static_cast<long long>(i) * ldo + (out_k_offset + kk) * 2 * P, tile[tx][r]);
  }
}

template <int P>
__global__ void zero_pad_kernel(std::uint16_t* __restrict__ out, long long ldo, int rows, long long from, long long to) {
  const long long pad = to - from;
  const long long total = static_cast<long long>(rows) * pad;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x)
    out[(idx / pad) * ldo + from + idx % pad] = 0;
}

// Source columns j = blockIdx.y, blockIdx.y + gridDim.y, ... (two expanded
// rows each); threads stride over k.
template <int P>
__global__ void pack_b_kernel(const Cx<double>* __restrict__ src, long long ldb, int k, int n,
                              std::uint16_t* __restrict__ out, long long ldo, long long kexp) {
  for (int j = blockIdx.y; j < n; j += gridDim.y) {
    const Cx<double>* in = src + static_cast<long long>(j) * ldb;
    std::uint16_t* row0 = out + (2LL * j) * ldo;
    std::uint16_t* row1 = row0 + ldo;
    for (int kk = blockIdx.x * blockDim.x + threadIdx.x; kk < k; kk += gridDim.x * blockDim.x) {
      const Cx<double> v = in[kk];
      std::uint16_t re[3], im[3];
      split3(v.re, re);
      split3(v.im, im);
      std::uint32_t p0[P], p1[P];
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const int t = term_b(p);
        p0[p] = pair(re[t], im[t] ^ 0x8000u);  // [Re, -Im] (sign flip is exact)
        p1[p] = pair(im[t], re[t]);            // [Im, Re]
      }
      store_pairs<P>(row0 + static_cast<long long>(kk) * 2 * P, p0);
      store_pairs<P>(row1 + static_cast<long long>(kk) * 2 * P, p1);
    }
    for (long long q = 2LL * P * k + blockIdx.x * blockDim.x + threadIdx.x; q < kexp;
         q += static_cast<long long>(gridDim.x) * blockDim.x) {
      row0[q] = 0;
      row1[q] = 0;
    }
  }
}

// Largest gridDim.y; kernels that put rows or columns on y stride past it.
constexpr int kMaxGridY = 65535;

// Blocks along a row of `length` entries when `rows` rows run side by side:
// enough CTAs in total for ~16 per SM, at least one per row.
unsigned row_blocks(long long length, int rows) {
  const long long per_row = std::max<long long>(1, (148LL * 16 + rows - 1) / rows);
  return static_cast<unsigned>(std::max<long long>(1, std::min<long long>(per_row, (length + 255) / 256)));
}

unsigned grid_for(long long total) {
  return static_cast<unsigned>(std::min<long long>(std::max<long long>(1, (total + 255) / 256), 148LL * 16));
}

// ---- tensor maps -----------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult status;
    SDFT_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &status));
    if (status != cudaDriverEntryPointSuccess || !ptr) throw CudaError("cuTensorMapEncodeTiled is unavailable");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  });
  return fn;
}

CUtensorMap kmajor_map(const std::uint16_t* base, long long rows, long long kexp, long long ld, int box_rows) {
  if (reinterpret_cast<std::uintptr_t>(base) % 16 != 0 || (ld * 2) % 16 != 0)
    throw InvalidArgument("BF16 operand base and row stride must be 16-byte aligned");
  CUtensorMap map;
  const cuuint64_t dims[2] = {static_cast<cuuint64_t>(kexp), static_cast<cuuint64_t>(rows)};
  const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld * 2)};
  const cuuint32_t box[2] = {static_cast<cuuint32_t>(BK), static_cast<cuuint32_t>(box_rows)};
  const cuuint32_t element_strides[2] = {1, 1};
  const CUresult r = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<std::uint16_t*>(base), dims,
                                 strides, box, element_strides, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed: " + std::to_string(static_cast<int>(r)));
  return map;
}

template <int BN>
void launch(const std::uint16_t* a, long long lda, const std::uint16_t* b, long long ldb, int m, int n2,
            long long kexp, const EpilogueArgs& ep_in, int splits, int k_blocks, int kpb, cudaStream_t stream) {
  constexpr int S = stages<BN>();
  const std::size_t smem = static_cast<std::size_t>(S) * (BM * BK * 2 + BN * BK * 2) + 1024 + 256;
  allow_dynamic_smem(umma_gemm_kernel<BN>, smem);
  const CUtensorMap map_a = kmajor_map(a, m, kexp, lda, BM);
  const CUtensorMap map_b = kmajor_map(b, n2, kexp, ldb, BN);
  if (ceil_div(m, BM) > 65535) throw InvalidArgument("tensor-core GEMM has more than 65535 row tiles");
  const dim3 grid(static_cast<unsigned>(ceil_div(n2, BN)), static_cast<unsigned>(ceil_div(m, BM)), splits);
  umma_gemm_kernel<BN><<<grid, kThreads, smem, stream>>>(map_a, map_b, k_blocks, kpb, ep_in);
  SDFT_LAUNCH("umma_gemm_kernel");
}

}  // namespace

bool umma_available() {
  int device = 0, major = 0;
  if (cudaGetDevice(&device) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess) return false;
  return major == 10;
}

void pack_a(Op aop, const Cx<double>* src, long long lds, int rows, int k, Split split, std::uint16_t* out,
            long long ldo, cudaStream_t stream) {
  const long long kexp = expanded_k(k, split);
  if (aop == Op::C) {
    const dim3 grid(row_blocks(std::max<long long>(k, kexp - 2LL * split_terms(split) * k), rows),
                    static_cast<unsigned>(std::min(rows, kMaxGridY)));
    if (split == Split::BF16x3)
      pack_a_direct_kernel<3, true><<<grid, 256, 0, stream>>>(src, lds, rows, k, out, ldo, kexp);
    else
      pack_a_direct_kernel<6, true><<<grid, 256, 0, stream>>>(src, lds, rows, k, out, ldo, kexp);
    SDFT_LAUNCH("pack_a_direct_kernel");
    return;
  }
  const dim3 grid(static_cast<unsigned>(ceil_div(rows, 32)), static_cast<unsigned>(ceil_div(k, 32)));
  if (split == Split::BF16x3)
    pack_a_transpose_kernel<3><<<grid, dim3(32, 8), 0, stream>>>(src, lds, rows, k, out, ldo, 0);
  else
    pack_a_transpose_kernel<6><<<grid, dim3(32, 8), 0, stream>>>(src, lds, rows, k, out, ldo, 0);
  SDFT_LAUNCH("pack_a_transpose_kernel");
  const long long from = 2LL * split_terms(split) * k;
  if (kexp > from) {
    zero_pad_kernel<3><<<grid_for(static_cast<long long>(rows) * (kexp - from)), 256, 0, stream>>>(out, ldo, rows,
                                                                                                  from, kexp);
    SDFT_LAUNCH("zero_pad_kernel");
  }
}

void pack_a_columns(const Cx<double>* src, long long lds, int rows, int first, int count, Split split,
                    std::uint16_t* out, long long ldo, cudaStream_t stream) {
  if (count <= 0) return;
  const dim3 grid(static_cast<unsigned>(ceil_div(rows, 32)), static_cast<unsigned>(ceil_div(count, 32)));
  const Cx<double>* s = src + static_cast<long long>(first) * lds;
  if (split == Split::BF16x3)
    pack_a_transpose_kernel<3><<<grid, dim3(32, 8), 0, stream>>>(s, lds, rows, count, out, ldo, first);
  else
    pack_a_transpose_kernel<6><<<grid, dim3(32, 8), 0, stream>>>(s, lds, rows, count, out, ldo, first);
  SDFT_LAUNCH("pack_a_transpose_kernel");
}

void pack_b(const Cx<double>* src, long long ldb, int k, int n, Split split, std::uint16_t* out, long long ldo,
            cudaStream_t stream) {
  const long long kexp = expanded_k(k, split);
  const dim3 grid(row_blocks(std::max<long long>(k, kexp - 2LL * split_terms(split) * k), n),
                  static_cast<unsigned>(std::min(n, kMaxGridY)));
  if (split == Split::BF16x3) pack_b_kernel<3><<<grid, 256, 0, stream>>>(src, ldb, k, n, out, ldo, kexp);
  else pack_b_kernel<6><<<grid, 256, 0, stream>>>(src, ldb, k, n, out, ldo, kexp);
  SDFT_LAUNCH("pack_b_kernel");
}

namespace {

// Column tile width of the cost model: the one of 128 / 160 / 256 that pads
// the 2n real columns least (the larger on ties).
int model_width(int n2) {
  int bn = 256;
  long long padded = ceil_div(n2, 256) * 256LL;
  for (int w : {160, 128}) {
    const long long p = ceil_div(n2, w) * static_cast<long long>(w);
    if (p < padded) {
      padded = p;
      bn = w;
    }
  }
  return bn;
}

int max_splits_for(int k_blocks) { return static_cast<int>(std::min<long long>(128, std::max(1, k_blocks / 8))); }

// Split-K count of the cost model for width bn: one CTA per SM is resident
// (the ring takes ~200 KB), so the time goes as waves x K blocks per CTA, plus
// the FP32 partials that a split writes and the reduction reads, counted in K
// blocks' worth of operand traffic spread over the SMs; the smallest split on
// ties, at least 8 K blocks per split.
int model_splits(int m, int n2, int k_blocks, int bn) {
  const long long tiles = static_cast<long long>(ceil_div(m, BM)) * static_cast<long long>(ceil_div(n2, bn));
  const double kblock_bytes = static_cast<double>(BM + bn) * BK * 2;
  double best_cost = -1;
  int splits = 1;
  for (long long s = 1; s <= max_splits_for(k_blocks); ++s) {
    const long long waves = (tiles * s + 147) / 148;
    const double partial = s > 1 ? 2.0 * 4.0 * static_cast<double>(m) * n2 * s / (148.0 * kblock_bytes) : 0.0;
    const double cost = static_cast<double>(waves * ((k_blocks + s - 1) / s)) + partial;
    if (best_cost < 0 || cost < best_cost) {
      best_cost = cost;
      splits = static_cast<int>(s);
    }
  }
  return splits;
}

// One product with the given tile width and split count.
void run_config(const std::uint16_t* a, long long lda, const std::uint16_t* b, long long ldb, int m, int n,
                long long kexp, Cx<double>* c, long long ldc, bool add, double alpha, int bn, int splits,
                Scratch& workspace, cudaStream_t stream) {
  const int n2 = 2 * n;
  const int k_blocks = static_cast<int>(kexp / BK);
  const int kpb = static_cast<int>(ceil_div(k_blocks, splits));
  splits = static_cast<int>(ceil_div(k_blocks, kpb));
  EpilogueArgs ep{m, n2, nullptr, c, ldc, alpha, add ? 1 : 0};
  if (splits > 1)
    ep.partial = static_cast<Cx<float>*>(workspace.reserve(sizeof(Cx<float>) * static_cast<std::size_t>(m) * n * splits));
  if (bn == 256) launch<256>(a, lda, b, ldb, m, n2, kexp, ep, splits, k_blocks, kpb, stream);
  else if (bn == 160) launch<160>(a, lda, b, ldb, m, n2, kexp, ep, splits, k_blocks, kpb, stream);
  else launch<128>(a, lda, b, ldb, m, n2, kexp, ep, splits, k_blocks, kpb, stream);
  if (splits > 1) {
    reduce_splits_kernel<<<dim3(static_cast<unsigned>(ceil_div(m, 256)), static_cast<unsigned>(std::min(n, kMaxGridY))),
                           256, 0, stream>>>(
        m, n, splits, ep.partial, c, ldc, add, alpha);
    SDFT_LAUNCH("reduce_splits_kernel");
  }
}

// Tile autotuner. Shapes are grouped into classes (row tiles of 128, real
// column count rounded up to 32, K blocks rounded up to a geometric grid of
// ratio 2^(1/8), so that operators whose plane-wave counts differ by a few
// per cent share their classes); the first product of a class times every
// candidate -- the three column widths, each with the cost model's split
// count and twice it, and no split -- on the caller's
// stream into a scratch output (CUDA events, one untimed run first) and keeps
// the fastest for the class, for the life of the process. Later products of
// the class, on any stream or thread, use that choice, so a given process
// computes every later product of a class with the same tiles and the same
// summation order. SDFT_B200_GEMM_AUTOTUNE=0 uses the cost model alone.
struct ShapeClass {
  int row_tiles, column_units, k_blocks;
  bool operator<(const ShapeClass& o) const {
    return std::tie(row_tiles, column_units, k_blocks) < std::tie(o.row_tiles, o.column_units, o.k_blocks);
  }
};
struct TileChoice {
  int bn, splits;
  float ms;
};
std::mutex g_tune_mutex;
std::map<ShapeClass, TileChoice> g_tuned;

bool autotune_enabled() {
  static const bool enabled = [] {
    const char* v = std::getenv("SDFT_B200_GEMM_AUTOTUNE");
    if (!v || std::string(v) == "1") return true;
    if (std::string(v) == "0") return false;
    throw InvalidArgument("SDFT_B200_GEMM_AUTOTUNE must be 0 or 1");
  }();
  return enabled;
}

TileChoice tuned_choice(const std::uint16_t* a, long long lda, const std::uint16_t* b, long long ldb, int m, int n,
                        long long kexp, Scratch& workspace, cudaStream_t stream) {
  const int n2 = 2 * n;
  const int k_blocks = static_cast<int>(kexp / BK);
  int k_class = 1;
  for (int j = 1; k_class < k_blocks; ++j) k_class = static_cast<int>(std::ceil(std::exp2(j / 8.0)));
  const ShapeClass key{static_cast<int>(ceil_div(m, BM)), static_cast<int>(ceil_div(n2, 32)), k_class};
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  auto found = g_tuned.find(key);
  if (found != g_tuned.end()) return found->second;
  std::vector<std::pair<int, int>> candidates;
  for (int bn : {128, 160, 256}) {
    const int s = model_splits(m, n2, k_blocks, bn);
    for (int split : {1, s, std::min(max_splits_for(k_blocks), 2 * s)})
      if (std::find(candidates.begin(), candidates.end(), std::make_pair(bn, split)) == candidates.end())
        candidates.emplace_back(bn, split);
  }
  static thread_local Scratch output, partials;
  auto* c = static_cast<Cx<double>*>(output.reserve(sizeof(Cx<double>) * static_cast<std::size_t>(m) * n));
  cudaEvent_t start = nullptr, stop = nullptr;
  SDFT_CUDA(cudaEventCreate(&start));
  SDFT_CUDA(cudaEventCreate(&stop));
  TileChoice best{model_width(n2), 0, -1.0f};
  best.splits = model_splits(m, n2, k_blocks, best.bn);
  try {
    for (const auto& [bn, splits] : candidates) {
      run_config(a, lda, b, ldb, m, n, kexp, c, m, false, 1.0, bn, splits, partials, stream);
      SDFT_CUDA(cudaEventRecord(start, stream));
      run_config(a, lda, b, ldb, m, n, kexp, c, m, false, 1.0, bn, splits, partials, stream);
      SDFT_CUDA(cudaEventRecord(stop, stream));
      SDFT_CUDA(cudaEventSynchronize(stop));
      float ms = 0;
      SDFT_CUDA(cudaEventElapsedTime(&ms, start, stop));
      if (best.ms < 0 || ms < best.ms) best = TileChoice{bn, splits, ms};
    }
  } catch (...) {
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
    throw;
  }
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  g_tuned.emplace(key, best);
  return best;
}

}  // namespace

void umma_complex_gemm(const std::uint16_t* a, long long lda, const std::uint16_t* b, long long ldb, int m, int n,
                       long long kexp, Cx<double>* c, long long ldc, bool add, double alpha, Scratch& workspace,
                       cudaStream_t stream) {
  if (m <= 0 || n <= 0 || kexp <= 0) return;
  if (kexp % BK != 0) throw InvalidArgument("expanded K must be a multiple of 64");
  int bn, splits;
  if (autotune_enabled()) {
    const TileChoice choice = tuned_choice(a, lda, b, ldb, m, n, kexp, workspace, stream);
    bn = choice.bn;
    splits = choice.splits;
  } else {
    bn = model_width(2 * n);
    splits = model_splits(m, 2 * n, static_cast<int>(kexp / BK), bn);
  }
  run_config(a, lda, b, ldb, m, n, kexp, c, ldc, add, alpha, bn, splits, workspace, stream);
}

std::size_t gemm_tuned_classes(std::size_t capacity, int* rows) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  std::size_t i = 0;
  for (const auto& [key, choice] : g_tuned) {
    if (i < capacity && rows) {
      int* r = rows + 5 * i;
      r[0] = key.row_tiles * BM;
      r[1] = key.column_units * 32;
      r[2] = key.k_blocks;
      r[3] = choice.bn;
      r[4] = choice.splits;
    }
    ++i;
  }
  return g_tuned.size();
}

Split search_split() {
  static const Split split = [] {
    const char* v = std::getenv("SDFT_B200_SPLIT");
    if (!v || std::string(v) == "x3") return Split::BF16x3;
    if (std::string(v) == "x6") return Split::BF16x6;
    throw InvalidArgument("SDFT_B200_SPLIT must be x3 or x6");
  }();
  return split;
}

void pack_persistent(Op aop, const Cx<double>* a, long long lda, int rows, int k, Split split, PackedA& out,
                     cudaStream_t stream) {
  release(out);
  out.ld = expanded_k(k, split);
  out.rows = rows;
  out.k = k;
  out.split = split;
  out.stream = stream;
  out.data = static_cast<std::uint16_t*>(
      stream_alloc(sizeof(std::uint16_t) * static_cast<std::size_t>(out.ld) * rows, stream));
  pack_a(aop, a, lda, rows, k, split, out.data, out.ld, stream);
}

void release(PackedA& packed) {
  stream_free(packed.data, packed.stream);
  packed = PackedA{};
}

void gemm_tc(Op aop, int m, int n, int k, const Cx<double>* a, long long lda, const PackedA* packed,
             const Cx<double>* b, long long ldb, Cx<double>* c, long long ldc, bool add, double alpha, Split split,
             TensorCoreWorkspace& ws, cudaStream_t stream) {
  if (m <= 0 || n <= 0 || k <= 0) return;
  const long long kexp = expanded_k(k, split);
  const std::uint16_t* pa;
  long long lda_p;
  if (packed) {
    if (packed->rows != m || packed->k != k || packed->split != split) throw InvalidArgument("packed operand shape mismatch");
    pa = packed->data;
    lda_p = packed->ld;
  } else {
    auto* buf = static_cast<std::uint16_t*>(ws.a.reserve(sizeof(std::uint16_t) * static_cast<std::size_t>(kexp) * m));
    pack_a(aop, a, lda, m, k, split, buf, kexp, stream);
    pa = buf;
    lda_p = kexp;
  }
  auto* pb = static_cast<std::uint16_t*>(ws.b.reserve(sizeof(std::uint16_t) * static_cast<std::size_t>(kexp) * 2 * n));
  pack_b(b, ldb, k, n, split, pb, kexp, stream);
  umma_complex_gemm(pa, lda_p, pb, kexp, m, n, kexp, c, ldc, add, alpha, ws.partial, stream);
}

unsigned int umma_error_flag() {
  unsigned int value = 0;
  SDFT_CUDA(cudaMemcpyFromSymbol(&value, g_umma_error, sizeof(value)));
  return value;
}

}  // namespace sdft_b200
