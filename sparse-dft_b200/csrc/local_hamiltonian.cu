// Fused local Hamiltonian (the reference's FFT loop, src/plane_wave_operator.cpp:237-257,
// and the CUDA scatter/cuFFT/multiply/cuFFT/gather chain, src/compute_cuda.cu:141-177)
// as three hand-written passes over a pruned slab:
//
//   plane_in   (one CTA per active grid row i0 and column): scatter the sphere
//              points of that plane into shared memory, backward FFT along
//              i2 on the active i1 rows, backward FFT along i1 on every i2
//              column, store the plane to the slab.
//   pencil     (one CTA per 32 (i1,i2) lines and column): load the active i0
//              entries, zero-pad to n0, backward FFT along i0, multiply by
//              V(r), forward FFT, store back only the active i0 entries.
//   plane_out  (per active i0 and column): forward FFT along i1 and i2, gather
//              the sphere points, y = T x + value/N.
//
// Rows i0 outside the sphere's span never reach HBM: the slab holds
// slots*n1*n2 complex values per column instead of n0*n1*n2.
#include <algorithm>
#include <cstring>
#include <limits>
#include <set>
#include <type_traits>

#include "local_hamiltonian.cuh"

namespace sdft_b200 {

namespace {

constexpr int kThreads = 256;
constexpr int kPencilLines = 32;
// Resident CTAs per SM the fixed plane and pencil kernels are compiled for:
// four in FP32 (64 registers; at N = 70 plane_out spills 144 B and still
// runs faster than at three CTAs: the passes are latency-bound), one in FP64,
// whose butterfly registers would spill under a tighter bound.
template <typename T>
constexpr int plane_blocks() {
  return sizeof(T) == 4 ? 4 : 1;
}

template <typename T>
struct LocalArgs {
  int n0, n1, n2, n2p, slots, krows;
  long long n12;
  const int* slot_row;
  const int* point_offset;
  const int* point_g;
  const int* point_smem;
  const int* krow;
  LinePlan p0, p1, p2;
  const Cx<T>* tw0;
  const Cx<T>* tw1;
  const Cx<T>* tw2;
};

template <typename T>
__global__ void __launch_bounds__(kThreads) plane_in_kernel(const Cx<double>* __restrict__ x, long long ldx,
                                                            LocalArgs<T> a, Cx<T>* __restrict__ slab) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* tw1 = reinterpret_cast<Cx<T>*>(smem_raw);
  Cx<T>* tw2 = tw1 + a.n1;
  const int plane_elems = a.n1 * a.n2p;
  Cx<T>* plane_a = tw2 + a.n2;
  Cx<T>* plane_b = plane_a + plane_elems;
  const int s = blockIdx.x, c = blockIdx.y;
  const int tid = threadIdx.x;
  for (int i = tid; i < a.n1; i += blockDim.x) tw1[i] = a.tw1[i];
  for (int i = tid; i < a.n2; i += blockDim.x) tw2[i] = a.tw2[i];
  for (int i = tid; i < 2 * plane_elems; i += blockDim.x) plane_a[i] = Cx<T>{0, 0};
  __syncthreads();
  const Cx<double>* xc = x + static_cast<long long>(c) * ldx;
  const int p_end = a.point_offset[s + 1];
  for (int p = a.point_offset[s] + tid; p < p_end; p += blockDim.x)
    plane_a[a.point_smem[p]] = cconvert<T>(xc[a.point_g[p]]);
  __syncthreads();
  // i2 along the active i1 rows, then i1 along every i2 column (rows outside
  // the active set stay zero in both buffers).
  Cx<T>* rows_done = fft_lines_pp<T, true>(plane_a, plane_b, a.krows, a.n2p, 1, a.krow, a.p2, tw2);
  Cx<T>* other = rows_done == plane_a ? plane_b : plane_a;
  Cx<T>* done = fft_lines_pp<T, true>(rows_done, other, a.n2, 1, a.n2p, nullptr, a.p1, tw1);
  Cx<T>* out = slab + (static_cast<long long>(c) * a.slots + s) * a.n12;
  for (int i = tid; i < a.n12; i += blockDim.x) {
    const int i1 = i / a.n2, i2 = i - i1 * a.n2;
    out[i] = done[i1 * a.n2p + i2];
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) pencil_kernel(Cx<T>* __restrict__ slab, LocalArgs<T> a,
                                                          const T* __restrict__ potential) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int TL = kPencilLines, STRIDE = TL + 1;
  Cx<T>* tw0 = reinterpret_cast<Cx<T>*>(smem_raw);
  Cx<T>* tile_a = tw0 + a.n0;
  Cx<T>* tile_b = tile_a + a.n0 * STRIDE;
  const long long kl0 = static_cast<long long>(blockIdx.x) * TL;
  const int c = blockIdx.y;
  const int lines = static_cast<int>(min(static_cast<long long>(TL), a.n12 - kl0));
  const int tid = threadIdx.x;
  for (int i = tid; i < a.n0; i += blockDim.x) tw0[i] = a.tw0[i];
  for (int i = tid; i < a.n0 * STRIDE; i += blockDim.x) tile_a[i] = Cx<T>{0, 0};
  __syncthreads();
  Cx<T>* base = slab + static_cast<long long>(c) * a.slots * a.n12 + kl0;
  for (int idx = tid; idx < a.slots * TL; idx += blockDim.x) {
    const int s = idx / TL, t = idx - s * TL;
    if (t < lines) tile_a[a.slot_row[s] * STRIDE + t] = base[static_cast<long long>(s) * a.n12 + t];
  }
  __syncthreads();
  Cx<T>* field = fft_lines_pp<T, true>(tile_a, tile_b, lines, 1, STRIDE, nullptr, a.p0, tw0);
  for (int idx = tid; idx < a.n0 * TL; idx += blockDim.x) {
    const int i = idx / TL, t = idx - i * TL;
    if (t < lines) {
      const T v = potential[static_cast<long long>(i) * a.n12 + kl0 + t];
      field[i * STRIDE + t] = cscale(field[i * STRIDE + t], v);
    }
  }
  __syncthreads();
  Cx<T>* back = fft_lines_pp<T, false>(field, field == tile_a ? tile_b : tile_a, lines, 1, STRIDE, nullptr, a.p0, tw0);
  for (int idx = tid; idx < a.slots * TL; idx += blockDim.x) {
    const int s = idx / TL, t = idx - s * TL;
    if (t < lines) base[static_cast<long long>(s) * a.n12 + t] = back[a.slot_row[s] * STRIDE + t];
  }
}

// pencil_kernel for a compile-time axis length N0: every entry of the tile is
// written once (slab value or zero), and the stages unroll with constant
// index arithmetic.
template <typename T, int N0>
__global__ void __launch_bounds__(kThreads, plane_blocks<T>()) pencil_fixed_kernel(Cx<T>* __restrict__ slab, LocalArgs<T> a,
                                                                const T* __restrict__ potential) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int TL = kPencilLines, STRIDE = TL + 1;
  Cx<T>* tw0 = reinterpret_cast<Cx<T>*>(smem_raw);
  Cx<T>* tile_a = tw0 + N0;
  Cx<T>* tile_b = tile_a + N0 * STRIDE;
  int* slot_of_row = reinterpret_cast<int*>(tile_b + N0 * STRIDE);
  const long long kl0 = static_cast<long long>(blockIdx.x) * TL;
  const int c = blockIdx.y;
  const int lines = static_cast<int>(min(static_cast<long long>(TL), a.n12 - kl0));
  const int tid = threadIdx.x;
  for (int i = tid; i < N0; i += kThreads) {
    tw0[i] = a.tw0[i];
    slot_of_row[i] = -1;
  }
  __syncthreads();
  for (int s = tid; s < a.slots; s += kThreads) slot_of_row[a.slot_row[s]] = s;
  __syncthreads();
  Cx<T>* base = slab + static_cast<long long>(c) * a.slots * a.n12 + kl0;
  // All of the thread's slab entries and V(r) values are loaded before the
  // first transform, so the loads are in flight together.
  constexpr int PER = (N0 * TL + kThreads - 1) / kThreads;
  Cx<T> entry[PER];
  T pot[PER];
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int idx = tid + q * kThreads;
    const int i = idx / TL, t = idx - i * TL;
    entry[q] = Cx<T>{0, 0};
    pot[q] = T(0);
    if (idx < N0 * TL && t < lines) {
      const int s = slot_of_row[i];
      if (s >= 0) entry[q] = base[static_cast<long long>(s) * a.n12 + t];
      pot[q] = potential[static_cast<long long>(i) * a.n12 + kl0 + t];
    }
  }
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int idx = tid + q * kThreads;
    if (idx < N0 * TL) tile_a[(idx / TL) * STRIDE + idx % TL] = entry[q];
  }
  __syncthreads();
  Cx<T>* field = fft_lines_fixed<T, true, N0, TL, kThreads>(tile_a, tile_b, 1, STRIDE, tw0);
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int idx = tid + q * kThreads;
    const int i = idx / TL, t = idx - i * TL;
    if (idx < N0 * TL && t < lines) field[i * STRIDE + t] = cscale(field[i * STRIDE + t], pot[q]);
  }
  __syncthreads();
  Cx<T>* back = fft_lines_fixed<T, false, N0, TL, kThreads>(field, field == tile_a ? tile_b : tile_a, 1, STRIDE, tw0);
  for (int idx = tid; idx < a.slots * TL; idx += kThreads) {
    const int s = idx / TL, t = idx - s * TL;
    if (t < lines) base[static_cast<long long>(s) * a.n12 + t] = back[a.slot_row[s] * STRIDE + t];
  }
}

// FP32 pencil pass with one thread per (i1, i2) line: the line's n0 values
// live in registers through both transforms (fft_line_registers), so no
// transform stage touches shared memory. The kernel is persistent: CTA k
// walks a contiguous range of units (block of 128 lines, column), column
// fastest. While a unit's transforms run, cp.async stages the next unit's
// slab rows into the other half of a double buffer, and V(r) of the line
// block is staged once per block (it is the same for every column), so no
// global load sits between the transforms. Thread t copies, reads and writes
// only line t of each staged row, so the pass needs no CTA barrier. The
// twiddles and the row -> slot map are kernel parameters.
constexpr int kRegisterPencilThreads = 128;

template <int N0>
struct PencilRegisterArgs {
  RegTwiddles<float, N0> tw;
  int slot_of_row[N0];  // slab slot of grid row i0, or -1 (row outside the sphere's span)
};

template <int BYTES>
__device__ __forceinline__ void copy_async(void* smem, const void* gmem) {
  const unsigned dst = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(dst), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void copy_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// Waits until at most one committed group of this thread is still pending.
__device__ __forceinline__ void copy_async_wait_all_but_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int N0>
__global__ void __launch_bounds__(kRegisterPencilThreads) pencil_registers_kernel(
    Cx<float>* __restrict__ slab, long long n12, int slots, int columns, long long units,
    const float* __restrict__ potential, const __grid_constant__ PencilRegisterArgs<N0> p) {
  constexpr int TL = kRegisterPencilThreads;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<float>* staged = reinterpret_cast<Cx<float>*>(smem_raw);     // [2][slots][TL]
  float* staged_v = reinterpret_cast<float*>(staged + 2 * slots * TL);  // [N0][TL]
  const int t = threadIdx.x;
  const long long begin = units * blockIdx.x / gridDim.x, end = units * (blockIdx.x + 1) / gridDim.x;
  auto stage_slab = [&](long long u) {
    const long long kl0 = (u / columns) * TL;
    const int c = static_cast<int>(u % columns);
    if (kl0 + t < n12) {
      const Cx<float>* src = slab + static_cast<long long>(c) * slots * n12 + kl0 + t;
      Cx<float>* dst = staged + (u & 1) * slots * TL + t;
      for (int s = 0; s < slots; ++s) copy_async<8>(dst + s * TL, src + s * n12);
    }
  };
  if (begin < end) stage_slab(begin);
  copy_async_commit();
  long long block = -1;
  for (long long u = begin; u < end; ++u) {
    const long long b = u / columns;
    const long long kl = b * TL + t;
    const bool live = kl < n12;
    if (b != block) {  // V(r) of the new line block
      block = b;
      if (live)
        for (int i = 0; i < N0; ++i) copy_async<4>(staged_v + i * TL + t, potential + i * n12 + kl);
      copy_async_commit();
    }
    if (u + 1 < end) stage_slab(u + 1);
    copy_async_commit();
    copy_async_wait_all_but_one();  // unit u's slab rows and the block's V(r) have landed
    const Cx<float>* mine = staged + (u & 1) * slots * TL + t;
    Cx<float> v[N0];
#pragma unroll
    for (int i = 0; i < N0; ++i) {
      const int s = p.slot_of_row[i];
      v[i] = s >= 0 ? mine[s * TL] : Cx<float>{0.0f, 0.0f};
    }
    fft_line_registers<float, true, N0>(v, p.tw.w);
#pragma unroll
    for (int i = 0; i < N0; ++i) v[i] = cscale(v[i], staged_v[i * TL + t]);
    fft_line_registers<float, false, N0>(v, p.tw.w);
    if (live) {
      Cx<float>* out = slab + static_cast<long long>(u % columns) * slots * n12 + kl;
#pragma unroll
      for (int i = 0; i < N0; ++i) {
        const int s = p.slot_of_row[i];
        if (s >= 0) out[s * n12] = v[i];
      }
    }
  }
}

// The same persistent pencil pass with pair-split lines (fft_pair_dif /
// fft_pair_dit) for even n0: lane pair (l, l ^ 16) of warp w holds line
// 16 w + (l & 15), the lower lane grid rows [0, n0/2), the upper one
// [n0/2, n0); V(r) multiplies the interleaved spectrum (lower rows 2m,
// upper 2m + 1). Half the registers of the one-thread form, so twice the
// resident warps. Each lane stages, reads and writes only its own rows of
// its own line: no CTA barrier.
constexpr int kPairPencilThreads = 128;
constexpr int kPairPencilLines = kPairPencilThreads / 2;
constexpr int kPairPencilBlocks = 2;  // resident CTAs per SM: up to 255 registers a thread, no spills
// Longest line the one-thread pencil holds in registers without spilling;
// longer (even) lines take the pair form.
constexpr int kRegisterPencilMax = 72;

template <int N0>
struct PencilPairArgs {
  RegTwiddles<float, N0> tw;
  RegTwiddles<float, N0 / 2> tw_half;
  int slot_of_row[N0];  // slab slot of grid row i0, or -1
};

template <int N0>
__global__ void __launch_bounds__(kPairPencilThreads, kPairPencilBlocks) pencil_pair_kernel(
    Cx<float>* __restrict__ slab, long long n12, int slots, int columns, long long units,
    const float* __restrict__ potential, const __grid_constant__ PencilPairArgs<N0> p) {
  constexpr int H = N0 / 2, TL = kPairPencilLines;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<float>* staged = reinterpret_cast<Cx<float>*>(smem_raw);           // [2][slots][TL]
  float* staged_v = reinterpret_cast<float*>(staged + 2 * slots * TL);  // [N0][TL]
  const int lane = threadIdx.x & (kWarp - 1);
  const bool upper = lane >= kPairXor;
  const int t = (threadIdx.x >> 5) * kPairXor + (lane & (kPairXor - 1));
  const int h = upper ? H : 0, odd = upper ? 1 : 0;
  const long long begin = units * blockIdx.x / gridDim.x, end = units * (blockIdx.x + 1) / gridDim.x;
  auto stage_slab = [&](long long u) {
    const long long kl0 = (u / columns) * TL;
    const int c = static_cast<int>(u % columns);
    if (kl0 + t < n12) {
      const Cx<float>* src = slab + static_cast<long long>(c) * slots * n12 + kl0 + t;
      Cx<float>* dst = staged + (u & 1) * slots * TL + t;
      for (int j = 0; j < H; ++j) {
        const int s = p.slot_of_row[j + h];
        if (s >= 0) copy_async<8>(dst + s * TL, src + s * n12);
      }
    }
  };
  if (begin < end) stage_slab(begin);
  copy_async_commit();
  long long block = -1;
  for (long long u = begin; u < end; ++u) {
    const long long b = u / columns;
    const long long kl = b * TL + t;
    const bool live = kl < n12;
    if (b != block) {  // V(r) rows 2m + odd of the new line block
      block = b;
      if (live)
        for (int m = 0; m < H; ++m)
          copy_async<4>(staged_v + (2 * m + odd) * TL + t, potential + (2 * m + odd) * n12 + kl);
      copy_async_commit();
    }
    if (u + 1 < end) stage_slab(u + 1);
    copy_async_commit();
    copy_async_wait_all_but_one();
    const Cx<float>* mine = staged + (u & 1) * slots * TL + t;
    Cx<float> v[H];
#pragma unroll
    for (int j = 0; j < H; ++j) {
      const int s = upper ? p.slot_of_row[j + H] : p.slot_of_row[j];
      v[j] = s >= 0 ? mine[s * TL] : Cx<float>{0.0f, 0.0f};
    }
    fft_pair_dif<float, true, N0>(v, upper, p.tw.w, p.tw_half.w);
#pragma unroll
    for (int m = 0; m < H; ++m) v[m] = cscale(v[m], staged_v[(2 * m + odd) * TL + t]);
    fft_pair_dit<float, false, N0>(v, upper, p.tw.w, p.tw_half.w);
    if (live) {
      Cx<float>* out = slab + static_cast<long long>(u % columns) * slots * n12 + kl;
#pragma unroll
      for (int k = 0; k < H; ++k) {
        const int s = upper ? p.slot_of_row[k + H] : p.slot_of_row[k];
        if (s >= 0) out[s * n12] = v[k];
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) plane_out_kernel(const Cx<T>* __restrict__ slab, LocalArgs<T> a,
                                                             const Cx<double>* __restrict__ x, long long ldx,
                                                             const double* __restrict__ kinetic, double count,
                                                             Cx<double>* __restrict__ y, long long ldy) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* tw1 = reinterpret_cast<Cx<T>*>(smem_raw);
  Cx<T>* tw2 = tw1 + a.n1;
  const int plane_elems = a.n1 * a.n2p;
  Cx<T>* plane_a = tw2 + a.n2;
  Cx<T>* plane_b = plane_a + plane_elems;
  const int s = blockIdx.x, c = blockIdx.y;
  const int tid = threadIdx.x;
  for (int i = tid; i < a.n1; i += blockDim.x) tw1[i] = a.tw1[i];
  for (int i = tid; i < a.n2; i += blockDim.x) tw2[i] = a.tw2[i];
  const Cx<T>* in = slab + (static_cast<long long>(c) * a.slots + s) * a.n12;
  for (int i = tid; i < a.n12; i += blockDim.x) {
    const int i1 = i / a.n2, i2 = i - i1 * a.n2;
    plane_a[i1 * a.n2p + i2] = in[i];
  }
  __syncthreads();
  Cx<T>* cols_done = fft_lines_pp<T, false>(plane_a, plane_b, a.n2, 1, a.n2p, nullptr, a.p1, tw1);
  Cx<T>* done = fft_lines_pp<T, false>(cols_done, cols_done == plane_a ? plane_b : plane_a, a.krows, a.n2p, 1,
                                       a.krow, a.p2, tw2);
  const Cx<double>* xc = x + static_cast<long long>(c) * ldx;
  Cx<double>* yc = y + static_cast<long long>(c) * ldy;
  const int p_end = a.point_offset[s + 1];
  for (int p = a.point_offset[s] + tid; p < p_end; p += blockDim.x) {
    const int g = a.point_g[p];
    const Cx<double> v = cconvert<double>(done[a.point_smem[p]]);
    const Cx<double> in_g = xc[g];
    const double t = kinetic[g];
    yc[g] = Cx<double>{t * in_g.re + v.re / count, t * in_g.im + v.im / count};
  }
}

// Lines along a strided axis: element e of line i at base + e*stride + i.
// GENERAL plans may hold prime radices above 7 (general lengths).
template <typename T, bool INV, int TL, bool GENERAL>
__global__ void __launch_bounds__(kThreads) fft_strided_kernel(Cx<T>* __restrict__ data, int n, long long stride,
                                                               long long inner, long long outer_stride, LinePlan p,
                                                               const Cx<T>* __restrict__ tw_global) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int STRIDE = TL + 1;
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  Cx<T>* tile_a = tw + n;
  Cx<T>* tile_b = tile_a + n * STRIDE;
  const long long i0 = static_cast<long long>(blockIdx.x) * TL;
  const int lines = static_cast<int>(min(static_cast<long long>(TL), inner - i0));
  Cx<T>* base = data + static_cast<long long>(blockIdx.y) * outer_stride + i0;
  const int tid = threadIdx.x;
  for (int i = tid; i < n; i += blockDim.x) tw[i] = tw_global[i];
  for (int idx = tid; idx < n * TL; idx += blockDim.x) {
    const int e = idx / TL, t = idx - e * TL;
    if (t < lines) tile_a[e * STRIDE + t] = base[e * stride + t];
  }
  __syncthreads();
  const Cx<T>* done = GENERAL ? fft_lines_pp_general<T, INV>(tile_a, tile_b, lines, 1, STRIDE, nullptr, p, tw)
                              : fft_lines_pp<T, INV>(tile_a, tile_b, lines, 1, STRIDE, nullptr, p, tw);
  for (int idx = tid; idx < n * TL; idx += blockDim.x) {
    const int e = idx / TL, t = idx - e * TL;
    if (t < lines) base[e * stride + t] = done[e * STRIDE + t];
  }
}

// Contiguous rows of length n (the innermost axis).
template <typename T, bool INV, int TR, bool GENERAL>
__global__ void __launch_bounds__(kThreads) fft_rows_kernel(Cx<T>* __restrict__ data, int n, int np, long long rows,
                                                            LinePlan p, const Cx<T>* __restrict__ tw_global) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  Cx<T>* tile_a = tw + n;
  Cx<T>* tile_b = tile_a + TR * np;
  const long long r0 = static_cast<long long>(blockIdx.x) * TR;
  const int count = static_cast<int>(min(static_cast<long long>(TR), rows - r0));
  Cx<T>* base = data + r0 * n;
  const int tid = threadIdx.x;
  for (int i = tid; i < n; i += blockDim.x) tw[i] = tw_global[i];
  for (int idx = tid; idx < count * n; idx += blockDim.x) {
    const int r = idx / n, e = idx - r * n;
    tile_a[r * np + e] = base[idx];
  }
  __syncthreads();
  const Cx<T>* done = GENERAL ? fft_lines_pp_general<T, INV>(tile_a, tile_b, count, np, 1, nullptr, p, tw)
                              : fft_lines_pp<T, INV>(tile_a, tile_b, count, np, 1, nullptr, p, tw);
  for (int idx = tid; idx < count * n; idx += blockDim.x) {
    const int r = idx / n, e = idx - r * n;
    base[idx] = done[r * np + e];
  }
}

template <typename Kernel>
void allow_smem(Kernel kernel, std::size_t bytes) {
  if (bytes > kMaxDynamicSmem) throw InvalidArgument("FFT tile does not fit in shared memory");
  allow_dynamic_smem(kernel, bytes);
}

// CTAs of `kernel` resident on the whole device at once (persistent grids).
template <typename Kernel>
long long resident_ctas(Kernel kernel, int threads, std::size_t smem) {
  int per_sm = 0, device = 0, sms = 0;
  SDFT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem));
  SDFT_CUDA(cudaGetDevice(&device));
  SDFT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  return static_cast<long long>(std::max(per_sm, 1)) * sms;
}

// plane_in_kernel for compile-time axis lengths N1 = N2 = N, one plane
// buffer (in-place stages): backward FFT along i2 on the active i1 rows, then
// along i1 on every i2 column.
template <typename T, int N>
__global__ void __launch_bounds__(kThreads, plane_blocks<T>()) plane_in_fixed_kernel(const Cx<double>* __restrict__ x, long long ldx,
                                                                  LocalArgs<T> a, Cx<T>* __restrict__ slab) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  const int np = a.n2p, plane_elems = N * np;
  Cx<T>* plane = tw + N;
  int* rows = reinterpret_cast<int*>(plane + plane_elems);
  const int s = blockIdx.x, c = blockIdx.y;
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += kThreads) tw[i] = a.tw2[i];
  for (int i = tid; i < a.krows; i += kThreads) rows[i] = a.krow[i];
  for (int i = tid; i < plane_elems; i += kThreads) plane[i] = Cx<T>{0, 0};
  __syncthreads();
  const Cx<double>* xc = x + static_cast<long long>(c) * ldx;
  const int p_end = a.point_offset[s + 1];
  for (int p = a.point_offset[s] + tid; p < p_end; p += kThreads)
    plane[a.point_smem[p]] = cconvert<T>(xc[a.point_g[p]]);
  __syncthreads();
  fft_inplace_fixed<T, true, N, true, kThreads>(plane, a.krows, rows, np, 1, tw);
  fft_inplace_fixed<T, true, N, false, kThreads>(plane, N, nullptr, 1, np, tw);
  Cx<T>* out = slab + (static_cast<long long>(c) * a.slots + s) * (N * N);
  for (int i = tid; i < N * N; i += kThreads) {
    const int i1 = i / N, i2 = i - i1 * N;
    out[i] = plane[i1 * np + i2];
  }
}

// plane_out_kernel for N1 = N2 = N, one plane buffer: forward FFT along i1
// on every column, along i2 on the active rows, gather, y = T x + value / count.
template <typename T, int N>
__global__ void __launch_bounds__(kThreads, plane_blocks<T>()) plane_out_fixed_kernel(const Cx<T>* __restrict__ slab, LocalArgs<T> a,
                                                                   const Cx<double>* __restrict__ x, long long ldx,
                                                                   const double* __restrict__ kinetic, double count,
                                                                   Cx<double>* __restrict__ y, long long ldy) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<T>* tw = reinterpret_cast<Cx<T>*>(smem_raw);
  const int np = a.n2p, plane_elems = N * np;
  Cx<T>* plane = tw + N;
  int* rows = reinterpret_cast<int*>(plane + plane_elems);
  const int s = blockIdx.x, c = blockIdx.y;
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += kThreads) tw[i] = a.tw2[i];
  for (int i = tid; i < a.krows; i += kThreads) rows[i] = a.krow[i];
  const Cx<T>* in = slab + (static_cast<long long>(c) * a.slots + s) * (N * N);
  // The plane's slab entries and the first points' x and T values are all
  // requested before the transforms (one round of memory latency).
  constexpr int PER = (N * N + kThreads - 1) / kThreads, POINTS = 4;
  {
    Cx<T> entry[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int i = tid + q * kThreads;
      entry[q] = i < N * N ? in[i] : Cx<T>{0, 0};
    }
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int i = tid + q * kThreads;
      if (i < N * N) plane[(i / N) * np + i % N] = entry[q];
    }
  }
  const Cx<double>* xc = x + static_cast<long long>(c) * ldx;
  Cx<double>* yc = y + static_cast<long long>(c) * ldy;
  const int p_begin = a.point_offset[s], p_end = a.point_offset[s + 1];
  int pg[POINTS], ps[POINTS];
  Cx<double> px[POINTS];
  double pt[POINTS];
#pragma unroll
  for (int q = 0; q < POINTS; ++q) {
    const int p = p_begin + tid + q * kThreads;
    pg[q] = -1;
    if (p < p_end) {
      pg[q] = a.point_g[p];
      ps[q] = a.point_smem[p];
      px[q] = xc[pg[q]];
      pt[q] = kinetic[pg[q]];
    }
  }
  __syncthreads();
  fft_inplace_fixed<T, false, N, false, kThreads>(plane, N, nullptr, 1, np, tw);
  fft_inplace_fixed<T, false, N, true, kThreads>(plane, a.krows, rows, np, 1, tw);
#pragma unroll
  for (int q = 0; q < POINTS; ++q)
    if (pg[q] >= 0) {
      const Cx<double> v = cconvert<double>(plane[ps[q]]);
      yc[pg[q]] = Cx<double>{pt[q] * px[q].re + v.re / count, pt[q] * px[q].im + v.im / count};
    }
  for (int p = p_begin + tid + POINTS * kThreads; p < p_end; p += kThreads) {
    const int g = a.point_g[p];
    const Cx<double> v = cconvert<double>(plane[a.point_smem[p]]);
    const Cx<double> in_g = xc[g];
    const double t = kinetic[g];
    yc[g] = Cx<double>{t * in_g.re + v.re / count, t * in_g.im + v.im / count};
  }
}

// FP32 plane passes with pair-split lines (fft_pair_dif / fft_pair_dit):
// one CTA per (slot, column) plane, lane pair (l, l ^ 16) of warp w on line
// 16 w + (l & 15). The i1 transform runs on the i2 columns, the i2 transform
// on the active i1 rows (row krow[line]); shared memory holds the plane once,
// for the transpose between the two directions and the sphere scatter /
// gather. Rows outside the active i1 set are zero in the column transform's
// input (plane_in) and never transformed along i2 (plane_out).
constexpr int kPointBatch = 8;

template <int N>
struct PlanePairArgs {
  RegTwiddles<float, N> tw;
  RegTwiddles<float, N / 2> tw_half;
  int row_active[N];  // 1 where grid row i1 holds sphere points in some slot
};

template <int N>
constexpr int plane_pair_threads() {
  return (N + 15) / 16 * kWarp;
}
// Resident CTAs per SM the pair plane kernels are compiled for: four up to
// 80 points (at most 96-128 registers a thread, no spills), two above (the
// 192-thread CTAs of 84-96 points would spill at a four-CTA bound).
template <int N>
constexpr int plane_pair_blocks() {
  return N <= 80 ? 4 : 2;
}

template <int N>
__global__ void __launch_bounds__(plane_pair_threads<N>(), plane_pair_blocks<N>()) plane_in_pair_kernel(
    const Cx<double>* __restrict__ x, long long ldx, LocalArgs<float> a, Cx<float>* __restrict__ slab,
    const __grid_constant__ PlanePairArgs<N> p) {
  constexpr int H = N / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<float>* plane = reinterpret_cast<Cx<float>*>(smem_raw);  // [N][np]
  const int np = a.n2p, s = blockIdx.x, c = blockIdx.y, tid = threadIdx.x;
  const int lane = tid & (kWarp - 1);
  const bool upper = lane >= kPairXor;
  const int line = (tid >> 5) * kPairXor + (lane & (kPairXor - 1));
  const int h = upper ? H : 0;
  for (int i = tid; i < a.krows * N; i += blockDim.x) {
    const int r = i / N, i2 = i - r * N;
    plane[__ldg(a.krow + r) * np + i2] = Cx<float>{0.0f, 0.0f};
  }
  __syncthreads();
  // Sphere points in rounds of kPointBatch per thread, every load of a round in flight together.
  const Cx<double>* xc = x + static_cast<long long>(c) * ldx;
  const int p_begin = a.point_offset[s], points = a.point_offset[s + 1] - p_begin;
  for (int first = tid; first < points; first += kPointBatch * blockDim.x) {
    int dst[kPointBatch], g[kPointBatch];
#pragma unroll
    for (int u = 0; u < kPointBatch; ++u) {
      const int i = first + u * blockDim.x;
      dst[u] = -1;
      if (i < points) {
        dst[u] = __ldg(a.point_smem + p_begin + i);
        g[u] = __ldg(a.point_g + p_begin + i);
      }
    }
    Cx<double> value[kPointBatch];
#pragma unroll
    for (int u = 0; u < kPointBatch; ++u)
      if (dst[u] >= 0) value[u] = xc[g[u]];
#pragma unroll
    for (int u = 0; u < kPointBatch; ++u)
      if (dst[u] >= 0) plane[dst[u]] = cconvert<float>(value[u]);
  }
  __syncthreads();
  Cx<float> v[H];
  {  // i2 along active row krow[line]: natural halves in, interleaved out
    const bool live = line < a.krows;
    Cx<float>* row = plane + (live ? __ldg(a.krow + line) : 0) * np;
#pragma unroll
    for (int j = 0; j < H; ++j) v[j] = live ? row[j + h] : Cx<float>{0.0f, 0.0f};
    fft_pair_dif<float, true, N>(v, upper, p.tw.w, p.tw_half.w);
    if (live) {
#pragma unroll
      for (int m = 0; m < H; ++m) row[2 * m + (upper ? 1 : 0)] = v[m];
    }
  }
  __syncthreads();
  {  // i1 along column i2 = line, straight to the slab rows 2m + upper
    const bool live = line < N;
    const int col = live ? line : 0;  // lanes past the last column read column 0 and store nothing
#pragma unroll
    for (int j = 0; j < H; ++j) {
      const int active = upper ? p.row_active[j + H] : p.row_active[j];
      v[j] = live && active ? plane[(j + h) * np + col] : Cx<float>{0.0f, 0.0f};
    }
    fft_pair_dif<float, true, N>(v, upper, p.tw.w, p.tw_half.w);
    if (live) {
      Cx<float>* out = slab + (static_cast<long long>(c) * a.slots + s) * (N * N) + col + (upper ? N : 0);
#pragma unroll
      for (int m = 0; m < H; ++m) out[2 * m * N] = v[m];
    }
  }
}

template <int N>
__global__ void __launch_bounds__(plane_pair_threads<N>(), plane_pair_blocks<N>()) plane_out_pair_kernel(
    const Cx<float>* __restrict__ slab, LocalArgs<float> a, const Cx<double>* __restrict__ x, long long ldx,
    const double* __restrict__ kinetic, double count, Cx<double>* __restrict__ y, long long ldy,
    const __grid_constant__ PlanePairArgs<N> p) {
  constexpr int H = N / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<float>* plane = reinterpret_cast<Cx<float>*>(smem_raw);  // [N][np]
  const int np = a.n2p, s = blockIdx.x, c = blockIdx.y, tid = threadIdx.x;
  const int lane = tid & (kWarp - 1);
  const bool upper = lane >= kPairXor;
  const int line = (tid >> 5) * kPairXor + (lane & (kPairXor - 1));
  const int h = upper ? H : 0;
  Cx<float> v[H];
  {  // i1 along column i2 = line: slab rows 2m + upper in, natural halves out
    const bool live = line < N;
    const int col = live ? line : 0;  // lanes past the last column read column 0 and store nothing
    const Cx<float>* in = slab + (static_cast<long long>(c) * a.slots + s) * (N * N) + col + (upper ? N : 0);
#pragma unroll
    for (int m = 0; m < H; ++m) v[m] = live ? in[2 * m * N] : Cx<float>{0.0f, 0.0f};
    fft_pair_dit<float, false, N>(v, upper, p.tw.w, p.tw_half.w);
    if (live) {
#pragma unroll
      for (int k = 0; k < H; ++k) {
        const int active = upper ? p.row_active[k + H] : p.row_active[k];
        if (active) plane[(k + h) * np + col] = v[k];
      }
    }
  }
  __syncthreads();
  {  // i2 along active row krow[line]: interleaved in, natural halves out
    const bool live = line < a.krows;
    Cx<float>* row = plane + (live ? __ldg(a.krow + line) : 0) * np;
#pragma unroll
    for (int m = 0; m < H; ++m) v[m] = live ? row[2 * m + (upper ? 1 : 0)] : Cx<float>{0.0f, 0.0f};
    fft_pair_dit<float, false, N>(v, upper, p.tw.w, p.tw_half.w);
    if (live) {
#pragma unroll
      for (int k = 0; k < H; ++k) row[k + h] = v[k];
    }
  }
  __syncthreads();
  const Cx<double>* xc = x + static_cast<long long>(c) * ldx;
  Cx<double>* yc = y + static_cast<long long>(c) * ldy;
  const int p_begin = a.point_offset[s], points = a.point_offset[s + 1] - p_begin;
  for (int first = tid; first < points; first += kPointBatch * blockDim.x) {
    int g[kPointBatch], at[kPointBatch];
#pragma unroll
    for (int u = 0; u < kPointBatch; ++u) {
      const int i = first + u * blockDim.x;
      g[u] = -1;
      if (i < points) {
        g[u] = __ldg(a.point_g + p_begin + i);
        at[u] = __ldg(a.point_smem + p_begin + i);
      }
    }
    Cx<double> in_g[kPointBatch];
    double t[kPointBatch];
#pragma unroll
    for (int u = 0; u < kPointBatch; ++u)
      if (g[u] >= 0) {
        in_g[u] = xc[g[u]];
        t[u] = __ldg(kinetic + g[u]);
      }
#pragma unroll
    for (int u = 0; u < kPointBatch; ++u)
      if (g[u] >= 0) {
        const Cx<double> value = cconvert<double>(plane[at[u]]);
        yc[g[u]] = Cx<double>{t[u] * in_g[u].re + value.re / count, t[u] * in_g[u].im + value.im / count};
      }
  }
}

// FP32 plane passes with the pair kernels for square planes of the even
// lengths they are compiled for; false otherwise.
template <typename T>
bool launch_planes_pair(const SpherePlan& plan, const LocalArgs<T>& a, bool inward, int columns,
                        const Cx<double>* x, long long ldx, Cx<T>* slab, const double* kinetic, double count,
                        Cx<double>* y, long long ldy, cudaStream_t stream) {
  if constexpr (!std::is_same_v<T, float>) {
    return false;
  } else {
    if (a.n1 != a.n2) return false;
    auto go = [&](auto length) {
      constexpr int N = decltype(length)::value;
      PlanePairArgs<N> p;
      for (int i = 0; i < N; ++i) p.tw.w[i] = plan.twiddles_host[1][i];
      for (int i = 0; i < N / 2; ++i) p.tw_half.w[i] = plan.twiddles_host[1][2 * i];
      for (int i = 0; i < N; ++i) p.row_active[i] = 0;
      for (int r : plan.krow_host) p.row_active[r] = 1;
      const std::size_t smem = sizeof(Cx<float>) * N * static_cast<std::size_t>(a.n2p);
      const dim3 grid(a.slots, columns);
      constexpr int threads = plane_pair_threads<N>();
      if (inward) {
        allow_smem(plane_in_pair_kernel<N>, smem);
        plane_in_pair_kernel<N><<<grid, threads, smem, stream>>>(x, ldx, a, slab, p);
        SDFT_LAUNCH("plane_in_pair_kernel");
      } else {
        allow_smem(plane_out_pair_kernel<N>, smem);
        plane_out_pair_kernel<N><<<grid, threads, smem, stream>>>(slab, a, x, ldx, kinetic, count, y, ldy, p);
        SDFT_LAUNCH("plane_out_pair_kernel");
      }
      return true;
    };
    switch (a.n1) {
      case 40: return go(std::integral_constant<int, 40>{});
      case 42: return go(std::integral_constant<int, 42>{});
      case 48: return go(std::integral_constant<int, 48>{});
      case 54: return go(std::integral_constant<int, 54>{});
      case 56: return go(std::integral_constant<int, 56>{});
      case 60: return go(std::integral_constant<int, 60>{});
      case 70: return go(std::integral_constant<int, 70>{});
      case 72: return go(std::integral_constant<int, 72>{});
      case 80: return go(std::integral_constant<int, 80>{});
      case 84: return go(std::integral_constant<int, 84>{});
      case 90: return go(std::integral_constant<int, 90>{});
      case 96: return go(std::integral_constant<int, 96>{});
      default: return false;
    }
  }
}

// Plane passes with the compile-time kernels for square planes of the common
// lengths; false when the plane has another shape.
template <typename T>
bool launch_planes_fixed(const LocalArgs<T>& a, bool inward, int columns, const Cx<double>* x, long long ldx,
                         Cx<T>* slab, const double* kinetic, double count, Cx<double>* y, long long ldy,
                         cudaStream_t stream) {
  if (a.n1 != a.n2) return false;
  const std::size_t smem = sizeof(Cx<T>) * (a.n1 + static_cast<std::size_t>(a.n1) * a.n2p) +
                           sizeof(int) * static_cast<std::size_t>(a.krows);
  const dim3 grid(a.slots, columns);
  auto go = [&](auto in_kernel, auto out_kernel) {
    if (inward) {
      allow_smem(in_kernel, smem);
      in_kernel<<<grid, kThreads, smem, stream>>>(x, ldx, a, slab);
      SDFT_LAUNCH("plane_in_fixed_kernel");
    } else {
      allow_smem(out_kernel, smem);
      out_kernel<<<grid, kThreads, smem, stream>>>(slab, a, x, ldx, kinetic, count, y, ldy);
      SDFT_LAUNCH("plane_out_fixed_kernel");
    }
    return true;
  };
#define SDFT_PLANES(N) \
  case N:              \
    return go(plane_in_fixed_kernel<T, N>, plane_out_fixed_kernel<T, N>);
  switch (a.n1) {
    SDFT_PLANES(24)
    SDFT_PLANES(35)
    SDFT_PLANES(36)
    SDFT_PLANES(45)
    SDFT_PLANES(48)
    SDFT_PLANES(60)
    SDFT_PLANES(64)
    SDFT_PLANES(70)
    SDFT_PLANES(72)
    SDFT_PLANES(80)
    SDFT_PLANES(81)
    SDFT_PLANES(84)
    SDFT_PLANES(90)
    SDFT_PLANES(96)
    default: return false;
  }
#undef SDFT_PLANES
}

// FP32 pencil pass with the register kernel where n0 has one; false otherwise.
template <typename T>
bool launch_pencil_registers(const SpherePlan& plan, int columns, const T* potential, Cx<T>* slab,
                             cudaStream_t stream) {
  if constexpr (!std::is_same_v<T, float>) {
    return false;
  } else {
    const long long n12 = static_cast<long long>(plan.n[1]) * plan.n[2];
    const long long units = static_cast<long long>(ceil_div(static_cast<std::size_t>(n12), kRegisterPencilThreads)) *
                            columns;
    auto go = [&](auto length) {
      constexpr int N0 = decltype(length)::value;
      if constexpr (N0 > kRegisterPencilMax) {
        const long long pair_units =
            static_cast<long long>(ceil_div(static_cast<std::size_t>(n12), kPairPencilLines)) * columns;
        PencilPairArgs<N0> p;
        for (int i = 0; i < N0; ++i) {
          p.tw.w[i] = plan.twiddles_host[0][i];
          p.slot_of_row[i] = plan.slot_of_row_host[i];
        }
        for (int i = 0; i < N0 / 2; ++i) p.tw_half.w[i] = plan.twiddles_host[0][2 * i];
        const std::size_t smem =
            sizeof(Cx<float>) * 2 * plan.slots * kPairPencilLines + sizeof(float) * N0 * kPairPencilLines;
        allow_smem(pencil_pair_kernel<N0>, smem);
        const long long grid =
            std::min<long long>(pair_units, resident_ctas(pencil_pair_kernel<N0>, kPairPencilThreads, smem));
        pencil_pair_kernel<N0><<<static_cast<unsigned>(grid), kPairPencilThreads, smem, stream>>>(
            slab, n12, plan.slots, columns, pair_units, potential, p);
        SDFT_LAUNCH("pencil_pair_kernel");
      } else {
        PencilRegisterArgs<N0> p;
        for (int i = 0; i < N0; ++i) {
          p.tw.w[i] = plan.twiddles_host[0][i];
          p.slot_of_row[i] = plan.slot_of_row_host[i];
        }
        const std::size_t smem =
            sizeof(Cx<float>) * 2 * plan.slots * kRegisterPencilThreads + sizeof(float) * N0 * kRegisterPencilThreads;
        allow_smem(pencil_registers_kernel<N0>, smem);
        const long long grid =
            std::min<long long>(units, resident_ctas(pencil_registers_kernel<N0>, kRegisterPencilThreads, smem));
        pencil_registers_kernel<N0><<<static_cast<unsigned>(grid), kRegisterPencilThreads, smem, stream>>>(
            slab, n12, plan.slots, columns, units, potential, p);
        SDFT_LAUNCH("pencil_registers_kernel");
      }
      return true;
    };
    switch (plan.n[0]) {
      case 35: return go(std::integral_constant<int, 35>{});
      case 40: return go(std::integral_constant<int, 40>{});
      case 42: return go(std::integral_constant<int, 42>{});
      case 45: return go(std::integral_constant<int, 45>{});
      case 48: return go(std::integral_constant<int, 48>{});
      case 49: return go(std::integral_constant<int, 49>{});
      case 54: return go(std::integral_constant<int, 54>{});
      case 56: return go(std::integral_constant<int, 56>{});
      case 60: return go(std::integral_constant<int, 60>{});
      case 63: return go(std::integral_constant<int, 63>{});
      case 70: return go(std::integral_constant<int, 70>{});
      case 72: return go(std::integral_constant<int, 72>{});
      case 80: return go(std::integral_constant<int, 80>{});
      case 84: return go(std::integral_constant<int, 84>{});
      case 90: return go(std::integral_constant<int, 90>{});
      case 96: return go(std::integral_constant<int, 96>{});
      default: return false;
    }
  }
}

// Pencil pass with the compile-time kernel for the common axis lengths.
template <typename T>
bool launch_pencil_fixed(const LocalArgs<T>& a, int columns, const T* potential, Cx<T>* slab, cudaStream_t stream) {
  const std::size_t smem =
      sizeof(Cx<T>) * (a.n0 + 2 * static_cast<std::size_t>(a.n0) * (kPencilLines + 1)) + sizeof(int) * a.n0;
  const dim3 grid(static_cast<unsigned>(ceil_div(static_cast<std::size_t>(a.n12), kPencilLines)), columns);
  auto go = [&](auto kernel) {
    allow_smem(kernel, smem);
    kernel<<<grid, kThreads, smem, stream>>>(slab, a, potential);
    SDFT_LAUNCH("pencil_fixed_kernel");
    return true;
  };
  switch (a.n0) {
    case 35: return go(pencil_fixed_kernel<T, 35>);
    case 36: return go(pencil_fixed_kernel<T, 36>);
    case 45: return go(pencil_fixed_kernel<T, 45>);
    case 48: return go(pencil_fixed_kernel<T, 48>);
    case 60: return go(pencil_fixed_kernel<T, 60>);
    case 64: return go(pencil_fixed_kernel<T, 64>);
    case 70: return go(pencil_fixed_kernel<T, 70>);
    case 72: return go(pencil_fixed_kernel<T, 72>);
    case 80: return go(pencil_fixed_kernel<T, 80>);
    case 81: return go(pencil_fixed_kernel<T, 81>);
    case 84: return go(pencil_fixed_kernel<T, 84>);
    case 90: return go(pencil_fixed_kernel<T, 90>);
    case 96: return go(pencil_fixed_kernel<T, 96>);
    default: return false;
  }
}


template <typename T>
LocalArgs<T> make_args(const SpherePlan& plan) {
  LocalArgs<T> a{};
  a.n0 = plan.n[0];
  a.n1 = plan.n[1];
  a.n2 = plan.n[2];
  a.n2p = plan.n2p;
  a.slots = plan.slots;
  a.krows = plan.krows;
  a.n12 = static_cast<long long>(plan.n[1]) * plan.n[2];
  a.slot_row = plan.slot_row;
  a.point_offset = plan.point_offset;
  a.point_g = plan.point_g;
  a.point_smem = plan.point_smem;
  a.krow = plan.krow;
  a.p0 = plan.line[0];
  a.p1 = plan.line[1];
  a.p2 = plan.line[2];
  a.tw0 = device_twiddles<T>(plan.n[0]);
  a.tw1 = device_twiddles<T>(plan.n[1]);
  a.tw2 = device_twiddles<T>(plan.n[2]);
  return a;
}

// Plane passes through the slab in global memory, for planes whose two
// shared-memory buffers do not fit (FP64 beyond ~118 points per axis, FP32
// beyond ~167, or lengths without a compiled plane kernel whose two buffers
// exceed the limit): scatter the sphere points into zeroed slab planes, then
// the i2 transform of every row of every plane (tiled rows kernel) and the
// i1 transform of every plane (strided kernel); plane_out runs the forward
// transforms in the opposite order and gathers. Rows without sphere points
// are transformed too (zeros): this path trades work for shared memory.
template <typename T>
__global__ void __launch_bounds__(kThreads) slab_scatter_kernel(const Cx<double>* __restrict__ x, long long ldx,
                                                                LocalArgs<T> a, Cx<T>* __restrict__ slab) {
  const int s = blockIdx.x, c = blockIdx.y;
  Cx<T>* plane = slab + (static_cast<long long>(c) * a.slots + s) * a.n12;
  for (long long i = threadIdx.x; i < a.n12; i += blockDim.x) plane[i] = Cx<T>{0, 0};
  __syncthreads();  // the zeros are in place before any point lands
  const Cx<double>* xc = x + static_cast<long long>(c) * ldx;
  for (int p = a.point_offset[s] + threadIdx.x; p < a.point_offset[s + 1]; p += blockDim.x) {
    const int at = a.point_smem[p], i1 = at / a.n2p, i2 = at - i1 * a.n2p;
    plane[static_cast<long long>(i1) * a.n2 + i2] = cconvert<T>(xc[a.point_g[p]]);
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) slab_gather_kernel(const Cx<T>* __restrict__ slab, LocalArgs<T> a,
                                                               const Cx<double>* __restrict__ x, long long ldx,
                                                               const double* __restrict__ kinetic, double count,
                                                               Cx<double>* __restrict__ y, long long ldy) {
  const int s = blockIdx.x, c = blockIdx.y;
  const Cx<T>* plane = slab + (static_cast<long long>(c) * a.slots + s) * a.n12;
  const Cx<double>* xc = x + static_cast<long long>(c) * ldx;
  Cx<double>* yc = y + static_cast<long long>(c) * ldy;
  for (int p = a.point_offset[s] + threadIdx.x; p < a.point_offset[s + 1]; p += blockDim.x) {
    const int g = a.point_g[p], at = a.point_smem[p], i1 = at / a.n2p, i2 = at - i1 * a.n2p;
    const Cx<double> v = cconvert<double>(plane[static_cast<long long>(i1) * a.n2 + i2]);
    const Cx<double> in_g = xc[g];
    const double t = kinetic[g];
    yc[g] = Cx<double>{t * in_g.re + v.re / count, t * in_g.im + v.im / count};
  }
}

// Rows of the slab planes along i2 (contiguous), tiles of the widest TR in
// {32, 16, 8} that fits.
template <typename T, bool INV>
void slab_rows(const LocalArgs<T>& a, int columns, Cx<T>* slab, cudaStream_t stream) {
  const int np = a.n2 | 1;
  const long long rows = static_cast<long long>(columns) * a.slots * a.n1;
  auto go = [&](auto tile) {
    constexpr int TR = decltype(tile)::value;
    const std::size_t smem = sizeof(Cx<T>) * (a.n2 + 2 * static_cast<std::size_t>(TR) * np);
    if (smem > kMaxDynamicSmem) return false;
    allow_smem(fft_rows_kernel<T, INV, TR, false>, smem);
    fft_rows_kernel<T, INV, TR, false><<<static_cast<unsigned>(ceil_div(rows, TR)), kThreads, smem, stream>>>(
        slab, a.n2, np, rows, a.p2, a.tw2);
    SDFT_LAUNCH("fft_rows_kernel slab planes");
    return true;
  };
  if (!go(std::integral_constant<int, 32>{}) && !go(std::integral_constant<int, 16>{}) &&
      !go(std::integral_constant<int, 8>{}))
    throw InvalidArgument("FFT tile does not fit in shared memory");
}

// Columns of the slab planes along i1 (stride n2), TL lines per tile.
template <typename T, bool INV>
void slab_columns(const LocalArgs<T>& a, int columns, Cx<T>* slab, cudaStream_t stream) {
  const long long planes = static_cast<long long>(columns) * a.slots;
  auto go = [&](auto tile) {
    constexpr int TL = decltype(tile)::value;
    const std::size_t smem = sizeof(Cx<T>) * (a.n1 + 2 * static_cast<std::size_t>(a.n1) * (TL + 1));
    if (smem > kMaxDynamicSmem) return false;
    allow_smem(fft_strided_kernel<T, INV, TL, false>, smem);
    // One plane per blockIdx.y, in launches of at most 65535 planes.
    for (long long first = 0; first < planes; first += 65535) {
      const dim3 blocks(static_cast<unsigned>(ceil_div(a.n2, TL)),
                        static_cast<unsigned>(std::min<long long>(65535, planes - first)));
      fft_strided_kernel<T, INV, TL, false><<<blocks, kThreads, smem, stream>>>(slab + first * a.n12, a.n1, a.n2,
                                                                               a.n2, a.n12, a.p1, a.tw1);
      SDFT_LAUNCH("fft_strided_kernel slab planes");
    }
    return true;
  };
  if (!go(std::integral_constant<int, 32>{}) && !go(std::integral_constant<int, 16>{}) &&
      !go(std::integral_constant<int, 8>{}))
    throw InvalidArgument("FFT tile does not fit in shared memory");
}

// The three passes: plane_in, pencil (V(r) multiply) and plane_out, each
// with its compile-time kernel where the lengths have one.
template <typename T>
void run_local_passes(const SpherePlan& plan, const LocalArgs<T>& a, double count, const Cx<double>* x, long long ldx, int columns,
                      const T* potential, const double* kinetic, Cx<double>* y, long long ldy, Cx<T>* slab,
                      cudaStream_t stream) {
  const std::size_t plane_smem = sizeof(Cx<T>) * (a.n1 + a.n2 + 2 * static_cast<std::size_t>(a.n1) * a.n2p);
  const std::size_t pencil_smem = sizeof(Cx<T>) * (a.n0 + 2 * static_cast<std::size_t>(a.n0) * (kPencilLines + 1));
  const dim3 planes(a.slots, columns);
  const bool planes_fit = plane_smem <= kMaxDynamicSmem;
  if (!launch_planes_pair<T>(plan, a, true, columns, x, ldx, slab, kinetic, count, y, ldy, stream) &&
      !launch_planes_fixed<T>(a, true, columns, x, ldx, slab, kinetic, count, y, ldy, stream)) {
    if (planes_fit) {
      allow_smem(plane_in_kernel<T>, plane_smem);
      plane_in_kernel<T><<<planes, kThreads, plane_smem, stream>>>(x, ldx, a, slab);
      SDFT_LAUNCH("plane_in_kernel");
    } else {
      slab_scatter_kernel<T><<<planes, kThreads, 0, stream>>>(x, ldx, a, slab);
      SDFT_LAUNCH("slab_scatter_kernel");
      slab_rows<T, true>(a, columns, slab, stream);
      slab_columns<T, true>(a, columns, slab, stream);
    }
  }
  if (!launch_pencil_registers<T>(plan, columns, potential, slab, stream) &&
      !launch_pencil_fixed<T>(a, columns, potential, slab, stream)) {
    const dim3 pencils(static_cast<unsigned>(ceil_div(static_cast<std::size_t>(a.n12), kPencilLines)), columns);
    allow_smem(pencil_kernel<T>, pencil_smem);
    pencil_kernel<T><<<pencils, kThreads, pencil_smem, stream>>>(slab, a, potential);
    SDFT_LAUNCH("pencil_kernel");
  }
  if (!launch_planes_pair<T>(plan, a, false, columns, x, ldx, slab, kinetic, count, y, ldy, stream) &&
      !launch_planes_fixed<T>(a, false, columns, x, ldx, slab, kinetic, count, y, ldy, stream)) {
    if (planes_fit) {
      allow_smem(plane_out_kernel<T>, plane_smem);
      plane_out_kernel<T><<<planes, kThreads, plane_smem, stream>>>(slab, a, x, ldx, kinetic, count, y, ldy);
      SDFT_LAUNCH("plane_out_kernel");
    } else {
      slab_columns<T, false>(a, columns, slab, stream);
      slab_rows<T, false>(a, columns, slab, stream);
      slab_gather_kernel<T><<<planes, kThreads, 0, stream>>>(slab, a, x, ldx, kinetic, count, y, ldy);
      SDFT_LAUNCH("slab_gather_kernel");
    }
  }
}

template <typename T>
void local_hamiltonian_impl(const SpherePlan& plan, const Cx<double>* x, long long ldx, int columns,
                            const T* potential, const double* kinetic, Cx<double>* y, long long ldy, Cx<T>* slab,
                            cudaStream_t stream) {
  const LocalArgs<T> a = make_args<T>(plan);
  run_local_passes<T>(plan, a, static_cast<double>(plan.count), x, ldx, columns, potential, kinetic, y, ldy, slab,
                      stream);
}

template <typename T, bool INV, int TL, bool GENERAL>
void fft3d_tiles(Cx<T>* grid, const int n[3], int batch, cudaStream_t stream) {
  const long long n12 = static_cast<long long>(n[1]) * n[2];
  const long long count = n12 * n[0];
  // axis 2: contiguous rows
  {
    const LinePlan p = make_line_plan(n[2], GENERAL);
    const int np = n[2] | 1;
    const std::size_t smem = sizeof(Cx<T>) * (n[2] + 2 * static_cast<std::size_t>(TL) * np);
    allow_smem(fft_rows_kernel<T, INV, TL, GENERAL>, smem);
    const long long rows = count / n[2] * batch;
    fft_rows_kernel<T, INV, TL, GENERAL><<<static_cast<unsigned>(ceil_div(rows, TL)), kThreads, smem, stream>>>(
        grid, n[2], np, rows, p, device_twiddles<T>(n[2]));
    SDFT_LAUNCH("fft_rows_kernel");
  }
  // axis 1: stride n2, n0*batch outer blocks
  {
    const LinePlan p = make_line_plan(n[1], GENERAL);
    const std::size_t smem = sizeof(Cx<T>) * (n[1] + 2 * static_cast<std::size_t>(n[1]) * (TL + 1));
    allow_smem(fft_strided_kernel<T, INV, TL, GENERAL>, smem);
    const dim3 blocks(static_cast<unsigned>(ceil_div(n[2], TL)), static_cast<unsigned>(n[0] * batch));
    fft_strided_kernel<T, INV, TL, GENERAL><<<blocks, kThreads, smem, stream>>>(grid, n[1], n[2], n[2], n12, p,
                                                                            device_twiddles<T>(n[1]));
    SDFT_LAUNCH("fft_strided_kernel axis1");
  }
  // axis 0: stride n1*n2
  {
    const LinePlan p = make_line_plan(n[0], GENERAL);
    const std::size_t smem = sizeof(Cx<T>) * (n[0] + 2 * static_cast<std::size_t>(n[0]) * (TL + 1));
    allow_smem(fft_strided_kernel<T, INV, TL, GENERAL>, smem);
    const dim3 blocks(static_cast<unsigned>(ceil_div(n12, TL)), static_cast<unsigned>(batch));
    fft_strided_kernel<T, INV, TL, GENERAL><<<blocks, kThreads, smem, stream>>>(grid, n[0], n12, n12, count, p,
                                                                            device_twiddles<T>(n[0]));
    SDFT_LAUNCH("fft_strided_kernel axis0");
  }
}

// Tile width: 32 lines when the widest axis fits in shared memory, else 16 or 8.
template <typename T, bool INV, bool GENERAL>
void fft3d_impl(Cx<T>* grid, const int n[3], int batch, cudaStream_t stream) {
  const std::size_t nmax = std::max({n[0], n[1], n[2]});
  auto fits = [&](std::size_t tl) { return sizeof(Cx<T>) * (nmax + 2 * nmax * (tl + 1)) <= 227 * 1024; };
  if (fits(32)) fft3d_tiles<T, INV, 32, GENERAL>(grid, n, batch, stream);
  else if (fits(16)) fft3d_tiles<T, INV, 16, GENERAL>(grid, n, batch, stream);
  else fft3d_tiles<T, INV, 8, GENERAL>(grid, n, batch, stream);
}

}  // namespace

void SpherePlan::build(const int shape[3], const std::vector<std::uint64_t>& indices, cudaStream_t on) {
  release();
  stream = on;
  for (int a = 0; a < 3; ++a) {
    if (shape[a] < 1 || !fft_length_supported(shape[a]))
      throw InvalidArgument("grid axis length must be a 2/3/5/7-smooth integer in [1,512]");
    n[a] = shape[a];
    line[a] = make_line_plan(shape[a]);
  }
  count = static_cast<std::size_t>(n[0]) * n[1] * n[2];
  if (indices.empty() || indices.size() > static_cast<std::size_t>(std::numeric_limits<int>::max()))
    throw InvalidArgument("plane-wave index map size out of range");
  npw = static_cast<int>(indices.size());
  n2p = n[2] | 1;
  const std::size_t n12 = static_cast<std::size_t>(n[1]) * n[2];
  std::vector<int> slot_of_row(n[0], -1);
  std::set<int> rows0, rows1;
  for (auto idx : indices) {
    if (idx >= count) throw InvalidArgument("plane-wave index outside the FFT grid");
    rows0.insert(static_cast<int>(idx / n12));
    rows1.insert(static_cast<int>((idx / n[2]) % n[1]));
  }
  std::vector<int> h_slot_row(rows0.begin(), rows0.end());
  slots = static_cast<int>(h_slot_row.size());
  for (int s = 0; s < slots; ++s) slot_of_row[h_slot_row[s]] = s;
  slot_of_row_host = slot_of_row;
  krow_host.assign(rows1.begin(), rows1.end());
  for (int a = 0; a < 3; ++a) {
    twiddles_host[a].resize(n[a]);
    host_twiddles<float>(n[a], twiddles_host[a].data());
  }
  std::vector<int> h_krow(rows1.begin(), rows1.end());
  krows = static_cast<int>(h_krow.size());
  std::vector<int> h_offset(slots + 1, 0);
  for (auto idx : indices) ++h_offset[slot_of_row[idx / n12] + 1];
  for (int s = 0; s < slots; ++s) h_offset[s + 1] += h_offset[s];
  std::vector<int> fill(h_offset.begin(), h_offset.end() - 1);
  std::vector<int> h_g(npw), h_smem(npw), h_compact(npw), kpos(n[1], -1);
  for (int k = 0; k < krows; ++k) kpos[h_krow[k]] = k;
  for (int g = 0; g < npw; ++g) {
    const auto idx = indices[g];
    const int s = slot_of_row[idx / n12];
    const int i1 = static_cast<int>((idx / n[2]) % n[1]);
    const int i2 = static_cast<int>(idx % n[2]);
    const int p = fill[s]++;
    h_g[p] = g;
    h_smem[p] = i1 * n2p + i2;
    h_compact[p] = kpos[i1] * n[2] + i2;
  }
  // Pageable host sources: each copy has staged its source when the call returns.
  auto upload = [&](int*& dst, const std::vector<int>& src) {
    dst = static_cast<int*>(stream_alloc(sizeof(int) * std::max<std::size_t>(1, src.size()), stream));
    if (!src.empty())
      SDFT_CUDA(cudaMemcpyAsync(dst, src.data(), sizeof(int) * src.size(), cudaMemcpyHostToDevice, stream));
  };
  upload(slot_row, h_slot_row);
  upload(point_offset, h_offset);
  upload(point_g, h_g);
  upload(point_smem, h_smem);
  upload(point_compact, h_compact);
  upload(krow, h_krow);
}

void SpherePlan::release() {
  for (int** p : {&slot_row, &point_offset, &point_g, &point_smem, &point_compact, &krow}) {
    stream_free(*p, stream);
    *p = nullptr;
  }
}

template <typename T>
void local_hamiltonian(const SpherePlan& plan, const Cx<double>* x, long long ldx, int columns, const T* potential,
                       const double* kinetic, Cx<double>* y, long long ldy, Cx<T>* slab, cudaStream_t stream) {
  if (columns <= 0) return;
  const int nmax = std::max({plan.n[0], plan.n[1], plan.n[2]});
  if (nmax > 128) throw InvalidArgument("operator FFT grid axes above 128 points are not supported");
  (void)nmax;
  local_hamiltonian_impl<T>(plan, x, ldx, columns, potential, kinetic, y, ldy, slab, stream);
}

template <typename T>
void fft3d(Cx<T>* grid, const int n[3], int batch, bool backward, cudaStream_t stream, bool general) {
  const int nmax = std::max({n[0], n[1], n[2]});
  if (nmax > kMaxLine) throw InvalidArgument("3D FFT axes above 512 points are not supported");
  // Smooth lengths keep the compiled-radix kernels even when general lengths are allowed.
  general = general && !(fft_length_supported(n[0]) && fft_length_supported(n[1]) && fft_length_supported(n[2]));
  if (general) {
    if (backward) fft3d_impl<T, true, true>(grid, n, batch, stream);
    else fft3d_impl<T, false, true>(grid, n, batch, stream);
  } else {
    if (backward) fft3d_impl<T, true, false>(grid, n, batch, stream);
    else fft3d_impl<T, false, false>(grid, n, batch, stream);
  }
}

template <typename T>
void local_hamiltonian_preset(const SpherePlan& plan, const Cx<double>* x, long long ldx, int columns,
                              const T* potential, const double* kinetic, Cx<double>* y, long long ldy,
                              Cx<T>* slab, const Cx<T>* const twiddle[3], cudaStream_t stream) {
  if (columns <= 0) return;
  if (std::max({plan.n[0], plan.n[1], plan.n[2]}) > 128)
    throw InvalidArgument("operator FFT grid axes above 128 points are not supported");
  LocalArgs<T> a{};
  a.n0 = plan.n[0];
  a.n1 = plan.n[1];
  a.n2 = plan.n[2];
  a.n2p = plan.n2p;
  a.slots = plan.slots;
  a.krows = plan.krows;
  a.n12 = static_cast<long long>(plan.n[1]) * plan.n[2];
  a.slot_row = plan.slot_row;
  a.point_offset = plan.point_offset;
  a.point_g = plan.point_g;
  a.point_smem = plan.point_smem;
  a.krow = plan.krow;
  a.p0 = plan.line[0];
  a.p1 = plan.line[1];
  a.p2 = plan.line[2];
  a.tw0 = twiddle[0];
  a.tw1 = twiddle[1];
  a.tw2 = twiddle[2];
  run_local_passes<T>(plan, a, static_cast<double>(plan.count), x, ldx, columns, potential, kinetic, y, ldy, slab,
                      stream);
}

template void local_hamiltonian_preset<float>(const SpherePlan&, const Cx<double>*, long long, int, const float*,
                                              const double*, Cx<double>*, long long, Cx<float>*,
                                              const Cx<float>* const[3], cudaStream_t);
template void local_hamiltonian_preset<double>(const SpherePlan&, const Cx<double>*, long long, int, const double*,
                                               const double*, Cx<double>*, long long, Cx<double>*,
                                               const Cx<double>* const[3], cudaStream_t);
template void local_hamiltonian<float>(const SpherePlan&, const Cx<double>*, long long, int, const float*,
                                       const double*, Cx<double>*, long long, Cx<float>*, cudaStream_t);
template void local_hamiltonian<double>(const SpherePlan&, const Cx<double>*, long long, int, const double*,
                                        const double*, Cx<double>*, long long, Cx<double>*, cudaStream_t);
template void fft3d<float>(Cx<float>*, const int[3], int, bool, cudaStream_t, bool);
template void fft3d<double>(Cx<double>*, const int[3], int, bool, cudaStream_t, bool);

}  // namespace sdft_b200
