// Device-resident plane-wave PAW operator: construction (the reference's
// PlaneWaveOperator constructor, src/plane_wave_operator.cpp:393-516) and the
// H~ / S~ / joint applications (src/plane_wave_operator.cpp:218-374).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <sstream>
#include <string>
#include <unordered_map>

#include "dense.cuh"
#include "operator.cuh"

namespace sdft_b200 {

namespace {
void check_solver(cusolverStatus_t status, const char* what) {
  if (status != CUSOLVER_STATUS_SUCCESS)
    throw CudaError(std::string("cuSOLVER error ") + std::to_string(static_cast<int>(status)) + " in " + what);
}
void check_blas(cublasStatus_t status, const char* what) {
  if (status != CUBLAS_STATUS_SUCCESS)
    throw CudaError(std::string("cuBLAS error ") + std::to_string(static_cast<int>(status)) + " in " + what);
}

std::uint64_t pack_key(int h, int k, int l) {
  const auto bias = [](int v) { return static_cast<std::uint64_t>(static_cast<std::int64_t>(v) + (1LL << 20)) & 0x1FFFFF; };
  return (bias(h) << 42) | (bias(k) << 21) | bias(l);
}

struct V3 {
  double x, y, z;
};
V3 vadd(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3 vscale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3 vcross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

using C = std::complex<double>;
double frobenius(const std::vector<C>& m) {
  double s = 0;
  for (const auto& v : m) s += std::norm(v);
  return std::sqrt(s);
}

// Row-major Sigma_np x NPW amplitudes (atom blocks of rows, the input layout)
// to the column-major device B (ld Sigma_np), through 32 x 32 shared-memory
// tiles so that both the reads and the writes are coalesced; a nonfinite entry
// raises *bad.
__global__ void paw_transpose_kernel(const Cx<double>* __restrict__ raw, int rows, int npw, Cx<double>* __restrict__ b,
                                     unsigned int* bad) {
  __shared__ Cx<double> tile[32][33];
  const int g0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
  unsigned int nonfinite = 0;
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int r = r0 + dy, g = g0 + threadIdx.x;
    if (r < rows && g < npw) {
      const Cx<double> v = raw[static_cast<std::size_t>(r) * npw + g];
      nonfinite |= !isfinite(v.re) || !isfinite(v.im);
      tile[dy][threadIdx.x] = v;
    }
  }
  __syncthreads();
  for (int dy = threadIdx.y; dy < 32; dy += blockDim.y) {
    const int g = g0 + dy, r = r0 + threadIdx.x;
    if (r < rows && g < npw) b[r + static_cast<std::size_t>(g) * rows] = tile[threadIdx.x][dy];
  }
  if (__any_sync(0xffffffffu, nonfinite) && (threadIdx.x & 31) == 0) atomicOr(bad, 1u);
}

// h_diag[g] += Re(b_g^H D b_g), s_diag[g] += Re(b_g^H Q b_g) per atom, one
// thread per plane wave, with the products and sums of the complex host loop
// (atoms, rows i, columns j: db_i = sum_j D(i,j) b_j, hd = sum_i conj(b_i) db_i)
// each rounded on its own, so the diagonals equal the host arithmetic's. The
// symmetrised blocks are column-major (D(i,j) at i + j*np) and uniform over
// the block's threads. The amplitudes are strided: the row-major input at
// construction (coalesced), or the resident column-major B when D and Q are
// replaced (each thread's column then stays in L1 across the block products).
__global__ void paw_diagonal_kernel(const Cx<double>* __restrict__ amplitudes, std::size_t row_stride,
                                    std::size_t column_stride, int npw, int atoms,
                                    const int* __restrict__ offsets, const long long* __restrict__ storage,
                                    const Cx<double>* __restrict__ d, const Cx<double>* __restrict__ q,
                                    double* __restrict__ h_diag, double* __restrict__ s_diag) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= npw) return;
  double hdiag = h_diag[g], sdiag = s_diag[g];
  for (int a = 0; a < atoms; ++a) {
    const int base = offsets[a], np = offsets[a + 1] - offsets[a];
    const Cx<double>* da = d + storage[a];
    const Cx<double>* qa = q + storage[a];
    const Cx<double>* col = amplitudes + static_cast<std::size_t>(base) * row_stride + static_cast<std::size_t>(g) * column_stride;
    double hr = 0, hi = 0, sr = 0, si = 0;
    for (int i = 0; i < np; ++i) {
      double dr = 0, di = 0, qr = 0, qi = 0;
      for (int j = 0; j < np; ++j) {
        const Cx<double> bj = col[static_cast<std::size_t>(j) * row_stride];
        const Cx<double> dij = da[i + static_cast<std::size_t>(j) * np], qij = qa[i + static_cast<std::size_t>(j) * np];
        dr = __dadd_rn(dr, __dsub_rn(__dmul_rn(dij.re, bj.re), __dmul_rn(dij.im, bj.im)));
        di = __dadd_rn(di, __dadd_rn(__dmul_rn(dij.re, bj.im), __dmul_rn(dij.im, bj.re)));
        qr = __dadd_rn(qr, __dsub_rn(__dmul_rn(qij.re, bj.re), __dmul_rn(qij.im, bj.im)));
        qi = __dadd_rn(qi, __dadd_rn(__dmul_rn(qij.re, bj.im), __dmul_rn(qij.im, bj.re)));
      }
      // conj(b_i) * db: real part b.re*db.re - (-b.im)*db.im, imaginary part
      // b.re*db.im + (-b.im)*db.re (only the real part reaches the diagonal,
      // the imaginary part is summed as on the host for the same operation count).
      const Cx<double> bi = col[static_cast<std::size_t>(i) * row_stride];
      hr = __dadd_rn(hr, __dsub_rn(__dmul_rn(bi.re, dr), __dmul_rn(-bi.im, di)));
      hi = __dadd_rn(hi, __dadd_rn(__dmul_rn(bi.re, di), __dmul_rn(-bi.im, dr)));
      sr = __dadd_rn(sr, __dsub_rn(__dmul_rn(bi.re, qr), __dmul_rn(-bi.im, qi)));
      si = __dadd_rn(si, __dadd_rn(__dmul_rn(bi.re, qi), __dmul_rn(-bi.im, qr)));
    }
    (void)hi;
    (void)si;
    hdiag = __dadd_rn(hdiag, hr);
    sdiag = __dadd_rn(sdiag, sr);
  }
  h_diag[g] = hdiag;
  s_diag[g] = sdiag;
}

// Adds the PAW terms to the diagonals; amplitude (row r, plane wave g) sits at
// amplitudes[r * row_stride + g * column_stride].
void paw_diagonals(const Cx<double>* amplitudes, std::size_t row_stride, std::size_t column_stride, int npw, int atoms,
                   const int* offsets, const long long* storage, const Cx<double>* d, const Cx<double>* q,
                   double* h_diag, double* s_diag, cudaStream_t stream) {
  paw_diagonal_kernel<<<(npw + 127) / 128, 128, 0, stream>>>(amplitudes, row_stride, column_stride, npw, atoms, offsets,
                                                             storage, d, q, h_diag, s_diag);
  SDFT_LAUNCH("paw_diagonal_kernel");
}

void paw_prepare(const Cx<double>* raw, int rows, int npw, int atoms, const int* offsets, const long long* storage,
                 const Cx<double>* d, const Cx<double>* q, Cx<double>* b, double* h_diag, double* s_diag,
                 unsigned int* bad, cudaStream_t stream) {
  const dim3 tiles((npw + 31) / 32, (rows + 31) / 32);
  if (tiles.y > 65535u) throw Overflow("PAW projector tiles exceed the grid limit");
  paw_transpose_kernel<<<tiles, dim3(32, 8), 0, stream>>>(raw, rows, npw, b, bad);
  SDFT_LAUNCH("paw_transpose_kernel");
  paw_diagonals(raw, npw, 1, npw, atoms, offsets, storage, d, q, h_diag, s_diag, stream);
}
}  // namespace

Context::Context(int dev, cudaStream_t s) : device(dev), stream(s) {
  SDFT_CUDA(cudaSetDevice(device));
  if (!stream) {
    SDFT_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    owns_stream = true;
  }
  for (Scratch* buffer : working_buffers()) buffer->stream = stream;
  for (Scratch* buffer : cache_buffers()) buffer->stream = stream;
  check_blas(cublasCreate(&blas), "cublasCreate");
  check_blas(cublasSetStream(blas, stream), "cublasSetStream");
  check_blas(cublasSetMathMode(blas, CUBLAS_DEFAULT_MATH), "cublasSetMathMode");  // true FP64, no TF32
  check_solver(cusolverDnCreate(&solver), "cusolverDnCreate");
  check_solver(cusolverDnSetStream(solver, stream), "cusolverDnSetStream");
}

Context::~Context() {
  // Everything stream-ordered on this stream is released before the stream goes.
  cudaStreamSynchronize(stream);
  for (Scratch* buffer : working_buffers()) buffer->release();
  for (Scratch* buffer : cache_buffers()) buffer->release();
  accel.plan.release();
  density.plan.release();
  release(accel.b_packed);
  release(accel.bh_packed);
  for (ImmutableLeft& entry : immutable.entries) release(entry.packed);
  // The frees above are stream-ordered: once they have run, the pool's
  // unused memory goes back to the device (a torn-down context leaves
  // nothing reserved beyond what other live objects hold).
  if (cudaStreamSynchronize(stream) == cudaSuccess && cudaSetDevice(device) == cudaSuccess) {
    try {
      trim_pool();
    } catch (...) {
    }
  }
  if (solver) cusolverDnDestroy(solver);
  if (blas) cublasDestroy(blas);
  if (owns_stream && stream) cudaStreamDestroy(stream);
}

void Context::synchronize() const { SDFT_CUDA(cudaStreamSynchronize(stream)); }

std::vector<Scratch*> Context::working_buffers() {
  std::vector<Scratch*> all = {&slab32, &slab64, &staging_in, &staging_out, &staging_aux, &projections, &onsite,
                               &tc.a, &tc.b, &tc.partial, &tc.adjoint};
  for (EigenWorkspace* w : {&eigen, &davidson.eigen})
    for (Scratch* s : {&w->tridiagonal, &w->vectors, &w->scalar, &w->product, &w->product2, &w->solver_work})
      all.push_back(s);
  DavidsonBuffers& d = davidson;
  for (Scratch* s : {&d.basis, &d.hbasis, &d.sbasis, &d.cached_h, &d.cached_s, &d.rr_a, &d.rr_b, &d.rr_w,
                     &d.rr_work, &d.info, &d.xs, &d.sxs, &d.hxs, &d.res, &d.block, &d.metric, &d.original,
                     &d.projections, &d.gram, &d.small, &d.order, &d.select, &d.pack_vc, &d.pack_vn, &d.pack_hn,
                     &d.pack_sn, &d.pack_hb, &d.pack_sb, &d.excluded, &d.polish, &d.polish_small,
                     &d.polish_values})
    all.push_back(s);
  CorrectionBuffers& c = davidson.corrections;
  for (Scratch* s : {&c.res, &c.z, &c.p, &c.hp, &c.xh, &c.sxh, &c.xl, &c.sxl, &c.coefficients, &c.scalars, &c.index})
    all.push_back(s);
  return all;
}

std::vector<Scratch*> Context::cache_buffers() {
  std::vector<Scratch*> all = {&accel.v64, &accel.v32, &accel.kinetic, &accel.b, &accel.d, &accel.q,
                               &density.rows, &density.planes, &density.grid, &density.meta};
  for (ImmutableLeft& entry : immutable.entries) all.push_back(&entry.fp64);
  return all;
}

void Context::recycle_scratch() {
  synchronize();
  for (Scratch* buffer : working_buffers()) buffer->release();
}

void Context::release_scratch() {
  recycle_scratch();
  synchronize();  // the stream-ordered frees have run: their blocks are unused
  trim_pool();
}

GVectorList enumerate_g_vectors(const double reciprocal[9], double cutoff_ev, const double kpoint[3],
                                double hartree_to_ev) {
  if (cutoff_ev <= 0.0 || !std::isfinite(cutoff_ev)) throw InvalidArgument("plane-wave cutoff must be finite and positive");
  if (hartree_to_ev <= 0 || !std::isfinite(hartree_to_ev)) throw InvalidArgument("invalid Hartree conversion");
  const V3 r0{reciprocal[0], reciprocal[1], reciprocal[2]}, r1{reciprocal[3], reciprocal[4], reciprocal[5]},
      r2{reciprocal[6], reciprocal[7], reciprocal[8]};
  const double gmax = std::sqrt(2.0 * cutoff_ev / hartree_to_ev);
  const double det = vdot(r0, vcross(r1, r2));
  if (std::abs(det) < 1e-12 || !std::isfinite(det)) throw InvalidArgument("reciprocal lattice is singular");
  const V3 d0 = vscale(vcross(r1, r2), 1.0 / det), d1 = vscale(vcross(r2, r0), 1.0 / det),
           d2 = vscale(vcross(r0, r1), 1.0 / det);
  const int hmax = static_cast<int>(std::ceil(gmax * std::sqrt(vdot(d0, d0)) + std::abs(kpoint[0]))) + 1;
  const int kmax = static_cast<int>(std::ceil(gmax * std::sqrt(vdot(d1, d1)) + std::abs(kpoint[1]))) + 1;
  const int lmax = static_cast<int>(std::ceil(gmax * std::sqrt(vdot(d2, d2)) + std::abs(kpoint[2]))) + 1;
  const V3 shift = vadd(vadd(vscale(r0, kpoint[0]), vscale(r1, kpoint[1])), vscale(r2, kpoint[2]));
  struct Entry {
    int h, k, l;
    V3 g;
    double kinetic;
  };
  std::vector<Entry> list;
  for (int h = -hmax; h <= hmax; ++h)
    for (int k = -kmax; k <= kmax; ++k)
      for (int l = -lmax; l <= lmax; ++l) {
        const V3 g = vadd(vadd(vscale(r0, h), vscale(r1, k)), vscale(r2, l));
        const V3 s = vadd(g, shift);
        const double g2 = vdot(s, s);
        if (0.5 * g2 <= cutoff_ev / hartree_to_ev + 1e-12) list.push_back({h, k, l, g, 0.5 * g2 * hartree_to_ev});
      }
  std::sort(list.begin(), list.end(), [](const Entry& a, const Entry& b) {
    if (a.kinetic != b.kinetic) return a.kinetic < b.kinetic;
    if (a.h != b.h) return a.h < b.h;
    if (a.k != b.k) return a.k < b.k;
    return a.l < b.l;
  });
  GVectorList out;
  for (const auto& e : list) {
    out.hkl.insert(out.hkl.end(), {e.h, e.k, e.l});
    out.cartesian.insert(out.cartesian.end(), {e.g.x, e.g.y, e.g.z});
    out.kinetic_ev.push_back(e.kinetic);
  }
  return out;
}

namespace {

// The retained local potential of an operator whose basis spans span[a] =
// high_a - low_a along each axis: its grid and V(r).
struct LocalPotential {
  int shape[3];
  double v0;                  // V(G = 0), added to the H diagonal
  std::vector<double> real;   // V(r), row-major grid
};

// Validation, grid rule and V(r) of the reference constructor
// (src/plane_wave_operator.cpp:400-475): finite and Hermitian V(G), the
// retained keys (|k_a| <= span_a) set the potential radius, the grid is the
// alias-free minimum rounded to a smooth length, and V(r) is one backward FFT
// of the retained keys on the device in FP64.
LocalPotential local_potential(Context& ctx, const int span[3], std::size_t potential_count, const int* potential_hkl,
                               const double* potential) {
  int radius[3] = {0, 0, 0};
  double max_potential = 0;
  std::unordered_map<std::uint64_t, std::size_t> keys;
  keys.reserve(potential_count * 2 + 1);
  for (std::size_t i = 0; i < potential_count; ++i) {
    const C v(potential[2 * i], potential[2 * i + 1]);
    if (!std::isfinite(v.real()) || !std::isfinite(v.imag())) throw InvalidArgument("nonfinite local potential");
    const int* k = potential_hkl + 3 * i;
    bool retained = true;
    for (int a = 0; a < 3; ++a) retained &= std::abs(k[a]) <= span[a];
    if (retained)
      for (int a = 0; a < 3; ++a) radius[a] = std::max(radius[a], std::abs(k[a]));
    max_potential = std::max(max_potential, std::abs(v));
    keys[pack_key(k[0], k[1], k[2])] = i;
  }
  // Hermitian V(G) (:438-444).
  for (std::size_t i = 0; i < potential_count; ++i) {
    const int* k = potential_hkl + 3 * i;
    const C v(potential[2 * i], potential[2 * i + 1]);
    const auto other = keys.find(pack_key(-k[0], -k[1], -k[2]));
    const C partner = other == keys.end() ? C{} : C(potential[2 * other->second], potential[2 * other->second + 1]);
    if (std::abs(v - std::conj(partner)) > 1e-10 * std::max(1., max_potential))
      throw InvalidArgument("local Fourier potential is not Hermitian");
  }
  // Grid rule (:445-457): alias-free minimum, rounded to a 2/3/5/7-smooth length.
  // SDFT_FFT_GRID=minimal keeps the minimum when it is smooth; the device FFT
  // only has smooth lengths, and every alias-free grid gives the same operator.
  const char* mode = std::getenv("SDFT_FFT_GRID");
  if (mode && std::string(mode) != "minimal" && std::string(mode) != "fast")
    throw InvalidArgument("SDFT_FFT_GRID must be minimal or fast");
  LocalPotential out;
  std::size_t count = 1;
  for (int a = 0; a < 3; ++a) {
    const int minimum = std::max(3, 2 * std::max(radius[a], span[a]) + 1);
    out.shape[a] = (mode && std::string(mode) == "minimal" && fft_length_supported(minimum)) ? minimum
                                                                                              : fast_fft_length(minimum);
    if (count > std::numeric_limits<std::size_t>::max() / out.shape[a]) throw Overflow("plane-wave FFT grid overflow");
    count *= out.shape[a];
  }
  const int* shape = out.shape;
  auto wrap = [](int x, int size) {
    int r = x % size;
    return r < 0 ? r + size : r;
  };
  auto index = [&](int h, int k, int l) {
    return (static_cast<std::uint64_t>(wrap(h, shape[0])) * shape[1] + wrap(k, shape[1])) * shape[2] + wrap(l, shape[2]);
  };
  // V(r) by one backward FFT of the retained keys, on the device in FP64 (:464-475).
  std::vector<Cx<double>> grid(count, Cx<double>{0, 0});
  for (std::size_t i = 0; i < potential_count; ++i) {
    const int* k = potential_hkl + 3 * i;
    bool retained = true;
    for (int a = 0; a < 3; ++a) retained &= std::abs(k[a]) <= span[a];
    if (!retained) continue;
    grid[index(k[0], k[1], k[2])] = Cx<double>{potential[2 * i], potential[2 * i + 1]};
  }
  Cx<double>* dgrid = static_cast<Cx<double>*>(stream_alloc(sizeof(Cx<double>) * count, ctx.stream));
  try {
    SDFT_CUDA(cudaMemcpyAsync(dgrid, grid.data(), sizeof(Cx<double>) * count, cudaMemcpyHostToDevice, ctx.stream));
    fft3d<double>(dgrid, out.shape, 1, true, ctx.stream);
    SDFT_CUDA(cudaMemcpyAsync(grid.data(), dgrid, sizeof(Cx<double>) * count, cudaMemcpyDeviceToHost, ctx.stream));
    SDFT_CUDA(cudaStreamSynchronize(ctx.stream));
  } catch (...) {
    stream_free(dgrid, ctx.stream);
    throw;
  }
  stream_free(dgrid, ctx.stream);
  out.real.resize(count);
  for (std::size_t i = 0; i < count; ++i) {
    if (std::abs(grid[i].im) > 1e-9 * std::max(1., std::abs(grid[i].re)))
      throw std::runtime_error("complex real-space local potential");
    out.real[i] = grid[i].re;
  }
  const auto zero = keys.find(pack_key(0, 0, 0));
  out.v0 = zero == keys.end() ? 0.0 : potential[2 * zero->second];
  return out;
}

// Per-atom D and Q (row-major np_a x np_a input) checked for finiteness and
// Hermiticity and stored symmetrised, column-major and concatenated
// (src/plane_wave_operator.cpp:484-509).
void symmetrised_blocks(const std::vector<std::uint64_t>& channels, const double* in_d, const double* in_q,
                        std::vector<Cx<double>>& d_blocks, std::vector<Cx<double>>& q_blocks) {
  std::size_t block_total = 0;
  for (auto np : channels) block_total += np * np;
  d_blocks.assign(block_total, Cx<double>{0, 0});
  q_blocks.assign(block_total, Cx<double>{0, 0});
  std::size_t blk_offset = 0;
  for (std::size_t a = 0; a < channels.size(); ++a) {
    const std::size_t np = channels[a];
    std::vector<C> d(np * np), q(np * np);
    for (std::size_t i = 0; i < np * np; ++i) {
      d[i] = C(in_d[2 * (blk_offset + i)], in_d[2 * (blk_offset + i) + 1]);
      q[i] = C(in_q[2 * (blk_offset + i)], in_q[2 * (blk_offset + i) + 1]);
    }
    for (const auto* m : {&d, &q})
      for (const auto& v : *m)
        if (!std::isfinite(v.real()) || !std::isfinite(v.imag())) throw InvalidArgument("nonfinite PAW projector/D/Q data");
    // row-major d[i*np + j] = D(i,j); Hermitian check and symmetrisation.
    std::vector<C> dd(np * np), qd(np * np);
    for (std::size_t i = 0; i < np; ++i)
      for (std::size_t j = 0; j < np; ++j) {
        dd[i * np + j] = d[i * np + j] - std::conj(d[j * np + i]);
        qd[i * np + j] = q[i * np + j] - std::conj(q[j * np + i]);
      }
    const double de = frobenius(dd), qe = frobenius(qd);
    if (de > 1e-10 * std::max(1., frobenius(d)) || qe > 1e-10 * std::max(1., frobenius(q))) {
      std::ostringstream reason;
      reason << "invalid Hermitian PAW blocks: atom=" << a << " D_norm=" << frobenius(d) << " D_asymmetry=" << de
             << " Q_norm=" << frobenius(q) << " Q_asymmetry=" << qe;
      throw InvalidArgument(reason.str());
    }
    // symmetrised, column-major device storage M(i,j) at i + j*np
    for (std::size_t i = 0; i < np; ++i)
      for (std::size_t j = 0; j < np; ++j) {
        const C ds = .5 * (d[i * np + j] + std::conj(d[j * np + i]));
        const C qs = .5 * (q[i * np + j] + std::conj(q[j * np + i]));
        d_blocks[blk_offset + i + j * np] = Cx<double>{ds.real(), ds.imag()};
        q_blocks[blk_offset + i + j * np] = Cx<double>{qs.real(), qs.imag()};
      }
    blk_offset += np * np;
  }
}

}  // namespace

DeviceOperator::DeviceOperator(Context& ctx, const OperatorInput& in) : ctx_(ctx) {
  SDFT_CUDA(cudaSetDevice(ctx.device));
  if (!in.npw || !std::isfinite(in.hartree_to_ev) || in.hartree_to_ev <= 0 || !std::isfinite(in.regularization) ||
      in.regularization < 0)
    throw InvalidArgument("invalid plane-wave operator dimensions or units");
  if (in.npw > static_cast<std::size_t>(std::numeric_limits<int>::max())) throw Overflow("plane-wave count exceeds int32");
  npw_ = static_cast<int>(in.npw);
  regularization_ = in.regularization;
  // Bounding box of the basis (:400-415).
  int low[3], high[3];
  for (int a = 0; a < 3; ++a) low[a] = high[a] = in.hkl[a];
  for (std::size_t g = 0; g < in.npw; ++g)
    for (int a = 0; a < 3; ++a) {
      low[a] = std::min(low[a], in.hkl[3 * g + a]);
      high[a] = std::max(high[a], in.hkl[3 * g + a]);
    }
  for (int a = 0; a < 3; ++a) span_[a] = high[a] - low[a];
  LocalPotential local = local_potential(ctx, span_, in.potential_count, in.potential_hkl, in.potential);
  const int* shape = local.shape;
  h_local_real_ = std::move(local.real);
  auto wrap = [](int x, int size) {
    int r = x % size;
    return r < 0 ? r + size : r;
  };
  auto index = [&](int h, int k, int l) {
    return (static_cast<std::uint64_t>(wrap(h, shape[0])) * shape[1] + wrap(k, shape[1])) * shape[2] + wrap(l, shape[2]);
  };
  // Basis maps and diagonals (:476-483).
  h_indices_.resize(in.npw);
  h_kinetic_.resize(in.npw);
  h_diag_.resize(in.npw);
  s_diag_.assign(in.npw, 1 + regularization_);
  for (std::size_t g = 0; g < in.npw; ++g) {
    if (!std::isfinite(in.kinetic_ev[g])) throw InvalidArgument("nonfinite kinetic energy");
    h_indices_[g] = index(in.hkl[3 * g], in.hkl[3 * g + 1], in.hkl[3 * g + 2]);
    h_kinetic_[g] = in.kinetic_ev[g] / in.hartree_to_ev;
    h_diag_[g] = in.kinetic_ev[g] / in.hartree_to_ev + local.v0;
  }
  {
    auto sorted = h_indices_;
    std::sort(sorted.begin(), sorted.end());
    if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
      throw InvalidArgument("duplicate plane-wave index");
  }
  // PAW blocks (:484-509): validate, symmetrise, diagonals, concatenated B.
  if (in.atoms > static_cast<std::size_t>(std::numeric_limits<int>::max())) throw Overflow("too many atoms");
  atoms_ = static_cast<int>(in.atoms);
  std::vector<int> offsets(atoms_ + 1, 0);
  std::vector<long long> storage(atoms_, 0);
  std::size_t total = 0, block_total = 0;
  for (int a = 0; a < atoms_; ++a) {
    const std::size_t np = in.projectors[a];
    if (!np || np > 256) throw InvalidArgument("invalid PAW low-rank operator dimensions");
    offsets[a] = static_cast<int>(total);
    storage[a] = static_cast<long long>(block_total);
    total += np;
    block_total += np * np;
    max_block_ = std::max<int>(max_block_, static_cast<int>(np));
  }
  offsets[atoms_] = static_cast<int>(total);
  if (total > 65536) throw InvalidArgument("too many PAW projectors");
  np_ = static_cast<int>(total);
  h_channels_.assign(in.projectors, in.projectors + in.atoms);
  std::vector<Cx<double>> d_blocks, q_blocks;
  symmetrised_blocks(h_channels_, in.d, in.q, d_blocks, q_blocks);
  // Device upload.
  upload_common(shape, d_blocks, q_blocks, offsets, storage);
  if (np_) {
    // B: the row-major per-atom amplitudes (the input layout) are uploaded as
    // they are, checked and transposed on the device into the column-major
    // Sigma_np x NPW matrix; the diagonals' PAW terms Re(b_g^H D b_g) and
    // Re(b_g^H Q b_g) are summed on the device in the host order (atoms, rows,
    // columns) with unfused products.
    const std::size_t entries = static_cast<std::size_t>(np_) * npw_;
    const cudaStream_t st = ctx.stream;
    Cx<double>* raw = static_cast<Cx<double>*>(stream_alloc(sizeof(Cx<double>) * entries, st));
    SDFT_CUDA(cudaMemcpyAsync(raw, in.amplitudes, sizeof(Cx<double>) * entries, cudaMemcpyHostToDevice, st));
    b_ = static_cast<Cx<double>*>(stream_alloc(sizeof(Cx<double>) * entries, st));
    double* diag = static_cast<double*>(stream_alloc(sizeof(double) * 2 * npw_ + 16, st));
    unsigned int* flag = reinterpret_cast<unsigned int*>(diag + 2 * npw_);
    SDFT_CUDA(cudaMemcpyAsync(diag, h_diag_.data(), sizeof(double) * npw_, cudaMemcpyHostToDevice, st));
    SDFT_CUDA(cudaMemcpyAsync(diag + npw_, s_diag_.data(), sizeof(double) * npw_, cudaMemcpyHostToDevice, st));
    SDFT_CUDA(cudaMemsetAsync(flag, 0, sizeof(unsigned int), st));
    paw_prepare(raw, np_, npw_, atoms_, block_offsets_, block_storage_, d_, q_, b_, diag, diag + npw_, flag,
                ctx.stream);
    unsigned int bad = 0;
    SDFT_CUDA(cudaMemcpyAsync(&bad, flag, sizeof(bad), cudaMemcpyDeviceToHost, ctx.stream));
    SDFT_CUDA(cudaMemcpyAsync(h_diag_.data(), diag, sizeof(double) * npw_, cudaMemcpyDeviceToHost, ctx.stream));
    SDFT_CUDA(cudaMemcpyAsync(s_diag_.data(), diag + npw_, sizeof(double) * npw_, cudaMemcpyDeviceToHost,
                              ctx.stream));
    SDFT_CUDA(cudaStreamSynchronize(ctx.stream));
    stream_free(raw, st);
    stream_free(diag, st);
    if (bad) throw InvalidArgument("nonfinite PAW projector/D/Q data");
    const Split split = search_split();
    pack_persistent(Op::N, b_, np_, np_, npw_, split, b_packed_, ctx.stream);
    pack_persistent(Op::C, b_, np_, npw_, np_, split, bh_packed_, ctx.stream);
  }
  SDFT_CUDA(cudaStreamSynchronize(ctx.stream));
}

namespace {
// Stream-ordered pool memory on `stream`; a pageable host source has been
// staged when the copy call returns, so it may go out of scope.
template <typename T>
void upload_array(T*& dst, const std::vector<T>& src, cudaStream_t stream) {
  dst = static_cast<T*>(stream_alloc(sizeof(T) * std::max<std::size_t>(1, src.size()), stream));
  if (!src.empty())
    SDFT_CUDA(cudaMemcpyAsync(dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, stream));
}
}  // namespace

void DeviceOperator::upload_common(const int shape[3], const std::vector<Cx<double>>& d_blocks,
                                   const std::vector<Cx<double>>& q_blocks, const std::vector<int>& offsets,
                                   const std::vector<long long>& storage) {
  plan_.build(shape, h_indices_, ctx_.stream);
  upload_array(kinetic_, h_kinetic_, ctx_.stream);
  upload_array(v64_, h_local_real_, ctx_.stream);
  std::vector<float> v32(h_local_real_.begin(), h_local_real_.end());
  upload_array(v32_, v32, ctx_.stream);
  if (np_) {
    upload_array(d_, d_blocks, ctx_.stream);
    upload_array(q_, q_blocks, ctx_.stream);
    upload_array(block_offsets_, offsets, ctx_.stream);
    upload_array(block_storage_, storage, ctx_.stream);
  }
}

// From a snapshot (the reference's load_solver_snapshot,
// src/plane_wave_operator.cpp:571-653): the arrays are the operator's own, so
// nothing is rebuilt; B is already column-major Sigma_np x NPW.
DeviceOperator::DeviceOperator(Context& ctx, const OperatorSnapshot& snap) : ctx_(ctx) {
  SDFT_CUDA(cudaSetDevice(ctx.device));
  if (snap.npw > static_cast<std::size_t>(std::numeric_limits<int>::max()) || snap.projectors > 65536 ||
      snap.channels.size() > static_cast<std::size_t>(std::numeric_limits<int>::max()))
    throw Overflow("solver snapshot dimensions exceed the device operator's limits");
  npw_ = static_cast<int>(snap.npw);
  regularization_ = snap.regularization;
  h_indices_ = snap.indices;
  h_kinetic_ = snap.kinetic;
  h_diag_ = snap.h_diagonal;
  s_diag_ = snap.s_diagonal;
  h_local_real_ = snap.local_real;
  atoms_ = static_cast<int>(snap.channels.size());
  std::vector<int> offsets(atoms_ + 1, 0);
  std::vector<long long> storage(atoms_, 0);
  std::size_t total = 0, block_total = 0;
  for (int a = 0; a < atoms_; ++a) {
    const std::size_t np = snap.channels[a];
    if (!np || np > 256) throw InvalidArgument("invalid PAW low-rank operator dimensions");
    offsets[a] = static_cast<int>(total);
    storage[a] = static_cast<long long>(block_total);
    total += np;
    block_total += np * np;
    max_block_ = std::max<int>(max_block_, static_cast<int>(np));
  }
  offsets[atoms_] = static_cast<int>(total);
  np_ = static_cast<int>(total);
  upload_common(snap.shape, snap.d, snap.q, offsets, storage);
  if (np_) {
    upload_array(b_, snap.all_b, ctx_.stream);
    const Split split = search_split();
    pack_persistent(Op::N, b_, np_, np_, npw_, split, b_packed_, ctx.stream);
    pack_persistent(Op::C, b_, np_, npw_, np_, split, bh_packed_, ctx.stream);
  }
  SDFT_CUDA(cudaStreamSynchronize(ctx.stream));
}

// SCF refresh: new V(G) and per-atom D/Q on the resident basis maps, plan,
// B and its tensor-core packing. The reference rebuilds the operator each SCF
// iteration and keeps only B's device copy through an immutable projector
// identity (src/scf_core.cpp:2312-2313, src/plane_wave_operator.cpp:395-397);
// here everything that depends on the basis and B stays, and the potential,
// blocks and diagonals are recomputed with the constructor's own checks and
// arithmetic. All validation happens before any state changes.
void DeviceOperator::update(std::size_t potential_count, const int* potential_hkl, const double* potential,
                            const double* d, const double* q) {
  if (span_[0] < 0)
    throw InvalidArgument("operator built from a solver snapshot has no G components; create a new operator");
  if (potential_count && (!potential_hkl || !potential)) throw InvalidArgument("null potential arrays");
  if (atoms_ && (!d || !q)) throw InvalidArgument("null PAW arrays");
  SDFT_CUDA(cudaSetDevice(ctx_.device));
  SDFT_CUDA(cudaStreamSynchronize(ctx_.stream));
  LocalPotential local = local_potential(ctx_, span_, potential_count, potential_hkl, potential);
  for (int a = 0; a < 3; ++a)
    if (local.shape[a] != plan_.n[a])
      throw InvalidArgument("SDFT_FFT_GRID changed the FFT grid since the operator was created; create a new operator");
  std::vector<Cx<double>> d_blocks, q_blocks;
  symmetrised_blocks(h_channels_, d, q, d_blocks, q_blocks);
  std::vector<double> h_diag(npw_), s_diag(npw_, 1 + regularization_);
  for (int g = 0; g < npw_; ++g) h_diag[g] = h_kinetic_[g] + local.v0;
  std::vector<float> v32(local.real.begin(), local.real.end());
  SDFT_CUDA(cudaMemcpyAsync(v64_, local.real.data(), sizeof(double) * local.real.size(), cudaMemcpyHostToDevice,
                            ctx_.stream));
  SDFT_CUDA(cudaMemcpyAsync(v32_, v32.data(), sizeof(float) * v32.size(), cudaMemcpyHostToDevice, ctx_.stream));
  if (np_) {
    SDFT_CUDA(cudaMemcpyAsync(d_, d_blocks.data(), sizeof(Cx<double>) * d_blocks.size(), cudaMemcpyHostToDevice,
                              ctx_.stream));
    SDFT_CUDA(cudaMemcpyAsync(q_, q_blocks.data(), sizeof(Cx<double>) * q_blocks.size(), cudaMemcpyHostToDevice,
                              ctx_.stream));
    auto* diag = static_cast<double*>(ctx_.staging_aux.reserve(sizeof(double) * 2 * npw_));
    SDFT_CUDA(cudaMemcpyAsync(diag, h_diag.data(), sizeof(double) * npw_, cudaMemcpyHostToDevice, ctx_.stream));
    SDFT_CUDA(cudaMemcpyAsync(diag + npw_, s_diag.data(), sizeof(double) * npw_, cudaMemcpyHostToDevice, ctx_.stream));
    paw_diagonals(b_, 1, static_cast<std::size_t>(np_), npw_, atoms_, block_offsets_, block_storage_, d_, q_, diag,
                  diag + npw_, ctx_.stream);
    SDFT_CUDA(cudaMemcpyAsync(h_diag.data(), diag, sizeof(double) * npw_, cudaMemcpyDeviceToHost, ctx_.stream));
    SDFT_CUDA(cudaMemcpyAsync(s_diag.data(), diag + npw_, sizeof(double) * npw_, cudaMemcpyDeviceToHost, ctx_.stream));
  }
  SDFT_CUDA(cudaStreamSynchronize(ctx_.stream));
  h_local_real_ = std::move(local.real);
  h_diag_ = std::move(h_diag);
  s_diag_ = std::move(s_diag);
  signature_ready_ = false;  // Q changed
}

namespace {
__global__ void clamped_root_columns_kernel(Cx<double>* __restrict__ v, int m, const double* __restrict__ lambda) {
  const long long total = static_cast<long long>(m) * m;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const double s = sqrt(fmax(lambda[i / m], 0.0));
    v[i] = Cx<double>{v[i].re * s, v[i].im * s};
  }
}

__global__ void shift_diagonal_kernel(Cx<double>* __restrict__ a, int m, double shift) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) a[i + static_cast<long long>(i) * m].re += shift;
}

// Ascending eigenvalues and eigenvectors (the lowest `wanted` of each) of
// the Hermitian m x m matrix a (lower triangle, ld m; overwritten) by cuSOLVER
// zheevd: a once-per-operator set-up step whose matrices (the projector Gram
// of a symmetric cell) carry large, nearly degenerate clusters.
void hermitian_eigen(Context& ctx, Cx<double>* a, int m, int wanted, double* values, Cx<double>* vectors) {
  int lwork = 0;
  auto* az = reinterpret_cast<cuDoubleComplex*>(a);
  auto* w = static_cast<double*>(ctx.eigen.product2.reserve(sizeof(double) * m));
  if (cusolverDnZheevd_bufferSize(ctx.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, az, m, w, &lwork) !=
      CUSOLVER_STATUS_SUCCESS)
    throw CudaError("cuSOLVER error in zheevd_bufferSize");
  auto* work = static_cast<cuDoubleComplex*>(
      ctx.eigen.solver_work.reserve(sizeof(cuDoubleComplex) * std::max(1, lwork) + sizeof(int)));
  int* info = reinterpret_cast<int*>(work + std::max(1, lwork));
  if (cusolverDnZheevd(ctx.solver, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, m, az, m, w, work, lwork, info) !=
      CUSOLVER_STATUS_SUCCESS)
    throw CudaError("cuSOLVER error in zheevd");
  int host_info = 0;
  SDFT_CUDA(cudaMemcpyAsync(&host_info, info, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
  SDFT_CUDA(cudaStreamSynchronize(ctx.stream));
  if (host_info) throw std::runtime_error("original PAW Gram decomposition failed");
  SDFT_CUDA(cudaMemcpyAsync(values, w, sizeof(double) * wanted, cudaMemcpyDeviceToDevice, ctx.stream));
  if (vectors != a) copy_block(a, m, vectors, m, m, wanted, ctx.stream);
}
}  // namespace

// The reference's overlap() signature (src/plane_wave_operator.cpp:702-717),
// FP64 on the device: Gram = B B^H; its eigendecomposition U diag(l) U^H;
// R = W U^H with W = U diag(sqrt(max(l, 0))); the lowest eigenvalue of
// (1+reg) I + R (Q R), the per-atom Q product compensated as in the applies.
const MetricSignature& DeviceOperator::metric_signature() {
  if (signature_ready_) return signature_;
  MetricSignature sig;
  sig.minimum = 1.0 + regularization_;
  if (np_ > 0) {
    SDFT_CUDA(cudaSetDevice(ctx_.device));
    const cudaStream_t st = ctx_.stream;
    const std::size_t pp = static_cast<std::size_t>(np_) * np_;
    auto* gram = static_cast<Cx<double>*>(ctx_.davidson.rr_a.reserve(sizeof(Cx<double>) * pp * 2));
    Cx<double>* herm = gram + pp;
    auto* root = static_cast<Cx<double>*>(ctx_.davidson.rr_b.reserve(sizeof(Cx<double>) * pp * 2));
    Cx<double>* qroot = root + pp;
    auto* values = static_cast<double*>(ctx_.davidson.rr_w.reserve(sizeof(double) * np_));
    zgemm(ctx_.blas, Op::N, Op::C, np_, np_, npw_, b_, np_, b_, np_, gram, np_, false);
    hermitian_part(gram, np_, herm, np_, np_, st);
    hermitian_eigen(ctx_, herm, np_, np_, values, gram);
    const unsigned blocks = static_cast<unsigned>(std::min<std::size_t>(ceil_div(pp, 256), 148 * 8));
    clamped_root_columns_kernel<<<blocks, 256, 0, st>>>(gram, np_, values);
    SDFT_LAUNCH("clamped_root_columns_kernel");
    zgemm(ctx_.blas, Op::N, Op::C, np_, np_, np_, gram, np_, herm, np_, root, np_, false);  // W U^H
    block_product(atoms_, block_offsets_, block_storage_, max_block_, q_, root, np_, np_, qroot, np_, st);
    zgemm(ctx_.blas, Op::N, Op::N, np_, np_, np_, root, np_, qroot, np_, gram, np_, false);
    shift_diagonal_kernel<<<static_cast<unsigned>(ceil_div(np_, 256)), 256, 0, st>>>(gram, np_,
                                                                                     1.0 + regularization_);
    SDFT_LAUNCH("shift_diagonal_kernel");
    hermitian_part(gram, np_, herm, np_, np_, st);
    double lowest = 0.0;
    if (np_ == 1) {
      Cx<double> one;
      SDFT_CUDA(cudaMemcpyAsync(&one, herm, sizeof(one), cudaMemcpyDeviceToHost, st));
      SDFT_CUDA(cudaStreamSynchronize(st));
      lowest = one.re;
    } else {
      hermitian_eigen(ctx_, herm, np_, 1, values, root);
      SDFT_CUDA(cudaMemcpyAsync(&lowest, values, sizeof(double), cudaMemcpyDeviceToHost, st));
      SDFT_CUDA(cudaStreamSynchronize(st));
    }
    if (!std::isfinite(lowest)) throw std::runtime_error("original PAW overlap signature failed");
    sig.minimum = std::min(sig.minimum, lowest);
  }
  sig.indefinite = sig.minimum < -1e-10;
  sig.singular = std::abs(sig.minimum) <= 1e-10;
  signature_ = sig;
  signature_ready_ = true;
  return signature_;
}

void DeviceOperator::require_positive_metric() {
  const MetricSignature& sig = metric_signature();
  if (sig.singular) throw std::runtime_error("original PAW overlap is numerically singular");
  if (sig.indefinite)
    throw Unsupported("original PAW overlap is indefinite: the reference solves this pencil with its "
                      "indefinite-metric Davidson, which this library does not provide");
}

DeviceOperator::~DeviceOperator() {
  plan_.release();
  release(b_packed_);
  release(bh_packed_);
  for (void* p : {static_cast<void*>(kinetic_), static_cast<void*>(v64_), static_cast<void*>(v32_),
                  static_cast<void*>(b_), static_cast<void*>(d_), static_cast<void*>(q_),
                  static_cast<void*>(block_offsets_), static_cast<void*>(block_storage_)})
    stream_free(p, ctx_.stream);
}

std::size_t DeviceOperator::device_bytes() const {
  std::size_t bytes = plan_.count * (sizeof(double) + sizeof(float)) + npw_ * (sizeof(double) + 2 * sizeof(int));
  bytes += static_cast<std::size_t>(np_) * npw_ * sizeof(Cx<double>);
  bytes += sizeof(std::uint16_t) * static_cast<std::size_t>(b_packed_.ld * b_packed_.rows + bh_packed_.ld * bh_packed_.rows);
  return bytes;
}

void DeviceOperator::local_part(const Cx<double>* x, int columns, Cx<double>* y, Precision precision) {
  if (precision == Precision::FP64) {
    auto* slab = static_cast<Cx<double>*>(ctx_.slab64.reserve(sizeof(Cx<double>) * plan_.slab_elements(columns)));
    local_hamiltonian<double>(plan_, x, npw_, columns, v64_, kinetic_, y, npw_, slab, ctx_.stream);
  } else {
    auto* slab = static_cast<Cx<float>*>(ctx_.slab32.reserve(sizeof(Cx<float>) * plan_.slab_elements(columns)));
    local_hamiltonian<float>(plan_, x, npw_, columns, v32_, kinetic_, y, npw_, slab, ctx_.stream);
  }
}

void DeviceOperator::project(const Cx<double>* x, int columns, Cx<double>* p, Precision precision) {
  if (!np_) throw InvalidArgument("invalid PAW projection buffers");
  if (precision == Precision::FP64)
    zgemm(ctx_.blas, Op::N, Op::N, np_, columns, npw_, b_, np_, x, npw_, p, np_, false);
  else
    gemm_tc(Op::N, np_, columns, npw_, b_, np_, &b_packed_, x, npw_, p, np_, false, 1.0, b_packed_.split, ctx_.tc,
            ctx_.stream);
}

void DeviceOperator::backproject(const Cx<double>* dp, int columns, Cx<double>* y, Precision precision) {
  if (precision == Precision::FP64)
    zgemm(ctx_.blas, Op::C, Op::N, npw_, columns, np_, b_, np_, dp, np_, y, npw_, true);
  else
    gemm_tc(Op::C, npw_, columns, np_, b_, np_, &bh_packed_, dp, np_, y, npw_, true, 1.0, bh_packed_.split, ctx_.tc,
            ctx_.stream);
}

void DeviceOperator::paw_add(const Cx<double>* p, int columns, bool overlap, Cx<double>* y, Precision precision) {
  auto* dp = static_cast<Cx<double>*>(ctx_.onsite.reserve(sizeof(Cx<double>) * static_cast<std::size_t>(np_) * columns));
  block_product(atoms_, block_offsets_, block_storage_, max_block_, overlap ? q_ : d_, p, np_, columns, dp, np_,
                ctx_.stream);
  backproject(dp, columns, y, precision);
}

void DeviceOperator::apply_hamiltonian(const Cx<double>* x, int columns, Cx<double>* y, Precision precision) {
  if (columns <= 0 || !x || !y || x == y) throw InvalidArgument("invalid direct plane-wave input/output buffers");
  local_part(x, columns, y, precision);
  if (np_) {
    auto* p = static_cast<Cx<double>*>(ctx_.projections.reserve(sizeof(Cx<double>) * static_cast<std::size_t>(np_) * columns));
    project(x, columns, p, precision);
    paw_add(p, columns, false, y, precision);
  }
}

void DeviceOperator::apply_overlap(const Cx<double>* x, int columns, Cx<double>* y, Precision precision) {
  if (columns <= 0 || !x || !y || x == y) throw InvalidArgument("invalid direct plane-wave input/output buffers");
  scale_copy(x, npw_, y, npw_, npw_, columns, 1.0 + regularization_, ctx_.stream);
  if (np_) {
    auto* p = static_cast<Cx<double>*>(ctx_.projections.reserve(sizeof(Cx<double>) * static_cast<std::size_t>(np_) * columns));
    project(x, columns, p, precision);
    paw_add(p, columns, true, y, precision);
  }
}

void DeviceOperator::apply_shifted(const Cx<double>* x, int columns, const double* shift, Cx<double>* y,
                                   Precision precision) {
  if (columns <= 0 || !x || !y || !shift || x == y) throw InvalidArgument("invalid shifted plane-wave buffers");
  local_part(x, columns, y, precision);
  shifted_axpy(x, npw_, y, npw_, npw_, columns, shift, 1.0 + regularization_, ctx_.stream);
  if (np_) {
    const std::size_t pc = static_cast<std::size_t>(np_) * columns;
    auto* p = static_cast<Cx<double>*>(ctx_.projections.reserve(sizeof(Cx<double>) * pc));
    auto* dp = static_cast<Cx<double>*>(ctx_.onsite.reserve(sizeof(Cx<double>) * pc));
    project(x, columns, p, precision);
    shifted_block_product(atoms_, block_offsets_, block_storage_, max_block_, d_, q_, shift, p, np_, columns, dp,
                          np_, ctx_.stream);
    backproject(dp, columns, y, precision);
  }
}

void DeviceOperator::apply_pair(const Cx<double>* x, int columns, Cx<double>* hy, Cx<double>* sy, Precision precision) {
  if (columns <= 0 || !x || !hy || !sy || x == hy || x == sy || hy == sy)
    throw InvalidArgument("invalid joint plane-wave input/output buffers");
  local_part(x, columns, hy, precision);
  scale_copy(x, npw_, sy, npw_, npw_, columns, 1.0 + regularization_, ctx_.stream);
  if (np_) {
    auto* p = static_cast<Cx<double>*>(ctx_.projections.reserve(sizeof(Cx<double>) * static_cast<std::size_t>(np_) * columns));
    project(x, columns, p, precision);  // one B x shared by H and S
    paw_add(p, columns, false, hy, precision);
    paw_add(p, columns, true, sy, precision);
  }
}

}  // namespace sdft_b200
