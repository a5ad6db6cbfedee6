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
}  // namespace

Context::Context(int dev, cudaStream_t s) : device(dev), stream(s) {
  SDFT_CUDA(cudaSetDevice(device));
  if (!stream) {
    SDFT_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    owns_stream = true;
  }
  check_blas(cublasCreate(&blas), "cublasCreate");
  check_blas(cublasSetStream(blas, stream), "cublasSetStream");
  check_blas(cublasSetMathMode(blas, CUBLAS_DEFAULT_MATH), "cublasSetMathMode");  // true FP64, no TF32
  check_solver(cusolverDnCreate(&solver), "cusolverDnCreate");
  check_solver(cusolverDnSetStream(solver, stream), "cusolverDnSetStream");
}

Context::~Context() {
  if (solver) cusolverDnDestroy(solver);
  if (blas) cublasDestroy(blas);
  for (Scratch* s : {&slab32, &slab64, &staging_in, &staging_out, &staging_aux, &projections, &onsite, &tc.a, &tc.b,
                     &tc.partial})
    s->release();
  if (owns_stream && stream) cudaStreamDestroy(stream);
}

void Context::synchronize() const { SDFT_CUDA(cudaStreamSynchronize(stream)); }

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

DeviceOperator::DeviceOperator(Context& ctx, const OperatorInput& in) : ctx_(ctx) {
  SDFT_CUDA(cudaSetDevice(ctx.device));
  if (!in.npw || !std::isfinite(in.hartree_to_ev) || in.hartree_to_ev <= 0 || !std::isfinite(in.regularization) ||
      in.regularization < 0)
    throw InvalidArgument("invalid plane-wave operator dimensions or units");
  if (in.npw > static_cast<std::size_t>(std::numeric_limits<int>::max())) throw Overflow("plane-wave count exceeds int32");
  npw_ = static_cast<int>(in.npw);
  regularization_ = in.regularization;
  // Bounding box of the basis and the retained potential radius (:400-415).
  int low[3], high[3], radius[3] = {0, 0, 0};
  for (int a = 0; a < 3; ++a) low[a] = high[a] = in.hkl[a];
  for (std::size_t g = 0; g < in.npw; ++g)
    for (int a = 0; a < 3; ++a) {
      low[a] = std::min(low[a], in.hkl[3 * g + a]);
      high[a] = std::max(high[a], in.hkl[3 * g + a]);
    }
  double max_potential = 0;
  std::unordered_map<std::uint64_t, std::size_t> keys;
  keys.reserve(in.potential_count * 2 + 1);
  for (std::size_t i = 0; i < in.potential_count; ++i) {
    const C v(in.potential[2 * i], in.potential[2 * i + 1]);
    if (!std::isfinite(v.real()) || !std::isfinite(v.imag())) throw InvalidArgument("nonfinite local potential");
    const int* k = in.potential_hkl + 3 * i;
    bool retained = true;
    for (int a = 0; a < 3; ++a) retained &= std::abs(k[a]) <= high[a] - low[a];
    if (retained)
      for (int a = 0; a < 3; ++a) radius[a] = std::max(radius[a], std::abs(k[a]));
    max_potential = std::max(max_potential, std::abs(v));
    keys[pack_key(k[0], k[1], k[2])] = i;
  }
  // Hermitian V(G) (:438-444).
  for (std::size_t i = 0; i < in.potential_count; ++i) {
    const int* k = in.potential_hkl + 3 * i;
    const C v(in.potential[2 * i], in.potential[2 * i + 1]);
    const auto other = keys.find(pack_key(-k[0], -k[1], -k[2]));
    const C partner = other == keys.end() ? C{} : C(in.potential[2 * other->second], in.potential[2 * other->second + 1]);
    if (std::abs(v - std::conj(partner)) > 1e-10 * std::max(1., max_potential))
      throw InvalidArgument("local Fourier potential is not Hermitian");
  }
  // Grid rule (:445-457): alias-free minimum, rounded to a 2/3/5/7-smooth length.
  // SDFT_FFT_GRID=minimal keeps the minimum when it is smooth; the device FFT
  // only has smooth lengths, and every alias-free grid gives the same operator.
  const char* mode = std::getenv("SDFT_FFT_GRID");
  if (mode && std::string(mode) != "minimal" && std::string(mode) != "fast")
    throw InvalidArgument("SDFT_FFT_GRID must be minimal or fast");
  int shape[3];
  std::size_t count = 1;
  for (int a = 0; a < 3; ++a) {
    const int minimum = std::max(3, 2 * std::max(radius[a], high[a] - low[a]) + 1);
    shape[a] = (mode && std::string(mode) == "minimal" && fft_length_supported(minimum)) ? minimum
                                                                                          : fast_fft_length(minimum);
    if (count > std::numeric_limits<std::size_t>::max() / shape[a]) throw Overflow("plane-wave FFT grid overflow");
    count *= shape[a];
  }
  auto wrap = [](int x, int size) {
    int r = x % size;
    return r < 0 ? r + size : r;
  };
  auto index = [&](int h, int k, int l) {
    return (static_cast<std::uint64_t>(wrap(h, shape[0])) * shape[1] + wrap(k, shape[1])) * shape[2] + wrap(l, shape[2]);
  };
  // V(r) by one backward FFT of the retained keys, on the device in FP64 (:464-475).
  {
    std::vector<Cx<double>> grid(count, Cx<double>{0, 0});
    for (std::size_t i = 0; i < in.potential_count; ++i) {
      const int* k = in.potential_hkl + 3 * i;
      bool retained = true;
      for (int a = 0; a < 3; ++a) retained &= std::abs(k[a]) <= high[a] - low[a];
      if (!retained) continue;
      grid[index(k[0], k[1], k[2])] = Cx<double>{in.potential[2 * i], in.potential[2 * i + 1]};
    }
    Cx<double>* dgrid = nullptr;
    SDFT_CUDA(cudaMalloc(&dgrid, sizeof(Cx<double>) * count));
    try {
      SDFT_CUDA(cudaMemcpyAsync(dgrid, grid.data(), sizeof(Cx<double>) * count, cudaMemcpyHostToDevice, ctx.stream));
      fft3d<double>(dgrid, shape, 1, true, ctx.stream);
      SDFT_CUDA(cudaMemcpyAsync(grid.data(), dgrid, sizeof(Cx<double>) * count, cudaMemcpyDeviceToHost, ctx.stream));
      SDFT_CUDA(cudaStreamSynchronize(ctx.stream));
    } catch (...) {
      cudaFree(dgrid);
      throw;
    }
    cudaFree(dgrid);
    h_local_real_.resize(count);
    for (std::size_t i = 0; i < count; ++i) {
      if (std::abs(grid[i].im) > 1e-9 * std::max(1., std::abs(grid[i].re)))
        throw std::runtime_error("complex real-space local potential");
      h_local_real_[i] = grid[i].re;
    }
  }
  // Basis maps and diagonals (:476-483).
  const auto zero = keys.find(pack_key(0, 0, 0));
  const double v0 = zero == keys.end() ? 0.0 : in.potential[2 * zero->second];
  h_indices_.resize(in.npw);
  h_kinetic_.resize(in.npw);
  h_diag_.resize(in.npw);
  s_diag_.assign(in.npw, 1 + regularization_);
  for (std::size_t g = 0; g < in.npw; ++g) {
    if (!std::isfinite(in.kinetic_ev[g])) throw InvalidArgument("nonfinite kinetic energy");
    h_indices_[g] = index(in.hkl[3 * g], in.hkl[3 * g + 1], in.hkl[3 * g + 2]);
    h_kinetic_[g] = in.kinetic_ev[g] / in.hartree_to_ev;
    h_diag_[g] = in.kinetic_ev[g] / in.hartree_to_ev + v0;
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
  std::vector<Cx<double>> all_b(static_cast<std::size_t>(np_) * in.npw), d_blocks(block_total), q_blocks(block_total);
  {
    std::size_t amp_offset = 0, blk_offset = 0;
    for (int a = 0; a < atoms_; ++a) {
      const std::size_t np = in.projectors[a];
      std::vector<C> b(np * in.npw), d(np * np), q(np * np);
      for (std::size_t i = 0; i < np * in.npw; ++i)
        b[i] = C(in.amplitudes[2 * (amp_offset + i)], in.amplitudes[2 * (amp_offset + i) + 1]);
      for (std::size_t i = 0; i < np * np; ++i) {
        d[i] = C(in.d[2 * (blk_offset + i)], in.d[2 * (blk_offset + i) + 1]);
        q[i] = C(in.q[2 * (blk_offset + i)], in.q[2 * (blk_offset + i) + 1]);
      }
      for (const auto& v : b)
        if (!std::isfinite(v.real()) || !std::isfinite(v.imag())) throw InvalidArgument("nonfinite PAW projector/D/Q data");
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
      std::vector<C> ds(np * np), qs(np * np);  // symmetrised, (i,j) row-major
      for (std::size_t i = 0; i < np; ++i)
        for (std::size_t j = 0; j < np; ++j) {
          ds[i * np + j] = .5 * (d[i * np + j] + std::conj(d[j * np + i]));
          qs[i * np + j] = .5 * (q[i * np + j] + std::conj(q[j * np + i]));
        }
      // column-major device storage, M(i,j) at i + j*np
      for (std::size_t i = 0; i < np; ++i)
        for (std::size_t j = 0; j < np; ++j) {
          d_blocks[blk_offset + i + j * np] = Cx<double>{ds[i * np + j].real(), ds[i * np + j].imag()};
          q_blocks[blk_offset + i + j * np] = Cx<double>{qs[i * np + j].real(), qs[i * np + j].imag()};
        }
      // diagonal contributions Re(b_g^H D b_g), Re(b_g^H Q b_g)
      for (std::size_t g = 0; g < in.npw; ++g) {
        C hd = 0, sd = 0;
        for (std::size_t i = 0; i < np; ++i) {
          C db = 0, qb = 0;
          for (std::size_t j = 0; j < np; ++j) {
            db += ds[i * np + j] * b[j * in.npw + g];
            qb += qs[i * np + j] * b[j * in.npw + g];
          }
          hd += std::conj(b[i * in.npw + g]) * db;
          sd += std::conj(b[i * in.npw + g]) * qb;
        }
        h_diag_[g] += hd.real();
        s_diag_[g] += sd.real();
      }
      for (std::size_t i = 0; i < np; ++i)
        for (std::size_t g = 0; g < in.npw; ++g) {
          const C v = b[i * in.npw + g];
          all_b[(offsets[a] + i) + g * static_cast<std::size_t>(np_)] = Cx<double>{v.real(), v.imag()};
        }
      amp_offset += np * in.npw;
      blk_offset += np * np;
    }
  }
  // Device upload.
  plan_.build(shape, h_indices_);
  auto upload = [&](auto*& dst, const auto& src) {
    using E = typename std::remove_reference_t<decltype(src)>::value_type;
    SDFT_CUDA(cudaMalloc(reinterpret_cast<void**>(&dst), sizeof(E) * std::max<std::size_t>(1, src.size())));
    if (!src.empty()) SDFT_CUDA(cudaMemcpy(dst, src.data(), sizeof(E) * src.size(), cudaMemcpyHostToDevice));
  };
  upload(kinetic_, h_kinetic_);
  upload(v64_, h_local_real_);
  std::vector<float> v32(h_local_real_.begin(), h_local_real_.end());
  upload(v32_, v32);
  if (np_) {
    upload(b_, all_b);
    const Split split = search_split();
    pack_persistent(Op::N, b_, np_, np_, npw_, split, b_packed_, ctx.stream);
    pack_persistent(Op::C, b_, np_, npw_, np_, split, bh_packed_, ctx.stream);
    upload(d_, d_blocks);
    upload(q_, q_blocks);
    upload(block_offsets_, offsets);
    upload(block_storage_, storage);
  }
  SDFT_CUDA(cudaStreamSynchronize(ctx.stream));
}

DeviceOperator::~DeviceOperator() {
  plan_.release();
  release(b_packed_);
  release(bh_packed_);
  for (void* p : {static_cast<void*>(kinetic_), static_cast<void*>(v64_), static_cast<void*>(v32_),
                  static_cast<void*>(b_), static_cast<void*>(d_), static_cast<void*>(q_),
                  static_cast<void*>(block_offsets_), static_cast<void*>(block_storage_)})
    if (p) cudaFree(p);
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
