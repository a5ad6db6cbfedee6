// extern "C" boundary (include/sdft_b200.h): converts exceptions into status
// codes and a thread-local message, and host pointers into staged device copies.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <new>
#include <string>

#include "../../include/sdft_b200.h"
#include "davidson.cuh"
#include "dense.cuh"
#include "eigensolver.cuh"
#include "band_density.cuh"
#include "band_groups.cuh"
#include "paw_density.cuh"
#include "operator.cuh"
#include "rmm_trial.cuh"
#include "server.cuh"
#include "xc_functional.cuh"

struct sdft_b200_context {
  std::unique_ptr<sdft_b200::Context> impl;
};
struct sdft_b200_operator {
  std::unique_ptr<sdft_b200::DeviceOperator> impl;
  std::unique_ptr<sdft_b200::DavidsonSolver> solver;  // workspace reused across solves
  std::unique_ptr<sdft_b200::RmmTrial> rmm;
  std::unique_ptr<sdft_b200::BandGroupSolver> groups;
};

struct sdft_b200_compensation {
  std::unique_ptr<sdft_b200::CompensationCharge> impl;
};
struct sdft_b200_server {
  std::unique_ptr<sdft_b200::SolveServer> impl;
};

namespace {
thread_local std::string last_error;

// Jacobi-Davidson CG steps for a Davidson request: MIXED takes the caller's
// positive count, 0 = SDFT_B200_CORRECTION_STEPS or 6, -1 = the reference's
// single preconditioner step; FP64 keeps the reference's step.
int correction_steps_of(const sdft_b200_davidson_options& o) {
  if (o.correction_steps < -1) throw sdft_b200::InvalidArgument("correction_steps must be -1, 0 or positive");
  if (o.precision != SDFT_B200_PRECISION_MIXED) {
    if (o.correction_steps > 0)
      throw sdft_b200::InvalidArgument("Jacobi-Davidson correction steps apply to the mixed form only");
    return 0;
  }
  if (o.correction_steps < 0) return 0;
  if (o.correction_steps > 0) return std::min(o.correction_steps, 64);
  static const int fallback = [] {
    const char* v = std::getenv("SDFT_B200_CORRECTION_STEPS");
    if (!v) return 6;
    char* end = nullptr;
    const long steps = std::strtol(v, &end, 10);
    if (end == v || *end || steps < 0 || steps > 64)
      throw sdft_b200::InvalidArgument("SDFT_B200_CORRECTION_STEPS must be an integer in [0, 64]");
    return static_cast<int>(steps);
  }();
  return fallback;
}

void copy_stats(const sdft_b200::DavidsonStats& st, sdft_b200_davidson_stats* stats) {
  stats->iterations = static_cast<size_t>(st.iterations);
  stats->converged = st.converged ? 1 : 0;
  stats->max_residual = st.max_residual;
  stats->seconds = st.seconds;
  stats->rayleigh_ritz_seconds = st.rr_seconds;
  stats->h_columns_search = static_cast<size_t>(st.h_columns_search);
  stats->h_columns_fp64 = static_cast<size_t>(st.h_columns_fp64);
  stats->s_columns_search = static_cast<size_t>(st.s_columns_search);
  stats->s_columns_fp64 = static_cast<size_t>(st.s_columns_fp64);
  stats->rayleigh_ritz_calls = st.rayleigh_ritz;
  stats->restarts = st.restarts;
  stats->fp64_refreshes = st.fp64_refreshes;
  stats->certifications = st.certifications;
  stats->handoff_iteration = st.handoff_iteration;
  stats->block_rank_fallbacks = st.block_rank_fallbacks;
  stats->correction_columns = static_cast<size_t>(st.correction_columns);
  stats->polish_steps = st.polish_steps;
  stats->polish_accepted = st.polish_accepted;
  stats->manifold_steps = st.manifold_steps;
  stats->manifold_accepted = st.manifold_accepted;
}

template <typename F>
sdft_b200_status guarded(F&& body) {
  try {
    body();
    return SDFT_B200_OK;
  } catch (const sdft_b200::InvalidArgument& e) {
    last_error = e.what();
    return SDFT_B200_INVALID_ARGUMENT;
  } catch (const std::invalid_argument& e) {
    last_error = e.what();
    return SDFT_B200_INVALID_ARGUMENT;
  } catch (const std::overflow_error& e) {
    last_error = e.what();
    return SDFT_B200_OVERFLOW;
  } catch (const sdft_b200::NonFinite& e) {
    last_error = e.what();
    return SDFT_B200_NONFINITE;
  } catch (const sdft_b200::Unsupported& e) {
    last_error = e.what();
    return SDFT_B200_UNSUPPORTED;
  } catch (const sdft_b200::CudaError& e) {
    last_error = e.what();
    return SDFT_B200_CUDA_ERROR;
  } catch (const std::bad_alloc&) {
    last_error = "out of memory";
    return SDFT_B200_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    last_error = e.what();
    return SDFT_B200_RUNTIME_ERROR;
  } catch (...) {
    last_error = "unknown error";
    return SDFT_B200_RUNTIME_ERROR;
  }
}

using sdft_b200::Cx;
using sdft_b200::Precision;

Precision precision_of(int p) {
  if (p == SDFT_B200_PRECISION_FP64) return Precision::FP64;
  if (p == SDFT_B200_PRECISION_MIXED) return Precision::Mixed;
  throw sdft_b200::InvalidArgument("precision must be SDFT_B200_PRECISION_FP64 or SDFT_B200_PRECISION_MIXED");
}

void require(bool condition, const char* message) {
  if (!condition) throw sdft_b200::InvalidArgument(message);
}

// Stage host data into context scratch (device), or pass device pointers through.
// A pointer the caller declares as device memory must be memory of the
// context's device (device or managed), checked before any launch: a host
// pointer, or another GPU's memory without peer access, would fault a kernel.
void require_device_memory(const void* p, int device, const char* what) {
  cudaPointerAttributes attributes{};
  const cudaError_t code = cudaPointerGetAttributes(&attributes, p);
  if (code != cudaSuccess) {
    cudaGetLastError();  // clear the error the failed query recorded
    throw sdft_b200::InvalidArgument(std::string(what) + " is not a CUDA device pointer");
  }
  const bool on_device = attributes.type == cudaMemoryTypeDevice || attributes.type == cudaMemoryTypeManaged;
  if (!on_device || attributes.device != device)
    throw sdft_b200::InvalidArgument(std::string(what) + " must be device memory of the context's device " +
                                     std::to_string(device));
}

struct Staged {
  sdft_b200::Context& ctx;
  int memory;
  Staged(sdft_b200::Context& c, int m) : ctx(c), memory(m) {
    require(m == SDFT_B200_MEMORY_HOST || m == SDFT_B200_MEMORY_DEVICE, "memory must be host or device");
  }
  const Cx<double>* in(const double* host, std::size_t complex_count, sdft_b200::Scratch& slot) {
    if (memory == SDFT_B200_MEMORY_DEVICE) {
      require_device_memory(host, ctx.device, "input");
      return reinterpret_cast<const Cx<double>*>(host);
    }
    auto* dst = static_cast<Cx<double>*>(slot.reserve(sizeof(Cx<double>) * complex_count));
    SDFT_CUDA(cudaMemcpyAsync(dst, host, sizeof(Cx<double>) * complex_count, cudaMemcpyHostToDevice, ctx.stream));
    return dst;
  }
  Cx<double>* out(double* host, std::size_t complex_count, sdft_b200::Scratch& slot) {
    if (memory == SDFT_B200_MEMORY_DEVICE) {
      require_device_memory(host, ctx.device, "output");
      return reinterpret_cast<Cx<double>*>(host);
    }
    return static_cast<Cx<double>*>(slot.reserve(sizeof(Cx<double>) * complex_count));
  }
  void back(double* host, const Cx<double>* dev, std::size_t complex_count) {
    if (memory == SDFT_B200_MEMORY_DEVICE) return;
    SDFT_CUDA(cudaMemcpyAsync(host, dev, sizeof(Cx<double>) * complex_count, cudaMemcpyDeviceToHost, ctx.stream));
  }
  // rows x cols block with leading dimension ld: only the block's own
  // entries are copied, so entries rows..ld-1 of each host column stay untouched.
  void matrix_in(Cx<double>* dev, const double* host, std::size_t rows, std::size_t cols, std::size_t ld) {
    if (memory == SDFT_B200_MEMORY_DEVICE) return;
    const std::size_t pitch = sizeof(Cx<double>) * ld;
    SDFT_CUDA(cudaMemcpy2DAsync(dev, pitch, host, pitch, sizeof(Cx<double>) * rows, cols, cudaMemcpyHostToDevice,
                                ctx.stream));
  }
  void matrix_back(double* host, const Cx<double>* dev, std::size_t rows, std::size_t cols, std::size_t ld) {
    if (memory == SDFT_B200_MEMORY_DEVICE) return;
    const std::size_t pitch = sizeof(Cx<double>) * ld;
    SDFT_CUDA(cudaMemcpy2DAsync(host, pitch, dev, pitch, sizeof(Cx<double>) * rows, cols, cudaMemcpyDeviceToHost,
                                ctx.stream));
  }
  void finish() {
    if (memory == SDFT_B200_MEMORY_HOST) ctx.synchronize();
  }
};
}  // namespace

extern "C" {

size_t sdft_b200_last_error(char* buffer, size_t length) {
  if (buffer && length) {
    const std::size_t count = std::min(length - 1, last_error.size());
    std::memcpy(buffer, last_error.data(), count);
    buffer[count] = 0;
  }
  return last_error.size();
}

const char* sdft_b200_version(void) { return "sdft_b200 0.1 sm_100a"; }

unsigned long long sdft_b200_kernel_launches(void) { return sdft_b200::launch_count(); }

sdft_b200_status sdft_b200_context_create(int device, void* stream, sdft_b200_context** out) {
  return guarded([&] {
    require(out != nullptr, "null context output");
    auto ctx = std::make_unique<sdft_b200_context>();
    ctx->impl = std::make_unique<sdft_b200::Context>(device, static_cast<cudaStream_t>(stream));
    *out = ctx.release();
  });
}

sdft_b200_status sdft_b200_context_destroy(sdft_b200_context* context) {
  return guarded([&] { delete context; });
}

sdft_b200_status sdft_b200_context_release_memory(sdft_b200_context* context) {
  return guarded([&] {
    require(context != nullptr, "null context");
    SDFT_CUDA(cudaSetDevice(context->impl->device));
    context->impl->release_scratch();
  });
}

sdft_b200_status sdft_b200_context_synchronize(sdft_b200_context* context) {
  return guarded([&] {
    require(context != nullptr, "null context");
    context->impl->synchronize();
  });
}

sdft_b200_status sdft_b200_enumerate_g_vectors(const double reciprocal[9], double cutoff_ev, const double kpoint[3],
                                               double hartree_to_ev, int32_t* hkl, double* cartesian,
                                               double* kinetic_ev, size_t capacity, size_t* count) {
  return guarded([&] {
    require(reciprocal && kpoint && count, "null enumeration argument");
    const auto list = sdft_b200::enumerate_g_vectors(reciprocal, cutoff_ev, kpoint, hartree_to_ev);
    *count = list.kinetic_ev.size();
    if (capacity >= list.kinetic_ev.size()) {
      if (hkl) std::memcpy(hkl, list.hkl.data(), sizeof(int32_t) * list.hkl.size());
      if (cartesian) std::memcpy(cartesian, list.cartesian.data(), sizeof(double) * list.cartesian.size());
      if (kinetic_ev) std::memcpy(kinetic_ev, list.kinetic_ev.data(), sizeof(double) * list.kinetic_ev.size());
    }
  });
}

sdft_b200_status sdft_b200_operator_create(sdft_b200_context* context, size_t npw, const int32_t* hkl,
                                           const double* kinetic_ev, size_t potential_count,
                                           const int32_t* potential_hkl, const double* potential, size_t atoms,
                                           const uint64_t* projectors, const double* amplitudes, const double* d,
                                           const double* q, double hartree_to_ev, double regularization,
                                           sdft_b200_operator** out) {
  return guarded([&] {
    require(context && out && hkl && kinetic_ev, "null operator argument");
    require(!potential_count || (potential_hkl && potential), "null potential arrays");
    require(!atoms || (projectors && amplitudes && d && q), "null PAW arrays");
    sdft_b200::OperatorInput in;
    in.npw = npw;
    in.hkl = hkl;
    in.kinetic_ev = kinetic_ev;
    in.potential_count = potential_count;
    in.potential_hkl = potential_hkl;
    in.potential = potential;
    in.atoms = atoms;
    in.projectors = projectors;
    in.amplitudes = amplitudes;
    in.d = d;
    in.q = q;
    in.hartree_to_ev = hartree_to_ev;
    in.regularization = regularization;
    auto op = std::make_unique<sdft_b200_operator>();
    op->impl = std::make_unique<sdft_b200::DeviceOperator>(*context->impl, in);
    *out = op.release();
  });
}

sdft_b200_status sdft_b200_operator_update(sdft_b200_operator* op, size_t potential_count,
                                           const int32_t* potential_hkl, const double* potential, const double* d,
                                           const double* q) {
  return guarded([&] {
    require(op != nullptr, "null operator");
    op->impl->update(potential_count, potential_hkl, potential, d, q);
  });
}

sdft_b200_status sdft_b200_operator_destroy(sdft_b200_operator* op) {
  return guarded([&] { delete op; });
}

sdft_b200_status sdft_b200_operator_info(const sdft_b200_operator* op, int32_t shape[3], size_t* grid_points,
                                         size_t* projectors, size_t* npw, size_t* active_rows) {
  return guarded([&] {
    require(op != nullptr, "null operator");
    const auto& plan = op->impl->plan();
    if (shape)
      for (int a = 0; a < 3; ++a) shape[a] = plan.n[a];
    if (grid_points) *grid_points = plan.count;
    if (projectors) *projectors = static_cast<size_t>(op->impl->projectors());
    if (npw) *npw = static_cast<size_t>(op->impl->npw());
    if (active_rows) *active_rows = static_cast<size_t>(plan.slots);
  });
}

sdft_b200_status sdft_b200_operator_metric_signature(sdft_b200_operator* op, double* minimum, int* indefinite) {
  return guarded([&] {
    require(op != nullptr, "null operator");
    const auto& sig = op->impl->metric_signature();
    if (minimum) *minimum = sig.minimum;
    if (indefinite) *indefinite = sig.indefinite ? 1 : 0;
    if (sig.singular) throw std::runtime_error("original PAW overlap is numerically singular");
  });
}

sdft_b200_status sdft_b200_apply_local(sdft_b200_operator* op, const double* x, size_t columns, double* y,
                                       int precision, int memory) {
  return guarded([&] {
    require(op && x && y && columns && x != y, "invalid direct plane-wave input/output buffers");
    require(columns <= static_cast<size_t>(INT32_MAX), "too many columns");
    auto& o = *op->impl;
    auto& ctx = o.context();
    SDFT_CUDA(cudaSetDevice(ctx.device));
    const std::size_t n = static_cast<std::size_t>(o.npw()) * columns;
    Staged stage(ctx, memory);
    const auto* dx = stage.in(x, n, ctx.staging_in);
    auto* dy = stage.out(y, n, ctx.staging_out);
    o.apply_local(dx, static_cast<int>(columns), dy, precision_of(precision));
    stage.back(y, dy, n);
    stage.finish();
  });
}

sdft_b200_status sdft_b200_apply_local_noalloc(sdft_b200_operator* op, const double* x, size_t columns, double* y,
                                               int precision) {
  return guarded([&] {
    require(op && x && y && columns && x != y, "invalid direct plane-wave input/output buffers");
    require(columns <= static_cast<size_t>(INT32_MAX), "too many columns");
    auto& o = *op->impl;
    SDFT_CUDA(cudaSetDevice(o.context().device));
    require_device_memory(x, o.context().device, "x");
    require_device_memory(y, o.context().device, "y");
    sdft_b200::apply_local_noalloc(o, reinterpret_cast<const Cx<double>*>(x), static_cast<int>(columns),
                                   reinterpret_cast<Cx<double>*>(y), precision_of(precision));
  });
}

sdft_b200_status sdft_b200_operator_arrays(const sdft_b200_operator* op, uint64_t* indices, double* kinetic,
                                           double* h_diagonal, double* s_diagonal, double* local_potential) {
  return guarded([&] {
    require(op != nullptr, "null operator");
    const auto& o = *op->impl;
    if (indices) std::memcpy(indices, o.indices().data(), sizeof(uint64_t) * o.indices().size());
    if (kinetic) std::memcpy(kinetic, o.kinetic().data(), sizeof(double) * o.kinetic().size());
    if (h_diagonal) std::memcpy(h_diagonal, o.h_diagonal().data(), sizeof(double) * o.h_diagonal().size());
    if (s_diagonal) std::memcpy(s_diagonal, o.s_diagonal().data(), sizeof(double) * o.s_diagonal().size());
    if (local_potential)
      std::memcpy(local_potential, o.local_real().data(), sizeof(double) * o.local_real().size());
  });
}

sdft_b200_status sdft_b200_apply(sdft_b200_operator* op, int which, const double* x, size_t columns, double* y,
                                 int precision, int memory) {
  return guarded([&] {
    require(op && x && y && columns, "invalid direct plane-wave input/output buffers");
    require(x != y, "invalid direct plane-wave input/output buffers");
    require(which == SDFT_B200_HAMILTONIAN || which == SDFT_B200_OVERLAP, "which must be HAMILTONIAN or OVERLAP");
    require(columns <= static_cast<size_t>(INT32_MAX), "too many columns");
    auto& o = *op->impl;
    auto& ctx = o.context();
    SDFT_CUDA(cudaSetDevice(ctx.device));
    const std::size_t n = static_cast<std::size_t>(o.npw()) * columns;
    Staged stage(ctx, memory);
    const auto* dx = stage.in(x, n, ctx.staging_in);
    auto* dy = stage.out(y, n, ctx.staging_out);
    if (which == SDFT_B200_HAMILTONIAN) o.apply_hamiltonian(dx, static_cast<int>(columns), dy, precision_of(precision));
    else o.apply_overlap(dx, static_cast<int>(columns), dy, precision_of(precision));
    stage.back(y, dy, n);
    stage.finish();
  });
}

sdft_b200_status sdft_b200_apply_pair(sdft_b200_operator* op, const double* x, size_t columns, double* hy,
                                      double* sy, int precision, int memory) {
  return guarded([&] {
    require(op && x && hy && sy && columns, "invalid joint plane-wave input/output buffers");
    require(x != hy && x != sy && hy != sy, "invalid joint plane-wave input/output buffers");
    require(columns <= static_cast<size_t>(INT32_MAX), "too many columns");
    auto& o = *op->impl;
    auto& ctx = o.context();
    SDFT_CUDA(cudaSetDevice(ctx.device));
    const std::size_t n = static_cast<std::size_t>(o.npw()) * columns;
    Staged stage(ctx, memory);
    const auto* dx = stage.in(x, n, ctx.staging_in);
    auto* dh = stage.out(hy, n, ctx.staging_out);
    auto* ds = stage.out(sy, n, ctx.staging_aux);
    o.apply_pair(dx, static_cast<int>(columns), dh, ds, precision_of(precision));
    stage.back(hy, dh, n);
    stage.back(sy, ds, n);
    stage.finish();
  });
}

sdft_b200_status sdft_b200_project(sdft_b200_operator* op, const double* x, size_t columns, double* p,
                                   int precision, int memory) {
  return guarded([&] {
    require(op && x && p && columns && x != p, "invalid PAW projection buffers");
    auto& o = *op->impl;
    require(o.projectors() > 0, "invalid PAW projection buffers");
    auto& ctx = o.context();
    SDFT_CUDA(cudaSetDevice(ctx.device));
    const std::size_t n = static_cast<std::size_t>(o.npw()) * columns;
    const std::size_t m = static_cast<std::size_t>(o.projectors()) * columns;
    Staged stage(ctx, memory);
    const auto* dx = stage.in(x, n, ctx.staging_in);
    auto* dp = stage.out(p, m, ctx.staging_out);
    o.project(dx, static_cast<int>(columns), dp, precision_of(precision));
    stage.back(p, dp, m);
    stage.finish();
  });
}

sdft_b200_status sdft_b200_local_hamiltonian(sdft_b200_context* context, const int32_t shape[3],
                                             const uint64_t* indices, size_t npw, const double* kinetic,
                                             const double* potential, const double* input, size_t columns,
                                             double* output, int precision, uint64_t operator_identity) {
  return guarded([&] {
    require(context && shape, "invalid accelerated FFT dimensions");
    auto& ctx = *context->impl;
    SDFT_CUDA(cudaSetDevice(ctx.device));
    const int s[3] = {shape[0], shape[1], shape[2]};
    sdft_b200::accelerator_local_hamiltonian(ctx, s, indices, npw, kinetic, potential, input, columns, output,
                                             precision_of(precision), operator_identity);
  });
}

sdft_b200_status sdft_b200_paw_pair(sdft_b200_context* context, uint64_t identity, size_t npw, size_t projectors,
                                    size_t columns, const double* b, const double* d, const double* q,
                                    const double* input, double* h, double* s, int precision,
                                    uint64_t projector_identity) {
  return guarded([&] {
    require(context != nullptr, "invalid CUDA PAW chain shape");
    auto& ctx = *context->impl;
    SDFT_CUDA(cudaSetDevice(ctx.device));
    sdft_b200::accelerator_paw_pair(ctx, identity, npw, projectors, columns, b, d, q, input, h, s,
                                    precision_of(precision), projector_identity ? projector_identity : identity);
  });
}

sdft_b200_status sdft_b200_pbe_points(sdft_b200_context* context, const double* density, const double* gradient,
                                      size_t count, double* out, int memory) {
  return guarded([&] {
    require(context && density && gradient && out && count, "invalid GPU PBE dimensions");
    auto& ctx = *context->impl;
    SDFT_CUDA(cudaSetDevice(ctx.device));
    if (memory == SDFT_B200_MEMORY_DEVICE) {
      sdft_b200::pbe_points(ctx, density, gradient, count, out);
      return;
    }
    require(memory == SDFT_B200_MEMORY_HOST, "memory must be host or device");
    auto* din = static_cast<double*>(ctx.staging_in.reserve(sizeof(double) * 2 * count));
    auto* dout = static_cast<double*>(ctx.staging_out.reserve(sizeof(double) * 7 * count));
    SDFT_CUDA(cudaMemcpyAsync(din, density, sizeof(double) * count, cudaMemcpyHostToDevice, ctx.stream));
    SDFT_CUDA(cudaMemcpyAsync(din + count, gradient, sizeof(double) * count, cudaMemcpyHostToDevice, ctx.stream));
    sdft_b200::pbe_points(ctx, din, din + count, count, dout);
    SDFT_CUDA(cudaMemcpyAsync(out, dout, sizeof(double) * 7 * count, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.synchronize();
  });
}

sdft_b200_status sdft_b200_band_density(sdft_b200_context* context, const int32_t* hkl, size_t npw,
                                        const double* psi, const double* occupations, size_t bands, double volume,
                                        const int32_t* support, size_t count, double* out, int memory) {
  return guarded([&] {
    require(context && hkl && psi && occupations && support && out && npw && bands && count,
            "invalid plane-wave FFT density dimensions");
    auto& ctx = *context->impl;
    SDFT_CUDA(cudaSetDevice(ctx.device));
    using C = sdft_b200::Cx<double>;
    if (memory == SDFT_B200_MEMORY_DEVICE) {
      sdft_b200::band_density(ctx, hkl, npw, reinterpret_cast<const C*>(psi), occupations, bands, volume, support,
                              count, reinterpret_cast<C*>(out));
      return;
    }
    require(memory == SDFT_B200_MEMORY_HOST, "memory must be host or device");
    auto* din = static_cast<C*>(ctx.staging_in.reserve(sizeof(C) * npw * bands));
    auto* dout = static_cast<C*>(ctx.staging_out.reserve(sizeof(C) * count));
    SDFT_CUDA(cudaMemcpyAsync(din, psi, sizeof(C) * npw * bands, cudaMemcpyHostToDevice, ctx.stream));
    sdft_b200::band_density(ctx, hkl, npw, din, occupations, bands, volume, support, count, dout);
    SDFT_CUDA(cudaMemcpyAsync(out, dout, sizeof(C) * count, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.synchronize();
  });
}

sdft_b200_status sdft_b200_onsite_density(sdft_b200_context* context, size_t rows, size_t atoms, size_t bands,
                                         const double* amplitudes, size_t stride, const double* occupations,
                                         double* out, int memory) {
  return guarded([&] {
    require(context && amplitudes && occupations && out && rows && atoms && bands && stride >= rows * atoms,
            "invalid projected onsite density dimensions");
    auto& ctx = *context->impl;
    SDFT_CUDA(cudaSetDevice(ctx.device));
    using C = sdft_b200::Cx<double>;
    const std::size_t outputs = atoms * rows * rows;
    if (memory == SDFT_B200_MEMORY_DEVICE) {
      sdft_b200::onsite_density(ctx, rows, atoms, bands, reinterpret_cast<const C*>(amplitudes), stride, occupations,
                                reinterpret_cast<C*>(out));
      return;
    }
    require(memory == SDFT_B200_MEMORY_HOST, "memory must be host or device");
    const std::size_t in_count = stride * (bands - 1) + rows * atoms;
    auto* din = static_cast<C*>(ctx.staging_in.reserve(sizeof(C) * in_count));
    auto* dout = static_cast<C*>(ctx.staging_out.reserve(sizeof(C) * outputs));
    SDFT_CUDA(cudaMemcpyAsync(din, amplitudes, sizeof(C) * in_count, cudaMemcpyHostToDevice, ctx.stream));
    sdft_b200::onsite_density(ctx, rows, atoms, bands, din, stride, occupations, dout);
    SDFT_CUDA(cudaMemcpyAsync(out, dout, sizeof(C) * outputs, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.synchronize();
  });
}

sdft_b200_status sdft_b200_compensation_create(sdft_b200_context* context, const double lattice[9], size_t atoms,
                                               const double* fractional, const int32_t* keys, size_t count,
                                               int max_l, size_t radial, const double* radial_grid,
                                               const double* compensation_r2, size_t dimension,
                                               const double* transform, sdft_b200_compensation** out) {
  return guarded([&] {
    require(context && out, "invalid PAW compensation dimensions");
    *out = nullptr;
    auto& ctx = *context->impl;
    SDFT_CUDA(cudaSetDevice(ctx.device));
    sdft_b200::CompensationInput in;
    in.lattice = lattice;
    in.atoms = atoms;
    in.fractional = fractional;
    in.keys = keys;
    in.count = count;
    in.max_l = max_l;
    in.radial = radial;
    in.radial_grid = radial_grid;
    in.compensation_r2 = compensation_r2;
    in.dimension = dimension;
    in.transform = transform;
    auto charge = std::make_unique<sdft_b200_compensation>();
    charge->impl = std::make_unique<sdft_b200::CompensationCharge>(ctx, in);
    *out = charge.release();
  });
}

sdft_b200_status sdft_b200_compensation_destroy(sdft_b200_compensation* charge) {
  return guarded([&] {
    if (!charge) return;
    SDFT_CUDA(cudaSetDevice(charge->impl->context().device));
    delete charge;
  });
}

sdft_b200_status sdft_b200_compensation_density(sdft_b200_compensation* charge, const double* onsite, double* out,
                                                int memory) {
  return guarded([&] {
    require(charge && onsite && out, "invalid PAW compensation dimensions");
    auto& c = *charge->impl;
    auto& ctx = c.context();
    SDFT_CUDA(cudaSetDevice(ctx.device));
    using C = sdft_b200::Cx<double>;
    if (memory == SDFT_B200_MEMORY_DEVICE) {
      c.density(reinterpret_cast<const C*>(onsite), reinterpret_cast<C*>(out));
      return;
    }
    require(memory == SDFT_B200_MEMORY_HOST, "memory must be host or device");
    const std::size_t in_count = c.atoms() * c.dimension() * c.dimension();
    auto* din = static_cast<C*>(ctx.staging_in.reserve(sizeof(C) * in_count));
    auto* dout = static_cast<C*>(ctx.staging_out.reserve(sizeof(C) * c.count()));
    SDFT_CUDA(cudaMemcpyAsync(din, onsite, sizeof(C) * in_count, cudaMemcpyHostToDevice, ctx.stream));
    c.density(din, dout);
    SDFT_CUDA(cudaMemcpyAsync(out, dout, sizeof(C) * c.count(), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.synchronize();
  });
}

sdft_b200_status sdft_b200_compensation_project(sdft_b200_compensation* charge, const double* potential,
                                                double* out, int memory) {
  return guarded([&] {
    require(charge && potential && out, "invalid PAW compensation dimensions");
    auto& c = *charge->impl;
    auto& ctx = c.context();
    SDFT_CUDA(cudaSetDevice(ctx.device));
    using C = sdft_b200::Cx<double>;
    if (memory == SDFT_B200_MEMORY_DEVICE) {
      c.project(reinterpret_cast<const C*>(potential), reinterpret_cast<C*>(out));
      return;
    }
    require(memory == SDFT_B200_MEMORY_HOST, "memory must be host or device");
    const std::size_t out_count = c.atoms() * c.dimension() * c.dimension();
    auto* din = static_cast<C*>(ctx.staging_in.reserve(sizeof(C) * c.count()));
    auto* dout = static_cast<C*>(ctx.staging_out.reserve(sizeof(C) * out_count));
    SDFT_CUDA(cudaMemcpyAsync(din, potential, sizeof(C) * c.count(), cudaMemcpyHostToDevice, ctx.stream));
    c.project(din, dout);
    SDFT_CUDA(cudaMemcpyAsync(out, dout, sizeof(C) * out_count, cudaMemcpyDeviceToHost, ctx.stream));
    ctx.synchronize();
  });
}

sdft_b200_status sdft_b200_density_functionals(sdft_b200_context* context, const double lattice[9], size_t count,
                                               const int32_t* hkl, const double* density, size_t core_count,
                                               const int32_t* core_hkl, const double* core, int quadrature_padding,
                                               int32_t* support_hkl, double* potential, double* xc_potential,
                                               size_t capacity, size_t* support_count,
                                               sdft_b200_functionals* result) {
  return guarded([&] {
    require(lattice && support_count, "null density functional argument");
    require(!count || (hkl && density), "null density arrays");
    require(!core_count || (core_hkl && core), "null core arrays");
    const auto support = sdft_b200::functional_support(lattice, count, hkl, density, core_count, core_hkl, core,
                                                       quadrature_padding);
    const std::size_t n = support.keys.size();
    *support_count = n;
    if (!capacity) return;
    require(capacity >= n, "density functional output capacity below the support size");
    require(context && support_hkl && potential && xc_potential && result, "null density functional outputs");
    for (std::size_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) support_hkl[3 * i + a] = support.keys[i][a];
    sdft_b200::FunctionalResult r;
    sdft_b200::density_functionals(*context->impl, support, reinterpret_cast<sdft_b200::Cx<double>*>(potential),
                                   reinterpret_cast<sdft_b200::Cx<double>*>(xc_potential), r);
    result->hartree_energy = r.hartree_energy;
    result->xc_energy = r.xc_energy;
    result->vxc_density = r.vxc_density;
    for (int k = 0; k < 9; ++k) {
      result->hartree_stress[k] = r.hartree_stress[k];
      result->xc_stress[k] = r.xc_stress[k];
    }
    result->sampled_electrons = r.sampled_electrons;
    result->minimum_density = r.minimum_density;
    result->clipped_density_points = r.clipped_density_points;
    result->grid_points = r.grid_points;
    for (int a = 0; a < 3; ++a) result->grid[a] = r.grid[a];
  });
}

sdft_b200_status sdft_b200_collinear_functionals(
    sdft_b200_context* context, const double lattice[9], size_t count_up, const int32_t* hkl_up, const double* up,
    size_t count_down, const int32_t* hkl_down, const double* down, size_t core_count, const int32_t* core_hkl,
    const double* core, int padding, int32_t* support_hkl, double* potential_up, double* potential_down,
    double* xc_potential_up, double* xc_potential_down, size_t capacity, size_t* support_count,
    sdft_b200_functionals result[2]) {
  return guarded([&] {
    require(lattice && support_count, "null density functional argument");
    require((!count_up || (hkl_up && up)) && (!count_down || (hkl_down && down)), "null spin density arrays");
    require(!core_count || (core_hkl && core), "null core arrays");
    const std::size_t counts[2] = {count_up, count_down};
    const int* const keys[2] = {hkl_up, hkl_down};
    const double* const values[2] = {up, down};
    const auto support =
        sdft_b200::collinear_support(lattice, counts, keys, values, core_count, core_hkl, core, padding);
    const std::size_t n = support.keys.size();
    *support_count = n;
    if (!capacity) return;
    require(capacity >= n, "density functional output capacity below the support size");
    require(context && support_hkl && potential_up && potential_down && xc_potential_up && xc_potential_down &&
                result,
            "null density functional outputs");
    for (std::size_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) support_hkl[3 * i + a] = support.keys[i][a];
    using C = sdft_b200::Cx<double>;
    C* const potential[2] = {reinterpret_cast<C*>(potential_up), reinterpret_cast<C*>(potential_down)};
    C* const xc[2] = {reinterpret_cast<C*>(xc_potential_up), reinterpret_cast<C*>(xc_potential_down)};
    sdft_b200::FunctionalResult r[2];
    sdft_b200::collinear_functionals(*context->impl, support, potential, xc, r);
    for (int c = 0; c < 2; ++c) {
      result[c].hartree_energy = r[c].hartree_energy;
      result[c].xc_energy = r[c].xc_energy;
      result[c].vxc_density = r[c].vxc_density;
      for (int k = 0; k < 9; ++k) {
        result[c].hartree_stress[k] = r[c].hartree_stress[k];
        result[c].xc_stress[k] = r[c].xc_stress[k];
      }
      result[c].sampled_electrons = r[c].sampled_electrons;
      result[c].minimum_density = r[c].minimum_density;
      result[c].clipped_density_points = r[c].clipped_density_points;
      result[c].grid_points = r[c].grid_points;
      for (int a = 0; a < 3; ++a) result[c].grid[a] = r[c].grid[a];
    }
  });
}

sdft_b200_status sdft_b200_rayleigh_ritz(sdft_b200_context* context, size_t n, size_t requested, const double* h,
                                        const double* s, double* values, double* vectors, int memory) {
  return guarded([&] {
    require(context && h && s && values && vectors && n && requested <= n, "invalid Rayleigh-Ritz dimensions");
    require(n <= 46340, "invalid Rayleigh-Ritz dimensions");
    require(memory == SDFT_B200_MEMORY_HOST || memory == SDFT_B200_MEMORY_DEVICE, "memory must be host or device");
    auto& ctx = *context->impl;
    SDFT_CUDA(cudaSetDevice(ctx.device));
    using C = sdft_b200::Cx<double>;
    const int m = static_cast<int>(n);
    const int count = requested ? static_cast<int>(requested) : m;
    const std::size_t mm = n * n;
    auto* buffers = static_cast<C*>(ctx.staging_in.reserve(sizeof(C) * 4 * mm));
    C* hw = buffers;
    C* sw = buffers + mm;
    C* staged = buffers + 2 * mm;
    auto* dvalues = static_cast<double*>(ctx.staging_out.reserve(sizeof(double) * n));
    const C* hin = reinterpret_cast<const C*>(h);
    const C* sin = reinterpret_cast<const C*>(s);
    if (memory == SDFT_B200_MEMORY_HOST) {
      SDFT_CUDA(cudaMemcpyAsync(staged, h, sizeof(C) * mm, cudaMemcpyHostToDevice, ctx.stream));
      SDFT_CUDA(cudaMemcpyAsync(staged + mm, s, sizeof(C) * mm, cudaMemcpyHostToDevice, ctx.stream));
      hin = staged;
      sin = staged + mm;
    }
    sdft_b200::hermitian_from_lower(hin, m, hw, m, m, ctx.stream);
    sdft_b200::hermitian_from_lower(sin, m, sw, m, m, ctx.stream);
    sdft_b200::generalized_lowest(ctx.blas, ctx.solver, hw, sw, m, count, dvalues, hw, ctx.eigen, sdft_b200::rr_mode(),
                                  ctx.stream);
    if (memory == SDFT_B200_MEMORY_HOST) {
      SDFT_CUDA(cudaMemcpyAsync(values, dvalues, sizeof(double) * count, cudaMemcpyDeviceToHost, ctx.stream));
      SDFT_CUDA(cudaMemcpyAsync(vectors, hw, sizeof(C) * n * count, cudaMemcpyDeviceToHost, ctx.stream));
    } else {
      SDFT_CUDA(cudaMemcpyAsync(values, dvalues, sizeof(double) * count, cudaMemcpyDeviceToDevice, ctx.stream));
      SDFT_CUDA(cudaMemcpyAsync(vectors, hw, sizeof(C) * n * count, cudaMemcpyDeviceToDevice, ctx.stream));
    }
    ctx.synchronize();
  });
}

sdft_b200_status sdft_b200_complex_gemm(sdft_b200_context* context, int aop, int bop, size_t m, size_t n, size_t k,
                                        const double* a, size_t lda, const double* b, size_t ldb, double* c,
                                        size_t ldc, int precision, int add, int memory) {
  return guarded([&] {
    require(context && a && b && c && m && n && k, "invalid complex GEMM shape/leading dimension");
    require((aop == SDFT_B200_OP_NORMAL || aop == SDFT_B200_OP_ADJOINT) &&
                (bop == SDFT_B200_OP_NORMAL || bop == SDFT_B200_OP_ADJOINT),
            "invalid complex GEMM operation");
    const std::size_t ar = aop == SDFT_B200_OP_NORMAL ? m : k, ac = aop == SDFT_B200_OP_NORMAL ? k : m;
    const std::size_t br = bop == SDFT_B200_OP_NORMAL ? k : n, bc = bop == SDFT_B200_OP_NORMAL ? n : k;
    require(lda >= ar && ldb >= br && ldc >= m, "invalid complex GEMM shape/leading dimension");
    if (std::max({m, n, k, lda, ldb, ldc}) > static_cast<size_t>(INT32_MAX))
      throw std::overflow_error("BLAS dimension overflow");
    const Precision p = precision_of(precision);
    auto& ctx = *context->impl;
    SDFT_CUDA(cudaSetDevice(ctx.device));
    Staged stage(ctx, memory);
    const auto* da = stage.in(a, lda * (ac - 1) + ar, ctx.staging_in);
    const auto* db = stage.in(b, ldb * (bc - 1) + br, ctx.staging_aux);
    if (p == Precision::Mixed && bop == SDFT_B200_OP_ADJOINT) {
      // The tensor cores take a normal right operand: form B^H (k x n) first.
      auto* adjoint = static_cast<Cx<double>*>(ctx.tc.adjoint.reserve(sizeof(Cx<double>) * k * n));
      sdft_b200::adjoint_block(db, static_cast<long long>(ldb), static_cast<int>(n), static_cast<int>(k), adjoint,
                               static_cast<long long>(k), ctx.stream);
      db = adjoint;
      ldb = k;
      bop = SDFT_B200_OP_NORMAL;
    }
    const std::size_t csize = ldc * (n - 1) + m;
    Cx<double>* dc = stage.out(c, csize, ctx.staging_out);
    if (add) stage.matrix_in(dc, c, m, n, ldc);
    const sdft_b200::Op ao = aop == SDFT_B200_OP_NORMAL ? sdft_b200::Op::N : sdft_b200::Op::C;
    const sdft_b200::Op bo = bop == SDFT_B200_OP_NORMAL ? sdft_b200::Op::N : sdft_b200::Op::C;
    if (p == Precision::FP64)
      sdft_b200::zgemm(ctx.blas, ao, bo, static_cast<int>(m), static_cast<int>(n), static_cast<int>(k), da,
                       static_cast<long long>(lda), db, static_cast<long long>(ldb), dc, static_cast<long long>(ldc),
                       add != 0);
    else
      sdft_b200::gemm_tc(ao, static_cast<int>(m), static_cast<int>(n), static_cast<int>(k), da,
                         static_cast<long long>(lda), nullptr, db, static_cast<long long>(ldb), dc,
                         static_cast<long long>(ldc), add != 0, 1.0, sdft_b200::search_split(), ctx.tc, ctx.stream);
    stage.matrix_back(c, dc, m, n, ldc);
    ctx.synchronize();
    if (sdft_b200::umma_error_flag()) throw sdft_b200::CudaError("tensor-core GEMM wait limit exceeded");
  });
}

sdft_b200_status sdft_b200_gemm_tuned_classes(size_t capacity, int32_t* rows, size_t* count) {
  return guarded([&] {
    require(count != nullptr && (rows != nullptr || capacity == 0), "invalid tuning table buffer");
    *count = sdft_b200::gemm_tuned_classes(capacity, rows);
  });
}

sdft_b200_status sdft_b200_complex_gemm_immutable_left(sdft_b200_context* context, uint64_t identity, int aop,
                                                       size_t m, size_t n, size_t k, const double* a, size_t lda,
                                                       const double* b, size_t ldb, double* c, size_t ldc,
                                                       int precision, int add, int memory) {
  return guarded([&] {
    require(context && identity && m && n && k && a && b && c && ldb >= k && ldc >= m &&
                (aop == SDFT_B200_OP_NORMAL || aop == SDFT_B200_OP_ADJOINT) &&
                lda >= (aop == SDFT_B200_OP_NORMAL ? m : k),
            "invalid immutable GEMM operand");
    if (std::max({m, n, k, lda, ldb, ldc}) > static_cast<size_t>(INT32_MAX))
      throw std::overflow_error("immutable BLAS dimension overflow");
    const Precision p = precision_of(precision);
    auto& ctx = *context->impl;
    SDFT_CUDA(cudaSetDevice(ctx.device));
    Staged stage(ctx, memory);
    const std::size_t ar = aop == SDFT_B200_OP_NORMAL ? m : k, ac = aop == SDFT_B200_OP_NORMAL ? k : m;
    const sdft_b200::Op ao = aop == SDFT_B200_OP_NORMAL ? sdft_b200::Op::N : sdft_b200::Op::C;
    auto& cache = ctx.immutable;
    sdft_b200::ImmutableLeft* entry = nullptr;
    for (auto& e : cache.entries)
      if (e.identity == identity && e.aop == aop && e.rows == ar && e.cols == ac) entry = &e;
    if (!entry) {
      entry = &cache.entries[0];
      for (auto& e : cache.entries)
        if (e.used < entry->used) entry = &e;
      entry->identity = 0;  // not valid until the copy below is queued
      sdft_b200::release(entry->packed);
      auto* dst = static_cast<Cx<double>*>(entry->fp64.reserve(sizeof(Cx<double>) * ar * ac));
      if (memory == SDFT_B200_MEMORY_DEVICE) require_device_memory(a, ctx.device, "a");
      SDFT_CUDA(cudaMemcpy2DAsync(dst, sizeof(Cx<double>) * ar, a, sizeof(Cx<double>) * lda, sizeof(Cx<double>) * ar,
                                  ac, memory == SDFT_B200_MEMORY_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                  ctx.stream));
      entry->identity = identity;
      entry->aop = aop;
      entry->rows = ar;
      entry->cols = ac;
    }
    entry->used = ++cache.clock;
    const auto* da = static_cast<const Cx<double>*>(entry->fp64.ptr);
    const auto* db = stage.in(b, ldb * (n - 1) + k, ctx.staging_aux);
    Cx<double>* dc = stage.out(c, ldc * (n - 1) + m, ctx.staging_out);
    if (add) stage.matrix_in(dc, c, m, n, ldc);
    if (p == Precision::FP64) {
      sdft_b200::zgemm(ctx.blas, ao, sdft_b200::Op::N, static_cast<int>(m), static_cast<int>(n), static_cast<int>(k),
                       da, static_cast<long long>(ar), db, static_cast<long long>(ldb), dc,
                       static_cast<long long>(ldc), add != 0);
    } else {
      const sdft_b200::Split split = sdft_b200::search_split();
      if (!entry->packed.data || entry->packed.split != split)
        sdft_b200::pack_persistent(ao, da, static_cast<long long>(ar), static_cast<int>(m), static_cast<int>(k),
                                   split, entry->packed, ctx.stream);
      sdft_b200::gemm_tc(ao, static_cast<int>(m), static_cast<int>(n), static_cast<int>(k), da,
                         static_cast<long long>(ar), &entry->packed, db, static_cast<long long>(ldb), dc,
                         static_cast<long long>(ldc), add != 0, 1.0, split, ctx.tc, ctx.stream);
    }
    stage.matrix_back(c, dc, m, n, ldc);
    ctx.synchronize();
    if (sdft_b200::umma_error_flag()) throw sdft_b200::CudaError("tensor-core GEMM wait limit exceeded");
  });
}

sdft_b200_status sdft_b200_complex_gemm_triple_right(sdft_b200_context* context, size_t m, size_t n, size_t k,
                                                     const double* const a[3], size_t lda, const double* b,
                                                     size_t ldb, double* const c[3], size_t ldc, int precision,
                                                     int memory) {
  return guarded([&] {
    require(context && a && c && b && m && n && k && lda >= m && ldb >= k && ldc >= m,
            "invalid joint Ritz rotation dimensions");
    for (int i = 0; i < 3; ++i) require(a[i] && c[i], "invalid joint Ritz rotation dimensions");
    if (std::max({m, n, k, lda, ldb, ldc}) > static_cast<size_t>(INT32_MAX))
      throw std::overflow_error("joint Ritz rotation BLAS dimensions overflow");
    // Address intervals of the operands, as the reference checks them
    // (src/compute_backend.cpp:262-282).
    auto interval = [](const void* p, std::size_t rows, std::size_t columns, std::size_t ld) {
      const auto first = reinterpret_cast<std::uintptr_t>(p);
      return std::make_pair(first, first + ((columns - 1) * ld + rows) * sizeof(Cx<double>));
    };
    auto overlaps = [](auto x, auto y) { return x.first < y.second && y.first < x.second; };
    const auto right = interval(b, k, n, ldb);
    for (int i = 0; i < 3; ++i) {
      const auto out = interval(c[i], m, n, ldc);
      require(!overlaps(out, right), "joint Ritz output aliases right operand");
      for (int j = 0; j < 3; ++j)
        require(!overlaps(out, interval(a[j], m, k, lda)) && (i == j || !overlaps(out, interval(c[j], m, n, ldc))),
                "joint Ritz outputs/inputs must be disjoint");
    }
    const Precision p = precision_of(precision);
    auto& ctx = *context->impl;
    SDFT_CUDA(cudaSetDevice(ctx.device));
    Staged stage(ctx, memory);
    const auto* db = stage.in(b, ldb * (n - 1) + k, ctx.staging_aux);
    const sdft_b200::Split split = sdft_b200::search_split();
    for (int i = 0; i < 3; ++i) {
      const auto* da = stage.in(a[i], lda * (k - 1) + m, ctx.staging_in);
      Cx<double>* dc = stage.out(c[i], ldc * (n - 1) + m, ctx.staging_out);
      if (p == Precision::FP64)
        sdft_b200::zgemm(ctx.blas, sdft_b200::Op::N, sdft_b200::Op::N, static_cast<int>(m), static_cast<int>(n),
                         static_cast<int>(k), da, static_cast<long long>(lda), db, static_cast<long long>(ldb), dc,
                         static_cast<long long>(ldc), false);
      else
        sdft_b200::gemm_tc(sdft_b200::Op::N, static_cast<int>(m), static_cast<int>(n), static_cast<int>(k), da,
                           static_cast<long long>(lda), nullptr, db, static_cast<long long>(ldb), dc,
                           static_cast<long long>(ldc), false, 1.0, split, ctx.tc, ctx.stream);
      stage.matrix_back(c[i], dc, m, n, ldc);
    }
    ctx.synchronize();
    if (sdft_b200::umma_error_flag()) throw sdft_b200::CudaError("tensor-core GEMM wait limit exceeded");
  });
}

sdft_b200_status sdft_b200_davidson(sdft_b200_operator* op, const sdft_b200_davidson_options* options,
                                   const double* initial, double* eigenvalues, double* eigenvectors,
                                   double* residuals, sdft_b200_davidson_stats* stats, int memory) {
  return guarded([&] {
    require(op && options && eigenvalues && residuals, "invalid matrix-free Davidson problem");
    require(memory == SDFT_B200_MEMORY_HOST || memory == SDFT_B200_MEMORY_DEVICE, "memory must be host or device");
    auto& o = *op->impl;
    auto& ctx = o.context();
    SDFT_CUDA(cudaSetDevice(ctx.device));
    require(options->roots >= 1 && options->roots <= static_cast<size_t>(o.npw()), "invalid matrix-free Davidson problem");
    require(options->max_iterations >= 1 && options->max_iterations <= 1000000, "invalid matrix-free Davidson problem");
    o.require_positive_metric();  // the overlap() signature checks, src/plane_wave_operator.cpp:702-717
    sdft_b200::DavidsonOptions d;
    d.roots = static_cast<int>(options->roots);
    d.max_iterations = static_cast<int>(options->max_iterations);
    d.tolerance = options->tolerance;
    d.precision = precision_of(options->precision);
    d.subspace_factor = options->subspace_factor ? options->subspace_factor : 8;
    d.handoff = options->handoff > 0 ? options->handoff : 1e-8;
    d.correction_steps = correction_steps_of(*options);
    const std::size_t block = static_cast<std::size_t>(o.npw()) * d.roots;
    const Cx<double>* warm = nullptr;
    if (initial) {
      Staged stage(ctx, memory);
      warm = stage.in(initial, block, ctx.staging_in);
    }
    if (!op->solver) op->solver = std::make_unique<sdft_b200::DavidsonSolver>(o);
    auto& solver = *op->solver;
    solver.solve(d, warm);
    const auto& values = solver.eigenvalues();
    const auto& res = solver.residuals();
    std::copy(values.begin(), values.end(), eigenvalues);
    std::copy(res.begin(), res.end(), residuals);
    if (eigenvectors) {
      // column-major npw x roots on the device is band-major roots x npw
      SDFT_CUDA(cudaMemcpyAsync(eigenvectors, solver.vectors(), sizeof(Cx<double>) * block,
                                memory == SDFT_B200_MEMORY_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                ctx.stream));
      ctx.synchronize();
    }
    if (stats) copy_stats(solver.stats(), stats);
  });
}

sdft_b200_status sdft_b200_rmm_trial(sdft_b200_operator* op, const sdft_b200_davidson_options* options,
                                     const double* initial, double* eigenvalues, double* eigenvectors,
                                     double* residuals, sdft_b200_davidson_stats* stats, int* trial_manifold,
                                     int memory) {
  return guarded([&] {
    require(op && options && initial && eigenvalues && residuals, "invalid RMM trial problem");
    require(memory == SDFT_B200_MEMORY_HOST || memory == SDFT_B200_MEMORY_DEVICE, "memory must be host or device");
    auto& o = *op->impl;
    auto& ctx = o.context();
    SDFT_CUDA(cudaSetDevice(ctx.device));
    require(options->roots >= 1 && options->roots <= static_cast<size_t>(o.npw()), "invalid RMM trial problem");
    require(options->max_iterations >= 1 && options->max_iterations <= 1000000, "invalid RMM trial problem");
    o.require_positive_metric();  // the overlap() signature checks, src/plane_wave_operator.cpp:702-717
    sdft_b200::DavidsonOptions d;
    d.roots = static_cast<int>(options->roots);
    d.max_iterations = static_cast<int>(options->max_iterations);
    d.tolerance = options->tolerance;
    d.precision = precision_of(options->precision);
    d.subspace_factor = options->subspace_factor ? options->subspace_factor : 8;
    d.handoff = options->handoff > 0 ? options->handoff : 1e-8;
    const std::size_t block = static_cast<std::size_t>(o.npw()) * d.roots;
    Staged stage(ctx, memory);
    const Cx<double>* warm = stage.in(initial, block, ctx.staging_in);
    if (!op->solver) op->solver = std::make_unique<sdft_b200::DavidsonSolver>(o);
    if (!op->rmm) op->rmm = std::make_unique<sdft_b200::RmmTrial>(o, *op->solver);
    const auto result = op->rmm->solve(d, warm);
    std::copy(result.eigenvalues.begin(), result.eigenvalues.end(), eigenvalues);
    std::copy(result.residuals.begin(), result.residuals.end(), residuals);
    if (eigenvectors) {
      SDFT_CUDA(cudaMemcpyAsync(eigenvectors, op->rmm->vectors(), sizeof(Cx<double>) * block,
                                memory == SDFT_B200_MEMORY_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                ctx.stream));
      ctx.synchronize();
    }
    if (trial_manifold) *trial_manifold = result.trial_manifold ? 1 : 0;
    if (stats) {
      sdft_b200::DavidsonStats st = result.fell_back ? result.fallback_stats : sdft_b200::DavidsonStats{};
      st.iterations = result.iterations;
      st.converged = result.converged;
      st.max_residual = result.residuals.empty() ? 0.0
                                                 : *std::max_element(result.residuals.begin(), result.residuals.end());
      copy_stats(st, stats);
    }
  });
}

sdft_b200_status sdft_b200_band_groups(sdft_b200_operator* op, const sdft_b200_davidson_options* options,
                                       const double* initial, double* eigenvalues, double* eigenvectors,
                                       double* residuals, sdft_b200_davidson_stats* stats, int memory) {
  return guarded([&] {
    require(op && options && eigenvalues && residuals, "invalid bounded band-group problem");
    require(memory == SDFT_B200_MEMORY_HOST || memory == SDFT_B200_MEMORY_DEVICE, "memory must be host or device");
    auto& o = *op->impl;
    auto& ctx = o.context();
    SDFT_CUDA(cudaSetDevice(ctx.device));
    require(options->roots >= 1 && options->roots <= static_cast<size_t>(o.npw()), "invalid bounded band-group problem");
    require(options->max_iterations >= 1 && options->max_iterations <= 1000000, "invalid bounded band-group problem");
    o.require_positive_metric();  // the overlap() signature checks, src/plane_wave_operator.cpp:702-717
    sdft_b200::DavidsonOptions d;
    d.roots = static_cast<int>(options->roots);
    d.max_iterations = static_cast<int>(options->max_iterations);
    d.tolerance = options->tolerance;
    d.precision = precision_of(options->precision);
    d.subspace_factor = options->subspace_factor ? options->subspace_factor : 8;
    d.handoff = options->handoff > 0 ? options->handoff : 1e-8;
    const std::size_t block = static_cast<std::size_t>(o.npw()) * d.roots;
    const Cx<double>* warm = nullptr;
    if (initial) {
      Staged stage(ctx, memory);
      warm = stage.in(initial, block, ctx.staging_in);
    }
    if (!op->solver) op->solver = std::make_unique<sdft_b200::DavidsonSolver>(o);
    if (!op->groups) op->groups = std::make_unique<sdft_b200::BandGroupSolver>(o, *op->solver);
    const auto result = op->groups->solve(d, warm);
    std::copy(result.eigenvalues.begin(), result.eigenvalues.end(), eigenvalues);
    std::copy(result.residuals.begin(), result.residuals.end(), residuals);
    if (eigenvectors) {
      SDFT_CUDA(cudaMemcpyAsync(eigenvectors, op->groups->vectors(), sizeof(Cx<double>) * block,
                                memory == SDFT_B200_MEMORY_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice,
                                ctx.stream));
      ctx.synchronize();
    }
    if (stats) {
      sdft_b200::DavidsonStats st;
      st.iterations = result.iterations;
      st.converged = result.converged;
      st.max_residual = result.residuals.empty() ? 0.0
                                                 : *std::max_element(result.residuals.begin(), result.residuals.end());
      copy_stats(st, stats);
    }
  });
}

sdft_b200_status sdft_b200_snapshot_read_info(const char* path, sdft_b200_snapshot_info* info) {
  return guarded([&] {
    require(path && info, "null snapshot argument");
    const auto snap = sdft_b200::read_operator_snapshot(path, true);
    info->npw = snap.npw;
    info->grid_points = snap.count;
    info->projectors = snap.projectors;
    info->atoms = snap.channels.size();
    info->roots = snap.roots;
    info->iterations = snap.iterations;
    info->initial_values = snap.initial_values;
    for (int a = 0; a < 3; ++a) info->shape[a] = snap.shape[a];
    info->regularization = snap.regularization;
    info->tolerance = snap.tolerance;
  });
}

sdft_b200_status sdft_b200_operator_from_snapshot(sdft_b200_context* context, const char* path,
                                                  sdft_b200_operator** out, double* initial) {
  return guarded([&] {
    require(context && path && out, "null snapshot argument");
    const auto snap = sdft_b200::read_operator_snapshot(path, false);
    auto op = std::make_unique<sdft_b200_operator>();
    op->impl = std::make_unique<sdft_b200::DeviceOperator>(*context->impl, snap);
    if (initial && !snap.initial.empty())
      std::memcpy(initial, snap.initial.data(), sizeof(Cx<double>) * snap.initial.size());
    *out = op.release();
  });
}

sdft_b200_status sdft_b200_server_create(int device, uint64_t memory_cap, int slots, sdft_b200_server** out) {
  return guarded([&] {
    require(out != nullptr, "null server output");
    auto server = std::make_unique<sdft_b200_server>();
    server->impl = std::make_unique<sdft_b200::SolveServer>(device, static_cast<std::size_t>(memory_cap), slots);
    *out = server.release();
  });
}

sdft_b200_status sdft_b200_server_destroy(sdft_b200_server* server) {
  return guarded([&] { delete server; });
}

sdft_b200_status sdft_b200_server_submit(sdft_b200_server* server, size_t npw, const int32_t* hkl,
                                         const double* kinetic_ev, size_t potential_count,
                                         const int32_t* potential_hkl, const double* potential, size_t atoms,
                                         const uint64_t* projectors, const double* amplitudes, const double* d,
                                         const double* q, double hartree_to_ev, double regularization,
                                         const sdft_b200_davidson_options* options, int want_vectors,
                                         uint64_t* ticket) {
  return guarded([&] {
    require(server && ticket && options && hkl && kinetic_ev && npw, "null solve request argument");
    require(!potential_count || (potential_hkl && potential), "null potential arrays");
    require(!atoms || (projectors && amplitudes && d && q), "null PAW arrays");
    require(options->max_iterations >= 1 && options->max_iterations <= 1000000, "invalid matrix-free Davidson problem");
    auto r = std::make_unique<sdft_b200::SolveRequest>();
    r->hkl.assign(hkl, hkl + 3 * npw);
    r->kinetic_ev.assign(kinetic_ev, kinetic_ev + npw);
    r->potential_hkl.assign(potential_hkl, potential_hkl + 3 * potential_count);
    r->potential.assign(potential, potential + 2 * potential_count);
    std::size_t rows = 0, block = 0;
    if (atoms) {
      r->projectors.assign(projectors, projectors + atoms);
      for (auto np : r->projectors) {
        require(np >= 1 && np <= 256, "invalid PAW low-rank operator dimensions");
        rows += np;
        block += np * np;
      }
      r->amplitudes.assign(amplitudes, amplitudes + 2 * rows * npw);
      r->d.assign(d, d + 2 * block);
      r->q.assign(q, q + 2 * block);
    }
    r->hartree_to_ev = hartree_to_ev;
    r->regularization = regularization;
    r->options.roots = static_cast<int>(options->roots);
    r->options.max_iterations = static_cast<int>(options->max_iterations);
    r->options.tolerance = options->tolerance;
    r->options.precision = precision_of(options->precision);
    r->options.subspace_factor = options->subspace_factor ? options->subspace_factor : 8;
    r->options.handoff = options->handoff > 0 ? options->handoff : 1e-8;
    r->options.correction_steps = correction_steps_of(*options);
    r->vectors = want_vectors != 0;
    *ticket = server->impl->submit(std::move(r));
  });
}

sdft_b200_status sdft_b200_server_wait(sdft_b200_server* server, uint64_t ticket, double timeout,
                                       double* eigenvalues, double* eigenvectors, double* residuals,
                                       sdft_b200_davidson_stats* stats, sdft_b200_solve_timing* timing) {
  sdft_b200::SolveResult result;
  bool finished = false;
  const sdft_b200_status waited = guarded([&] {
    require(server != nullptr, "null server");
    finished = server->impl->wait(ticket, timeout, result);
  });
  if (waited != SDFT_B200_OK) return waited;
  if (!finished) {
    last_error = "the solve has not finished";
    return SDFT_B200_NOT_READY;
  }
  if (timing) {
    timing->slot = result.slot;
    timing->footprint = result.footprint;
    timing->submitted = result.submitted;
    timing->started = result.started;
    timing->finished = result.finished;
  }
  if (result.status != SDFT_B200_OK) {
    last_error = result.error;
    return static_cast<sdft_b200_status>(result.status);
  }
  if (eigenvalues) std::copy(result.eigenvalues.begin(), result.eigenvalues.end(), eigenvalues);
  if (residuals) std::copy(result.residuals.begin(), result.residuals.end(), residuals);
  if (eigenvectors && !result.vectors.empty()) std::copy(result.vectors.begin(), result.vectors.end(), eigenvectors);
  if (stats) copy_stats(result.stats, stats);
  return SDFT_B200_OK;
}

sdft_b200_status sdft_b200_server_memory(const sdft_b200_server* server, uint64_t* cap, uint64_t* in_use,
                                         uint64_t* peak) {
  return guarded([&] {
    require(server != nullptr, "null server");
    if (cap) *cap = server->impl->memory_cap();
    if (in_use) *in_use = server->impl->in_use();
    if (peak) *peak = server->impl->peak_in_use();
  });
}

sdft_b200_status sdft_b200_solve_footprint(size_t npw, const int32_t* hkl, size_t projectors_total, size_t roots,
                                           int subspace_factor, uint64_t* bytes) {
  return guarded([&] {
    require(bytes != nullptr && roots >= 1 && roots <= npw, "invalid solve footprint arguments");
    *bytes = sdft_b200::solve_footprint(npw, hkl, projectors_total, static_cast<int>(roots), subspace_factor);
  });
}

}  // extern "C"
