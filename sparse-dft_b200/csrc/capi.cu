// extern "C" boundary (include/sdft_b200.h): converts exceptions into status
// codes and a thread-local message, and host pointers into staged device copies.
#include <cstring>
#include <new>
#include <string>

#include "../../include/sdft_b200.h"
#include "operator.cuh"

struct sdft_b200_context {
  std::unique_ptr<sdft_b200::Context> impl;
};
struct sdft_b200_operator {
  std::unique_ptr<sdft_b200::DeviceOperator> impl;
};

namespace {
thread_local std::string last_error;

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
struct Staged {
  sdft_b200::Context& ctx;
  int memory;
  Staged(sdft_b200::Context& c, int m) : ctx(c), memory(m) {
    require(m == SDFT_B200_MEMORY_HOST || m == SDFT_B200_MEMORY_DEVICE, "memory must be host or device");
  }
  const Cx<double>* in(const double* host, std::size_t complex_count, sdft_b200::Scratch& slot) {
    if (memory == SDFT_B200_MEMORY_DEVICE) return reinterpret_cast<const Cx<double>*>(host);
    auto* dst = static_cast<Cx<double>*>(slot.reserve(sizeof(Cx<double>) * complex_count));
    SDFT_CUDA(cudaMemcpyAsync(dst, host, sizeof(Cx<double>) * complex_count, cudaMemcpyHostToDevice, ctx.stream));
    return dst;
  }
  Cx<double>* out(double* host, std::size_t complex_count, sdft_b200::Scratch& slot) {
    if (memory == SDFT_B200_MEMORY_DEVICE) return reinterpret_cast<Cx<double>*>(host);
    return static_cast<Cx<double>*>(slot.reserve(sizeof(Cx<double>) * complex_count));
  }
  void back(double* host, const Cx<double>* dev, std::size_t complex_count) {
    if (memory == SDFT_B200_MEMORY_DEVICE) return;
    SDFT_CUDA(cudaMemcpyAsync(host, dev, sizeof(Cx<double>) * complex_count, cudaMemcpyDeviceToHost, ctx.stream));
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

sdft_b200_status sdft_b200_operator_destroy(sdft_b200_operator* op) {
  return guarded([&] { delete op; });
}

sdft_b200_status sdft_b200_operator_info(const sdft_b200_operator* op, int32_t shape[3], size_t* grid_points,
                                         size_t* projectors, size_t* npw) {
  return guarded([&] {
    require(op != nullptr, "null operator");
    const auto& plan = op->impl->plan();
    if (shape)
      for (int a = 0; a < 3; ++a) shape[a] = plan.n[a];
    if (grid_points) *grid_points = plan.count;
    if (projectors) *projectors = static_cast<size_t>(op->impl->projectors());
    if (npw) *npw = static_cast<size_t>(op->impl->npw());
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

}  // extern "C"
