// Solve server (continuous batching of independent Davidson solves).
#include <algorithm>
#include <cmath>
#include <stdexcept>

#include "fft.cuh"
#include "server.cuh"
#include "umma_gemm.cuh"

namespace sdft_b200 {

namespace {

// Status codes of the C ABI (sdft_b200_status).
enum : int { kOk = 0, kInvalid = 1, kOverflow = 2, kRuntime = 3, kCuda = 4, kMemory = 5, kNonFinite = 6 };

int status_of(std::exception_ptr error, std::string& message) {
  try {
    std::rethrow_exception(error);
  } catch (const InvalidArgument& e) {
    message = e.what();
    return kInvalid;
  } catch (const std::invalid_argument& e) {
    message = e.what();
    return kInvalid;
  } catch (const std::overflow_error& e) {
    message = e.what();
    return kOverflow;
  } catch (const NonFinite& e) {
    message = e.what();
    return kNonFinite;
  } catch (const CudaError& e) {
    message = e.what();
    return kCuda;
  } catch (const std::bad_alloc&) {
    message = "out of memory";
    return kMemory;
  } catch (const std::exception& e) {
    message = e.what();
    return kRuntime;
  } catch (...) {
    message = "unknown error";
    return kRuntime;
  }
}

}  // namespace

std::size_t solve_footprint(std::size_t npw, const int* hkl, std::size_t projectors_total, int roots,
                            int subspace_factor) {
  if (!npw || !hkl || roots < 1) throw InvalidArgument("invalid solve request dimensions");
  // Grid: the operator's rule with every retained potential key inside the
  // basis span, N_a = fast(max(3, 2 width_a + 1)).
  double grid = 1.0;
  for (int a = 0; a < 3; ++a) {
    int low = hkl[a], high = hkl[a];
    for (std::size_t g = 0; g < npw; ++g) {
      low = std::min(low, hkl[3 * g + a]);
      high = std::max(high, hkl[3 * g + a]);
    }
    grid *= fast_fft_length(std::max(3, 2 * (high - low) + 1));
  }
  const double n = static_cast<double>(npw), p = static_cast<double>(projectors_total);
  const int factor = subspace_factor ? subspace_factor : 8;
  const double cap = std::min<double>(n, std::max(factor * roots, 64));
  const double kmax = std::min<double>(cap, std::max(3 * roots, 2));
  const double r = std::min<double>(roots, n);
  const double cx = 16.0;  // complex128
  double bytes = 0;
  // Operator: V(r) in FP64 and FP32, maps and diagonals, B, both packed B operands (BF16x6).
  bytes += 12.0 * grid + 40.0 * n + cx * p * n + 2.0 * 24.0 * p * n;
  // Davidson: basis and images, Ritz block and residuals, correction blocks,
  // projected pencil, Rayleigh-Ritz and eigensolver matrices, Gram blocks.
  bytes += 3.0 * cx * n * cap + 4.0 * cx * n * r + 3.0 * cx * n * kmax + 10.0 * cx * cap * cap +
           cx * cap * kmax + 4.0 * cx * kmax * kmax;
  // Largest apply (a full basis refresh): FP64 and FP32 grid slabs, PAW
  // projections, packed tensor-core operands and split-K partials.
  bytes += (cx + 8.0) * grid * cap + 3.0 * cx * p * cap + 24.0 * n * cap + 48.0 * n * kmax + 8.0 * cap * kmax * 64.0;
  // Mixed search: BF16x6 copies of V^H, HV and SV as right factors, V, HV, SV as left factors.
  bytes += 192.0 * n * cap;
  bytes = bytes * 1.1 + 64.0 * 1024 * 1024;  // allocator rounding and handles
  if (!std::isfinite(bytes) || bytes > 1e18) throw Overflow("solve footprint overflow");
  return static_cast<std::size_t>(bytes);
}

SolveServer::SolveServer(int device, std::size_t memory_cap, int slots)
    : device_(device), cap_(memory_cap), start_(std::chrono::steady_clock::now()) {
  if (slots < 1 || slots > 64) throw InvalidArgument("server slots must be in [1, 64]");
  if (!memory_cap) throw InvalidArgument("server memory cap must be positive");
  int count = 0;
  SDFT_CUDA(cudaGetDeviceCount(&count));
  if (device < 0 || device >= count) throw InvalidArgument("invalid CUDA device");
  workers_.reserve(slots);
  try {
    for (int s = 0; s < slots; ++s) workers_.emplace_back(&SolveServer::worker, this, s);
  } catch (...) {
    {
      std::lock_guard<std::mutex> lock(mutex_);
      stopping_ = true;
    }
    work_.notify_all();
    for (auto& t : workers_) t.join();
    throw;
  }
}

SolveServer::~SolveServer() {
  {
    std::lock_guard<std::mutex> lock(mutex_);
    stopping_ = true;
  }
  work_.notify_all();
  for (auto& t : workers_)
    if (t.joinable()) t.join();
}

double SolveServer::now() const {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - start_).count();
}

std::size_t SolveServer::in_use() const {
  std::lock_guard<std::mutex> lock(mutex_);
  return in_use_;
}

std::size_t SolveServer::peak_in_use() const {
  std::lock_guard<std::mutex> lock(mutex_);
  return peak_;
}

std::uint64_t SolveServer::submit(std::unique_ptr<SolveRequest> request) {
  if (!request) throw InvalidArgument("null solve request");
  const std::size_t npw = request->kinetic_ev.size();
  if (!npw || request->hkl.size() != 3 * npw) throw InvalidArgument("solve request basis arrays disagree");
  std::uint64_t projectors_total = 0;
  for (auto np : request->projectors) projectors_total += np;
  const auto& o = request->options;
  if (o.roots < 1 || static_cast<std::size_t>(o.roots) > npw) throw InvalidArgument("invalid matrix-free Davidson problem");
  const std::size_t footprint = solve_footprint(npw, request->hkl.data(), projectors_total, o.roots, o.subspace_factor);
  if (footprint > cap_)
    throw InvalidArgument("solve footprint " + std::to_string(footprint) + " bytes exceeds the server memory cap " +
                          std::to_string(cap_));
  std::uint64_t ticket;
  {
    std::lock_guard<std::mutex> lock(mutex_);
    if (stopping_) throw std::runtime_error("solve server is stopping");
    ticket = next_ticket_++;
    pending_.insert(ticket);
    queue_.push_back(Entry{ticket, std::move(request), footprint, now()});
  }
  work_.notify_all();
  return ticket;
}

bool SolveServer::wait(std::uint64_t ticket, double timeout, SolveResult& out) {
  std::unique_lock<std::mutex> lock(mutex_);
  if (!pending_.count(ticket)) throw InvalidArgument("unknown solve ticket");
  auto ready = [&] { return results_.count(ticket) != 0; };
  if (timeout < 0) {
    done_.wait(lock, ready);
  } else if (!done_.wait_for(lock, std::chrono::duration<double>(timeout), ready)) {
    return false;
  }
  auto found = results_.find(ticket);
  out = std::move(found->second);
  results_.erase(found);
  pending_.erase(ticket);
  return true;
}

void SolveServer::worker(int slot) {
  std::unique_ptr<Context> ctx;
  std::string context_error;
  int context_status = kOk;
  try {
    SDFT_CUDA(cudaSetDevice(device_));
    ctx = std::make_unique<Context>(device_, nullptr);
  } catch (...) {
    context_status = status_of(std::current_exception(), context_error);
  }
  while (true) {
    Entry entry;
    {
      std::unique_lock<std::mutex> lock(mutex_);
      // FIFO admission: the queue's head starts once its footprint fits.
      work_.wait(lock, [&] { return stopping_ || (!queue_.empty() && in_use_ + queue_.front().footprint <= cap_); });
      if (stopping_ && queue_.empty()) break;
      if (stopping_) {
        // Requests still queued at shutdown are answered with an error.
        entry = std::move(queue_.front());
        queue_.pop_front();
        SolveResult r;
        r.status = kRuntime;
        r.error = "solve server stopped before the request started";
        r.submitted = entry.submitted;
        results_[entry.ticket] = std::move(r);
        done_.notify_all();
        continue;
      }
      entry = std::move(queue_.front());
      queue_.pop_front();
      in_use_ += entry.footprint;
      peak_ = std::max(peak_, in_use_);
    }
    work_.notify_all();  // the next head may fit beside this one
    SolveResult result;
    result.footprint = entry.footprint;
    result.slot = slot;
    result.submitted = entry.submitted;
    result.started = now();
    if (context_status != kOk) {
      result.status = context_status;
      result.error = context_error;
    } else {
      try {
        const SolveRequest& q = *entry.request;
        OperatorInput in;
        in.npw = q.kinetic_ev.size();
        in.hkl = q.hkl.data();
        in.kinetic_ev = q.kinetic_ev.data();
        in.potential_count = q.potential.size() / 2;
        in.potential_hkl = q.potential_hkl.data();
        in.potential = q.potential.data();
        in.atoms = q.projectors.size();
        in.projectors = q.projectors.data();
        in.amplitudes = q.amplitudes.data();
        in.d = q.d.data();
        in.q = q.q.data();
        in.hartree_to_ev = q.hartree_to_ev;
        in.regularization = q.regularization;
        {
          DeviceOperator op(*ctx, in);
          op.require_positive_metric();
          DavidsonSolver solver(op);
          solver.solve(q.options, nullptr);
          result.eigenvalues = solver.eigenvalues();
          result.residuals = solver.residuals();
          result.stats = solver.stats();
          if (q.vectors) {
            const std::size_t count = in.npw * static_cast<std::size_t>(q.options.roots);
            result.vectors.resize(2 * count);
            SDFT_CUDA(cudaMemcpyAsync(result.vectors.data(), solver.vectors(), sizeof(Cx<double>) * count,
                                      cudaMemcpyDeviceToHost, ctx->stream));
          }
          ctx->synchronize();
        }
        ctx->recycle_scratch();
      } catch (...) {
        result.status = status_of(std::current_exception(), result.error);
        try {
          ctx->recycle_scratch();
        } catch (...) {
        }
      }
    }
    result.finished = now();
    {
      std::lock_guard<std::mutex> lock(mutex_);
      in_use_ -= entry.footprint;
      results_[entry.ticket] = std::move(result);
    }
    done_.notify_all();
    work_.notify_all();
  }
}

}  // namespace sdft_b200
