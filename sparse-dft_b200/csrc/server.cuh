// Solve server: continuous batching of independent Davidson solves on one
// device. Each request (one operator, one k-point) is copied in, waits in a
// FIFO queue, and is admitted when a worker slot is free and its estimated
// device footprint fits under the memory cap next to the solves already
// running. Every worker owns a context (stream, cuBLAS and cuSOLVER handles,
// scratch), so admitted solves overlap on the device; a solve's result does
// not depend on what else runs (same kernels, same inputs, own buffers).
// A request's operator and working buffers are stream-ordered allocations
// from the library's memory pool on the worker's stream: they return to the
// pool when the request ends and serve the next request's allocations, so
// no request start or end synchronises the device.
#pragma once
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "davidson.cuh"

namespace sdft_b200 {

struct SolveRequest {
  std::vector<int> hkl;
  std::vector<double> kinetic_ev;
  std::vector<int> potential_hkl;
  std::vector<double> potential;
  std::vector<std::uint64_t> projectors;
  std::vector<double> amplitudes, d, q;
  double hartree_to_ev = 27.211386245988;
  double regularization = 1e-12;
  DavidsonOptions options;
  bool vectors = false;
};

struct SolveResult {
  int status = 0;  // sdft_b200_status
  std::string error;
  std::vector<double> eigenvalues, residuals, vectors;  // vectors: band-major roots x npw, interleaved complex
  DavidsonStats stats;
  std::size_t footprint = 0;
  int slot = -1;
  double submitted = 0, started = 0, finished = 0;  // seconds since the server started
};

// Device bytes a solve is budgeted at: operator arrays, the packed projector
// operands, the Davidson basis and its images, the projected pencil and the
// eigensolver workspace, and the largest apply's grid slab and packed
// operands (every term an upper bound).
std::size_t solve_footprint(std::size_t npw, const int* hkl, std::size_t projectors_total, int roots,
                            int subspace_factor);

class SolveServer {
 public:
  SolveServer(int device, std::size_t memory_cap, int slots);
  ~SolveServer();
  SolveServer(const SolveServer&) = delete;
  SolveServer& operator=(const SolveServer&) = delete;

  // Queues a request; throws InvalidArgument when it can never fit the cap.
  std::uint64_t submit(std::unique_ptr<SolveRequest> request);
  // Waits up to timeout seconds; true (and the result moved out) when done.
  bool wait(std::uint64_t ticket, double timeout, SolveResult& out);
  std::size_t memory_cap() const { return cap_; }
  std::size_t in_use() const;
  std::size_t peak_in_use() const;

 private:
  struct Entry {
    std::uint64_t ticket;
    std::unique_ptr<SolveRequest> request;
    std::size_t footprint;
    double submitted;
  };
  void worker(int slot);
  double now() const;

  int device_;
  std::size_t cap_;
  mutable std::mutex mutex_;
  std::condition_variable work_, done_;
  std::deque<Entry> queue_;
  std::unordered_map<std::uint64_t, SolveResult> results_;
  std::unordered_set<std::uint64_t> pending_;  // submitted, result not yet collected
  std::size_t in_use_ = 0, peak_ = 0;
  std::uint64_t next_ticket_ = 1;
  bool stopping_ = false;
  std::vector<std::thread> workers_;
  std::chrono::steady_clock::time_point start_;
};

}  // namespace sdft_b200
