// Host-side FFT planning: radix factorisation and cached twiddle tables.
#include "fft.cuh"

#include <cmath>
#include <limits>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include <atomic>

namespace sdft_b200 {

namespace {
std::atomic<unsigned long long> launches{0};
}
void count_launch() { launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long launch_count() { return launches.load(std::memory_order_relaxed); }

LinePlan make_line_plan(int n, bool general) {
  if (n < 1 || n > kMaxLine) throw InvalidArgument("FFT length out of the supported range [1, 512]");
  LinePlan plan;
  plan.n = n;
  int rest = n;
  auto push = [&](int r) {
    if (plan.stages >= kMaxStages) throw InvalidArgument("FFT length has too many factors");
    plan.radix[plan.stages++] = r;
    rest /= r;
  };
  while (rest % 4 == 0) push(4);
  for (int p : {2, 3, 5, 7})
    while (rest % p == 0) push(p);
  if (general)
    for (int p = 11; rest > 1; p += 2)
      while (rest % p == 0) push(p);
  if (rest != 1) throw InvalidArgument("FFT length must be 2/3/5/7-smooth: " + std::to_string(n));
  return plan;
}

bool fft_length_supported(int n) {
  if (n < 1 || n > kMaxLine) return false;
  for (int p : {2, 3, 5, 7})
    while (n % p == 0) n /= p;
  return n == 1;
}

int fast_fft_length(int minimum) {
  if (minimum < 1) throw InvalidArgument("invalid FFT length");
  for (int n = minimum;; ++n) {
    int r = n;
    for (int p : {2, 3, 5, 7})
      while (r % p == 0) r /= p;
    if (r == 1) return n;
    if (n == std::numeric_limits<int>::max()) throw Overflow("FFT length overflow");
  }
}

namespace {
std::mutex table_mutex;
// key: (device, n, bytes per real)
std::map<std::tuple<int, int, int>, void*>& tables() {
  static std::map<std::tuple<int, int, int>, void*> t;
  return t;
}
}  // namespace

template <typename T>
const Cx<T>* device_twiddles(int n) {
  int device = 0;
  SDFT_CUDA(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lock(table_mutex);
  const auto key = std::make_tuple(device, n, static_cast<int>(sizeof(T)));
  auto found = tables().find(key);
  if (found != tables().end()) return static_cast<const Cx<T>*>(found->second);
  std::vector<Cx<T>> host(static_cast<std::size_t>(n));
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < n; ++m) {
    const long double angle = two_pi * static_cast<long double>(m) / static_cast<long double>(n);
    host[m] = Cx<T>{static_cast<T>(std::cos(angle)), static_cast<T>(-std::sin(angle))};
  }
  void* ptr = nullptr;
  SDFT_CUDA(cudaMalloc(&ptr, sizeof(Cx<T>) * n));
  SDFT_CUDA(cudaMemcpy(ptr, host.data(), sizeof(Cx<T>) * n, cudaMemcpyHostToDevice));
  tables()[key] = ptr;  // lives until process exit, shared by all operators on the device
  return static_cast<const Cx<T>*>(ptr);
}

template <typename T>
void host_twiddles(int n, Cx<T>* out) {
  const long double two_pi = 6.283185307179586476925286766559005768L;
  for (int m = 0; m < n; ++m) {
    const long double angle = two_pi * static_cast<long double>(m) / static_cast<long double>(n);
    out[m] = Cx<T>{static_cast<T>(std::cos(angle)), static_cast<T>(-std::sin(angle))};
  }
}

template void host_twiddles<float>(int, Cx<float>*);
template void host_twiddles<double>(int, Cx<double>*);
template const Cx<float>* device_twiddles<float>(int);
template const Cx<double>* device_twiddles<double>(int);

}  // namespace sdft_b200
