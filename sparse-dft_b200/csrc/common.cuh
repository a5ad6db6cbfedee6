// Shared device/host utilities for the sm_100a plane-wave PAW library.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace sdft_b200 {

// Errors carry the reference's exception classes across the C ABI as codes.
struct InvalidArgument : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};
struct Overflow : std::overflow_error {
  using std::overflow_error::overflow_error;
};
struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct NonFinite : std::runtime_error {
  using std::runtime_error::runtime_error;
};
// A case the reference routes to a solver this library does not provide (the
// caller keeps the reference's own route for it).
struct Unsupported : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void check_cuda(cudaError_t code, const char* what) {
  if (code != cudaSuccess) throw CudaError(std::string("CUDA: ") + what + ": " + cudaGetErrorString(code));
}
// Counts this library's own kernel launches (library GEMMs/eigensolvers excluded).
void count_launch();
unsigned long long launch_count();
#define SDFT_CUDA(call) ::sdft_b200::check_cuda((call), #call)
#define SDFT_LAUNCH(what) (::sdft_b200::count_launch(), ::sdft_b200::check_cuda(cudaGetLastError(), what))

// Stream-ordered device memory from the library's pool on the current device
// (device_memory.cu): neither call synchronises the device. The memory is
// valid for work ordered after the allocation on `stream` (or after the
// stream has been synchronised); a freed block returns to the pool and is
// kept there for the next allocation. trim_pool() hands the pool's unused
// memory back to the device.
void* stream_alloc(std::size_t bytes, cudaStream_t stream);
void stream_free(void* ptr, cudaStream_t stream);
void trim_pool();

// Largest dynamic shared memory a kernel here may take (B200 opt-in limit).
constexpr std::size_t kMaxDynamicSmem = 227 * 1024;

// Opts a kernel in to all the dynamic shared memory its static shared memory
// leaves of kMaxDynamicSmem. The attribute is one value per kernel for the
// whole process, so every call sets the same maximum: solvers on other
// threads launch the same kernel with other sizes.
template <typename Kernel>
void allow_dynamic_smem(Kernel kernel, std::size_t bytes) {
  cudaFuncAttributes attributes;
  SDFT_CUDA(cudaFuncGetAttributes(&attributes, kernel));
  const std::size_t limit = kMaxDynamicSmem - std::min(kMaxDynamicSmem, attributes.sharedSizeBytes);
  if (bytes > limit) throw InvalidArgument("kernel tile does not fit in shared memory");
  SDFT_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(limit)));
}

// Interleaved complex in precision T (float2/double2 layout).
template <typename T>
struct alignas(2 * sizeof(T)) Cx {
  T re, im;
};

template <typename T>
__host__ __device__ __forceinline__ Cx<T> cx(T re, T im) {
  return Cx<T>{re, im};
}
template <typename T>
__host__ __device__ __forceinline__ Cx<T> operator+(Cx<T> a, Cx<T> b) {
  return {a.re + b.re, a.im + b.im};
}
template <typename T>
__host__ __device__ __forceinline__ Cx<T> operator-(Cx<T> a, Cx<T> b) {
  return {a.re - b.re, a.im - b.im};
}
template <typename T>
__host__ __device__ __forceinline__ Cx<T> cmul(Cx<T> a, Cx<T> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <typename T>
__host__ __device__ __forceinline__ Cx<T> cscale(Cx<T> a, T s) {
  return {a.re * s, a.im * s};
}

template <typename To, typename From>
__host__ __device__ __forceinline__ Cx<To> cconvert(Cx<From> a) {
  return {static_cast<To>(a.re), static_cast<To>(a.im)};
}

constexpr int kWarp = 32;
constexpr int kSmCount = 148;  // B200: 2 dies x 74 SMs

inline std::size_t ceil_div(std::size_t a, std::size_t b) { return (a + b - 1) / b; }

}  // namespace sdft_b200
