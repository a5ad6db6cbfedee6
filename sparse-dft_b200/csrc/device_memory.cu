// Stream-ordered device memory from one library pool per device.
#include <cstdint>
#include <mutex>

#include "common.cuh"

namespace sdft_b200 {

namespace {

constexpr int kMaxDevices = 64;
std::once_flag pool_once[kMaxDevices];
cudaMemPool_t pools[kMaxDevices] = {};

cudaMemPool_t current_pool() {
  int device = 0;
  SDFT_CUDA(cudaGetDevice(&device));
  if (device < 0 || device >= kMaxDevices) throw CudaError("device ordinal outside the library's pool table");
  std::call_once(pool_once[device], [device] {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    SDFT_CUDA(cudaMemPoolCreate(&pool, &props));
    // Freed blocks stay in the pool (no release at synchronisation points),
    // so a released buffer's memory serves the next allocation on any stream
    // of this device without mapping new memory.
    std::uint64_t keep = UINT64_MAX;
    SDFT_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[device] = pool;
  });
  return pools[device];
}

}  // namespace

void* stream_alloc(std::size_t bytes, cudaStream_t stream) {
  void* ptr = nullptr;
  SDFT_CUDA(cudaMallocFromPoolAsync(&ptr, std::max<std::size_t>(bytes, 1), current_pool(), stream));
  return ptr;
}

void stream_free(void* ptr, cudaStream_t stream) {
  if (ptr) cudaFreeAsync(ptr, stream);
}

void trim_pool() {
  SDFT_CUDA(cudaMemPoolTrimTo(current_pool(), 0));
}

}  // namespace sdft_b200
