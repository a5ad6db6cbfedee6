// Fused local H~psi on device arrays with no allocation of any kind in the
// call: the slab between the plane and pencil passes and the three twiddle
// tables live in one file-scope device array of fixed size, whose address is
// looked up once per device with cudaGetSymbolAddress.
//
// For callers that must not allocate: a serving loop that has reserved the
// device's memory up front (pools sized to HBM), or one that cannot accept the
// device-wide synchronisation that cudaMalloc/cudaFree imply. The regular
// entry point grows its slab with cudaMalloc on first use of a larger block.
//
// Scratch contract:
//   - capacity kNoAllocScratchBytes (32 MiB) per device; the twiddle tables
//     take the first kTwiddleBytes, the slab the rest. A call whose slab
//     (slots * n1 * n2 * columns complex values) does not fit is rejected.
//   - nothing in it has to start at zero: each call writes the tables (from a
//     kernel parameter, so no host buffer is read by the device), and the
//     plane pass writes every slab entry before the pencil pass reads it.
//   - all calls on one device share it: two calls whose work overlaps in time
//     (different streams, threads or contexts on the same device) race on it.
//     Calls issued on one stream are ordered and safe.
#include <mutex>
#include <string>

#include "operator.cuh"

namespace sdft_b200 {

namespace {

constexpr std::size_t kNoAllocScratchBytes = std::size_t(32) << 20;
constexpr std::size_t kTwiddleBytes = 32 * 1024;  // 3 tables x 512 x 16 B, rounded up
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_address[kMaxDevices] = {};

// Once per device, with that device current. The first call on a device does
// this look-up, so it must come before any stream capture on that device.
// The address belongs to the device's primary context, the one the CUDA
// runtime makes current: the cache assumes that context for the life of the
// process (a cudaDeviceReset, or a caller that switches to a context of its
// own through the driver API, would need a new look-up).
unsigned char* scratch_for(int device) {
  if (device < 0 || device >= kMaxDevices) throw InvalidArgument("device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_address[device]) {
    void* address = nullptr;
    SDFT_CUDA(cudaGetSymbolAddress(&address, g_noalloc_scratch));
    g_scratch_address[device] = address;
  }
  return static_cast<unsigned char*>(g_scratch_address[device]);
}

// The three axes' twiddle tables, packed in the layout the scratch array
// holds them in, travel as one kernel parameter (24 KiB at most; parameters
// above 4 KiB need CUDA 12.1 and sm_70 or newer), so the device never reads a
// host buffer: each table starts at a kMaxLine boundary.
struct TwiddleTables {
  // Storage for three tables of Cx<T> entries, table a from entry a * kMaxLine
  // (Cx<float> tables fill the first half of the bytes).
  Cx<double> values[3 * kMaxLine];
};
static_assert(sizeof(TwiddleTables) <= 24 * 1024, "twiddle tables exceed the parameter budget");
static_assert(sizeof(TwiddleTables) <= kTwiddleBytes, "twiddle tables exceed their part of the scratch");

__global__ void write_twiddles_kernel(const TwiddleTables tables, int bytes, unsigned char* __restrict__ dst) {
  const auto* src = reinterpret_cast<const unsigned char*>(tables.values);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < bytes / 16; i += gridDim.x * blockDim.x)
    reinterpret_cast<uint4*>(dst)[i] = reinterpret_cast<const uint4*>(src)[i];
}

template <typename T>
void run(DeviceOperator& op, const Cx<double>* x, int columns, Cx<double>* y, const T* potential) {
  Context& ctx = op.context();
  const SpherePlan& plan = op.plan();
  const std::size_t per_column = sizeof(Cx<T>) * plan.slab_elements(1);
  const std::size_t capacity = kNoAllocScratchBytes - kTwiddleBytes;
  if (per_column * static_cast<std::size_t>(columns) > capacity)
    throw InvalidArgument("no-allocation local apply: " + std::to_string(columns) + " columns need " +
                          std::to_string(per_column * static_cast<std::size_t>(columns)) +
                          " slab bytes, above the 32 MiB static scratch; at most " +
                          std::to_string(capacity / per_column) + " columns per call for this operator");
  unsigned char* scratch = scratch_for(ctx.device);
  // Same table values as the cached tables of the regular path.
  TwiddleTables tables{};
  auto* packed = reinterpret_cast<Cx<T>*>(tables.values);
  const Cx<T>* twiddle[3];
  for (int a = 0; a < 3; ++a) {
    host_twiddles<T>(plan.n[a], packed + static_cast<std::size_t>(a) * kMaxLine);
    twiddle[a] = reinterpret_cast<const Cx<T>*>(scratch) + static_cast<std::size_t>(a) * kMaxLine;
  }
  const int bytes = static_cast<int>(sizeof(Cx<T>) * 3 * kMaxLine);
  write_twiddles_kernel<<<8, 256, 0, ctx.stream>>>(tables, bytes, scratch);
  SDFT_LAUNCH("write_twiddles_kernel");
  auto* slab = reinterpret_cast<Cx<T>*>(scratch + kTwiddleBytes);
  local_hamiltonian_preset<T>(plan, x, op.npw(), columns, potential, op.device_kinetic(), y, op.npw(), slab, twiddle,
                              ctx.stream);
}

}  // namespace

void apply_local_noalloc(DeviceOperator& op, const Cx<double>* x, int columns, Cx<double>* y, Precision precision) {
  if (columns <= 0) throw InvalidArgument("invalid direct plane-wave input/output buffers");
  if (precision == Precision::FP64) run<double>(op, x, columns, y, op.device_potential64());
  else run<float>(op, x, columns, y, op.device_potential32());
}

}  // namespace sdft_b200
