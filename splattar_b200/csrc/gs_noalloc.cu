// Radix sort for callers that cannot let a library allocate device memory.
//
// gs_radix_sort_pairs takes its ping-pong buffers from the stream-ordered
// allocator on every call. Some callers cannot allow that: hosts that own
// every byte of device memory through their own pool or budget, loops that
// must not pay an allocation's latency or its implicit synchronisation, and
// bindings that forbid hidden allocations behind an FFI call. This variant
// allocates nothing: its scratch is a fixed array in the library's device
// image, sized for at most NOALLOC_MAX_PAIRS (key, value) pairs, which every
// GPU that loads the library holds until the process exits.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "gs_cuda.h"
#include "gs_kernels.h"

namespace gs {
namespace {

constexpr uint64_t NOALLOC_MAX_PAIRS = 1ull << 20;  // 1,048,576 pairs
// Per-pass digit histograms (256 bins x SORT_GRID blocks) plus the block
// sums of the histogram scan; must cover sort_scratch_bytes().
constexpr size_t NOALLOC_SORT_SCRATCH = sizeof(uint32_t) * 256 * SORT_GRID + sizeof(unsigned long long) * SCAN_GRID;
constexpr size_t NOALLOC_BYTES = 2 * NOALLOC_MAX_PAIRS * sizeof(uint32_t) + NOALLOC_SORT_SCRATCH;

// The scratch: alternate keys, alternate values, then the pass scratch.
// Every pass writes each scratch word it later reads, so nothing needs
// clearing between calls; the last call's contents simply remain.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[MAX_DEVICES] = {};

// Device address of the scratch array on the current device. In host code
// the array's name is only a host-side stand-in, so its device address is
// looked up once per device (with that device current) and cached for the
// life of the process: a caller that resets the device (cudaDeviceReset)
// destroys the context that address belongs to and must not call this entry
// point afterwards.
gs_status noalloc_scratch(unsigned char** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_error_message(std::string("gs_radix_sort_pairs_noalloc: cudaGetDevice: ") + cudaGetErrorString(e));
    return GS_ERR_CUDA;
  }
  if (dev < 0 || dev >= MAX_DEVICES) {
    set_error_message("gs_radix_sort_pairs_noalloc: device index out of range");
    return GS_ERR_INVALID_ARG;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    if (sort_scratch_bytes() > NOALLOC_SORT_SCRATCH) {
      set_error_message("gs_radix_sort_pairs_noalloc: pass scratch larger than the static array");
      return GS_ERR_CAPACITY;
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_error_message(std::string("gs_radix_sort_pairs_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      return GS_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return GS_OK;
}

}  // namespace
}  // namespace gs

using namespace gs;

extern "C" gs_status gs_radix_sort_pairs_noalloc(uint32_t* keys, uint32_t* vals, uint64_t n, uint32_t key_bits,
                                                  void* stream) {
  if (n == 0) return GS_OK;
  if (!keys || !vals || key_bits == 0 || key_bits > 32) {
    set_error_message("gs_radix_sort_pairs_noalloc: null array or key_bits outside 1..32");
    return GS_ERR_INVALID_ARG;
  }
  if (n > NOALLOC_MAX_PAIRS) {
    set_error_message("gs_radix_sort_pairs_noalloc: " + std::to_string(n) + " pairs exceed the maximum of " +
                      std::to_string(NOALLOC_MAX_PAIRS) + " (use gs_radix_sort_pairs)");
    return GS_ERR_CAPACITY;
  }
  unsigned char* base = nullptr;
  gs_status s = noalloc_scratch(&base);
  if (s) return s;
  uint32_t* k1 = reinterpret_cast<uint32_t*>(base);
  uint32_t* v1 = k1 + NOALLOC_MAX_PAIRS;
  void* pass_scratch = v1 + NOALLOC_MAX_PAIRS;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  int in1 = 0;
  int le = launch_radix_sort(keys, vals, k1, v1, n, nullptr, (int)key_bits, pass_scratch, &in1, st);
  if (!le && in1) {
    le = (int)cudaMemcpyAsync(keys, k1, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
    if (!le) le = (int)cudaMemcpyAsync(vals, v1, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st);
  }
  if (le) {
    set_error_message(std::string("gs_radix_sort_pairs_noalloc: ") + cudaGetErrorString((cudaError_t)le));
    return GS_ERR_CUDA;
  }
  return GS_OK;
}
