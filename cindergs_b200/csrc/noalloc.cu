// A pair sort that allocates nothing: cgs_sort_pairs_u32_noalloc.
//
// Some callers cannot let this library call cudaMalloc. A host engine that
// owns every device allocation through its own pool or memory budget (a
// renderer embedding the splat pipeline as a plug-in, a Rust host whose GPU
// memory is managed by its own allocator) must not see a library grow the
// process's footprint behind its back, and a real-time loop cannot call
// cudaMalloc mid-frame because an allocation can synchronise the whole device
// and stall the frame. For them this entry point runs the same stable LSD
// radix sort as cgs_sort_pairs_u32 (radix_sort.cu), but every scratch buffer
// it needs -- the alternate key/value buffers, the digit histograms, the
// chained look-back words and the counters -- lives in one file-scope
// __device__ array of fixed size, so the call itself allocates nothing. The
// caller still provides the keys and values (sorted in place).
//
// The array (kScratchBytes, 9 MiB + 8.25 KiB) is part of the library image: every
// GPU that loads the library holds it until the process exits. Every call
// shares it and it keeps the last call's contents, so the parts that must
// start at zero are cleared with cudaMemsetAsync at the start of each call;
// calls whose work overlaps on the GPU (different streams or host threads at
// the same time) race on it and must be serialised by the caller.
#include <mutex>

#include "cgs.h"
#include "kernels.h"

namespace cgs {
namespace {

constexpr uint64_t kMaxPairs = CGS_NOALLOC_SORT_MAX_PAIRS;
constexpr size_t kMaxTiles = (kMaxPairs + 4095) / 4096;  // 4096 keys per sort tile
// Layout: [alt keys | alt values | 8 x 256 histogram words | look-back words
// for up to 8 passes of 16 digits or 4 passes of 256 digits | 64 counter words]
constexpr size_t kAltBytes = kMaxPairs * 4;
constexpr size_t kHistBytes = 8 * 256 * 4;
constexpr size_t kStatusBytes = 4 * kMaxTiles * 256 * 4;  // = 8 * tiles * 16 * 4 * 8
constexpr size_t kWordsBytes = 256;
constexpr size_t kScratchBytes = 2 * kAltBytes + kHistBytes + kStatusBytes + kWordsBytes;
static_assert(kStatusBytes >= 8 * kMaxTiles * 16 * 4, "look-back area too small for 4-bit digits");

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device. In host code the
// array's name is only a host-side stand-in, so the address is looked up once
// per device with that device current.
int scratch_for_current_device(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return CGS_E_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return CGS_E_CAPACITY;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return CGS_E_CUDA;
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return CGS_OK;
}

}  // namespace
}  // namespace cgs

#pragma GCC visibility push(default)
extern "C" int cgs_sort_pairs_u32_noalloc(uint32_t* d_keys, uint32_t* d_vals, uint64_t n,
                                          uint32_t key_bits, int32_t digit_bits, void* stream) {
  using namespace cgs;
  if (digit_bits != 0 && digit_bits != 4 && digit_bits != 8) return CGS_E_ARG;
  if (key_bits == 0 || key_bits > 32) return CGS_E_ARG;
  if (n > kMaxPairs) return CGS_E_CAPACITY;
  if (n > 0 && (!d_keys || !d_vals)) return CGS_E_ARG;
  if (n <= 1) return CGS_OK;
  void* base = nullptr;
  const int rc = scratch_for_current_device(&base);
  if (rc != CGS_OK) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  char* b = static_cast<char*>(base);
  uint32_t* alt_keys = reinterpret_cast<uint32_t*>(b);
  uint32_t* alt_vals = reinterpret_cast<uint32_t*>(b + kAltBytes);
  uint32_t* hist = reinterpret_cast<uint32_t*>(b + 2 * kAltBytes);
  uint32_t* status = reinterpret_cast<uint32_t*>(b + 2 * kAltBytes + kHistBytes);
  uint32_t* words = reinterpret_cast<uint32_t*>(b + 2 * kAltBytes + kHistBytes + kStatusBytes);
  // words[0] = n, words[1] = status bits, words[2..] = per-pass tile counters
  if (cudaMemsetAsync(hist, 0, kHistBytes + kStatusBytes + kWordsBytes, s) != cudaSuccess)
    return CGS_E_CUDA;
  const uint32_t n32 = (uint32_t)n;
  if (cudaMemcpyAsync(words, &n32, 4, cudaMemcpyHostToDevice, s) != cudaSuccess) return CGS_E_CUDA;
  const uint32_t rb = digit_bits == 0 ? 8u : (uint32_t)digit_bits;
  if (launch_histogram(d_keys, words, n32, 0, key_bits, rb, hist, s) != cudaSuccess)
    return CGS_E_CUDA;
  SortArgs sa{};
  sa.keys[0] = d_keys;
  sa.keys[1] = alt_keys;
  sa.vals[0] = d_vals;
  sa.vals[1] = alt_vals;
  sa.n_ptr = words;
  sa.capacity = n32;
  sa.first_bit = 0;
  sa.num_bits = key_bits;
  sa.radix_bits = rb;
  sa.hist = hist;
  sa.status = status;
  sa.tile_ctr = words + 2;
  sa.status_word = words + 1;
  sa.src = 0;
  int src = 0;
  if (run_radix_sort(sa, &src, s) != cudaSuccess) return CGS_E_CUDA;
  if (src == 1) {
    if (cudaMemcpyAsync(d_keys, alt_keys, n * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(d_vals, alt_vals, n * 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
      return CGS_E_CUDA;
  }
  uint32_t st = 0;
  if (cudaMemcpyAsync(&st, words + 1, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return CGS_E_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return CGS_E_CUDA;
  if (st & kStatusLookbackTimeout) return CGS_E_TIMEOUT;
  if (st & kStatusCapacity) return CGS_E_CAPACITY;
  return CGS_OK;
}
#pragma GCC visibility pop
