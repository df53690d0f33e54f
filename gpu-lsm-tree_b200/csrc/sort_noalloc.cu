// gpulsm_sort_pairs_noalloc: the onesweep radix sort of gpulsm_sort_pairs
// without any device allocation, for callers that are not allowed to
// allocate device memory - for example a process whose device memory is
// entirely reserved by another allocator under a fixed budget (a serving
// stack with its own pool), or a latency-critical path that cannot risk an
// allocator call that may block or fail under memory pressure.
//
// Its scratch (ping-pong buffers, digit histograms, look-back words) is one
// file-scope __device__ array of kNoallocScratchBytes, held by every GPU that
// loads the library until the process exits.  The caller still passes the
// input and output buffers.  Limits and rules:
//   - at most kNoallocMaxKeys (2^20) keys per call; larger counts are
//     rejected with GPULSM_ERR_LENGTH before any work is enqueued;
//   - every call on a device shares the one array and it keeps the last
//     call's contents; each call clears the parts that must start at zero,
//     and calls that overlap on the GPU (different streams without ordering,
//     or different host threads) race on it - serialise them;
//   - the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (host code cannot use the symbol itself: in host
//     code it is only a stand-in for the device array) - make that first call
//     before any stream capture on that device;
//   - keys_in may be keys_out (and values_in values_out): the sort then runs
//     in place; a partial overlap of an input with an output is rejected;
//   - the call returns once the sort has finished: it copies the passes'
//     status word into a host variable and reports a look-back wait that gave
//     up as GPULSM_ERR_TIMEOUT (the output is then not sorted).
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

#include "common.cuh"
#include "radix_sort.cuh"
#include "sort_noalloc.h"

namespace gpulsm {

namespace {
constexpr size_t kKeyBytes = size_t(kNoallocMaxKeys) * 8;  // 64-bit keys at most
constexpr size_t kValBytes = size_t(kNoallocMaxKeys) * 4;
constexpr size_t kWorkBytes = (size_t(radix::kMaxPasses) * radix::kDigits + 64 +
                               size_t(radix::kMaxPasses) * ((kNoallocMaxKeys + radix::kTile - 1) / radix::kTile) *
                                   radix::kDigits) * 4;
constexpr size_t kStatusBytes = 256;
constexpr size_t kNoallocScratchBytes = kKeyBytes + kValBytes + kWorkBytes + kStatusBytes;

// The scratch array itself (device memory, shared by every call on a device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void *g_scratch_addr[kMaxDevices] = {};

// Once per device, with that device current: the device address of the array.
void *scratch_for_current_device() {
  int dev = 0;
  GPULSM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device ordinal out of range for the scratch table");
  std::lock_guard<std::mutex> g(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      (void)cudaGetLastError();
      throw std::runtime_error(std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                               cudaGetErrorString(e));
    }
    g_scratch_addr[dev] = p;
  }
  return g_scratch_addr[dev];
}

template <typename KeyT>
void sort_in_static_scratch(const void *keys_in, const uint32_t *values_in, void *keys_out, uint32_t *values_out,
                            uint32_t n, uint32_t begin_bit, uint32_t end_bit, cudaStream_t s) {
  char *base = static_cast<char *>(scratch_for_current_device());
  KeyT *scratch_keys = reinterpret_cast<KeyT *>(base);
  uint32_t *scratch_vals = reinterpret_cast<uint32_t *>(base + kKeyBytes);
  uint32_t *work = reinterpret_cast<uint32_t *>(base + kKeyBytes + kValBytes);
  uint32_t *status = reinterpret_cast<uint32_t *>(base + kKeyBytes + kValBytes + kWorkBytes);
  int dev = 0, sms = 148;
  GPULSM_CUDA(cudaGetDevice(&dev));
  GPULSM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const bool vals = values_in != nullptr;
  // the sort ping-pongs between the caller's output and the static scratch;
  // an in-place call (input == output) needs no first copy
  GPULSM_CUDA(cudaMemsetAsync(status, 0, 4, s));
  if (keys_out != keys_in)
    GPULSM_CUDA(cudaMemcpyAsync(keys_out, keys_in, size_t(n) * sizeof(KeyT), cudaMemcpyDeviceToDevice, s));
  if (vals && values_out != values_in)
    GPULSM_CUDA(cudaMemcpyAsync(values_out, values_in, size_t(n) * 4, cudaMemcpyDeviceToDevice, s));
  KeyT *kk[2] = {static_cast<KeyT *>(keys_out), scratch_keys};
  uint32_t *vv[2] = {values_out, scratch_vals};
  // radix::sort zeroes the histogram / look-back words it needs (kept from the previous call)
  const int cur = vals ? radix::sort<KeyT, true>(kk, vv, n, int(begin_bit), int(end_bit), work, status, sms, s)
                       : radix::sort<KeyT, false>(kk, vv, n, int(begin_bit), int(end_bit), work, status, sms, s);
  if (cur == 1) {
    GPULSM_CUDA(cudaMemcpyAsync(keys_out, scratch_keys, size_t(n) * sizeof(KeyT), cudaMemcpyDeviceToDevice, s));
    if (vals) GPULSM_CUDA(cudaMemcpyAsync(values_out, scratch_vals, size_t(n) * 4, cudaMemcpyDeviceToDevice, s));
  }
  // the status word lives in the shared array; it is copied into a host
  // variable on this thread's stack (no allocation) and the call waits for it
  uint32_t status_word = 0;
  GPULSM_CUDA(cudaMemcpyAsync(&status_word, status, 4, cudaMemcpyDeviceToHost, s));
  GPULSM_CUDA(cudaStreamSynchronize(s));
  if (status_word & kDevWaitTimeout)
    throw std::runtime_error(
        "gpulsm_sort_pairs_noalloc: a radix pass timed out waiting on its look-back; output invalid");
}
}  // namespace

size_t noalloc_scratch_bytes() { return kNoallocScratchBytes; }

void sort_pairs_noalloc(const void *keys_in, const uint32_t *values_in, void *keys_out, uint32_t *values_out,
                        uint64_t count, uint32_t key_bits, uint32_t begin_bit, uint32_t end_bit, cudaStream_t s) {
  if (count > kNoallocMaxKeys)
    throw std::length_error("gpulsm_sort_pairs_noalloc sorts at most " + std::to_string(kNoallocMaxKeys) +
                            " keys per call (its scratch is a fixed static array); got " + std::to_string(count));
  if (!count) return;
  if (key_bits == 32)
    sort_in_static_scratch<uint32_t>(keys_in, values_in, keys_out, values_out, uint32_t(count), begin_bit, end_bit, s);
  else
    sort_in_static_scratch<unsigned long long>(keys_in, values_in, keys_out, values_out, uint32_t(count), begin_bit,
                                               end_bit, s);
}

}  // namespace gpulsm
