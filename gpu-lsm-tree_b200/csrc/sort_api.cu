// Standalone entry to the onesweep radix sort (gpulsm_sort_pairs).  The call
// returns once the sort has finished: it reads back the passes' status word.
#include <algorithm>
#include <stdexcept>

#include "common.cuh"
#include "radix_sort.cuh"
#include "sort_api.h"

namespace gpulsm {

namespace {
template <typename KeyT>
void sort_typed(const void *keys_in, const uint32_t *values_in, void *keys_out,
                uint32_t *values_out, uint64_t count, uint32_t begin_bit, uint32_t end_bit,
                cudaStream_t s) {
  int dev = 0, sms = 148;
  GPULSM_CUDA(cudaGetDevice(&dev));
  GPULSM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int passes = int((end_bit - begin_bit + 7) / 8);
  const size_t ws_bytes = radix::workspace_bytes(count, passes) + 256;
  const bool vals = values_in != nullptr;
  const size_t kb = count * sizeof(KeyT), vb = vals ? count * 4 : 0;
  char *block = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void **>(&block), ws_bytes + 2 * kb + 2 * vb + 1024, s) !=
      cudaSuccess) {
    (void)cudaGetLastError();
    throw std::bad_alloc();
  }
  uint32_t *ws = reinterpret_cast<uint32_t *>(block);
  uint32_t *status = ws + (ws_bytes - 256) / 4;
  KeyT *k0 = reinterpret_cast<KeyT *>(block + ((ws_bytes + 255) & ~size_t(255)));
  KeyT *k1 = reinterpret_cast<KeyT *>(reinterpret_cast<char *>(k0) + ((kb + 255) & ~size_t(255)));
  uint32_t *v0 = reinterpret_cast<uint32_t *>(reinterpret_cast<char *>(k1) + ((kb + 255) & ~size_t(255)));
  uint32_t *v1 = v0 + ((vb + 255) & ~size_t(255)) / 4;
  GPULSM_CUDA(cudaMemsetAsync(status, 0, 4, s));
  GPULSM_CUDA(cudaMemcpyAsync(k0, keys_in, kb, cudaMemcpyDeviceToDevice, s));
  if (vals) GPULSM_CUDA(cudaMemcpyAsync(v0, values_in, vb, cudaMemcpyDeviceToDevice, s));
  KeyT *kk[2] = {k0, k1};
  uint32_t *vv[2] = {v0, v1};
  int cur;
  if (vals)
    cur = radix::sort<KeyT, true>(kk, vv, uint32_t(count), int(begin_bit), int(end_bit), ws, status,
                                  sms, s);
  else
    cur = radix::sort<KeyT, false>(kk, vv, uint32_t(count), int(begin_bit), int(end_bit), ws,
                                   status, sms, s);
  GPULSM_CUDA(cudaMemcpyAsync(keys_out, kk[cur], kb, cudaMemcpyDeviceToDevice, s));
  if (vals) GPULSM_CUDA(cudaMemcpyAsync(values_out, vv[cur], vb, cudaMemcpyDeviceToDevice, s));
  // the passes' status word: a look-back wait that gave up leaves the output
  // unsorted, so the call waits for the sort and reports it
  uint32_t status_word = 0;
  GPULSM_CUDA(cudaMemcpyAsync(&status_word, status, 4, cudaMemcpyDeviceToHost, s));
  GPULSM_CUDA(cudaFreeAsync(block, s));
  GPULSM_CUDA(cudaStreamSynchronize(s));
  if (status_word & kDevWaitTimeout)
    throw std::runtime_error("gpulsm_sort_pairs: a radix pass timed out waiting on its look-back; output invalid");
}
}  // namespace

void sort_pairs_any(const void *keys_in, const uint32_t *values_in, void *keys_out,
                    uint32_t *values_out, uint64_t count, uint32_t key_bits, uint32_t begin_bit,
                    uint32_t end_bit, cudaStream_t s) {
  if (key_bits == 32)
    sort_typed<uint32_t>(keys_in, values_in, keys_out, values_out, count, begin_bit, end_bit, s);
  else
    sort_typed<unsigned long long>(keys_in, values_in, keys_out, values_out, count, begin_bit,
                                   end_bit, s);
}

}  // namespace gpulsm
