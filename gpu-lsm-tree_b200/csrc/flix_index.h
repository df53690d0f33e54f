// Host engine of the FliX-style bucket layer: the B200 counterpart of
// cg_rtx_index_updates' bucket-layer surface (FliX/impl_cg_rtx_index_updates.cuh:1711-2677).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>

namespace gpulsm {

struct FlixConfig {
  uint32_t key_bits = 64;
  uint32_t node_size = 0;
  uint32_t fill_percent = 0;
  uint32_t search_mode = 0;
  uint64_t max_elements = 0;
};

class FlixIndex {
 public:
  explicit FlixIndex(const FlixConfig &config);
  ~FlixIndex();
  FlixIndex(const FlixIndex &) = delete;
  FlixIndex &operator=(const FlixIndex &) = delete;

  void build(const void *keys, const uint32_t *values, uint64_t n, uint64_t max_n, cudaStream_t s);
  void insert(const void *keys, const uint32_t *values, uint64_t n, cudaStream_t s);
  void remove(const void *keys, uint64_t n, cudaStream_t s);
  void lookups_ordered(const void *sorted_probes, uint64_t n, uint32_t *out, cudaStream_t s);
  void lookups_successor(const void *sorted_probes, uint64_t n, void *out_keys, cudaStream_t s);
  void lookup(const void *probes, uint64_t n, uint32_t *out, cudaStream_t s);
  void successor(const void *probes, uint64_t n, void *out_keys, cudaStream_t s);
  void rebuild(cudaStream_t s);
  uint64_t resident_bytes();
  uint64_t size();
  uint32_t status();
  void allocation_state(uint64_t *used, uint64_t *total, uint64_t *buckets, uint32_t *grows);

  struct Impl;

 private:
  std::unique_ptr<Impl> impl_;
  std::mutex mu_;
};

}  // namespace gpulsm
