// Multi-tenant batched dictionary: many independent u32 dictionaries updated
// in rounds with a handful of launches per round for all tenants together.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <vector>

#include "tenant_types.h"

namespace gpulsm {

class TenantPool {
 public:
  // capacities: host array, max live keys per tenant; max_round_keys bounds
  // the total batch of one round; tile / fan_in / fanout are the tunables.
  TenantPool(uint32_t tenants, const uint64_t *capacities, uint64_t max_round_keys, uint32_t tile,
             uint32_t fan_in, uint32_t fanout);
  ~TenantPool();
  TenantPool(const TenantPool &) = delete;
  TenantPool &operator=(const TenantPool &) = delete;

  void set_tuning(uint32_t tile, uint32_t fan_in, uint32_t fanout);
  // one round: keys/values concatenated per tenant, offsets[tenants + 1] (device)
  void insert_round(const uint32_t *keys, const uint32_t *values, const uint64_t *offsets, cudaStream_t s);
  // the same round replayed from a CUDA graph captured for these buffers
  void round_graph(const uint32_t *keys, const uint32_t *values, const uint64_t *offsets, cudaStream_t s);
  void lookup(const uint32_t *tenant_ids, const uint32_t *keys, uint64_t n, uint32_t *out_values,
              uint8_t *out_found, cudaStream_t s);
  void sizes(uint64_t *out_rows);
  uint32_t status();
  uint64_t resident_bytes() const;
  uint32_t tenants() const { return tenants_; }

 private:
  struct Graph {
    const uint32_t *keys;
    const uint32_t *values;
    const uint64_t *offsets;
    bool flush;
    cudaGraphExec_t exec;
  };
  uint32_t tenant_bits() const;
  void enqueue_round(const uint32_t *keys, const uint32_t *values, const uint64_t *offsets, bool flush,
                     cudaStream_t s);
  void merge(uint32_t kind, cudaStream_t s);
  void fences(uint32_t which, cudaStream_t s);
  void refresh_fences(cudaStream_t s);

  uint32_t tenants_;
  uint64_t max_round_;
  uint32_t tile_ = 2048, fan_in_ = 4, fanout_ = 16;
  uint64_t rounds_ = 0;
  bool fences_stale_ = false;
  int num_sms_ = 148;
  std::vector<uint64_t> caps_;
  tenants::TenantMeta *meta_ = nullptr;
  tenants::Arena arena_{};
  unsigned long long arena_rows_ = 0, fence_words_ = 0, max_tiles_ = 0;
  char *work_ = nullptr;
  size_t work_bytes_ = 0, zero_bytes_ = 0;
  unsigned long long *words_[2] = {nullptr, nullptr};
  uint32_t *wvals_[2] = {nullptr, nullptr};
  uint32_t *bkeys_ = nullptr, *bvals_ = nullptr, *btenant_ = nullptr;
  unsigned long long *bstart_ = nullptr, *tiles_ = nullptr, *tile_off_ = nullptr;
  uint32_t *out_n_ = nullptr, *misc_ = nullptr;
  char *zero_ = nullptr;
  uint32_t *radix_ws_ = nullptr, *dedup_ctr_ = nullptr;
  unsigned long long *dedup_lb_ = nullptr;
  uint32_t *merge_ctr_[2] = {nullptr, nullptr};
  unsigned long long *merge_lb_[2] = {nullptr, nullptr};
  std::vector<Graph> graphs_;
  cudaEvent_t op_done_ = nullptr;
  std::mutex mu_;
};

}  // namespace gpulsm
