// gpulsmopt_b200.cuh - the reference-side drop-in for GPULSMOpt over the C ABI.
//
// A C++ caller of the reference's GPULSMOpt (GPULSMOpt.cuh:5599-5881), such as
// FliX's index adapter (FliX/impl_gpulsmopt.cuh:137-311) or the paper sweep
// (FliX/paper_lsmu_sweep.cu), replaces its one `#include "GPULSMOpt.cuh"` with
// `#include "gpulsmopt_b200.cuh"` and links libgpulsm.so; nothing else in the
// caller changes.  The class keeps the reference's name, its adapter structs
// (gpu_dictionary_adapter.cuh, included unchanged from the caller's tree), its
// method names and argument meaning, and its exception classes:
//   invalid_argument (null pointers, bad sizes), length_error, bad_alloc,
//   runtime_error (capacity, publication, CUDA errors, device wait time-outs).
// Updates complete in the caller's stream as the reference's do: insert and
// erase join the dictionary's merge stream before returning.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <new>
#include <stdexcept>
#include <string>

#include "gpu_dictionary_adapter.cuh"
#include "gpulsm.h"

// The two reference constants the FliX adapter reports in its parameter list
// (FliX/impl_gpulsmopt.cuh:69,180-183; GPULSMOpt.cuh:41-42).  They describe the
// reference's own layout; this engine's levels are set by DictionaryConfig.
namespace gpulsmopt2_detail {
constexpr std::uint32_t kMaximumLevels = 64u;
constexpr std::uint32_t kBatchesPerEpoch = 16u;
}  // namespace gpulsmopt2_detail

class GPULSMOpt {
 public:
  struct DeviceKeyBatch {
    const std::uint32_t *keys = nullptr;
    std::size_t count = 0;
  };

  explicit GPULSMOpt(const DictionaryConfig &c) {
    gpulsm_dict_config g{};
    g.max_elements = c.max_elements;
    g.batch_capacity = c.batch_capacity;
    g.level_zero_capacity = c.level_zero_capacity;
    check(gpulsm_dict_create(&g, &d_));
  }
  ~GPULSMOpt() { gpulsm_dict_destroy(d_); }
  GPULSMOpt(const GPULSMOpt &) = delete;
  GPULSMOpt &operator=(const GPULSMOpt &) = delete;

  void clear(cudaStream_t s) { check(gpulsm_dict_clear(d_, s)); }

  void bulk_build(const std::uint32_t *keys, const std::uint32_t *values, std::size_t count, cudaStream_t s) {
    check(gpulsm_dict_bulk_build(d_, keys, values, count, s));
  }

  void insert(const DeviceKeyValueBatch &b, cudaStream_t s) {
    check(gpulsm_dict_insert(d_, b.keys, b.values, b.count, s));
    check(gpulsm_dict_join(d_, s));
  }

  void erase(const DeviceKeyBatch &b, cudaStream_t s) {
    check(gpulsm_dict_erase(d_, b.keys, b.count, s));
    check(gpulsm_dict_join(d_, s));
  }

  // quotients_grouped is a hint of the reference's quotient layout; lookups
  // here need no grouping, so it is accepted and ignored
  void lookup(const DeviceLookupBatch &b, cudaStream_t s, bool quotients_grouped = false) {
    (void)quotients_grouped;
    check(gpulsm_dict_lookup(d_, b.queries, b.count, b.out_values, b.out_found, s));
  }

  void range(const DeviceRangeOutputBatch &b, cudaStream_t s) {
    check(gpulsm_dict_range_sum(d_, b.lo, b.hi, b.query_count, b.out_sums, s));
  }

  void successor(const DeviceSuccessorBatch &b, cudaStream_t s) {
    check(gpulsm_dict_successor(d_, b.queries, b.count, b.out_keys, s));
  }

  std::uint32_t canonical_carry_status() const {
    std::uint32_t v = 0;
    check(gpulsm_dict_status(d_, &v));
    return v;
  }

  std::size_t gpu_resident_bytes() const {
    std::uint64_t v = 0;
    check(gpulsm_dict_resident_bytes(d_, &v));
    return static_cast<std::size_t>(v);
  }

 private:
  static void check(int rc) {
    if (rc == GPULSM_OK) return;
    const std::string m = gpulsm_last_error();
    if (rc == GPULSM_ERR_INVALID_ARGUMENT) throw std::invalid_argument(m);
    if (rc == GPULSM_ERR_LENGTH) throw std::length_error(m);
    if (rc == GPULSM_ERR_OUT_OF_MEMORY) throw std::bad_alloc();
    throw std::runtime_error(m);
  }

  gpulsm_dict *d_ = nullptr;
};
