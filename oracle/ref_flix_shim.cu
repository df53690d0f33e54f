// C-ABI shim over the reference's own FliX bucket layer.  TEST INFRASTRUCTURE ONLY.
//
// This translation unit contains no reference code: it #includes
// FliX/impl_cg_rtx_index_updates.cuh in place (the include path points at the
// read-only reference checkout) and wraps the bucket-layer methods of
// class cg_rtx_index_updates in extern "C" functions, so tests can drive the
// reference's FliX kernels on a B200 as a GPU parity oracle and time them
// beside ours.  The OptiX names the header mentions come from
// flix_shim/optix_decls.h as declarations only; the library is linked with
// -z defs, so it cannot reference any OptiX function.
//
// The instantiation follows the reference's published update experiments
// (FliX/build/runscripts_experiments/LookupsSorted_VaryingRounds.sh:36-50 with
// NodeSizeInput 5): node_size_log 5 (32 keys per node), cache_line 0, initial
// fill 50%, compiled with TILE_INSERTS TILE_INSERTS_C INSERTS_TILE_BULK_ONLY
// TILE_DELETES DELETES_TILE_BULK, MAX_NODE 32 and tile size 32 (see Makefile).
// Built by oracle/Makefile into oracle/_ref/ only.
//
// Known defect of the reference for 64-bit keys: its tiled ordered lookup and
// tiled bulk delete read a node entry's value with extract_offset_node<smallsize>
// (FliX/coarse_granular_lookups_tile_bulk.cuh:403,
// FliX/coarse_granular_deletes_tiles.cuh:1201), which places the value as if
// keys were 4 bytes wide (FliX/coarse_granular_inserts.cuh:51-55).  With 8-byte
// keys it reads bytes of a key instead, and deletes move those bytes into the
// value slots.  Only build, insert and successor are correct for 64-bit keys
// in this instantiation; 32-bit keys (the published configuration) are exact.
#include "optix_decls.h"
#include "impl_cg_rtx_index_updates.cuh"

#include <cstdint>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>

// the header declares it `extern` (FliX/impl_cg_rtx_index_updates.cuh:52); the
// bucket layer never reads it
optix_wrapper optix;

namespace {
thread_local std::string g_last_error;

template <class F> int guarded(F &&f) {
  try {
    f();
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
      g_last_error = cudaGetErrorString(e);
      return 4;
    }
    return 0;
  } catch (const std::invalid_argument &e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::bad_alloc &e) {
    g_last_error = e.what();
    return 6;
  } catch (const std::runtime_error &e) {
    g_last_error = e.what();
    return 3;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return 5;
  }
}

struct FlixRef {
  virtual ~FlixRef() = default;
  virtual void build(const void *keys, size_t n, size_t max_n) = 0;
  virtual void rebuild() = 0;
  virtual void insert(const void *keys, const uint32_t *values, size_t n, cudaStream_t s) = 0;
  virtual void remove(const void *keys, size_t n, cudaStream_t s) = 0;
  virtual void lookups_ordered(const void *keys, uint32_t *out, size_t n, cudaStream_t s) = 0;
  virtual void lookups_successor(const void *keys, void *out, size_t n, cudaStream_t s) = 0;
  virtual size_t total_keys(cudaStream_t s) = 0;
  virtual size_t resident_bytes() = 0;
  virtual uint64_t next_free() = 0;
  virtual uint64_t allocation_nodes() = 0;
  virtual uint64_t bucket_count() = 0;
};

template <typename K> struct FlixRefT final : FlixRef {
  using Index = cg_rtx_index_updates<K, 0, 5, 50>;
  Index index;
  ~FlixRefT() override { index.destroy(); }
  void build(const void *keys, size_t n, size_t max_n) override {
    double ms = 0;
    size_t bytes = 0;
    index.build_bucket_layer_only(static_cast<const K *>(keys), n, max_n, 0, &ms, &bytes);
  }
  void rebuild() override {
    double ms = 0;
    size_t bytes = 0;
    index.rebuild_bucket_layer_only(&ms, &bytes);
  }
  void insert(const void *keys, const uint32_t *values, size_t n, cudaStream_t s) override {
    index.insert(static_cast<const K *>(keys), values, n, s);
  }
  void remove(const void *keys, size_t n, cudaStream_t s) override {
    index.remove(static_cast<const K *>(keys), n, s);
  }
  void lookups_ordered(const void *keys, uint32_t *out, size_t n, cudaStream_t s) override {
    index.lookups_ordered(static_cast<const K *>(keys), out, n, s);
  }
  void lookups_successor(const void *keys, void *out, size_t n, cudaStream_t s) override {
    index.lookups_successor(static_cast<const K *>(keys), static_cast<K *>(out), n, s);
  }
  // compute_total_size bounds its chain walks by the host's copy of the next
  // free allocation-region node, refreshed only by allocation_buffer_next_free
  // (FliX/impl_cg_rtx_index_updates.cuh:1657-1700); refresh it first
  size_t total_keys(cudaStream_t s) override {
    index.allocation_buffer_next_free();
    return index.compute_total_size(s);
  }
  size_t resident_bytes() override { return index.gpu_resident_bytes(); }
  uint64_t next_free() override { return index.allocation_buffer_next_free(); }
  uint64_t allocation_nodes() override { return index.allocation_buffer_total_nodes(); }
  uint64_t bucket_count() override { return index.partition_count_with_overflow; }
};

FlixRef *as_ref(void *h) {
  if (!h) throw std::invalid_argument("null FliX reference handle");
  return static_cast<FlixRef *>(h);
}
}  // namespace

extern "C" {

const char *reff_last_error(void) { return g_last_error.c_str(); }

int reff_create(int key_bits, void **out) {
  return guarded([&] {
    if (!out) throw std::invalid_argument("null output handle");
    if (key_bits == 32)
      *out = new FlixRefT<uint32_t>();
    else if (key_bits == 64)
      *out = new FlixRefT<uint64_t>();
    else
      throw std::invalid_argument("key_bits must be 32 or 64");
  });
}

int reff_destroy(void *h) {
  return guarded([&] { delete as_ref(h); });
}

int reff_build(void *h, const void *keys, uint64_t n, uint64_t max_n) {
  return guarded([&] { as_ref(h)->build(keys, n, max_n); });
}

int reff_rebuild(void *h) {
  return guarded([&] { as_ref(h)->rebuild(); });
}

int reff_insert(void *h, const void *keys, const uint32_t *values, uint64_t n, void *stream) {
  return guarded([&] { as_ref(h)->insert(keys, values, n, static_cast<cudaStream_t>(stream)); });
}

int reff_remove(void *h, const void *keys, uint64_t n, void *stream) {
  return guarded([&] { as_ref(h)->remove(keys, n, static_cast<cudaStream_t>(stream)); });
}

int reff_lookups_ordered(void *h, const void *keys, uint32_t *out, uint64_t n, void *stream) {
  return guarded([&] { as_ref(h)->lookups_ordered(keys, out, n, static_cast<cudaStream_t>(stream)); });
}

int reff_lookups_successor(void *h, const void *keys, void *out, uint64_t n, void *stream) {
  return guarded([&] { as_ref(h)->lookups_successor(keys, out, n, static_cast<cudaStream_t>(stream)); });
}

int reff_total_keys(void *h, void *stream, uint64_t *out) {
  return guarded([&] { *out = as_ref(h)->total_keys(static_cast<cudaStream_t>(stream)); });
}

int reff_resident_bytes(void *h, uint64_t *out) {
  return guarded([&] { *out = as_ref(h)->resident_bytes(); });
}

int reff_allocation_state(void *h, uint64_t *next_free, uint64_t *total_nodes, uint64_t *buckets) {
  return guarded([&] {
    FlixRef *r = as_ref(h);
    *next_free = r->next_free();
    *total_nodes = r->allocation_nodes();
    *buckets = r->bucket_count();
  });
}

}  // extern "C"
