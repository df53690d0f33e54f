// extern "C" boundary (include/gpulsm.h): maps C++ exceptions of the engines
// to gpulsm_status codes, as a C caller (ctypes / cgo / JNI) needs.
#include "../../include/gpulsm.h"

#include <cuda_runtime.h>

#include <new>
#include <stdexcept>
#include <string>

#include "common.cuh"
#include "flix_index.h"
#include "lsm_dictionary.h"
#include "radix_sort.cuh"
#include "model_api.h"
#include "serving.h"
#include "sort_api.h"
#include "sort_noalloc.h"
#include "tenants.h"

struct gpulsm_dict {
  gpulsm::LsmDictionary impl;
  explicit gpulsm_dict(const gpulsm::DictConfig &c) : impl(c) {}
};

struct gpulsm_flix {
  gpulsm::FlixIndex impl;
  explicit gpulsm_flix(const gpulsm::FlixConfig &c) : impl(c) {}
};

struct gpulsm_tenants {
  gpulsm::TenantPool impl;
  gpulsm_tenants(uint32_t t, const uint64_t *caps, uint64_t max_round, uint32_t tile, uint32_t fan_in,
                 uint32_t fanout)
      : impl(t, caps, max_round, tile, fan_in, fanout) {}
};

struct gpulsm_server {
  gpulsm::Server impl;
  gpulsm_server(const gpulsm::DictConfig &c, uint64_t budget, uint32_t round, uint32_t depth)
      : impl(c, budget, round, depth) {}
};

namespace {
thread_local std::string g_error;

template <class F> int guarded(F &&f) {
  try {
    f();
    return GPULSM_OK;
  } catch (const std::invalid_argument &e) {
    g_error = e.what();
    return GPULSM_ERR_INVALID_ARGUMENT;
  } catch (const std::length_error &e) {
    g_error = e.what();
    return GPULSM_ERR_LENGTH;
  } catch (const std::bad_alloc &e) {
    g_error = std::string("out of device memory: ") + e.what();
    return GPULSM_ERR_OUT_OF_MEMORY;
  } catch (const gpulsm::CudaError &e) {
    g_error = e.what();
    return e.code == cudaErrorMemoryAllocation ? GPULSM_ERR_OUT_OF_MEMORY : GPULSM_ERR_CUDA;
  } catch (const std::runtime_error &e) {
    g_error = e.what();
    const std::string m = e.what();
    if (m.find("capacity") != std::string::npos) return GPULSM_ERR_CAPACITY;
    if (m.find("timed out") != std::string::npos) return GPULSM_ERR_TIMEOUT;
    return GPULSM_ERR_PUBLICATION;
  } catch (const std::exception &e) {
    g_error = e.what();
    return GPULSM_ERR_CUDA;
  }
}

inline cudaStream_t S(void *s) { return static_cast<cudaStream_t>(s); }

template <class T> void need(T *p, const char *what) {
  if (!p) throw std::invalid_argument(std::string("null ") + what);
}

// Rejects a non-null pointer the GPU cannot dereference (pageable host memory,
// an integer passed in a pointer slot) before any kernel can touch it, so a
// caller mistake becomes GPULSM_ERR_INVALID_ARGUMENT instead of a device fault.
// Null pointers are left to the engines' own argument checks.
void device_accessible(const void *p, const char *what) {
  if (!p) return;
  cudaPointerAttributes a{};
  const cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw std::invalid_argument(std::string(what) + " is not a CUDA pointer");
  }
  if (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) return;
  if (a.type == cudaMemoryTypeHost && a.devicePointer) return;  // mapped pinned host memory
  throw std::invalid_argument(std::string(what) + " is not device-accessible memory");
}

void device_accessible(std::initializer_list<std::pair<const void *, const char *>> ptrs) {
  for (const auto &p : ptrs) device_accessible(p.first, p.second);
}

// The sort entries accept an output equal to its input (in place) but no
// partial overlap between any two of the four buffers.
bool ranges_overlap(const void *a, size_t an, const void *b, size_t bn) {
  if (!a || !b || !an || !bn) return false;
  const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return x < y + bn && y < x + an;
}

void no_partial_overlap(const void *ki, const void *ko, size_t kbytes, const void *vi, const void *vo,
                        size_t vbytes) {
  if (ki != ko && ranges_overlap(ki, kbytes, ko, kbytes))
    throw std::invalid_argument("keys_in and keys_out overlap partially (only keys_in == keys_out is allowed)");
  if (vi != vo && ranges_overlap(vi, vbytes, vo, vbytes))
    throw std::invalid_argument("values_in and values_out overlap partially (only values_in == values_out is allowed)");
  if (ranges_overlap(ko, kbytes, vo, vbytes) || ranges_overlap(ki, kbytes, vo, vbytes) ||
      ranges_overlap(ko, kbytes, vi, vbytes))
    throw std::invalid_argument("a key buffer overlaps a value buffer");
}

gpulsm::DictConfig dict_config(const gpulsm_dict_config &config) {
  gpulsm::DictConfig c;
  c.max_elements = config.max_elements;
  c.batch_capacity = config.batch_capacity;
  c.level_zero_capacity = config.level_zero_capacity;
  c.fan_in = config.fan_in;
  c.rows_per_bucket_log2 = config.rows_per_bucket_log2;
  c.search_mode = config.search_mode;
  return c;
}

void copy_stats(const gpulsm::ServeStats &s, gpulsm_serve_stats *o) {
  o->completed = s.completed;
  o->rejected = s.rejected;
  o->rounds = s.rounds;
  o->keys = s.keys;
  o->p50_us = s.p50_us;
  o->p99_us = s.p99_us;
  o->max_us = s.max_us;
  o->mean_us = s.mean_us;
  o->mean_round_keys = s.mean_round_keys;
  o->wall_s = s.wall_s;
  o->gpu_busy_s = s.gpu_busy_s;
  o->host_launch_s = s.host_launch_s;
  o->graph_rounds = s.graph_rounds;
  for (int k = 0; k < 4; ++k) o->kind_gpu_s[k] = s.kind_gpu_s[k];
  o->host_copy_s = s.host_copy_s;
  o->host_scatter_s = s.host_scatter_s;
  o->graph_updates = s.graph_updates;
  o->stage_flushes = s.stage_flushes;
  o->max_round_gpu_us = s.max_round_gpu_us;
  o->max_launch_us = s.max_launch_us;
}
}  // namespace

extern "C" {

const char *gpulsm_last_error(void) { return g_error.c_str(); }
const char *gpulsm_version(void) { return "gpulsm-b200 0.1 (sm_100a)"; }
uint64_t gpulsm_launch_count(void) { return gpulsm::launch_counter().load(); }

// ---------------------------------------------------------------- LSM dictionary
int gpulsm_dict_create(const gpulsm_dict_config *config, gpulsm_dict **out) {
  return guarded([&] {
    need(config, "config");
    need(out, "out");
    *out = new gpulsm_dict(dict_config(*config));
  });
}

int gpulsm_dict_destroy(gpulsm_dict *d) {
  return guarded([&] { delete d; });
}

int gpulsm_dict_clear(gpulsm_dict *d, void *stream) {
  return guarded([&] {
    need(d, "dict");
    d->impl.clear(S(stream));
  });
}

int gpulsm_dict_join(gpulsm_dict *d, void *stream) {
  return guarded([&] {
    need(d, "dict");
    d->impl.join(S(stream));
  });
}

int gpulsm_dict_bulk_build(gpulsm_dict *d, const uint32_t *keys, const uint32_t *values,
                           uint64_t count, void *stream) {
  return guarded([&] {
    need(d, "dict");
    device_accessible({{keys, "keys"}, {values, "values"}});
    d->impl.bulk_build(keys, values, count, S(stream));
  });
}

int gpulsm_dict_insert(gpulsm_dict *d, const uint32_t *keys, const uint32_t *values,
                       uint64_t count, void *stream) {
  return guarded([&] {
    need(d, "dict");
    device_accessible({{keys, "keys"}, {values, "values"}});
    d->impl.insert(keys, values, count, S(stream));
  });
}

int gpulsm_dict_erase(gpulsm_dict *d, const uint32_t *keys, uint64_t count, void *stream) {
  return guarded([&] {
    need(d, "dict");
    device_accessible({{keys, "keys"}});
    d->impl.erase(keys, count, S(stream));
  });
}

int gpulsm_dict_update(gpulsm_dict *d, const uint32_t *keys, const uint32_t *values, const uint8_t *erase,
                       uint64_t count, void *stream) {
  return guarded([&] {
    need(d, "dict");
    device_accessible({{keys, "keys"}, {values, "values"}, {erase, "erase"}});
    d->impl.update(keys, values, erase, count, S(stream));
  });
}

int gpulsm_dict_lookup(gpulsm_dict *d, const uint32_t *queries, uint64_t count,
                       uint32_t *out_values, uint8_t *out_found, void *stream) {
  return guarded([&] {
    need(d, "dict");
    device_accessible({{queries, "queries"}, {out_values, "out_values"}, {out_found, "out_found"}});
    d->impl.lookup(queries, count, out_values, out_found, S(stream));
  });
}

int gpulsm_dict_range_sum(gpulsm_dict *d, const uint32_t *lo, const uint32_t *hi, uint64_t count,
                          uint32_t *out_sums, void *stream) {
  return guarded([&] {
    need(d, "dict");
    device_accessible({{lo, "lo"}, {hi, "hi"}, {out_sums, "out_sums"}});
    d->impl.range_sum(lo, hi, count, out_sums, S(stream));
  });
}

int gpulsm_dict_range_count(gpulsm_dict *d, const uint32_t *lo, const uint32_t *hi,
                            uint64_t count, uint32_t *out_counts, void *stream) {
  return guarded([&] {
    need(d, "dict");
    device_accessible({{lo, "lo"}, {hi, "hi"}, {out_counts, "out_counts"}});
    d->impl.range_count(lo, hi, count, out_counts, S(stream));
  });
}

int gpulsm_dict_range_offsets(gpulsm_dict *d, const uint32_t *lo, const uint32_t *hi,
                              uint64_t count, uint64_t *offsets, void *stream) {
  return guarded([&] {
    need(d, "dict");
    device_accessible({{lo, "lo"}, {hi, "hi"}, {offsets, "offsets"}});
    d->impl.range_offsets(lo, hi, count, offsets, S(stream));
  });
}

int gpulsm_dict_range_pairs(gpulsm_dict *d, const uint32_t *lo, const uint32_t *hi,
                            uint64_t count, const uint64_t *offsets, uint32_t *out_keys,
                            uint32_t *out_values, void *stream) {
  return guarded([&] {
    need(d, "dict");
    device_accessible({{lo, "lo"}, {hi, "hi"}, {offsets, "offsets"}, {out_keys, "out_keys"}, {out_values, "out_values"}});
    d->impl.range_pairs(lo, hi, count, offsets, out_keys, out_values, S(stream));
  });
}

int gpulsm_dict_successor(gpulsm_dict *d, const uint32_t *queries, uint64_t count,
                          uint32_t *out_keys, void *stream) {
  return guarded([&] {
    need(d, "dict");
    device_accessible({{queries, "queries"}, {out_keys, "out_keys"}});
    d->impl.successor(queries, count, out_keys, S(stream));
  });
}

int gpulsm_dict_status(gpulsm_dict *d, uint32_t *out_status) {
  return guarded([&] {
    need(d, "dict");
    need(out_status, "out_status");
    *out_status = d->impl.status();
  });
}

int gpulsm_dict_resident_bytes(gpulsm_dict *d, uint64_t *out_bytes) {
  return guarded([&] {
    need(d, "dict");
    need(out_bytes, "out_bytes");
    *out_bytes = d->impl.resident_bytes();
  });
}

int gpulsm_dict_kernel_timing(gpulsm_dict *d, int enable) {
  return guarded([&] {
    need(d, "dict");
    d->impl.set_kernel_timing(enable != 0);
  });
}

int gpulsm_dict_kernel_timing_read(gpulsm_dict *d, uint64_t *out_launches, double *out_ms, double *out_bytes) {
  return guarded([&] {
    need(d, "dict");
    d->impl.kernel_timing(out_launches, out_ms, out_bytes);
  });
}

int gpulsm_dict_cleanup(gpulsm_dict *d, void *stream, uint64_t *out_live_keys) {
  return guarded([&] {
    need(d, "dict");
    const uint64_t n = d->impl.cleanup(S(stream));
    if (out_live_keys) *out_live_keys = n;
  });
}

int gpulsm_dict_size(gpulsm_dict *d, uint64_t *out_rows, uint32_t *out_levels) {
  return guarded([&] {
    need(d, "dict");
    d->impl.size(out_rows, out_levels);
  });
}

// ---------------------------------------------------------------- FliX
int gpulsm_flix_create(const gpulsm_flix_config *config, gpulsm_flix **out) {
  return guarded([&] {
    need(config, "config");
    need(out, "out");
    gpulsm::FlixConfig c;
    c.key_bits = config->key_bits;
    c.node_size = config->node_size;
    c.fill_percent = config->fill_percent;
    c.search_mode = config->search_mode;
    c.max_elements = config->max_elements;
    *out = new gpulsm_flix(c);
  });
}

int gpulsm_flix_destroy(gpulsm_flix *f) {
  return guarded([&] { delete f; });
}

int gpulsm_flix_build(gpulsm_flix *f, const void *keys, const uint32_t *values, uint64_t count,
                      uint64_t max_count, void *stream) {
  return guarded([&] {
    need(f, "index");
    device_accessible({{keys, "keys"}, {values, "values"}});
    f->impl.build(keys, values, count, max_count, S(stream));
  });
}

int gpulsm_flix_insert(gpulsm_flix *f, const void *keys, const uint32_t *values, uint64_t count,
                       void *stream) {
  return guarded([&] {
    need(f, "index");
    device_accessible({{keys, "keys"}, {values, "values"}});
    f->impl.insert(keys, values, count, S(stream));
  });
}

int gpulsm_flix_remove(gpulsm_flix *f, const void *keys, uint64_t count, void *stream) {
  return guarded([&] {
    need(f, "index");
    device_accessible({{keys, "keys"}});
    f->impl.remove(keys, count, S(stream));
  });
}

int gpulsm_flix_lookups_ordered(gpulsm_flix *f, const void *sorted_probes, uint64_t count,
                                uint32_t *out_values, void *stream) {
  return guarded([&] {
    need(f, "index");
    device_accessible({{sorted_probes, "probes"}, {out_values, "out_values"}});
    f->impl.lookups_ordered(sorted_probes, count, out_values, S(stream));
  });
}

int gpulsm_flix_lookups_successor(gpulsm_flix *f, const void *sorted_probes, uint64_t count,
                                  void *out_keys, void *stream) {
  return guarded([&] {
    need(f, "index");
    device_accessible({{sorted_probes, "probes"}, {out_keys, "out_keys"}});
    f->impl.lookups_successor(sorted_probes, count, out_keys, S(stream));
  });
}

int gpulsm_flix_lookup(gpulsm_flix *f, const void *probes, uint64_t count, uint32_t *out_values,
                       void *stream) {
  return guarded([&] {
    need(f, "index");
    device_accessible({{probes, "probes"}, {out_values, "out_values"}});
    f->impl.lookup(probes, count, out_values, S(stream));
  });
}

int gpulsm_flix_successor(gpulsm_flix *f, const void *probes, uint64_t count, void *out_keys,
                          void *stream) {
  return guarded([&] {
    need(f, "index");
    device_accessible({{probes, "probes"}, {out_keys, "out_keys"}});
    f->impl.successor(probes, count, out_keys, S(stream));
  });
}

int gpulsm_flix_rebuild(gpulsm_flix *f, void *stream) {
  return guarded([&] {
    need(f, "index");
    f->impl.rebuild(S(stream));
  });
}

int gpulsm_flix_resident_bytes(gpulsm_flix *f, uint64_t *out_bytes) {
  return guarded([&] {
    need(f, "index");
    need(out_bytes, "out_bytes");
    *out_bytes = f->impl.resident_bytes();
  });
}

int gpulsm_flix_size(gpulsm_flix *f, uint64_t *out_keys) {
  return guarded([&] {
    need(f, "index");
    need(out_keys, "out_keys");
    *out_keys = f->impl.size();
  });
}

int gpulsm_flix_allocation_state(gpulsm_flix *f, uint64_t *out_used_nodes, uint64_t *out_region_nodes,
                                 uint64_t *out_buckets, uint32_t *out_grows) {
  return guarded([&] {
    need(f, "index");
    need(out_used_nodes, "out_used_nodes");
    need(out_region_nodes, "out_region_nodes");
    need(out_buckets, "out_buckets");
    need(out_grows, "out_grows");
    f->impl.allocation_state(out_used_nodes, out_region_nodes, out_buckets, out_grows);
  });
}

int gpulsm_flix_status(gpulsm_flix *f, uint32_t *out_status) {
  return guarded([&] {
    need(f, "index");
    need(out_status, "out_status");
    *out_status = f->impl.status();
  });
}

// ---------------------------------------------------------------- tenants
int gpulsm_tenants_create(uint32_t tenants, const uint64_t *capacities, uint64_t max_round_keys, uint32_t tile,
                          uint32_t fan_in, uint32_t fanout, gpulsm_tenants **out) {
  return guarded([&] {
    need(out, "out");
    need(capacities, "capacities");
    *out = new gpulsm_tenants(tenants, capacities, max_round_keys, tile, fan_in, fanout);
  });
}

int gpulsm_tenants_destroy(gpulsm_tenants *p) {
  return guarded([&] { delete p; });
}

int gpulsm_tenants_set_tuning(gpulsm_tenants *p, uint32_t tile, uint32_t fan_in, uint32_t fanout) {
  return guarded([&] {
    need(p, "pool");
    p->impl.set_tuning(tile, fan_in, fanout);
  });
}

int gpulsm_tenants_insert_round(gpulsm_tenants *p, const uint32_t *keys, const uint32_t *values,
                                const uint64_t *offsets, void *stream) {
  return guarded([&] {
    need(p, "pool");
    device_accessible({{keys, "keys"}, {values, "values"}, {offsets, "offsets"}});
    p->impl.insert_round(keys, values, offsets, S(stream));
  });
}

int gpulsm_tenants_round_graph(gpulsm_tenants *p, const uint32_t *keys, const uint32_t *values,
                               const uint64_t *offsets, void *stream) {
  return guarded([&] {
    need(p, "pool");
    device_accessible({{keys, "keys"}, {values, "values"}, {offsets, "offsets"}});
    p->impl.round_graph(keys, values, offsets, S(stream));
  });
}

int gpulsm_tenants_lookup(gpulsm_tenants *p, const uint32_t *tenant_ids, const uint32_t *keys, uint64_t count,
                          uint32_t *out_values, uint8_t *out_found, void *stream) {
  return guarded([&] {
    need(p, "pool");
    device_accessible({{tenant_ids, "tenant_ids"}, {keys, "keys"}, {out_values, "out_values"},
                       {out_found, "out_found"}});
    p->impl.lookup(tenant_ids, keys, count, out_values, out_found, S(stream));
  });
}

int gpulsm_tenants_sizes(gpulsm_tenants *p, uint64_t *out_rows) {
  return guarded([&] {
    need(p, "pool");
    need(out_rows, "out_rows");
    p->impl.sizes(out_rows);
  });
}

int gpulsm_tenants_status(gpulsm_tenants *p, uint32_t *out_status) {
  return guarded([&] {
    need(p, "pool");
    need(out_status, "out_status");
    *out_status = p->impl.status();
  });
}

int gpulsm_tenants_resident_bytes(gpulsm_tenants *p, uint64_t *out_bytes) {
  return guarded([&] {
    need(p, "pool");
    need(out_bytes, "out_bytes");
    *out_bytes = p->impl.resident_bytes();
  });
}

// ---------------------------------------------------------------- learned model
uint64_t gpulsm_model_bytes(uint32_t segments) { return gpulsm::learned::bytes_for(segments); }

int gpulsm_model_fit(const void *sorted_keys, uint64_t count, uint32_t key_bits, uint32_t segments,
                     uint32_t iters, void *model, float *loss_history, void *stream) {
  return guarded([&] {
    if (key_bits != 32 && key_bits != 64) throw std::invalid_argument("key_bits must be 32 or 64");
    if (count && !sorted_keys) throw std::invalid_argument("null keys");
    need(model, "model");
    if (!segments || segments > (1u << 24)) throw std::invalid_argument("segments must be in [1, 2^24]");
    if (count > 0xffffffffull) throw std::length_error("model fit limited to 2^32-1 keys");
    device_accessible({{sorted_keys, "sorted_keys"}, {model, "model"}, {loss_history, "loss_history"}});
    if (key_bits == 32)
      gpulsm::learned::fit(static_cast<const uint32_t *>(sorted_keys), count, segments, iters, model,
                           loss_history, S(stream));
    else
      gpulsm::learned::fit(static_cast<const unsigned long long *>(sorted_keys), count, segments, iters, model,
                           loss_history, S(stream));
  });
}

int gpulsm_model_gradients(const void *sorted_keys, uint64_t count, uint32_t key_bits, uint32_t segments,
                           void *model, float *grad, float *loss, void *stream) {
  return guarded([&] {
    if (key_bits != 32 && key_bits != 64) throw std::invalid_argument("key_bits must be 32 or 64");
    need(model, "model");
    need(grad, "grad");
    device_accessible({{sorted_keys, "sorted_keys"}, {model, "model"}, {grad, "grad"}, {loss, "loss"}});
    if (key_bits == 32)
      gpulsm::learned::gradients(static_cast<const uint32_t *>(sorted_keys), count, segments, model, grad, loss,
                                 S(stream));
    else
      gpulsm::learned::gradients(static_cast<const unsigned long long *>(sorted_keys), count, segments, model,
                                 grad, loss, S(stream));
  });
}

int gpulsm_model_lower_bound(const void *sorted_keys, uint64_t count, uint32_t key_bits, uint32_t segments,
                             const void *model, const void *queries, uint64_t query_count, uint64_t *out,
                             void *stream) {
  return guarded([&] {
    if (key_bits != 32 && key_bits != 64) throw std::invalid_argument("key_bits must be 32 or 64");
    if (!query_count) return;
    need(model, "model");
    need(queries, "queries");
    need(out, "out");
    device_accessible({{sorted_keys, "sorted_keys"}, {model, "model"}, {queries, "queries"}, {out, "out"}});
    auto *o = reinterpret_cast<unsigned long long *>(out);
    if (key_bits == 32)
      gpulsm::learned::lower_bound(static_cast<const uint32_t *>(sorted_keys), count, segments, model,
                                   static_cast<const uint32_t *>(queries), query_count, o, S(stream));
    else
      gpulsm::learned::lower_bound(static_cast<const unsigned long long *>(sorted_keys), count, segments, model,
                                   static_cast<const unsigned long long *>(queries), query_count, o, S(stream));
  });
}

int gpulsm_binary_lower_bound(const void *sorted_keys, uint64_t count, uint32_t key_bits, const void *queries,
                              uint64_t query_count, uint64_t *out, void *stream) {
  return guarded([&] {
    if (key_bits != 32 && key_bits != 64) throw std::invalid_argument("key_bits must be 32 or 64");
    if (!query_count) return;
    need(queries, "queries");
    need(out, "out");
    device_accessible({{sorted_keys, "sorted_keys"}, {queries, "queries"}, {out, "out"}});
    auto *o = reinterpret_cast<unsigned long long *>(out);
    if (key_bits == 32)
      gpulsm::learned::binary_lower_bound(static_cast<const uint32_t *>(sorted_keys), count,
                                          static_cast<const uint32_t *>(queries), query_count, o, S(stream));
    else
      gpulsm::learned::binary_lower_bound(static_cast<const unsigned long long *>(sorted_keys), count,
                                          static_cast<const unsigned long long *>(queries), query_count, o,
                                          S(stream));
  });
}

// ---------------------------------------------------------------- building blocks
int gpulsm_sort_pairs(const void *keys_in, const uint32_t *values_in, void *keys_out,
                      uint32_t *values_out, uint64_t count, uint32_t key_bits, uint32_t begin_bit,
                      uint32_t end_bit, void *stream) {
  return guarded([&] {
    if (key_bits != 32 && key_bits != 64) throw std::invalid_argument("key_bits must be 32 or 64");
    if (begin_bit >= end_bit || end_bit > key_bits) throw std::invalid_argument("bad bit range");
    if (count > gpulsm::radix::kMaxKeys) throw std::length_error("sort limited to 2^30-1 keys");
    if (!count) return;
    need(keys_in, "keys_in");
    need(keys_out, "keys_out");
    if (values_in) need(values_out, "values_out");
    no_partial_overlap(keys_in, keys_out, count * (key_bits / 8), values_in, values_out, values_in ? count * 4 : 0);
    device_accessible({{keys_in, "keys_in"}, {values_in, "values_in"}, {keys_out, "keys_out"}, {values_out, "values_out"}});
    gpulsm::sort_pairs_any(keys_in, values_in, keys_out, values_out, count, key_bits, begin_bit,
                           end_bit, S(stream));
  });
}

}  // extern "C"

// ---------------------------------------------------------------- serving loop
extern "C" {
int gpulsm_server_create(const gpulsm_dict_config *config, uint64_t budget_bytes, uint32_t max_round_keys,
                         uint32_t depth, gpulsm_server **out) {
  return guarded([&] {
    need(config, "config");
    need(out, "out");
    *out = new gpulsm_server(dict_config(*config), budget_bytes, max_round_keys, depth);
  });
}

int gpulsm_server_destroy(gpulsm_server *server) {
  return guarded([&] { delete server; });
}

int gpulsm_server_bulk_build(gpulsm_server *server, const uint32_t *keys, const uint32_t *values, uint64_t count,
                             void *stream) {
  return guarded([&] {
    need(server, "server");
    device_accessible({{keys, "keys"}, {values, "values"}});
    server->impl.drain();
    server->impl.dict().bulk_build(keys, values, count, S(stream));
    GPULSM_CUDA(cudaStreamSynchronize(S(stream)));
  });
}

int gpulsm_server_submit(gpulsm_server *server, uint32_t kind, const uint32_t *keys, const uint32_t *aux,
                         uint64_t count, uint32_t *out, uint8_t *out_found, uint64_t *out_ticket) {
  return guarded([&] {
    need(server, "server");
    need(out_ticket, "out_ticket");
    *out_ticket = server->impl.submit(kind, keys, aux, count, out, out_found);
  });
}

int gpulsm_server_poll(gpulsm_server *server, uint64_t ticket, int32_t *out_state) {
  return guarded([&] {
    need(server, "server");
    need(out_state, "out_state");
    *out_state = server->impl.poll(ticket);
  });
}

int gpulsm_server_wait(gpulsm_server *server, uint64_t ticket, int32_t *out_state) {
  return guarded([&] {
    need(server, "server");
    need(out_state, "out_state");
    *out_state = server->impl.wait(ticket);
  });
}

int gpulsm_server_wait_round(gpulsm_server *server, uint64_t ticket, int32_t *out_state, uint64_t *out_round) {
  return guarded([&] {
    need(server, "server");
    need(out_state, "out_state");
    need(out_round, "out_round");
    *out_state = server->impl.wait(ticket, out_round);
  });
}

int gpulsm_server_drain(gpulsm_server *server) {
  return guarded([&] {
    need(server, "server");
    server->impl.drain();
  });
}

int gpulsm_server_stats(gpulsm_server *server, gpulsm_serve_stats *out) {
  return guarded([&] {
    need(server, "server");
    need(out, "out");
    copy_stats(server->impl.stats(), out);
  });
}

int gpulsm_server_set_staged_updates(gpulsm_server *server, int staged) {
  return guarded([&] {
    need(server, "server");
    server->impl.set_staged_updates(staged != 0);
  });
}

int gpulsm_server_reset_stats(gpulsm_server *server) {
  return guarded([&] {
    need(server, "server");
    server->impl.reset_stats();
  });
}

int gpulsm_server_run_load(gpulsm_server *server, const gpulsm_load_spec *spec, gpulsm_serve_stats *out) {
  return guarded([&] {
    need(server, "server");
    need(spec, "spec");
    need(out, "out");
    gpulsm::LoadSpec l;
    l.rate_per_s = spec->rate_per_s;
    l.seconds = spec->seconds;
    for (int i = 0; i < 4; ++i) l.mix[i] = spec->mix[i];
    l.zipf_s = spec->zipf_s;
    l.max_outstanding = spec->max_outstanding ? spec->max_outstanding : 64;
    l.min_keys = spec->min_keys;
    l.max_keys = spec->max_keys;
    l.range_width_max = spec->range_width_max ? spec->range_width_max : (1u << 16);
    l.seed = spec->seed;
    l.universe = spec->universe;
    l.universe_n = spec->universe_n;
    gpulsm::ServeStats st;
    server->impl.run_load(l, &st);
    copy_stats(st, out);
  });
}

int gpulsm_server_resident_bytes(gpulsm_server *server, uint64_t *out_bytes) {
  return guarded([&] {
    need(server, "server");
    need(out_bytes, "out_bytes");
    *out_bytes = server->impl.dict().resident_bytes() + server->impl.device_bytes();
  });
}
}  // extern "C"

// Allocation-free sort (see sort_noalloc.cu): same checks as gpulsm_sort_pairs.
extern "C" int gpulsm_sort_pairs_noalloc(const void *keys_in, const uint32_t *values_in, void *keys_out,
                                         uint32_t *values_out, uint64_t count, uint32_t key_bits,
                                         uint32_t begin_bit, uint32_t end_bit, void *stream) {
  return guarded([&] {
    if (key_bits != 32 && key_bits != 64) throw std::invalid_argument("key_bits must be 32 or 64");
    if (begin_bit >= end_bit || end_bit > key_bits) throw std::invalid_argument("bad bit range");
    if (count > gpulsm::kNoallocMaxKeys)
      throw std::length_error("gpulsm_sort_pairs_noalloc sorts at most 2^20 keys per call");
    if (!count) return;
    need(keys_in, "keys_in");
    need(keys_out, "keys_out");
    if (values_in) need(values_out, "values_out");
    no_partial_overlap(keys_in, keys_out, count * (key_bits / 8), values_in, values_out, values_in ? count * 4 : 0);
    device_accessible({{keys_in, "keys_in"}, {values_in, "values_in"}, {keys_out, "keys_out"},
                       {values_out, "values_out"}});
    gpulsm::sort_pairs_noalloc(keys_in, values_in, keys_out, values_out, count, key_bits, begin_bit, end_bit,
                               S(stream));
  });
}

extern "C" uint64_t gpulsm_sort_noalloc_scratch_bytes(void) { return gpulsm::noalloc_scratch_bytes(); }

