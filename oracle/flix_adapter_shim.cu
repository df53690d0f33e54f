// The reference's own FliX index adapter for GPULSMOpt (class gpulsmopt,
// FliX/impl_gpulsmopt.cuh:137-311), compiled against include/gpulsmopt_b200.cuh
// instead of the reference's GPULSMOpt.cuh and linked to libgpulsm.so: the
// boundary proof that a reference-side caller builds and runs unchanged over
// the C ABI.  TEST INFRASTRUCTURE ONLY.
//
// This file contains no reference code.  oracle/Makefile compiles it with the
// include path pointing at a temporary copy of FliX/impl_gpulsmopt.cuh in which
// the one line `#include "../GPULSMOpt.cuh"` reads `#include "gpulsmopt_b200.cuh"`
// (the edit a maintainer makes), and at the reference checkout for the rest;
// the copy is deleted after the compile and only the library lands in oracle/_ref.
#include "utilities.cuh"        // FliX's parameters_type, used by the adapter
#include "impl_gpulsmopt.cuh"   // the adapter, over gpulsmopt_b200.cuh

#include <exception>
#include <string>

namespace {
thread_local std::string g_err;
using Adapter = gpulsmopt<key32>;

template <class F> int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (const std::invalid_argument &e) {
    g_err = e.what();
    return 1;
  } catch (const std::length_error &e) {
    g_err = e.what();
    return 7;
  } catch (const std::bad_alloc &e) {
    g_err = e.what();
    return 6;
  } catch (const std::exception &e) {
    g_err = e.what();
    return 3;
  }
}
}  // namespace

extern "C" {
const char *adapter_last_error(void) { return g_err.c_str(); }
int adapter_create(void **out) {
  return guarded([&] { *out = new Adapter(); });
}
int adapter_destroy(void *h) {
  return guarded([&] {
    auto *a = static_cast<Adapter *>(h);
    a->destroy();
    delete a;
  });
}
// build: values are the input positions (FliX/impl_gpulsmopt.cuh:222-229)
int adapter_build(void *h, const uint32_t *keys, uint64_t n, uint64_t max_n) {
  return guarded([&] {
    double ms = 0;
    size_t bytes = 0;
    static_cast<Adapter *>(h)->build(keys, n, max_n, 0, &ms, &bytes);
  });
}
int adapter_insert(void *h, const uint32_t *keys, const uint32_t *values, uint64_t n, void *s) {
  return guarded([&] { static_cast<Adapter *>(h)->insert(keys, values, n, static_cast<cudaStream_t>(s)); });
}
int adapter_remove(void *h, const uint32_t *keys, uint64_t n, void *s) {
  return guarded([&] { static_cast<Adapter *>(h)->remove(keys, n, static_cast<cudaStream_t>(s)); });
}
int adapter_lookup(void *h, const uint32_t *keys, uint32_t *out, uint64_t n, void *s) {
  return guarded([&] { static_cast<Adapter *>(h)->lookup(keys, out, n, static_cast<cudaStream_t>(s)); });
}
int adapter_range_lookup_sum(void *h, const uint32_t *lo, const uint32_t *hi, uint32_t *out, uint64_t n,
                             void *s) {
  return guarded(
      [&] { static_cast<Adapter *>(h)->range_lookup_sum(lo, hi, out, n, static_cast<cudaStream_t>(s)); });
}
int adapter_lookups_successor(void *h, const uint32_t *keys, uint32_t *out, uint64_t n, void *s) {
  return guarded([&] { static_cast<Adapter *>(h)->lookups_successor(keys, out, n, static_cast<cudaStream_t>(s)); });
}
int adapter_resident_bytes(void *h, uint64_t *out) {
  return guarded([&] { *out = static_cast<Adapter *>(h)->gpu_resident_bytes(); });
}
}  // extern "C"
