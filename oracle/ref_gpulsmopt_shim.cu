// C-ABI shim over the reference's own GPULSMOpt engine.  TEST INFRASTRUCTURE ONLY.
//
// This translation unit contains no reference code: it #includes the
// reference header GPULSMOpt.cuh in place (the include path points at the
// read-only reference checkout) and wraps the public methods of
// class GPULSMOpt (GPULSMOpt.cuh:5599-5881) in extern "C" functions so tests
// can drive the reference kernels on a B200 as a GPU parity oracle and time
// them beside ours.  Built by oracle/Makefile into oracle/_ref/ only.
#include "GPULSMOpt.cuh"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>

namespace {
thread_local std::string g_last_error;

template <class F> int guarded(F &&f) {
  try {
    f();
    return 0;
  } catch (const std::invalid_argument &e) {
    g_last_error = e.what();
    return 1;
  } catch (const std::length_error &e) {
    g_last_error = e.what();
    return 7;
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
}  // namespace

extern "C" {

const char *ref_last_error(void) { return g_last_error.c_str(); }

int ref_create(std::uint64_t max_elements, std::uint64_t batch_capacity,
               std::uint64_t level_zero_capacity, void **out) {
  return guarded([&] {
    DictionaryConfig c;
    c.max_elements = max_elements;
    c.batch_capacity = batch_capacity;
    c.level_zero_capacity = level_zero_capacity;
    *out = new GPULSMOpt(c);
  });
}

int ref_destroy(void *d) {
  return guarded([&] { delete static_cast<GPULSMOpt *>(d); });
}

int ref_clear(void *d, void *stream) {
  return guarded([&] { static_cast<GPULSMOpt *>(d)->clear(static_cast<cudaStream_t>(stream)); });
}

int ref_bulk_build(void *d, const std::uint32_t *keys, const std::uint32_t *values,
                   std::uint64_t n, void *stream) {
  return guarded([&] {
    static_cast<GPULSMOpt *>(d)->bulk_build(keys, values, n, static_cast<cudaStream_t>(stream));
  });
}

int ref_insert(void *d, const std::uint32_t *keys, const std::uint32_t *values,
               std::uint64_t n, void *stream) {
  return guarded([&] {
    static_cast<GPULSMOpt *>(d)->insert(DeviceKeyValueBatch{keys, values, n},
                                        static_cast<cudaStream_t>(stream));
  });
}

int ref_erase(void *d, const std::uint32_t *keys, std::uint64_t n, void *stream) {
  return guarded([&] {
    static_cast<GPULSMOpt *>(d)->erase(GPULSMOpt::DeviceKeyBatch{keys, n},
                                       static_cast<cudaStream_t>(stream));
  });
}

int ref_lookup(void *d, const std::uint32_t *queries, std::uint64_t n,
               std::uint32_t *out_values, std::uint8_t *out_found, int grouped,
               void *stream) {
  return guarded([&] {
    static_cast<GPULSMOpt *>(d)->lookup(
        DeviceLookupBatch{queries, n, out_values, out_found},
        static_cast<cudaStream_t>(stream), grouped != 0);
  });
}

int ref_range(void *d, const std::uint32_t *lo, const std::uint32_t *hi, std::uint64_t n,
              std::uint32_t *out_sums, void *stream) {
  return guarded([&] {
    static_cast<GPULSMOpt *>(d)->range(DeviceRangeOutputBatch{lo, hi, n, out_sums},
                                       static_cast<cudaStream_t>(stream));
  });
}

int ref_successor(void *d, const std::uint32_t *queries, std::uint64_t n,
                  std::uint32_t *out_keys, void *stream) {
  return guarded([&] {
    static_cast<GPULSMOpt *>(d)->successor(DeviceSuccessorBatch{queries, n, out_keys},
                                           static_cast<cudaStream_t>(stream));
  });
}

int ref_status(void *d, std::uint32_t *out) {
  return guarded([&] { *out = static_cast<GPULSMOpt *>(d)->canonical_carry_status(); });
}

int ref_resident_bytes(void *d, std::uint64_t *out) {
  return guarded([&] { *out = static_cast<GPULSMOpt *>(d)->gpu_resident_bytes(); });
}

}  // extern "C"
