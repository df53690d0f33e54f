// Allocation-free variant of the radix sort entry (see sort_noalloc.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace gpulsm {
constexpr uint64_t kNoallocMaxKeys = uint64_t{1} << 20;
// Bytes of the static device scratch array every GPU holds for this entry.
size_t noalloc_scratch_bytes();
void sort_pairs_noalloc(const void *keys_in, const uint32_t *values_in, void *keys_out, uint32_t *values_out,
                        uint64_t count, uint32_t key_bits, uint32_t begin_bit, uint32_t end_bit, cudaStream_t s);
}  // namespace gpulsm
