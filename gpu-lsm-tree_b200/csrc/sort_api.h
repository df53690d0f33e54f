// Host entry to the onesweep radix sort used by gpulsm_sort_pairs.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace gpulsm {
// Stable sort of (key, optional u32 value) by key bits [begin_bit, end_bit);
// inputs untouched, scratch allocated stream-ordered.
void sort_pairs_any(const void *keys_in, const uint32_t *values_in, void *keys_out,
                    uint32_t *values_out, uint64_t count, uint32_t key_bits, uint32_t begin_bit,
                    uint32_t end_bit, cudaStream_t s);
}  // namespace gpulsm
