// FliX bucket layer engine (placeholder until the tiled kernels land).
#include <stdexcept>

#include "flix_index.h"

namespace gpulsm {

struct FlixIndex::Impl {};

FlixIndex::FlixIndex(const FlixConfig &) { throw std::invalid_argument("FliX mode is not available in this build"); }
FlixIndex::~FlixIndex() = default;
void FlixIndex::build(const void *, const uint32_t *, uint64_t, uint64_t, cudaStream_t) {}
void FlixIndex::insert(const void *, const uint32_t *, uint64_t, cudaStream_t) {}
void FlixIndex::remove(const void *, uint64_t, cudaStream_t) {}
void FlixIndex::lookups_ordered(const void *, uint64_t, uint32_t *, cudaStream_t) {}
void FlixIndex::lookups_successor(const void *, uint64_t, void *, cudaStream_t) {}
void FlixIndex::lookup(const void *, uint64_t, uint32_t *, cudaStream_t) {}
void FlixIndex::successor(const void *, uint64_t, void *, cudaStream_t) {}
void FlixIndex::rebuild(cudaStream_t) {}
uint64_t FlixIndex::resident_bytes() { return 0; }
uint64_t FlixIndex::size() { return 0; }
uint32_t FlixIndex::status() { return 0; }

}  // namespace gpulsm
