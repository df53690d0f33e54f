// Host API of the learned position model (learned.cuh).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace gpulsm {
namespace learned {
// Device bytes of a model with `segments` segments (rounded up to a power of two).
size_t bytes_for(uint32_t segments);
// Fit on sorted keys: interpolation init, `iters` preconditioned gradient steps
// (forward/backward kernels), then per-segment maximum error.  loss_hist
// (device, iters + 1 floats, may be null) receives the mean squared error
// before each step and after the last one.
// n_dev (optional): the exact count on the device; n is then an upper bound.
template <typename K>
void fit(const K *keys, uint64_t n, uint32_t segments, uint32_t iters, void *model, float *loss_hist,
         cudaStream_t s, const unsigned long long *n_dev = nullptr);
// dL/da_s, dL/db_s interleaved per segment (device, 2 * segments floats) and
// the mean squared error, for the model's current parameters.
template <typename K>
void gradients(const K *keys, uint64_t n, uint32_t segments, void *model, float *grad, float *loss,
               cudaStream_t s);
template <typename K>
void lower_bound(const K *keys, uint64_t n, uint32_t segments, const void *model, const K *q, uint64_t count,
                 unsigned long long *out, cudaStream_t s);
template <typename K>
void binary_lower_bound(const K *keys, uint64_t n, const K *q, uint64_t count, unsigned long long *out,
                        cudaStream_t s);
}  // namespace learned
}  // namespace gpulsm
