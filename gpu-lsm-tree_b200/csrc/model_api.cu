// Host side of the learned position model (learned.cuh): fit, gradient
// export for checking against the CPU, and exact lower-bound queries.
#include <algorithm>
#include <stdexcept>

#include "learned.cuh"
#include "model_api.h"

namespace gpulsm {
namespace learned {

namespace {
uint32_t pow2_at_least(uint32_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

struct Parts {
  ModelHeader *h;
  Segment *seg;
  float *acc;
};

Parts parts(void *model, uint32_t segments) {
  char *p = static_cast<char *>(model);
  Parts r;
  r.h = reinterpret_cast<ModelHeader *>(p);
  r.seg = reinterpret_cast<Segment *>(p + sizeof(ModelHeader));
  r.acc = reinterpret_cast<float *>(p + sizeof(ModelHeader) + (size_t(segments) + 1) * sizeof(Segment));
  return r;
}

template <typename K>
__global__ void export_gradients_kernel(const ModelHeader *__restrict__ hp, const float *__restrict__ acc,
                                        const float *__restrict__ sq, float *__restrict__ grad,
                                        float *__restrict__ loss, uint32_t segments) {
  const ModelHeader h = *hp;
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  const float scale = h.n ? 2.f / float(h.n) : 0.f;
  if (s < segments) {
    grad[2 * s] = s < h.nseg ? acc[3 * s] * scale : 0.f;
    grad[2 * s + 1] = s < h.nseg ? acc[3 * s + 1] * scale : 0.f;
  }
  if (s == 0 && loss) *loss = h.n ? *sq / float(h.n) : 0.f;
}

template <typename K>
__global__ void scale_loss_kernel(const ModelHeader *__restrict__ hp, float *__restrict__ loss, uint32_t count) {
  const uint32_t i = threadIdx.x + blockIdx.x * blockDim.x;
  const ModelHeader h = *hp;
  if (i < count && h.n) loss[i] /= float(h.n);
}
}  // namespace

size_t bytes_for(uint32_t segments) { return model_bytes(pow2_at_least(segments)); }

template <typename K>
void fit(const K *keys, uint64_t n, uint32_t segments, uint32_t iters, void *model, float *loss_hist,
         cudaStream_t s, const unsigned long long *n_dev) {
  segments = pow2_at_least(std::max<uint32_t>(segments, 1));
  Parts p = parts(model, segments);
  model_header_kernel<K><<<1, 1, 0, s>>>(keys, n, segments, p.h, n_dev); note_launch();
  model_init_scan_kernel<K><<<grid_for(std::max<uint64_t>(n, segments + 1), 256), 256, 0, s>>>(keys, p.h, p.seg);
  note_launch();
  model_init_params_kernel<K><<<grid_for(segments, 256), 256, 0, s>>>(p.h, p.seg); note_launch();
  GPULSM_CUDA(cudaMemsetAsync(p.acc, 0, size_t(segments) * 16, s));
  if (loss_hist) GPULSM_CUDA(cudaMemsetAsync(loss_hist, 0, size_t(iters + 1) * 4, s));
  const unsigned grid = grid_for(std::max<uint64_t>(n, 1), 256);
  for (uint32_t t = 0; t < iters; ++t) {
    model_forward_backward_kernel<K><<<grid, 256, 0, s>>>(keys, p.h, p.seg, p.acc,
                                                          loss_hist ? loss_hist + t : p.acc + 3 * segments);
    note_launch();
    model_update_kernel<K><<<grid_for(segments, 256), 256, 0, s>>>(p.h, p.seg, p.acc, 0.5f); note_launch();
  }
  if (loss_hist) {
    // loss after the last step (forward only: the accumulators are cleared again below)
    model_forward_backward_kernel<K><<<grid, 256, 0, s>>>(keys, p.h, p.seg, p.acc, loss_hist + iters);
    note_launch();
    GPULSM_CUDA(cudaMemsetAsync(p.acc, 0, size_t(segments) * 12, s));
    scale_loss_kernel<K><<<grid_for(iters + 1, 256), 256, 0, s>>>(p.h, loss_hist, iters + 1); note_launch();
  }
  model_error_kernel<K><<<grid, 256, 0, s>>>(keys, p.h, p.seg); note_launch();
  GPULSM_CUDA(cudaGetLastError());
}

template <typename K>
void gradients(const K *keys, uint64_t n, uint32_t segments, void *model, float *grad, float *loss,
               cudaStream_t s) {
  segments = pow2_at_least(std::max<uint32_t>(segments, 1));
  Parts p = parts(model, segments);
  float *sq = p.acc + 3 * segments;  // spare word after the accumulators
  GPULSM_CUDA(cudaMemsetAsync(p.acc, 0, size_t(segments) * 16, s));
  model_forward_backward_kernel<K><<<grid_for(std::max<uint64_t>(n, 1), 256), 256, 0, s>>>(keys, p.h, p.seg,
                                                                                            p.acc, sq);
  note_launch();
  export_gradients_kernel<K><<<grid_for(segments, 256), 256, 0, s>>>(p.h, p.acc, sq, grad, loss, segments);
  note_launch();
  GPULSM_CUDA(cudaMemsetAsync(p.acc, 0, size_t(segments) * 16, s));
  GPULSM_CUDA(cudaGetLastError());
}

template <typename K>
void lower_bound(const K *keys, uint64_t n, uint32_t segments, const void *model, const K *q, uint64_t count,
                 unsigned long long *out, cudaStream_t s) {
  segments = pow2_at_least(std::max<uint32_t>(segments, 1));
  Parts p = parts(const_cast<void *>(model), segments);
  (void)n;
  model_lower_bound_kernel<K><<<grid_for(count, 256), 256, 0, s>>>(keys, p.h, p.seg, q, count, out);
  note_launch();
  GPULSM_CUDA(cudaGetLastError());
}

template <typename K>
void binary_lower_bound(const K *keys, uint64_t n, const K *q, uint64_t count, unsigned long long *out,
                        cudaStream_t s) {
  binary_lower_bound_kernel<K><<<grid_for(count, 256), 256, 0, s>>>(keys, n, q, count, out); note_launch();
  GPULSM_CUDA(cudaGetLastError());
}

template void fit<uint32_t>(const uint32_t *, uint64_t, uint32_t, uint32_t, void *, float *, cudaStream_t,
                            const unsigned long long *);
template void fit<unsigned long long>(const unsigned long long *, uint64_t, uint32_t, uint32_t, void *, float *,
                                      cudaStream_t, const unsigned long long *);
template void gradients<uint32_t>(const uint32_t *, uint64_t, uint32_t, void *, float *, float *, cudaStream_t);
template void gradients<unsigned long long>(const unsigned long long *, uint64_t, uint32_t, void *, float *,
                                            float *, cudaStream_t);
template void lower_bound<uint32_t>(const uint32_t *, uint64_t, uint32_t, const void *, const uint32_t *,
                                    uint64_t, unsigned long long *, cudaStream_t);
template void lower_bound<unsigned long long>(const unsigned long long *, uint64_t, uint32_t, const void *,
                                              const unsigned long long *, uint64_t, unsigned long long *,
                                              cudaStream_t);
template void binary_lower_bound<uint32_t>(const uint32_t *, uint64_t, const uint32_t *, uint64_t,
                                           unsigned long long *, cudaStream_t);
template void binary_lower_bound<unsigned long long>(const unsigned long long *, uint64_t,
                                                     const unsigned long long *, uint64_t, unsigned long long *,
                                                     cudaStream_t);

}  // namespace learned
}  // namespace gpulsm
