// Learned position model for one sorted key array (an LSM level, or FliX's
// bucket maxima): a piecewise-linear CDF with equal-width segments in key
// space, fp32 parameters, trained on the GPU by the forward/backward kernels
// below and made exact by a per-segment maximum error.
//
//   segment s covers keys kmin + [s << shift, (s + 1) << shift)
//   xhat  = ((key - kmin) - (s << shift)) / 2^shift - 1/2  in [-1/2, 1/2)
//   pred  = b_s + a_s * xhat                                (fp32, a_s >= 0)
// (the centred feature decouples slope and intercept, so the preconditioned
// gradient steps below converge in a few iterations)
//   loss  = (1/N) sum_i (pred(key_i) - i)^2
//   dL/da_s = (2/N) sum_{i in s} r_i xhat_i,  dL/db_s = (2/N) sum_{i in s} r_i
//
// Lookup: lower_bound(x) lies in [first_s, first_{s+1}]; with p = floor(pred)
// clamped to that range and err_s = max over the segment's keys of
// |floor(pred(key_i)) - i|, monotonicity of pred (a_s >= 0, IEEE rounding is
// monotone) puts it in [p - err_s - 1, p + err_s + 1], so a binary search of
// that window is exact for members and non-members alike.
#pragma once

#include "common.cuh"

namespace gpulsm {
namespace learned {

struct Segment {
  float a;
  float b;
  uint32_t err;
  uint32_t first;  // lower_bound of the segment's first key value
};
static_assert(sizeof(Segment) == 16, "segment layout");

struct ModelHeader {
  unsigned long long n;
  unsigned long long kmin;
  unsigned long long kmax;
  uint32_t shift;
  uint32_t nseg;
  uint32_t iters;
  uint32_t pad[3];
};
static_assert(sizeof(ModelHeader) == 48, "header layout");

// Device memory of a model: header, then nseg + 1 segments (the last one only
// carries first = n), then training accumulators (3 floats per segment).
inline size_t model_bytes(uint32_t segments) {
  return sizeof(ModelHeader) + (size_t(segments) + 1) * sizeof(Segment) + size_t(segments) * 16;
}

template <typename K>
struct ModelView {
  const ModelHeader *h;
  const Segment *seg;
};

template <typename K>
__device__ __forceinline__ float seg_xhat(K x, K kmin, uint32_t shift, uint32_t s) {
  const unsigned long long d = (unsigned long long)(x - kmin) - ((unsigned long long)s << shift);
  return float(d) * __uint_as_float((127u - shift) << 23) - 0.5f;  // d * 2^-shift - 1/2
}

template <typename K>
__device__ __forceinline__ uint32_t seg_of(K x, K kmin, uint32_t shift, uint32_t nseg) {
  const unsigned long long s = (unsigned long long)(x - kmin) >> shift;
  return s < nseg ? uint32_t(s) : nseg - 1;
}

template <typename K>
__device__ __forceinline__ uint64_t lower_bound_range(const K *keys, uint64_t lo, uint64_t hi, K x) {
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (keys[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Exact lower_bound through the model (first index with keys[i] >= x).
template <typename K>
__device__ __forceinline__ uint64_t model_lower_bound(const ModelHeader &h, const Segment *seg, const K *keys,
                                                     K x) {
  if (h.n == 0 || x <= K(h.kmin)) return 0;
  if (x > K(h.kmax)) return h.n;
  const uint32_t s = seg_of<K>(x, K(h.kmin), h.shift, h.nseg);
  const Segment g = seg[s];
  const uint64_t lo_b = g.first, hi_b = seg[s + 1].first;
  const float pred = g.b + g.a * seg_xhat<K>(x, K(h.kmin), h.shift, s);
  int64_t p = int64_t(floorf(pred));
  p = p < int64_t(lo_b) ? int64_t(lo_b) : (p > int64_t(hi_b) ? int64_t(hi_b) : p);
  const int64_t e = int64_t(g.err) + 1;
  const uint64_t lo = p - e > int64_t(lo_b) ? uint64_t(p - e) : lo_b;
  const uint64_t hi = p + e + 1 < int64_t(hi_b) ? uint64_t(p + e + 1) : hi_b;
  return lower_bound_range(keys, lo, hi, x);
}

// ---------------------------------------------------------------------------
// fit, step 0: header (key range, segment width) - one thread
template <typename K>
__global__ void model_header_kernel(const K *__restrict__ keys, uint64_t n, uint32_t segments,
                                    ModelHeader *__restrict__ h, const unsigned long long *__restrict__ n_dev) {
  if (threadIdx.x || blockIdx.x) return;
  if (n_dev) n = *n_dev;  // a count produced on the device (an LSM level's row count)
  ModelHeader m{};
  m.n = n;
  m.kmin = n ? (unsigned long long)keys[0] : 1ull;
  m.kmax = n ? (unsigned long long)keys[n - 1] : 0ull;
  const unsigned long long range = n ? m.kmax - m.kmin : 0ull;
  uint32_t bits = 0;
  while (bits < 64 && (range >> bits)) ++bits;  // bits needed for range
  uint32_t sbits = 0;
  while ((1u << sbits) < segments) ++sbits;     // segments rounded to a power of two
  m.shift = bits > sbits ? bits - sbits : 0;
  m.nseg = uint32_t((range >> m.shift) + 1);
  *h = m;
}

// step 1: first index of every segment, interpolation init (a = count,
// b = first + count / 2: the line through the segment's end points)
template <typename K>
__global__ void model_init_kernel(const K *__restrict__ keys, const ModelHeader *__restrict__ hp,
                                  Segment *__restrict__ seg) {
  const ModelHeader h = *hp;
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s > h.nseg) return;
  uint64_t first;
  if (s == h.nseg) {
    first = h.n;
  } else {
    const unsigned long long start = h.kmin + ((unsigned long long)s << h.shift);
    first = lower_bound_range<K>(keys, 0, h.n, K(start));
  }
  seg[s].first = uint32_t(first);
  seg[s].err = 0;
}

// step 1 (linear): first index of every segment from one pass over the keys:
// key i starts the segments (seg(key i-1), seg(key i)]; the last key closes
// the array (first[nseg] = n).  Same result as a lower_bound per segment.
template <typename K>
__global__ void __launch_bounds__(256) model_init_scan_kernel(const K *__restrict__ keys,
                                                              const ModelHeader *__restrict__ hp,
                                                              Segment *__restrict__ seg) {
  const ModelHeader h = *hp;
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (h.n == 0) {
    if (i <= h.nseg) {
      seg[i].first = 0;
      seg[i].err = 0;
    }
    return;
  }
  if (i >= h.n) return;
  const int64_t si = seg_of<K>(keys[i], K(h.kmin), h.shift, h.nseg);
  const int64_t sp = i ? int64_t(seg_of<K>(keys[i - 1], K(h.kmin), h.shift, h.nseg)) : -1;
  for (int64_t s = sp + 1; s <= si; ++s) {
    seg[s].first = uint32_t(i);
    seg[s].err = 0;
  }
  if (i + 1 == h.n)
    for (int64_t s = si + 1; s <= int64_t(h.nseg); ++s) {
      seg[s].first = uint32_t(h.n);
      seg[s].err = 0;
    }
}

template <typename K>
__global__ void model_init_params_kernel(const ModelHeader *__restrict__ hp, Segment *__restrict__ seg) {
  const ModelHeader h = *hp;
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= h.nseg) return;
  const float first = float(seg[s].first), next = float(seg[s + 1].first);
  seg[s].b = 0.5f * (first + next);
  seg[s].a = next - first;
}

// forward + backward: residuals of every key, per-segment gradient sums
// (acc[3s] = sum r*xhat, acc[3s+1] = sum r, acc[3s+2] = sum xhat^2) and the
// total squared error.  Keys are sorted, so a warp mostly shares one segment:
// peers are found with __match_any_sync and reduced before one atomic.
template <typename K>
__global__ void __launch_bounds__(256) model_forward_backward_kernel(
    const K *__restrict__ keys, const ModelHeader *__restrict__ hp, const Segment *__restrict__ seg,
    float *__restrict__ acc, float *__restrict__ loss) {
  const ModelHeader h = *hp;
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const bool valid = i < h.n;
  uint32_t s = 0xffffffffu;
  float ra = 0.f, rb = 0.f, xx = 0.f, sq = 0.f;
  if (valid) {
    const K x = keys[i];
    s = seg_of<K>(x, K(h.kmin), h.shift, h.nseg);
    const float xh = seg_xhat<K>(x, K(h.kmin), h.shift, s);
    const Segment g = seg[s];
    const float r = (g.b + g.a * xh) - float(i);
    ra = r * xh;
    rb = r;
    xx = xh * xh;
    sq = r * r;
  }
  // Sorted keys: every segment occupies a contiguous interval of lanes, so a
  // shuffle-down segmented sum leaves each interval's total in its first lane.
  const uint32_t lane = threadIdx.x & 31;
  float sa = ra, sb = rb, sx = xx;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const float ya = __shfl_down_sync(0xffffffffu, sa, o);
    const float yb = __shfl_down_sync(0xffffffffu, sb, o);
    const float yx = __shfl_down_sync(0xffffffffu, sx, o);
    const uint32_t other = __shfl_down_sync(0xffffffffu, s, o);
    if (lane + o < 32 && other == s) {
      sa += ya;
      sb += yb;
      sx += yx;
    }
  }
  const uint32_t prev = __shfl_up_sync(0xffffffffu, s, 1);
  if (valid && (lane == 0 || prev != s)) {
    atomicAdd(&acc[3 * s], sa);
    atomicAdd(&acc[3 * s + 1], sb);
    atomicAdd(&acc[3 * s + 2], sx);
  }
  float t = sq;
#pragma unroll
  for (int o = 16; o; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  if (lane == 0 && t != 0.f) atomicAdd(loss, t);
}

// optimizer step: gradient descent with a diagonal preconditioner per
// segment (learning rate eta / sum xhat^2 for a, eta / count for b); clears
// the accumulators for the next pass.  a is kept >= 0 (monotone model).
template <typename K>
__global__ void model_update_kernel(const ModelHeader *__restrict__ hp, Segment *__restrict__ seg,
                                    float *__restrict__ acc, float eta) {
  const ModelHeader h = *hp;
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= h.nseg) return;
  const float cnt = float(seg[s + 1].first - seg[s].first);
  const float ga = acc[3 * s], gb = acc[3 * s + 1], xx = acc[3 * s + 2];
  acc[3 * s] = 0.f;
  acc[3 * s + 1] = 0.f;
  acc[3 * s + 2] = 0.f;
  if (cnt == 0.f) return;
  Segment g = seg[s];
  g.a -= eta * ga / fmaxf(xx, 1e-6f);
  g.b -= eta * gb / cnt;
  if (g.a < 0.f) g.a = 0.f;
  seg[s].a = g.a;
  seg[s].b = g.b;
}

// maximum |floor(pred(key_i)) - i| per segment (warp-aggregated atomicMax)
template <typename K>
__global__ void __launch_bounds__(256) model_error_kernel(const K *__restrict__ keys,
                                                          const ModelHeader *__restrict__ hp,
                                                          Segment *__restrict__ seg) {
  const ModelHeader h = *hp;
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= h.n) return;
  const K x = keys[i];
  const uint32_t s = seg_of<K>(x, K(h.kmin), h.shift, h.nseg);
  const Segment g = seg[s];
  const float pred = g.b + g.a * seg_xhat<K>(x, K(h.kmin), h.shift, s);
  const int64_t d = int64_t(floorf(pred)) - int64_t(i);
  const uint32_t e = uint32_t(d < 0 ? -d : d);
  const uint32_t peers = __match_any_sync(__activemask(), s);
  const uint32_t m = __reduce_max_sync(peers, e);
  if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicMax(&seg[s].err, m);
}

// exact lower bounds of a query batch through the model
template <typename K>
__global__ void __launch_bounds__(256) model_lower_bound_kernel(const K *__restrict__ keys,
                                                                const ModelHeader *__restrict__ hp,
                                                                const Segment *__restrict__ seg,
                                                                const K *__restrict__ q, uint64_t count,
                                                                unsigned long long *__restrict__ out) {
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const ModelHeader h = *hp;
  out[i] = model_lower_bound<K>(h, seg, keys, q[i]);
}

// plain binary search over the whole array: the method without the model
template <typename K>
__global__ void __launch_bounds__(256) binary_lower_bound_kernel(const K *__restrict__ keys, uint64_t n,
                                                                 const K *__restrict__ q, uint64_t count,
                                                                 unsigned long long *__restrict__ out) {
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  out[i] = lower_bound_range<K>(keys, 0, n, q[i]);
}

}  // namespace learned
}  // namespace gpulsm
