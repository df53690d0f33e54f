// Onesweep-style LSD radix sort (8-bit digits) for 32/64-bit keys with an
// optional u32 payload.  One upfront histogram pass computes the digit counts
// of every pass; each pass then ranks a 4096-key tile in registers with
// ballot-built peer groups (match_any_bits), publishes its digit counts through a
// decoupled look-back (bounded spin, never a hang), stages the tile in shared
// memory in digit order and writes it out in coalesced runs.  Stable, so a
// later "keep the last of each equal-key run" pass sees input order.
#pragma once

#include "common.cuh"

namespace gpulsm {
namespace radix {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kDigits = 256;
constexpr int kItems = 16;
constexpr uint32_t kTile = kThreads * kItems;  // 4096 keys per tile
constexpr int kMaxPasses = 8;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kFlagMask = 3u << 30;
constexpr uint32_t kCountMask = (1u << 30) - 1u;
constexpr uint32_t kMaxKeys = kCountMask;  // look-back counts are 30-bit

inline uint32_t tiles_for(uint64_t n) { return static_cast<uint32_t>((n + kTile - 1) / kTile); }

// Workspace: [hist passes*256][counters 64][lookback passes*tiles*256], u32.
inline size_t workspace_words(uint64_t n, int passes) {
  return size_t(passes) * kDigits + 64 + size_t(passes) * tiles_for(n ? n : 1) * kDigits;
}
inline size_t workspace_bytes(uint64_t n, int passes) { return workspace_words(n, passes) * 4; }

// Digit mask of pass p over bits [begin_bit, end_bit): 8 bits, except a last
// pass that reaches past end_bit, which sorts only the bits below end_bit.
__host__ __device__ inline uint32_t digit_mask(uint32_t begin_bit, uint32_t end_bit, uint32_t p) {
  const uint32_t width = end_bit - (begin_bit + 8 * p);
  return width >= 8 ? 0xffu : ((1u << width) - 1u);
}

template <typename KeyT>
__global__ void __launch_bounds__(kThreads) histogram_kernel(const KeyT *__restrict__ keys, uint32_t n,
                                                             uint32_t begin_bit, uint32_t end_bit,
                                                             uint32_t passes, uint32_t *__restrict__ hist) {
  __shared__ uint32_t s[kMaxPasses][kDigits];
  for (uint32_t i = threadIdx.x; i < kMaxPasses * kDigits; i += kThreads) (&s[0][0])[i] = 0;
  __syncthreads();
  for (uint32_t i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
    const KeyT k = keys[i];
    for (uint32_t p = 0; p < passes; ++p)
      atomicAdd(&s[p][uint32_t(k >> (begin_bit + 8 * p)) & digit_mask(begin_bit, end_bit, p)], 1u);
  }
  __syncthreads();
  for (uint32_t p = 0; p < passes; ++p) {
    const uint32_t c = s[p][threadIdx.x];
    if (c) atomicAdd(&hist[p * kDigits + threadIdx.x], c);
  }
}

template <typename KeyT, bool kValues>
struct OnesweepSmem {
  static constexpr size_t bytes = size_t(kTile) * (sizeof(KeyT) + (kValues ? 4 : 0));
};

template <typename KeyT, bool kValues>
__global__ void __launch_bounds__(kThreads) onesweep_kernel(
    const KeyT *__restrict__ kin, const uint32_t *__restrict__ vin, KeyT *__restrict__ kout,
    uint32_t *__restrict__ vout, uint32_t n_host, uint32_t shift, uint32_t dmask,
    const uint32_t *__restrict__ pass_hist,
    uint32_t *__restrict__ lookback, uint32_t *__restrict__ tile_counter,
    uint32_t *__restrict__ status, const uint32_t *__restrict__ n_dev) {
  // n_dev (optional) carries a count produced on the device; the grid is then
  // sized for n_host, an upper bound, and tiles past the count leave at once
  const uint32_t n = n_dev ? *n_dev : n_host;
  extern __shared__ __align__(16) unsigned char dyn[];
  KeyT *s_keys = reinterpret_cast<KeyT *>(dyn);
  uint32_t *s_vals = reinterpret_cast<uint32_t *>(dyn + size_t(kTile) * sizeof(KeyT));
  __shared__ uint32_t warp_hist[kWarps * kDigits];
  __shared__ uint32_t s_local_start[kDigits];
  __shared__ uint32_t s_offset[kDigits];
  __shared__ uint32_t s_scan[kWarps];
  __shared__ uint32_t s_total;
  __shared__ uint32_t s_tile;

  if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
  for (uint32_t i = threadIdx.x; i < kWarps * kDigits; i += kThreads) warp_hist[i] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t tile_base = tile * kTile;
  if (tile_base >= n) return;  // past a device-side count: no later tile waits on this one
  const uint32_t warp_base = tile_base + warp * 32 * kItems;

  KeyT keys[kItems];
  uint32_t vals[kItems];
  uint32_t digits[kItems];
  uint32_t ranks[kItems];
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const uint32_t idx = warp_base + i * 32 + lane;
    const bool valid = idx < n;
    keys[i] = valid ? kin[idx] : KeyT(0);
    if (kValues) vals[i] = valid ? vin[idx] : 0u;
    digits[i] = valid ? (uint32_t(keys[i] >> shift) & dmask) : 256u;
  }
  uint32_t *my_hist = warp_hist + warp * kDigits;
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const uint32_t d = digits[i];
    const uint32_t peers = match_any_bits<9>(d);  // digits 0..255, 256 = no key
    const uint32_t leader = 31u - __clz(peers);
    uint32_t base = 0;
    if (lane == leader && d < kDigits) {
      base = my_hist[d];
      my_hist[d] = base + __popc(peers);
    }
    base = __shfl_sync(0xffffffffu, base, leader);
    ranks[i] = base + __popc(peers & lt);
    __syncwarp();
  }
  __syncthreads();

  // Thread d owns digit d: exclusive offsets of each warp, tile total.
  const uint32_t d = threadIdx.x;
  uint32_t total = 0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) {
    const uint32_t c = warp_hist[w * kDigits + d];
    warp_hist[w * kDigits + d] = total;
    total += c;
  }
  uint32_t *my_lb = lookback + size_t(tile) * kDigits + d;
  st_relaxed_u32(my_lb, (tile == 0 ? kFlagInc : kFlagAgg) | total);

  const uint32_t gbase = block_exclusive_scan<kThreads>(pass_hist[d], s_scan, &s_total);
  const uint32_t local_start = block_exclusive_scan<kThreads>(total, s_scan, &s_total);

  uint32_t excl = 0;
  if (tile > 0) {
    int32_t t = int32_t(tile) - 1;
    uint32_t spins = 0;
    while (true) {
      const uint32_t v = ld_relaxed_u32(lookback + size_t(t) * kDigits + d);
      const uint32_t flag = v & kFlagMask;
      if (flag == 0u) {
        if (++spins > kMaxSpins) {
          atomicOr(status, kDevWaitTimeout);
          break;
        }
        continue;
      }
      excl += v & kCountMask;
      if (flag == kFlagInc || t == 0) break;
      --t;
    }
    st_relaxed_u32(my_lb, kFlagInc | ((excl + total) & kCountMask));
  }
  s_local_start[d] = local_start;
  s_offset[d] = gbase + excl - local_start;
  __syncthreads();

#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const uint32_t dd = digits[i];
    if (dd < kDigits) {
      const uint32_t pos = s_local_start[dd] + my_hist[dd] + ranks[i];
      s_keys[pos] = keys[i];
      if (kValues) s_vals[pos] = vals[i];
    }
  }
  __syncthreads();
  const uint32_t valid_count = min(kTile, n - tile_base);
  for (uint32_t j = threadIdx.x; j < valid_count; j += kThreads) {
    const KeyT k = s_keys[j];
    const uint32_t o = s_offset[uint32_t(k >> shift) & dmask] + j;
    if (o < n) {  // always true unless a look-back wait timed out (status bit set)
      kout[o] = k;
      if (kValues) vout[o] = s_vals[j];
    }
  }
}

// Runs the digit passes over [begin_bit, end_bit).  The workspace must be
// zeroed and its histogram filled (histogram_kernel, or a fused producer that
// counts the same digits, digit_mask included) before the call.  keys[0]/vals[0] hold the input; returns the index of the
// buffer that holds the sorted output.
template <typename KeyT, bool kValues>
int run_passes(KeyT *keys[2], uint32_t *vals[2], uint32_t n, int begin_bit, int end_bit,
               uint32_t *workspace, uint32_t *status, cudaStream_t stream,
               const uint32_t *n_dev = nullptr) {
  const int passes = (end_bit - begin_bit + 7) / 8;
  const uint32_t tiles = tiles_for(n);
  const size_t smem = OnesweepSmem<KeyT, kValues>::bytes;
  GPULSM_CUDA(cudaFuncSetAttribute(onesweep_kernel<KeyT, kValues>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  uint32_t *hist = workspace;
  uint32_t *counters = workspace + size_t(passes) * kDigits;
  uint32_t *lookback = counters + 64;
  int cur = 0;
  for (int p = 0; p < passes; ++p) {
    onesweep_kernel<KeyT, kValues><<<tiles, kThreads, smem, stream>>>(
        keys[cur], kValues ? vals[cur] : nullptr, keys[cur ^ 1], kValues ? vals[cur ^ 1] : nullptr,
        n, uint32_t(begin_bit + 8 * p), digit_mask(uint32_t(begin_bit), uint32_t(end_bit), uint32_t(p)),
        hist + p * kDigits, lookback + size_t(p) * tiles * kDigits,
        counters + p, status, n_dev); note_launch();
    cur ^= 1;
  }
  GPULSM_CUDA(cudaGetLastError());
  return cur;
}

// Full sort: zero workspace, histogram, passes.
template <typename KeyT, bool kValues>
int sort(KeyT *keys[2], uint32_t *vals[2], uint32_t n, int begin_bit, int end_bit,
         uint32_t *workspace, uint32_t *status, int num_sms, cudaStream_t stream) {
  if (n == 0) return 0;
  const int passes = (end_bit - begin_bit + 7) / 8;
  GPULSM_CUDA(cudaMemsetAsync(workspace, 0, workspace_bytes(n, passes), stream));
  const unsigned blocks = std::min<unsigned>(grid_for(n, kTile), unsigned(num_sms) * 4u);
  histogram_kernel<KeyT><<<blocks, kThreads, 0, stream>>>(keys[0], n, uint32_t(begin_bit), uint32_t(end_bit),
                                                          uint32_t(passes), workspace); note_launch();
  return run_passes<KeyT, kValues>(keys, vals, n, begin_bit, end_bit, workspace, status, stream);
}

}  // namespace radix
}  // namespace gpulsm
