// Batch admission by top-byte buckets: the sorted, deduplicated level run of
// one update batch (GPULSMOpt.cuh:2578-2633 sorts the batch, ages the
// duplicates and keeps the newest) in three launches instead of a four-pass
// LSD sort plus a dedup pass:
//
//   1. pack_histogram_kernel   words (key << 32 | value) in input order and
//                              the key-byte histograms (lsm_kernels.cuh)
//   2. one onesweep pass       stable partition of the words by the key's top
//                              byte (radix_sort.cuh)
//   3. admit_bucket_kernel     one CTA per top-byte bucket, in bucket order:
//                              sorts the bucket's varying low key bits in
//                              shared memory (a stable 8-bit LSD pass per
//                              varying byte), keeps the last row of every
//                              equal-key run (input order survives both
//                              stable sorts, so the last row is the newest),
//                              chains its row count to the earlier buckets by
//                              decoupled look-back and writes the level rows
//                              plus its share of the radix directory.  A
//                              bucket larger than shared memory is sorted
//                              through global memory by the same CTA in
//                              chunks (correct for any skew, slower).
//
// The level's key bounds are the top-byte span of the batch
// [first << 24, last << 24 | 0xffffff]: every search uses kmin/kmax only as
// bounds, so they need not be the exact extreme keys.
#pragma once

#include "lsm_kernels.cuh"

namespace gpulsm {
namespace lsm {
namespace admit {

constexpr int kThreads = 512;
constexpr int kItems = 12;
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kCap = uint32_t(kThreads) * kItems;  // rows one bucket sorts in shared memory
constexpr uint32_t kBuckets = 256;
constexpr uint64_t kMaxKeys = uint64_t(1) << 20;  // larger batches take the four-pass sort

__device__ __forceinline__ uint32_t word_key(unsigned long long w) { return uint32_t(w >> 32); }

struct RankSmem {
  uint16_t cnt[kWarps][256];  // per warp and digit: count, then exclusive offset
  uint32_t dstart[257];       // first chunk position of each digit; dstart[256] = chunk rows
  uint32_t scan[kWarps];
  uint32_t total;
};

// Lanes of the warp whose 8-bit digit equals this lane's, among the lanes in
// `valid` (eight ballots instead of match.any, which issues on a slow pipe).
__device__ __forceinline__ uint32_t digit_peers(uint32_t d, uint32_t valid) {
  uint32_t peers = valid;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    const uint32_t m = __ballot_sync(0xffffffffu, (d >> b) & 1u);
    peers &= ((d >> b) & 1u) ? m : ~m;
  }
  return peers;
}

__device__ __forceinline__ uint32_t digit_of(unsigned long long w, uint32_t bit) {
  return (word_key(w) >> bit) & 0xffu;
}

// Stable rank of one chunk of up to kCap words held warp-striped in
// registers (item i of lane l in warp w is chunk element w*32*keff + i*32 + l)
// by the 8-bit key digit at `bit`.  pos[i] = the element's position in the
// chunk sorted by that digit.  keff is block-uniform.
__device__ __forceinline__ void rank_chunk(const unsigned long long (&it)[kItems], uint32_t keff, uint32_t cnt,
                                           uint32_t bit, RankSmem &sm, uint32_t (&pos)[kItems]) {
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  for (uint32_t d = lane; d < 256; d += 32) sm.cnt[w][d] = 0;
  __syncwarp();
  const uint32_t wbase = w * 32u * keff;
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    pos[i] = 0;
    if (uint32_t(i) < keff) {
      const bool valid = wbase + uint32_t(i) * 32u + lane < cnt;
      const uint32_t d = digit_of(it[i], bit);
      const uint32_t peers = digit_peers(d, __ballot_sync(0xffffffffu, valid));
      if (valid) pos[i] = sm.cnt[w][d] + __popc(peers & lt);
      __syncwarp();
      if (valid && (__ffs(peers) - 1) == int(lane)) sm.cnt[w][d] = uint16_t(sm.cnt[w][d] + __popc(peers));
      __syncwarp();
    }
  }
  __syncthreads();
  uint32_t tot = 0;
  if (threadIdx.x < 256) {
#pragma unroll
    for (int ww = 0; ww < kWarps; ++ww) {
      const uint32_t c = sm.cnt[ww][threadIdx.x];
      sm.cnt[ww][threadIdx.x] = uint16_t(tot);
      tot += c;
    }
  }
  const uint32_t ds = block_exclusive_scan<kThreads>(tot, sm.scan, &sm.total);
  if (threadIdx.x < 256) sm.dstart[threadIdx.x] = ds;
  if (threadIdx.x == 0) sm.dstart[256] = cnt;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kItems; ++i)
    if (uint32_t(i) < keff && wbase + uint32_t(i) * 32u + lane < cnt) {
      const uint32_t d = digit_of(it[i], bit);
      pos[i] += sm.dstart[d] + sm.cnt[w][d];
    }
}

__device__ __forceinline__ void load_striped(const unsigned long long *src, uint32_t keff, uint32_t cnt,
                                             unsigned long long (&it)[kItems]) {
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint32_t wbase = w * 32u * keff;
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const uint32_t e = wbase + uint32_t(i) * 32u + lane;
    it[i] = (uint32_t(i) < keff && e < cnt) ? src[e] : 0ull;
  }
}

__device__ __forceinline__ bool run_end(const unsigned long long *src, uint32_t j, uint32_t cnt) {
  return j + 1 == cnt || word_key(src[j]) != word_key(src[j + 1]);
}

// Distinct keys of a sorted sequence.
__device__ __forceinline__ uint32_t count_distinct(const unsigned long long *src, uint32_t cnt, RankSmem &sm) {
  uint32_t c = 0;
  for (uint32_t j = threadIdx.x; j < cnt; j += kThreads) c += run_end(src, j, cnt) ? 1u : 0u;
  (void)block_exclusive_scan<kThreads>(c, sm.scan, &sm.total);
  return sm.total;
}

// Write the last row of every equal-key run of the sorted sequence
// src[0, cnt) to out[g0 ...], in chunks of kCap read striped (element
// c0 + i*kThreads + t): per item a warp ballot counts the kept rows, one block
// scan over the (item, warp) counts gives every warp its output offset, and
// consecutive lanes store consecutive rows.
__device__ __forceinline__ void write_rows(const unsigned long long *src, uint32_t cnt, int tombstone,
                                           uint32_t *out_keys, uint32_t *out_vals, uint8_t *out_flags,
                                           unsigned long long g0, RankSmem &rs) {
  static_assert(kItems * kWarps <= 256, "one scan slot per (item, warp)");
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
  const uint32_t lt = lanemask_lt();
  uint32_t *slot = rs.dstart;  // kItems * kWarps counts, then their offsets
  unsigned long long written = 0;
  for (uint32_t c0 = 0; c0 < cnt; c0 += kCap) {
    const uint32_t cc = min(kCap, cnt - c0);
    uint32_t ends[kItems];
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      const uint32_t e = c0 + uint32_t(i) * kThreads + threadIdx.x;
      ends[i] = __ballot_sync(0xffffffffu, e < c0 + cc && run_end(src, e, cnt));
      if (lane == 0) slot[i * kWarps + w] = __popc(ends[i]);
    }
    __syncthreads();
    const uint32_t v = threadIdx.x < uint32_t(kItems * kWarps) ? slot[threadIdx.x] : 0u;
    const uint32_t ex = block_exclusive_scan<kThreads>(v, rs.scan, &rs.total);
    const uint32_t chunk_kept = rs.total;
    if (threadIdx.x < uint32_t(kItems * kWarps)) slot[threadIdx.x] = ex;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kItems; ++i)
      if ((ends[i] >> lane) & 1u) {
        const uint32_t e = c0 + uint32_t(i) * kThreads + threadIdx.x;
        const unsigned long long w64 = src[e];
        const unsigned long long r = g0 + written + slot[i * kWarps + w] + __popc(ends[i] & lt);
        out_keys[r] = word_key(w64);
        out_vals[r] = uint32_t(w64);  // the tombstone value was packed for erase batches
        out_flags[r] = tombstone ? kFlagTomb : uint8_t(0);
      }
    __syncthreads();
    written += chunk_kept;
  }
}

// Varying key bits (OR ^ AND over the keys) of a sequence.
__device__ __forceinline__ uint32_t varying_bits(const unsigned long long *src, uint32_t cnt, RankSmem &sm) {
  uint32_t o = 0u, a = 0xffffffffu;
  for (uint32_t j = threadIdx.x; j < cnt; j += kThreads) {
    const uint32_t k = word_key(src[j]);
    o |= k;
    a &= k;
  }
#pragma unroll
  for (int s = 16; s; s >>= 1) {
    o |= __shfl_xor_sync(0xffffffffu, o, s);
    a &= __shfl_xor_sync(0xffffffffu, a, s);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) {
    sm.dstart[warp] = o;
    sm.dstart[kWarps + warp] = a;
  }
  __syncthreads();
  o = 0u;
  a = 0xffffffffu;
  for (int w = 0; w < kWarps; ++w) {
    o |= sm.dstart[w];
    a &= sm.dstart[kWarps + w];
  }
  __syncthreads();
  return o ^ a;
}

// Stable sort of a bucket larger than shared memory through global memory:
// per varying byte, a histogram pass then chunks ranked stably in shared
// memory and scattered to the digit's running offset.  Returns the buffer
// holding the sorted rows (a or b).
__device__ __noinline__ unsigned long long *sort_global(unsigned long long *a, unsigned long long *b, uint32_t cnt,
                                                       uint32_t vary, RankSmem &sm, uint32_t *s_off) {
  unsigned long long *src = a, *dst = b;
  for (uint32_t bit = 0; bit < 32; bit += 8) {
    if (((vary >> bit) & 0xffu) == 0u) continue;
    for (uint32_t d = threadIdx.x; d < 256; d += kThreads) s_off[d] = 0;
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < cnt; j += kThreads) atomicAdd(&s_off[(word_key(src[j]) >> bit) & 0xffu], 1u);
    __syncthreads();
    const uint32_t v = threadIdx.x < 256 ? s_off[threadIdx.x] : 0u;
    const uint32_t ex = block_exclusive_scan<kThreads>(v, sm.scan, &sm.total);
    if (threadIdx.x < 256) s_off[threadIdx.x] = ex;
    __syncthreads();
    for (uint32_t c0 = 0; c0 < cnt; c0 += kCap) {
      const uint32_t cc = min(kCap, cnt - c0);
      const uint32_t keff = (cc + kThreads - 1) / kThreads;
      unsigned long long it[kItems];
      uint32_t pos[kItems];
      load_striped(src + c0, keff, cc, it);
      rank_chunk(it, keff, cc, bit, sm, pos);
      const uint32_t wbase = (threadIdx.x >> 5) * 32u * keff;
#pragma unroll
      for (int i = 0; i < kItems; ++i)
        if (uint32_t(i) < keff && wbase + uint32_t(i) * 32u + (threadIdx.x & 31u) < cc) {
          const uint32_t d = digit_of(it[i], bit);
          dst[s_off[d] + pos[i] - sm.dstart[d]] = it[i];
        }
      __syncthreads();
      if (threadIdx.x < 256) s_off[threadIdx.x] += sm.dstart[threadIdx.x + 1] - sm.dstart[threadIdx.x];
      __syncthreads();
    }
    unsigned long long *t = src;
    src = dst;
    dst = t;
  }
  return src;
}

struct BucketSmem {
  unsigned long long words[kCap];
  RankSmem rank;
  uint32_t start[kBuckets + 1];
  uint32_t off[256];
  uint32_t first, last, tile;
  unsigned long long g0;
};
constexpr size_t kBucketSmemBytes = sizeof(BucketSmem);

// One CTA per nonempty top-byte bucket (ticket t -> bucket first + t).
// words0: the batch partitioned by top byte (stable); words1: scratch of the
// same size for oversized buckets; top_hist: rows per top byte.
__global__ void __launch_bounds__(kThreads, 2) admit_bucket_kernel(
    unsigned long long *__restrict__ words0, unsigned long long *__restrict__ words1,
    const uint32_t *__restrict__ top_hist, uint32_t n, int tombstone, uint32_t *__restrict__ out_keys,
    uint32_t *__restrict__ out_vals, uint8_t *__restrict__ out_flags, LevelDesc *__restrict__ out_desc,
    uint32_t *__restrict__ out_dir, uint32_t dir_bits, uint32_t rows_log2, unsigned long long *__restrict__ lb,
    uint32_t *__restrict__ tile_counter, uint32_t *__restrict__ status) {
  extern __shared__ __align__(16) unsigned char dyn[];
  BucketSmem &sm = *reinterpret_cast<BucketSmem *>(dyn);
  if (threadIdx.x == 0) {
    sm.tile = atomicAdd(tile_counter, 1u);
    sm.first = kBuckets;
    sm.last = 0;
  }
  __syncthreads();
  // bucket starts (exclusive scan of the top-byte counts) and the nonempty span
  const uint32_t c = threadIdx.x < kBuckets ? top_hist[threadIdx.x] : 0u;
  const uint32_t ex = block_exclusive_scan<kThreads>(c, sm.rank.scan, &sm.rank.total);
  if (threadIdx.x < kBuckets) {
    sm.start[threadIdx.x] = ex;
    if (c) {
      atomicMin(&sm.first, threadIdx.x);
      atomicMax(&sm.last, threadIdx.x);
    }
  }
  if (threadIdx.x == 0) sm.start[kBuckets] = n;
  __syncthreads();
  const uint32_t first = sm.first, last = sm.last;
  if (first > last) return;  // empty batch
  const uint32_t tile = sm.tile, b = first + tile;
  if (b > last) return;  // later tickets: no bucket waits on them
  const uint32_t s0 = sm.start[b];
  const uint32_t cnt = sm.start[b + 1] - s0;
  if (s0 > n || cnt > n - s0) {  // histogram inconsistent with the batch: refuse
    atomicOr(status, kDevBadInput);
    return;
  }
  const unsigned long long *sorted;
  if (cnt <= kCap) {
    for (uint32_t j = threadIdx.x; j < cnt; j += kThreads) sm.words[j] = words0[s0 + j];
    __syncthreads();
    const uint32_t vary = cnt > 1 ? varying_bits(sm.words, cnt, sm.rank) : 0u;
    const uint32_t keff = (cnt + kThreads - 1) / kThreads;
    for (uint32_t bit = 0; bit < 24; bit += 8) {
      if (((vary >> bit) & 0xffu) == 0u) continue;
      unsigned long long it[kItems];
      uint32_t pos[kItems];
      load_striped(sm.words, keff, cnt, it);
      rank_chunk(it, keff, cnt, bit, sm.rank, pos);  // its barriers order the loads before the stores
      const uint32_t wbase = (threadIdx.x >> 5) * 32u * keff;
#pragma unroll
      for (int i = 0; i < kItems; ++i)
        if (uint32_t(i) < keff && wbase + uint32_t(i) * 32u + (threadIdx.x & 31u) < cnt) sm.words[pos[i]] = it[i];
      __syncthreads();
    }
    sorted = sm.words;
  } else {
    const uint32_t vary = varying_bits(words0 + s0, cnt, sm.rank) & 0x00ffffffu;
    sorted = sort_global(words0 + s0, words1 + s0, cnt, vary, sm.rank, sm.off);
    __syncthreads();
  }
  const uint32_t kept = count_distinct(sorted, cnt, sm.rank);
  if (threadIdx.x < 32) {
    const unsigned long long e = warp_lookback(lb, tile, kept, status);
    if (threadIdx.x == 0) sm.g0 = e;
  }
  __syncthreads();
  const unsigned long long g0 = sm.g0;
  if (g0 + kept > n) {  // only after a timed-out look-back (status bit set)
    atomicOr(status, kDevWaitTimeout);
    return;
  }
  write_rows(sorted, cnt, tombstone, out_keys, out_vals, out_flags, g0, sm.rank);
  __syncthreads();
  // directory share: the bucket consumed the keys [b << 24, b << 24 | 0xffffff]
  const uint32_t kmin = first << 24, kmax = (last << 24) | 0x00ffffffu;
  const DirGeom g = dir_geometry(kmin, kmax, n, dir_bits, rows_log2);
  const uint32_t *rows = out_keys + g0;
  fill_directory(out_dir, g, b > first, (b << 24) - 1u, (b << 24) | 0x00ffffffu, b == last, g0, kept, g0 + kept,
                 [&](uint32_t j) { return rows[j]; });
  if (b == first && threadIdx.x == 0) {
    out_desc->kmin = g.kmin;
    out_desc->kmax = g.kmax;
    out_desc->shift = g.shift;
    out_desc->nbuckets = g.nbuckets;
  }
  if (b == last && threadIdx.x == 0) out_desc->n = g0 + kept;
}

}  // namespace admit
}  // namespace lsm
}  // namespace gpulsm
