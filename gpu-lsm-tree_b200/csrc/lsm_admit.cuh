// Batch admission by top-byte buckets: the sorted, deduplicated level run of
// one update batch (GPULSMOpt.cuh:2578-2633 sorts the batch, ages the
// duplicates and keeps the newest) in four launches instead of a four-pass
// LSD sort plus a dedup pass:
//
//   1. part_hist_kernel     per 2048-key tile, the counts of the key's top byte
//   2. part_scan_kernel     per top byte, the exclusive scan over the tiles
//   3. part_scatter_kernel  words (key << 32 | value) written to their top-byte
//                           bucket in input order (a stable partition); a
//                           batch of inserts and erases packs the input
//                           position instead of the value
//   4. admit_bucket_kernel  one CTA per top-byte bucket, in bucket order:
//                           sorts the bucket by (key, input position) in
//                           shared memory (a 12-bit counting sort plus an
//                           insertion sort of every bin, or stable 8-bit LSD
//                           passes when a bin is large), keeps the last row of
//                           every equal-key run (the newest), chains its row
//                           count to the earlier buckets by decoupled look-back
//                           and writes the level rows plus its share of the
//                           radix directory.  A bucket larger than shared
//                           memory is sorted through global memory by the
//                           same CTA in chunks (correct for any skew, slower).
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

// Lanes of the warp whose 8-bit digit equals this lane's, among the lanes in `valid`.
__device__ __forceinline__ uint32_t digit_peers(uint32_t d, uint32_t valid) {
  return match_any_bits<8>(d) & valid;
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

// Where a kept row's value and flag come from.  Insert and erase batches
// packed the value into the sort word (erase: the tombstone value); a mixed
// batch packed the row's input position instead, and the row reads its value
// and its erase mark from the batch by that position.
struct RowSource {
  const uint32_t *vals;  // mixed batches: the batch's values (erased rows ignore theirs)
  const uint8_t *erase;  // mixed batches: nonzero = the row erases its key; null otherwise
  int tombstone;         // erase batches
};

__device__ __forceinline__ void resolve_row(const RowSource &src, unsigned long long w, uint32_t &v, uint8_t &f) {
  if (src.erase) {
    const uint32_t i = uint32_t(w);
    const bool er = src.erase[i] != 0;
    v = er ? kTombValue : src.vals[i];
    f = er ? kFlagTomb : uint8_t(0);
  } else {
    v = uint32_t(w);
    f = src.tombstone ? kFlagTomb : uint8_t(0);
  }
}

// at(j): the j-th word of a sorted sequence (an array, or an index into one)
template <typename At>
__device__ __forceinline__ bool run_end(const At &at, uint32_t j, uint32_t cnt) {
  return j + 1 == cnt || word_key(at(j)) != word_key(at(j + 1));
}

// Distinct keys of a sorted sequence.
template <typename At>
__device__ __forceinline__ uint32_t count_distinct(const At &at, uint32_t cnt, RankSmem &sm) {
  uint32_t c = 0;
  for (uint32_t j = threadIdx.x; j < cnt; j += kThreads) c += run_end(at, j, cnt) ? 1u : 0u;
  (void)block_exclusive_scan<kThreads>(c, sm.scan, &sm.total);
  return sm.total;
}

// Write the last row of every equal-key run of the sorted sequence
// at(0 .. cnt) to out[g0 ...], in chunks of kCap read striped (element
// c0 + i*kThreads + t): per item a warp ballot counts the kept rows, one block
// scan over the (item, warp) counts gives every warp its output offset, and
// consecutive lanes store consecutive rows.  The first element of every
// equal-key run writes the radix-directory entries its run's row starts: the
// buckets after the bucket of the previous distinct key (bp before the first
// row) up to its own, pointing at the row (= run ends before the element).
template <typename At>
__device__ __forceinline__ void write_rows(const At &at, uint32_t cnt, const RowSource &src, uint32_t *out_keys,
                                           uint32_t *out_vals, uint8_t *out_flags, unsigned long long g0,
                                           RankSmem &rs, uint32_t *__restrict__ dir, const DirGeom &g,
                                           int64_t bp) {
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
      ends[i] = __ballot_sync(0xffffffffu, e < c0 + cc && run_end(at, e, cnt));
      if (lane == 0) slot[i * kWarps + w] = __popc(ends[i]);
    }
    __syncthreads();
    const uint32_t v = threadIdx.x < uint32_t(kItems * kWarps) ? slot[threadIdx.x] : 0u;
    const uint32_t ex = block_exclusive_scan<kThreads>(v, rs.scan, &rs.total);
    const uint32_t chunk_kept = rs.total;
    if (threadIdx.x < uint32_t(kItems * kWarps)) slot[threadIdx.x] = ex;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      const uint32_t e = c0 + uint32_t(i) * kThreads + threadIdx.x;
      if (e >= c0 + cc) continue;
      // run ends before e = the output row of e's run (its last element is kept)
      const unsigned long long r = g0 + written + slot[i * kWarps + w] + __popc(ends[i] & lt);
      const unsigned long long w64 = at(e);
      const uint32_t k = word_key(w64);
      if ((ends[i] >> lane) & 1u) {
        uint32_t v;
        uint8_t f;
        resolve_row(src, w64, v, f);
        out_keys[r] = k;
        out_vals[r] = v;
        out_flags[r] = f;
      }
      // the first element of a run writes the directory entries its row starts
      // (no directory: it is built when a read first needs it)
      const uint32_t kp = e > 0 ? word_key(at(e - 1)) : 0u;
      if (dir && (e == 0 || kp != k)) {
        const int64_t bprev = e > 0 ? int64_t((kp - g.kmin) >> g.shift) : bp;
        const int64_t bj = int64_t((k - g.kmin) >> g.shift);
        for (int64_t b = bprev + 1; b <= bj; ++b)
          if (GPULSM_OK(b >= 0 && b < int64_t(g.nbuckets), 10, b)) dir[b] = uint32_t(r);
      }
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

// ---------------------------------------------------------------------------
// Stable partition of a batch by the key's top byte without a look-back chain
// (reduce, then scan, then scatter), reading keys and values directly:
//   part_hist_kernel    per tile of kPartTile keys: its 256 top-byte counts,
//                       stored byte-major (cnt[byte * tiles + tile])
//   part_scan_kernel    per byte: exclusive scan over the tiles, and the
//                       byte's total
//   part_scatter_kernel per tile: byte bases from the totals, a stable rank
//                       inside the tile (ballot peer groups), then the words
//                       (key << 32 | value) staged by byte and written in runs
constexpr int kPartThreads = 256;
constexpr int kPartItems = 8;
constexpr uint32_t kPartTile = uint32_t(kPartThreads) * kPartItems;  // 2048 keys
constexpr int kPartWarps = kPartThreads / 32;

inline uint32_t part_tiles(uint64_t n) { return uint32_t((n + kPartTile - 1) / kPartTile); }

__global__ void __launch_bounds__(kPartThreads) part_hist_kernel(const uint32_t *__restrict__ keys, uint32_t n,
                                                                 uint32_t tiles, uint32_t *__restrict__ cnt,
                                                                 unsigned long long *__restrict__ zero,
                                                                 uint32_t zero_words) {
  __shared__ uint32_t h[256];
  chain_wait();
  // the bucket kernel's ticket counter and look-back slots start at zero
  for (uint32_t i = blockIdx.x * kPartThreads + threadIdx.x; i < zero_words; i += gridDim.x * kPartThreads)
    zero[i] = 0ull;
  const uint32_t base = blockIdx.x * kPartTile;
  uint32_t k[kPartItems];
#pragma unroll
  for (int i = 0; i < kPartItems; ++i) {  // all loads in flight before the first atomic
    const uint32_t e = base + uint32_t(i) * kPartThreads + threadIdx.x;
    k[i] = e < n ? keys[e] : 0u;
  }
  h[threadIdx.x] = 0;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kPartItems; ++i)
    if (base + uint32_t(i) * kPartThreads + threadIdx.x < n) atomicAdd(&h[k[i] >> 24], 1u);
  __syncthreads();
  cnt[threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

// one block per top byte; prefix[byte * tiles + tile] = rows of that byte in
// earlier tiles, total[byte] = the byte's rows
__global__ void __launch_bounds__(kPartThreads) part_scan_kernel(const uint32_t *__restrict__ cnt, uint32_t tiles,
                                                                 uint32_t *__restrict__ prefix,
                                                                 uint32_t *__restrict__ total) {
  __shared__ uint32_t s_scan[kPartWarps];
  __shared__ uint32_t s_total;
  chain_wait();
  const uint32_t b = blockIdx.x;
  uint32_t carry = 0;
  for (uint32_t t0 = 0; t0 < tiles; t0 += kPartThreads) {
    const uint32_t t = t0 + threadIdx.x;
    const uint32_t c = t < tiles ? cnt[b * tiles + t] : 0u;
    const uint32_t ex = block_exclusive_scan<kPartThreads>(c, s_scan, &s_total);
    if (t < tiles) prefix[b * tiles + t] = carry + ex;
    carry += s_total;
  }
  if (threadIdx.x == 0) total[b] = carry;
}

__global__ void __launch_bounds__(kPartThreads) part_scatter_kernel(
    const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals, uint32_t n, uint32_t tiles,
    const uint32_t *__restrict__ prefix, const uint32_t *__restrict__ total, unsigned long long *__restrict__ out,
    int pack_index) {
  __shared__ unsigned long long s_words[kPartTile];
  __shared__ uint32_t warp_hist[kPartWarps][256];
  __shared__ uint32_t s_start[256];   // first staged position of each byte in the tile
  __shared__ uint32_t s_dst[256];     // global position of the tile's first row of each byte
  __shared__ uint32_t s_scan[kPartWarps];
  __shared__ uint32_t s_total;
  chain_wait();
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, tile = blockIdx.x;
  // the tile's keys and values, then the byte bases: all loads are in flight
  // before the first shared-memory step waits on any of them
  const uint32_t wbase = tile * kPartTile + warp * 32u * kPartItems;
  unsigned long long w[kPartItems];
  uint32_t d[kPartItems], rank[kPartItems];
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int i = 0; i < kPartItems; ++i) {
    const uint32_t e = wbase + uint32_t(i) * 32u + lane;
    const bool valid = e < n;
    const uint32_t k = valid ? keys[e] : 0u;
    const uint32_t v = pack_index ? e : vals ? (valid ? vals[e] : 0u) : kTombValue;
    w[i] = (static_cast<unsigned long long>(k) << 32) | v;
    d[i] = valid ? (k >> 24) : 256u;
  }
  const uint32_t tot = total[threadIdx.x];
  const uint32_t pre = prefix[threadIdx.x * tiles + tile];
  for (uint32_t i = lane; i < 256; i += 32) warp_hist[warp][i] = 0;
  // byte bases: exclusive scan of the totals (every tile repeats this 256-entry scan)
  const uint32_t base = block_exclusive_scan<kPartThreads>(tot, s_scan, &s_total);
  s_dst[threadIdx.x] = base + pre;
  __syncwarp();
#pragma unroll
  for (int i = 0; i < kPartItems; ++i) {  // stable rank per warp, items in element order
    const uint32_t peers = match_any_bits<9>(d[i]);
    const uint32_t leader = 31u - __clz(peers);
    uint32_t r = 0;
    if (lane == leader && d[i] < 256u) {
      r = warp_hist[warp][d[i]];
      warp_hist[warp][d[i]] = r + __popc(peers);
    }
    rank[i] = __shfl_sync(0xffffffffu, r, leader) + __popc(peers & lt);
    __syncwarp();
  }
  __syncthreads();
  // thread b: exclusive offsets of each warp for byte b, then byte starts in the tile
  uint32_t run = 0;
#pragma unroll
  for (int ww = 0; ww < kPartWarps; ++ww) {
    const uint32_t c = warp_hist[ww][threadIdx.x];
    warp_hist[ww][threadIdx.x] = run;
    run += c;
  }
  const uint32_t st = block_exclusive_scan<kPartThreads>(run, s_scan, &s_total);
  s_start[threadIdx.x] = st;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kPartItems; ++i)
    if (d[i] < 256u) s_words[s_start[d[i]] + warp_hist[warp][d[i]] + rank[i]] = w[i];
  __syncthreads();
  const uint32_t count = min(kPartTile, n - tile * kPartTile);
  for (uint32_t j = threadIdx.x; j < count; j += kPartThreads) {
    const unsigned long long x = s_words[j];
    const uint32_t b = uint32_t(x >> 56);
    out[s_dst[b] + (j - s_start[b])] = x;
  }
}

// Exclusive prefix of a bucket's row count over the earlier buckets.  Every
// bucket publishes its own count (never an inclusive prefix) and reads all the
// earlier counts at once, one thread per bucket, so once they are published
// the wait is one round trip instead of a walk of distance / 32 round trips.
// Waits are bounded: a count that never appears sets the timeout bit and
// reads as 0 (the host then fails the dictionary).
static_assert(kBuckets <= kThreads, "one thread per earlier bucket");
__device__ __forceinline__ uint32_t bucket_prefix(unsigned long long *lb, uint32_t tile, uint32_t kept,
                                                  uint32_t *status, RankSmem &rs) {
  if (threadIdx.x == 0) st_relaxed_u64(lb + tile, kLbAgg | kept);
  uint32_t v = 0;
  if (threadIdx.x < tile) {
    uint32_t spins = 0;
    unsigned long long x;
    while (((x = ld_relaxed_u64(lb + threadIdx.x)) & ~kLbMask) == 0ull) {
      if (++spins > kMaxSpins) {
        atomicOr(status, kDevWaitTimeout);
        x = kLbAgg;
        break;
      }
      __nanosleep(32);
    }
    v = uint32_t(x & kLbMask);
  }
  (void)block_exclusive_scan<kThreads>(v, rs.scan, &rs.total);
  return rs.total;
}

constexpr uint32_t kBins = 4096;   // counting-sort bins of the fast path (12 key bits)
constexpr uint32_t kMaxBin = 32;   // larger bins (skew) take the LSD passes instead

struct BucketSmem {
  unsigned long long words[kCap];  // the bucket's words in input order
  uint16_t idx[kCap];              // input position of each element, in sorted order
  uint32_t sk[kCap];               // counting-sort output: in-bin key bits << 13 | input position
  uint32_t bins[kBins];            // bin counts, then bin ends
  RankSmem rank;
  uint32_t start[kBuckets + 1];
  uint32_t off[256];
  uint32_t first, last, tile, maxbin;
  unsigned long long g0;
};

// Fast in-bucket sort: one counting pass on the 12 highest varying key bits
// (shared atomics: order inside a bin is arbitrary), then every element
// finds its place inside its bin - about one other element on uniform keys -
// by counting the bin's elements that order before it by (key, input
// position), which restores input order among equal keys; the words are then
// permuted into that order in place (through registers).  Inside a bin the
// keys differ only in the bits below the bin bits (ds <= 12 of them), so
// (those bits << 13 | input position) orders a bin in one 32-bit compare.
// Returns false (nothing changed) when a bin exceeds kMaxBin.
static_assert(kCap <= (1u << 13), "input positions fit 13 bits");
__device__ __forceinline__ bool bin_sort(BucketSmem &sm, uint32_t cnt, uint32_t vary) {
  const uint32_t hb = 31u - __clz(vary);
  const uint32_t ds = hb >= 11u ? hb - 11u : 0u;
  const uint32_t low = (1u << ds) - 1u;
  for (uint32_t d = threadIdx.x; d < kBins; d += kThreads) sm.bins[d] = 0;
  if (threadIdx.x == 0) sm.maxbin = 0;
  __syncthreads();
  for (uint32_t e = threadIdx.x; e < cnt; e += kThreads) atomicAdd(&sm.bins[(word_key(sm.words[e]) >> ds) & (kBins - 1)], 1u);
  __syncthreads();
  // exclusive scan of the bins: thread t owns the 8 consecutive bins [8t, 8t + 8),
  // read and written as two 16-byte vectors
  static_assert(kBins == 8u * kThreads, "8 bins per thread");
  uint4 *bv = reinterpret_cast<uint4 *>(sm.bins);
  const uint4 lo4 = bv[2 * threadIdx.x], hi4 = bv[2 * threadIdx.x + 1];
  uint32_t c[8] = {lo4.x, lo4.y, lo4.z, lo4.w, hi4.x, hi4.y, hi4.z, hi4.w};
  uint32_t sum = 0, mx = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    sum += c[j];
    mx = max(mx, c[j]);
  }
  uint32_t run = block_exclusive_scan<kThreads>(sum, sm.rank.scan, &sm.rank.total);
  if (mx) atomicMax(&sm.maxbin, mx);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const uint32_t x = c[j];
    c[j] = run;
    run += x;
  }
  bv[2 * threadIdx.x] = make_uint4(c[0], c[1], c[2], c[3]);
  bv[2 * threadIdx.x + 1] = make_uint4(c[4], c[5], c[6], c[7]);
  __syncthreads();
  if (sm.maxbin > kMaxBin) return false;  // uniform across the block
  for (uint32_t e = threadIdx.x; e < cnt; e += kThreads) {
    const uint32_t k = word_key(sm.words[e]);
    const uint32_t p = atomicAdd(&sm.bins[(k >> ds) & (kBins - 1)], 1u);
    sm.sk[p] = ((k & low) << 13) | e;
  }
  __syncthreads();  // bins[d] now holds the end of bin d
  const uint32_t keff = (cnt + kThreads - 1) / kThreads;
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const uint32_t p = uint32_t(i) * kThreads + threadIdx.x;
    if (uint32_t(i) >= keff || p >= cnt) continue;
    const uint32_t x = sm.sk[p], e = x & 0x1fffu;
    const uint32_t bin = (word_key(sm.words[e]) >> ds) & (kBins - 1);
    const uint32_t b0 = bin ? sm.bins[bin - 1] : 0u, b1 = sm.bins[bin];
    uint32_t r = 0;
    for (uint32_t q = b0; q < b1; ++q) r += sm.sk[q] < x ? 1u : 0u;  // at most kMaxBin
    sm.idx[b0 + r] = uint16_t(e);
  }
  __syncthreads();
  unsigned long long t[kItems];
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const uint32_t j = uint32_t(i) * kThreads + threadIdx.x;
    t[i] = uint32_t(i) < keff && j < cnt ? sm.words[sm.idx[j]] : 0ull;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kItems; ++i) {
    const uint32_t j = uint32_t(i) * kThreads + threadIdx.x;
    if (uint32_t(i) < keff && j < cnt) sm.words[j] = t[i];
  }
  __syncthreads();
  return true;
}
constexpr size_t kBucketSmemBytes = sizeof(BucketSmem);

// One CTA per nonempty top-byte bucket (ticket t -> bucket first + t).
// words0: the batch partitioned by top byte (stable); words1: scratch of the
// same size for oversized buckets; top_hist: rows per top byte.
__global__ void __launch_bounds__(kThreads, 2) admit_bucket_kernel(
    unsigned long long *__restrict__ words0, unsigned long long *__restrict__ words1,
    const uint32_t *__restrict__ top_hist, uint32_t n, RowSource src, uint32_t *__restrict__ out_keys,
    uint32_t *__restrict__ out_vals, uint8_t *__restrict__ out_flags, LevelDesc *__restrict__ out_desc,
    uint32_t *__restrict__ out_dir, uint32_t dir_bits, uint32_t rows_log2, unsigned long long *__restrict__ lb,
    uint32_t *__restrict__ tile_counter, uint32_t *__restrict__ status) {
  extern __shared__ __align__(16) unsigned char dyn[];
  BucketSmem &sm = *reinterpret_cast<BucketSmem *>(dyn);
  chain_wait();
  // the top-byte counts load while the ticket is taken
  const uint32_t c = threadIdx.x < kBuckets ? top_hist[threadIdx.x] : 0u;
  if (threadIdx.x == 0) {
    sm.tile = atomicAdd(tile_counter, 1u);
    sm.first = kBuckets;
    sm.last = 0;
  }
  __syncthreads();
  // bucket starts (exclusive scan of the top-byte counts) and the nonempty span
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
    if (threadIdx.x == 0) {
      atomicOr(status, kDevBadInput);
      st_relaxed_u64(lb + tile, kLbAgg);  // later buckets need not wait for it
    }
    return;
  }
  const unsigned long long *sorted;  // the bucket's words sorted by (key, input position)
  if (cnt <= kCap) {
    {  // every thread issues all its loads before its shared stores
      unsigned long long t[kItems];
#pragma unroll
      for (int i = 0; i < kItems; ++i) {
        const uint32_t j = uint32_t(i) * kThreads + threadIdx.x;
        t[i] = j < cnt ? words0[s0 + j] : 0ull;
      }
#pragma unroll
      for (int i = 0; i < kItems; ++i) {
        const uint32_t j = uint32_t(i) * kThreads + threadIdx.x;
        if (j < cnt) sm.words[j] = t[i];
      }
    }
    __syncthreads();
    const uint32_t vary = cnt > 1 ? varying_bits(sm.words, cnt, sm.rank) & 0x00ffffffu : 0u;
    if (!(vary && bin_sort(sm, cnt, vary))) {
      // no varying bits (one key, input order kept) or a skewed bucket: LSD passes
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
          if (uint32_t(i) < keff && wbase + uint32_t(i) * 32u + (threadIdx.x & 31u) < cnt)
            sm.words[pos[i]] = it[i];
        __syncthreads();
      }
    }
    sorted = sm.words;
  } else {
    const uint32_t vary = varying_bits(words0 + s0, cnt, sm.rank) & 0x00ffffffu;
    sorted = sort_global(words0 + s0, words1 + s0, cnt, vary, sm.rank, sm.off);
    __syncthreads();
  }
  // directory share: the bucket consumed the keys [b << 24, b << 24 | 0xffffff];
  // its rows start the buckets after bucket((b << 24) - 1) (the previous
  // bucket's last key) and it closes the range up to bucket(b << 24 | 0xffffff)
  const uint32_t kmin = first << 24, kmax = (last << 24) | 0x00ffffffu;
  const DirGeom g = dir_geometry(kmin, kmax, n, dir_bits, rows_log2);
  const int32_t bp = b > first ? int32_t((((b << 24) - 1u) - g.kmin) >> g.shift) : -1;
  const int32_t bl = b == last ? int32_t(g.nbuckets) - 1 : int32_t((((b << 24) | 0x00ffffffu) - g.kmin) >> g.shift);
  uint32_t kept;
  unsigned long long g0;
  if (cnt <= kCap) {
    // one ballot pass marks the last row of every equal-key run; a block scan
    // gives every kept row its offset and the bucket its row count, which is
    // published before the bucket reads the earlier buckets' counts
    const unsigned long long *w = sm.words;
    const uint32_t keff = (cnt + kThreads - 1) / kThreads;
    const uint32_t lane = threadIdx.x & 31u, wi = threadIdx.x >> 5, lt = lanemask_lt();
    uint32_t *slot = sm.rank.dstart;  // kItems * kWarps counts, then their offsets
    static_assert(kItems * kWarps <= kBuckets, "one scan slot per (item, warp)");
    uint32_t ends[kItems];
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      ends[i] = 0u;
      if (uint32_t(i) < keff) {
        const uint32_t e = uint32_t(i) * kThreads + threadIdx.x;
        ends[i] = __ballot_sync(0xffffffffu, e < cnt && (e + 1 == cnt || word_key(w[e]) != word_key(w[e + 1])));
      }
      if (lane == 0) slot[i * kWarps + wi] = __popc(ends[i]);
    }
    __syncthreads();
    const uint32_t v = threadIdx.x < uint32_t(kItems * kWarps) ? slot[threadIdx.x] : 0u;
    const uint32_t ex = block_exclusive_scan<kThreads>(v, sm.rank.scan, &sm.rank.total);
    kept = sm.rank.total;
    if (threadIdx.x < uint32_t(kItems * kWarps)) slot[threadIdx.x] = ex;
    g0 = bucket_prefix(lb, tile, kept, status, sm.rank);  // its block scan orders the slot stores
    if (g0 + kept > n) {  // only after a timed-out wait (status bit set)
      atomicOr(status, kDevWaitTimeout);
      return;
    }
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
      const uint32_t e = uint32_t(i) * kThreads + threadIdx.x;
      if (uint32_t(i) >= keff || e >= cnt) continue;
      // run ends before e = the output row of e's run (its last element is kept)
      const unsigned long long r = g0 + slot[i * kWarps + wi] + __popc(ends[i] & lt);
      const unsigned long long w64 = w[e];
      const uint32_t k = word_key(w64);
      if ((ends[i] >> lane) & 1u) {
        uint32_t v;
        uint8_t f;
        resolve_row(src, w64, v, f);
        out_keys[r] = k;
        out_vals[r] = v;
        out_flags[r] = f;
      }
      // the first element of a run writes the directory entries its row starts
      // (no directory: it is built when a read first needs it)
      const uint32_t kp = e > 0 ? word_key(w[e - 1]) : 0u;
      if (out_dir && (e == 0 || kp != k)) {
        const int32_t bprev = e > 0 ? int32_t((kp - g.kmin) >> g.shift) : bp;
        const int32_t bj = int32_t((k - g.kmin) >> g.shift);
        for (int32_t bb = bprev + 1; bb <= bj; ++bb)
          if (GPULSM_OK(bb >= 0 && bb < int32_t(g.nbuckets), 10, bb)) out_dir[bb] = uint32_t(r);
      }
    }
  } else {
    const auto by_array = [sorted](uint32_t j) { return sorted[j]; };
    kept = count_distinct(by_array, cnt, sm.rank);
    g0 = bucket_prefix(lb, tile, kept, status, sm.rank);
    if (g0 + kept > n) {  // only after a timed-out wait (status bit set)
      atomicOr(status, kDevWaitTimeout);
      return;
    }
    write_rows(by_array, cnt, src, out_keys, out_vals, out_flags, g0, sm.rank, out_dir, g, int64_t(bp));
  }
  if (out_dir && threadIdx.x == 0) {
    // an empty bucket between the first and the last one only closes its range
    const int32_t blast = cnt ? int32_t((word_key(sorted[cnt - 1]) - g.kmin) >> g.shift) : bp;
    for (int32_t bb = blast + 1; bb <= bl; ++bb)
      if (GPULSM_OK(bb >= 0 && bb < int32_t(g.nbuckets), 13, bb)) out_dir[bb] = uint32_t(g0 + kept);
    if (b == last) out_dir[g.nbuckets] = uint32_t(g0 + kept);
  }
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
