// Kernels of the LSM dictionary (GPULSMOpt semantics, u32 keys / u32 values).
//
// HBM layout of one level (a sorted run of unique keys, newest version only):
//   keys   u32[n]   sorted ascending
//   vals   u32[n]   value, or 0xffffffff for a tombstone
//   flags  u8[n]    bit 0 = tombstone (read only when the value is 0xffffffff)
//   dir    u32[nbuckets+1]  radix directory: dir[b] = first row whose
//          (key - kmin) >> shift >= b, so bucket b spans [dir[b], dir[b+1]).
//   desc   LevelDesc {n, kmin, kmax, shift, nbuckets} written on the device.
// Levels are ordered newest (index 0) to oldest; the first level holding a key
// decides its visible version (the reference's lower level id = newer rule,
// GPULSMOpt.cuh:4714-4750).
#pragma once

#include "common.cuh"
#include "learned.cuh"

namespace gpulsm {
namespace lsm {

constexpr int kMaxLevels = 16;
constexpr uint32_t kTombValue = 0xffffffffu;
constexpr uint8_t kFlagTomb = 1u;

struct LevelDesc {
  unsigned long long n;
  uint32_t kmin, kmax, shift, nbuckets;
  uint32_t pad[2];
};
static_assert(sizeof(LevelDesc) == 32, "LevelDesc layout");

// How a level is searched: its radix directory (dir), its learned position
// model (mh/ms, search mode 1) or, with neither, binary search over all rows.
__device__ __forceinline__ LevelDesc load_desc(const LevelDesc *p) {
  LevelDesc d;
  d.n = __ldg(&p->n);
  d.kmin = __ldg(&p->kmin);
  d.kmax = __ldg(&p->kmax);
  d.shift = __ldg(&p->shift);
  d.nbuckets = __ldg(&p->nbuckets);
  return d;
}

struct LevelView {
  const uint32_t *keys;
  const uint32_t *vals;
  const uint8_t *flags;
  const uint32_t *dir;
  const LevelDesc *desc;
  const learned::ModelHeader *mh = nullptr;
  const learned::Segment *ms = nullptr;
  const uint32_t *live = nullptr;  // live-value prefix (range sums over levels), u32 modulo 2^32
};

struct LevelSet {
  LevelView lv[kMaxLevels];
  uint32_t count;
};

// Receipt of an update, written into mapped pinned host memory by the kernel
// that finishes it: the row count of every level afterwards and the status
// word, each one 8-byte word tagged with the update's sequence number
// (count | seq << 33, status | seq << 32), so the host validates every word
// on its own and neither a fence nor an event is needed.
struct ReceiptSrc {
  const LevelDesc *desc[kMaxLevels];
  unsigned long long *out;  // kMaxLevels counts, then the status
  const uint32_t *status;
  uint32_t count;
  int32_t self;             // level whose count is the writing kernel's own output
  uint32_t seq;
};
constexpr int kReceiptWords = kMaxLevels + 1;
constexpr unsigned long long kReceiptCountMask = (1ull << 33) - 1ull;

// Run by the first warp of the finishing CTA.
__device__ __forceinline__ void write_receipt(const ReceiptSrc &r, unsigned long long self_n) {
  const uint32_t i = threadIdx.x & 31u;
  if (i < uint32_t(kMaxLevels)) {
    unsigned long long n = 0;
    if (int32_t(i) == r.self) n = self_n;
    else if (i < r.count && r.desc[i]) n = r.desc[i]->n;
    r.out[i] = (n & kReceiptCountMask) | (static_cast<unsigned long long>(r.seq & 0x7fffffffu) << 33);
  } else if (i == uint32_t(kMaxLevels)) {
    r.out[i] = static_cast<unsigned long long>(*r.status) | (static_cast<unsigned long long>(r.seq) << 32);
  }
}

// ---------------------------------------------------------------------------
// Admission: pack (key, value) into one u64 word (key in the high half so an
// LSD sort on bits 32..63 orders by key and keeps input order among equal
// keys) and count the key bytes of the four sort passes.
// kTopOnly: count only the top key byte (hist[3 * 256 ...]), for admission
// by top-byte buckets.
template <bool kTopOnly>
__global__ void __launch_bounds__(256) pack_histogram_kernel(const uint32_t *__restrict__ keys,
                                                             const uint32_t *__restrict__ vals,
                                                             uint32_t n,
                                                             unsigned long long *__restrict__ words,
                                                             uint32_t *__restrict__ hist) {
  __shared__ uint32_t s[4][256];
  for (uint32_t i = threadIdx.x; i < 4 * 256; i += 256) (&s[0][0])[i] = 0;
  __syncthreads();
  for (uint32_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += gridDim.x * 256) {
    const uint32_t k = keys[i];
    const uint32_t v = vals ? vals[i] : kTombValue;
    words[i] = (static_cast<unsigned long long>(k) << 32) | v;
    if (!kTopOnly) {
      atomicAdd(&s[0][k & 0xffu], 1u);
      atomicAdd(&s[1][(k >> 8) & 0xffu], 1u);
      atomicAdd(&s[2][(k >> 16) & 0xffu], 1u);
    }
    atomicAdd(&s[3][k >> 24], 1u);
  }
  __syncthreads();
  for (int p = kTopOnly ? 3 : 0; p < 4; ++p) {
    const uint32_t c = s[p][threadIdx.x];
    if (c) atomicAdd(&hist[p * 256 + threadIdx.x], c);
  }
}

// ---------------------------------------------------------------------------
// Radix directory built by the kernel that writes the run.  Its geometry is
// fixed before the rows exist from a key range [kmin, kmax] that bounds every
// output row (dedup and tombstone drops only remove rows) and the host's upper
// bound of the row count: about 2^rows_log2 rows per bucket, at most
// 2^dir_bits buckets.
struct DirGeom {
  uint32_t kmin, kmax, shift, nbuckets;
};

__device__ __forceinline__ DirGeom dir_geometry(uint32_t kmin, uint32_t kmax, unsigned long long n_upper,
                                                uint32_t dir_bits, uint32_t rows_log2) {
  const uint32_t range = kmax - kmin;
  const uint32_t nl2 = ceil_log2_u64(n_upper ? n_upper : 1);
  const uint32_t want = min(nl2 > rows_log2 ? nl2 - rows_log2 : 0u, dir_bits);
  const uint32_t range_bits = range ? 32u - __clz(range) : 0u;
  const uint32_t shift = range_bits > want ? range_bits - want : 0u;
  return DirGeom{kmin, kmax, shift, (range >> shift) + 1u};
}

// A tile that consumed the input keys in (prev_key, last_key] (no prev for the
// first tile) and kept `cnt` rows - keys key_at(0..cnt) at global positions
// g0.. - owns the directory buckets (bucket(prev_key), bucket(last_key)]: each
// gets the position of the tile's first kept row in or after it, or g0 + cnt
// (where the next tile's rows start) when no kept row of the tile reaches it.
// Consecutive tiles own consecutive bucket ranges, so every entry is written
// exactly once; the last tile also closes the range and writes dir[nbuckets].
template <typename KeyAt>
__device__ __forceinline__ void fill_directory(uint32_t *__restrict__ dir, const DirGeom &g, bool has_prev,
                                               uint32_t prev_key, uint32_t last_key, bool last_tile,
                                               unsigned long long g0, uint32_t cnt, unsigned long long n_out,
                                               KeyAt key_at) {
  const int64_t bp = has_prev ? int64_t((prev_key - g.kmin) >> g.shift) : -1;
  const int64_t bl = last_tile ? int64_t(g.nbuckets) - 1 : int64_t((last_key - g.kmin) >> g.shift);
  for (uint32_t j = threadIdx.x; j < cnt; j += blockDim.x) {
    const int64_t bj = int64_t((key_at(j) - g.kmin) >> g.shift);
    const int64_t bprev = j ? int64_t((key_at(j - 1) - g.kmin) >> g.shift) : bp;
    for (int64_t b = bprev + 1; b <= bj; ++b)
      if (GPULSM_OK(b >= 0 && b < int64_t(g.nbuckets), 10, b)) dir[b] = uint32_t(g0 + j);
  }
  if (threadIdx.x == 0) {
    const int64_t blast = cnt ? int64_t((key_at(cnt - 1) - g.kmin) >> g.shift) : bp;
    for (int64_t b = blast + 1; b <= bl; ++b)
      if (GPULSM_OK(b >= 0 && b < int64_t(g.nbuckets), 13, b)) dir[b] = uint32_t(g0 + cnt);
    if (last_tile) dir[g.nbuckets] = uint32_t(n_out);
  }
}

__device__ __forceinline__ void write_empty_desc(LevelDesc *d, uint32_t *dir) {
  d->n = 0;
  d->kmin = 1u;
  d->kmax = 0u;
  d->shift = 0u;
  d->nbuckets = 1u;
  if (dir) {
    dir[0] = 0u;
    dir[1] = 0u;
  }
}

// The radix directory of a level whose merge skipped it: entry b is the first
// row whose key's bucket is at least b (n when none) and entry nbuckets is n -
// the entries the merge kernel writes when it builds the directory itself.
// Geometry from the level's descriptor; rows past desc->n are not read.
// Each thread takes 8 consecutive rows (two 16-byte loads: run buffers are
// 16-byte aligned) and the key before them.
constexpr uint32_t kDirRows = 8;

__global__ void __launch_bounds__(256) build_directory_kernel(const uint32_t *__restrict__ keys,
                                                              const LevelDesc *__restrict__ desc,
                                                              uint32_t *__restrict__ dir) {
  const uint64_t n = desc->n;
  const uint32_t kmin = desc->kmin, shift = desc->shift, nb = desc->nbuckets;
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  const uint64_t t0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  // the buckets after the last row's (all of them for an empty level) close at n
  const int64_t blast = n ? int64_t((keys[n - 1] - kmin) >> shift) : -1;
  for (uint64_t b = uint64_t(blast + 1) + t0; b <= nb; b += stride) dir[b] = uint32_t(n);
  for (uint64_t j0 = t0 * kDirRows; j0 < n; j0 += stride * kDirRows) {
    uint32_t k[kDirRows];
    if (j0 + kDirRows <= n) {
      const uint4 *v = reinterpret_cast<const uint4 *>(keys + j0);
      const uint4 x = __ldg(v), y = __ldg(v + 1);
      k[0] = x.x, k[1] = x.y, k[2] = x.z, k[3] = x.w, k[4] = y.x, k[5] = y.y, k[6] = y.z, k[7] = y.w;
    } else {
#pragma unroll
      for (uint32_t i = 0; i < kDirRows; ++i) k[i] = j0 + i < n ? keys[j0 + i] : 0u;
    }
    int64_t bp = j0 ? int64_t((keys[j0 - 1] - kmin) >> shift) : -1;
#pragma unroll
    for (uint32_t i = 0; i < kDirRows; ++i) {
      if (j0 + i >= n) break;
      const int64_t bj = int64_t((k[i] - kmin) >> shift);
      for (int64_t b = bp + 1; b <= bj; ++b) dir[b] = uint32_t(j0 + i);
      bp = bj;
    }
  }
}

// Keep the LAST word of every equal-key run of a stably sorted batch (the
// highest input index wins, GPULSMOpt.cuh:2578-2598 ages + :2633 keep-last)
// and split it into a level (keys, vals, flags, directory).  Single pass: tile
// counts are chained by decoupled look-back.
constexpr int kCompactThreads = 256;
constexpr int kCompactItems = 8;
constexpr uint32_t kCompactTile = kCompactThreads * kCompactItems;

__global__ void __launch_bounds__(kCompactThreads) dedup_last_kernel(
    const unsigned long long *__restrict__ words, uint32_t n, int tombstone,
    uint32_t *__restrict__ out_keys, uint32_t *__restrict__ out_vals, uint8_t *__restrict__ out_flags,
    LevelDesc *__restrict__ out_desc, uint32_t *__restrict__ out_dir, uint32_t dir_bits, uint32_t rows_log2,
    unsigned long long *__restrict__ lb, uint32_t *__restrict__ tile_counter, uint32_t *__restrict__ status) {
  __shared__ unsigned long long s_words[kCompactTile + 1];
  __shared__ uint32_t s_scan[kCompactThreads / 32];
  __shared__ uint32_t s_total;
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_base;
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint32_t base = tile * kCompactTile;
  const uint32_t count = base < n ? min(kCompactTile, n - base) : 0u;
  for (uint32_t j = threadIdx.x; j <= count; j += kCompactThreads) {
    const uint32_t g = base + j;
    s_words[j] = g < n ? words[g] : ~0ull;  // one word past the tile decides keep-last
  }
  __syncthreads();
  uint32_t keep_mask = 0, kept = 0;
#pragma unroll
  for (int i = 0; i < kCompactItems; ++i) {
    const uint32_t j = threadIdx.x * kCompactItems + i;
    if (j < count) {
      const bool last = (base + j + 1 == n) || ((s_words[j] >> 32) != (s_words[j + 1] >> 32));
      if (last) {
        keep_mask |= 1u << i;
        ++kept;
      }
    }
  }
  const uint32_t local = block_exclusive_scan<kCompactThreads>(kept, s_scan, &s_total);
  const uint32_t tile_kept = s_total;
  if (threadIdx.x < 32) {
    const unsigned long long lb_excl = warp_lookback(lb, tile, tile_kept, status);
    if (threadIdx.x == 0) s_base = lb_excl;
  }
  // stage the kept words compactly (reuse the buffer after everyone has read it)
  unsigned long long mine[kCompactItems];
#pragma unroll
  for (int i = 0; i < kCompactItems; ++i) mine[i] = s_words[threadIdx.x * kCompactItems + i];
  __syncthreads();
  uint32_t o = local;
#pragma unroll
  for (int i = 0; i < kCompactItems; ++i)
    if (keep_mask & (1u << i)) s_words[o++] = mine[i];
  __syncthreads();
  const unsigned long long gbase = s_base;
  for (uint32_t j = threadIdx.x; j < tile_kept; j += kCompactThreads) {
    const unsigned long long w = s_words[j];
    if (gbase + j >= n) break;  // only after a timed-out look-back (status bit set)
    out_keys[gbase + j] = uint32_t(w >> 32);
    out_vals[gbase + j] = tombstone ? kTombValue : uint32_t(w);
    out_flags[gbase + j] = tombstone ? kFlagTomb : 0u;
  }
  // directory over the batch's key range (the sorted input's first and last key)
  const DirGeom g = dir_geometry(uint32_t(words[0] >> 32), uint32_t(words[n - 1] >> 32), n, dir_bits, rows_log2);
  const bool last_tile = base + kCompactTile >= n;
  const unsigned long long kept_total = gbase + tile_kept;
  fill_directory(out_dir, g, base > 0, base > 0 ? uint32_t(words[base - 1] >> 32) : 0u,
                 uint32_t(words[base + count - 1] >> 32), last_tile, gbase, tile_kept, kept_total,
                 [&](uint32_t j) { return uint32_t(s_words[j] >> 32); });
  if (tile == 0 && threadIdx.x == 0) {
    out_desc->kmin = g.kmin;
    out_desc->kmax = g.kmax;
    out_desc->shift = g.shift;
    out_desc->nbuckets = g.nbuckets;
  }
  if (last_tile && threadIdx.x == 0) out_desc->n = kept_total;
}

// ---------------------------------------------------------------------------
// Merge of a newer run A into an older run B (both sorted, unique keys).
// Merge-path tiles of kMergeTile outputs; ties put A first, so a B row whose
// key was just taken from A is shadowed and dropped (newest level wins).  With
// drop_tombstones (the output becomes the oldest level) tombstones disappear.
//
// The tile's input slices (keys, values, flags) arrive in shared memory by
// bulk copies.  Each thread merges kMergeItems consecutive outputs with the
// two run heads cached in registers and records the tile-local source index
// of every kept row; a block scan compacts them; the kept rows are gathered
// in striped order, staged at the alignment of their output position and
// written by bulk stores (plus a few unaligned head and tail rows).  An odd
// item count keeps the threads' starting diagonals in distinct banks.
constexpr int kMergeThreads = 256;
constexpr int kMergeItems = 15;
constexpr uint32_t kMergeTile = kMergeThreads * kMergeItems;  // 3840 outputs per tile

__device__ __forceinline__ uint64_t merge_path(const uint32_t *a, uint64_t na, const uint32_t *b,
                                               uint64_t nb, uint64_t diag) {
  uint64_t lo = diag > nb ? diag - nb : 0, hi = diag < na ? diag : na;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (a[mid] <= b[diag - 1 - mid]) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// merge_path on tile-local (32-bit) lengths, for shared-memory segments
__device__ __forceinline__ uint32_t merge_path32(const uint32_t *a, uint32_t na, const uint32_t *b, uint32_t nb,
                                                 uint32_t diag) {
  uint32_t lo = diag > nb ? diag - nb : 0, hi = diag < na ? diag : na;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (a[mid] <= b[diag - 1 - mid]) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Split points of every merge tile: parts[i] = A rows before diagonal
// min(i * kMergeTile, na + nb), one warp per split.  The merge-path predicate
// P(k) = A[k] <= B[d-1-k] is true then false along k; each step probes 32
// evenly spaced k at once (one round trip) and keeps the interval where P
// turns false, so a split costs about log32(na) dependent loads instead of
// log2(na).
__global__ void __launch_bounds__(256) merge_partition_kernel(const uint32_t *__restrict__ ak,
                                                              const LevelDesc *__restrict__ adesc,
                                                              const uint32_t *__restrict__ bk,
                                                              const LevelDesc *__restrict__ bdesc,
                                                              unsigned long long *__restrict__ parts,
                                                              uint32_t max_parts,
                                                              unsigned long long *__restrict__ zero,
                                                              uint32_t zero_words) {
  chain_wait();
  // the merge's ticket counter and look-back slots start at zero
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < zero_words; i += gridDim.x * blockDim.x) zero[i] = 0ull;
  const uint32_t split = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  if (split >= max_parts) return;  // whole warps leave together
  const uint64_t na = adesc->n, nb = bdesc->n, total = na + nb;
  const uint64_t d = min(uint64_t(split) * kMergeTile, total);
  uint64_t lo = d > nb ? d - nb : 0, hi = d < na ? d : na;  // the answer lies in [lo, hi]
  while (hi > lo) {
    const uint64_t span = hi - lo;
    const uint64_t step = span <= 32 ? 1 : (span + 31) / 32;
    const uint64_t k = lo + (uint64_t(lane) + 1) * step - 1;  // probe P(k)
    const bool t = k < hi && ak[k] <= bk[d - 1 - k];
    const uint32_t trues = __popc(__ballot_sync(0xffffffffu, t));  // a prefix of the lanes
    const uint64_t nlo = lo + uint64_t(trues) * step;  // P holds below nlo
    hi = min(hi, nlo + step - 1);                      // and fails at the first false probe
    lo = nlo;
  }
  if (lane == 0) parts[split] = lo;
}

// Shared memory of one merge tile.  The two input slices arrive by bulk
// copies (16-byte aligned chunks, so a slice starts 0-3 keys / 0-15 flags into
// its chunk); after the gather the same arrays stage the output rows at the
// alignment of their global position, for bulk stores of the aligned middle.
struct MergeSmem {
  // A chunk, then B chunk (each at most slice + 6 keys, + 30 flags); the tails
  // leave room for the serial merge's reads past a slice's end (up to
  // kMergeItems + 1 keys past B's slice), whose values it never uses
  uint32_t key[kMergeTile + 32];
  uint32_t val[kMergeTile + 16];
  uint8_t flag[kMergeTile + 80];
  uint16_t src[kMergeTile];       // tile-local source index of each kept row
  uint32_t scan[kMergeThreads / 32];
  uint32_t total;
  uint32_t tile;
  unsigned long long base;
  unsigned long long bar;         // mbarrier of the input copies
};
constexpr size_t kMergeSmemBytes = sizeof(MergeSmem);

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void bulk_store(void *dst, const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// One potentially blocking probe of the phase: the thread is suspended in
// hardware until the phase completes or a time limit of the implementation
// passes (no polling instructions are issued meanwhile).
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the input copies; false (and the status bit) on timeout.
// The probes suspend the waiting warps, so the CTAs that share the SM keep
// its issue slots while the copies are in flight.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t *status) {
  for (uint32_t tries = 0; !mbar_try(bar, 0); ++tries) {
    if (tries > kMaxTryWaits) {
      atomicOr(status, kDevWaitTimeout);
      return false;
    }
  }
  return true;
}

template <bool kDropTombstones>
__global__ void __launch_bounds__(kMergeThreads, 4) merge_kernel(
    const uint32_t *__restrict__ ak, const uint32_t *__restrict__ av, const uint8_t *__restrict__ af,
    const LevelDesc *__restrict__ adesc, const uint32_t *__restrict__ bk,
    const uint32_t *__restrict__ bv, const uint8_t *__restrict__ bf,
    const LevelDesc *__restrict__ bdesc, uint32_t *__restrict__ ok, uint32_t *__restrict__ ov,
    uint8_t *__restrict__ of, LevelDesc *__restrict__ odesc, uint32_t *__restrict__ odir, uint32_t dir_bits,
    uint32_t rows_log2, unsigned long long out_upper, unsigned long long out_capacity,
    const unsigned long long *__restrict__ parts, unsigned long long *__restrict__ lb,
    uint32_t *__restrict__ tile_counter, uint32_t *__restrict__ status, unsigned long long *__restrict__ trace,
    ReceiptSrc rcpt) {
  extern __shared__ __align__(128) unsigned char merge_dyn[];
  MergeSmem &sm = *reinterpret_cast<MergeSmem *>(merge_dyn);
  chain_wait();
  if (threadIdx.x == 0) sm.tile = atomicAdd(tile_counter, 1u);
  // the inputs' descriptors load while the ticket is taken
  LevelDesc da, db;
  da.n = adesc->n;
  da.kmin = adesc->kmin;
  da.kmax = adesc->kmax;
  db.n = bdesc->n;
  db.kmin = bdesc->kmin;
  db.kmax = bdesc->kmax;
  __syncthreads();
  const uint64_t na = da.n, nb = db.n, total = na + nb;
  const uint32_t tile = sm.tile;
  const uint64_t d0 = uint64_t(tile) * kMergeTile;
  if (total == 0) {
    if (tile == 0 && threadIdx.x == 0) write_empty_desc(odesc, odir);
    return;
  }
  if (d0 >= total) return;  // beyond the merged length (grid sized for an upper bound)
  const uint64_t d1 = min(d0 + kMergeTile, total);
  const uint64_t a0 = parts[tile], a1 = parts[tile + 1], b0 = d0 - a0, b1 = d1 - a1;
  const uint32_t alen = uint32_t(a1 - a0), blen = uint32_t(b1 - b0), len = alen + blen;
  // input chunks: [x0 & ~3, (x1 + 3) & ~3) keys/values and [x0 & ~15, (x1 + 15) & ~15)
  // flags; every run buffer's capacity is a multiple of 16 rows, so the
  // rounded-up ends stay inside the allocations
  const uint32_t oa = uint32_t(a0) & 3u, ob = uint32_t(b0) & 3u, fa = uint32_t(a0) & 15u, fb = uint32_t(b0) & 15u;
  const uint32_t la = alen ? uint32_t(((a1 + 3) & ~3ull) - (a0 & ~3ull)) : 0u;
  const uint32_t lbn = blen ? uint32_t(((b1 + 3) & ~3ull) - (b0 & ~3ull)) : 0u;
  const uint32_t fla = alen ? uint32_t(((a1 + 15) & ~15ull) - (a0 & ~15ull)) : 0u;
  const uint32_t flb = blen ? uint32_t(((b1 + 15) & ~15ull) - (b0 & ~15ull)) : 0u;
  const uint32_t bar = smem_addr(&sm.bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    const uint32_t bytes = 8u * (la + lbn) + fla + flb;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
    if (alen) {
      bulk_load(sm.key, ak + (a0 & ~3ull), 4u * la, bar);
      bulk_load(sm.val, av + (a0 & ~3ull), 4u * la, bar);
      bulk_load(sm.flag, af + (a0 & ~15ull), fla, bar);
    }
    if (blen) {
      bulk_load(sm.key + la, bk + (b0 & ~3ull), 4u * lbn, bar);
      bulk_load(sm.val + la, bv + (b0 & ~3ull), 4u * lbn, bar);
      bulk_load(sm.flag + fla, bf + (b0 & ~15ull), flb, bar);
    }
  }
  // while the copies fly: the keys around the tile, the output geometry
  // every output key lies in the union of the inputs' key ranges
  const uint32_t kmin = na == 0 ? db.kmin : nb == 0 ? da.kmin : min(da.kmin, db.kmin);
  const uint32_t kmax = na == 0 ? db.kmax : nb == 0 ? da.kmax : max(da.kmax, db.kmax);
  const DirGeom geom = dir_geometry(kmin, kmax, out_upper, dir_bits, rows_log2);
  // key of the A row just before this tile (shadows a leading B row); the
  // largest key consumed before / by this tile bounds its directory buckets
  const bool has_prev_a = a0 > 0;
  const uint32_t prev_a_global = has_prev_a ? ak[a0 - 1] : 0u;
  const bool has_prev = a0 > 0 || b0 > 0;
  const uint32_t prev_key = max(has_prev_a ? prev_a_global : 0u, b0 > 0 ? bk[b0 - 1] : 0u);
  const uint32_t last_key = max(a1 > 0 ? ak[a1 - 1] : 0u, b1 > 0 ? bk[b1 - 1] : 0u);
  __syncthreads();  // the barrier is initialised before anyone waits on it
  if (!mbar_wait(bar, status)) {
    (void)mbar_wait(bar, status);  // a second bounded wait for copies still in flight
    return;
  }
  const uint32_t *sA = sm.key + oa, *sB = sm.key + la + ob;
  const uint32_t *vA = sm.val + oa, *vB = sm.val + la + ob;
  const uint8_t *gA = sm.flag + fa, *gB = sm.flag + fla + fb;
  // serial merge of this thread's outputs, branch-free: one shared load per
  // output (the new head of the side that advanced).  A head read at or past
  // its slice's end (ai == alen; bi >= blen) is never used: ka only counts
  // while ai < alen, kb only while bi < blen, and items past my_n (where bi
  // may run up to blen + kMergeItems) keep nothing - MergeSmem's padding
  // keeps those reads inside the arrays.
  const uint32_t my_d = min(uint32_t(threadIdx.x) * kMergeItems, len);
  const uint32_t my_n = min(uint32_t(kMergeItems), len - my_d);
  uint32_t ai = merge_path32(sA, alen, sB, blen, my_d);
  uint32_t bi = my_d - ai;
  bool hp = ai > 0 ? true : has_prev_a;
  uint32_t prev = ai > 0 ? sA[ai - 1] : prev_a_global;
  uint32_t ka = sA[ai], kb = sB[bi];
  uint16_t src[kMergeItems];
  uint32_t keep_mask = 0;
#pragma unroll
  for (int i = 0; i < kMergeItems; ++i) {
    const bool ta = ai < alen && (bi >= blen || ka <= kb);
    const uint32_t idx = ta ? ai : alen + bi;
    const bool shadow = !ta && hp && prev == kb;
    bool keep = uint32_t(i) < my_n && !shadow;
    if (kDropTombstones) keep = keep && !(*(ta ? gA + ai : gB + bi) & kFlagTomb);
    hp = hp || ta;
    prev = ta ? ka : prev;
    ai += ta ? 1u : 0u;
    bi += ta ? 0u : 1u;
    const uint32_t nxt = *(ta ? sA + ai : sB + bi);
    ka = ta ? nxt : ka;
    kb = ta ? kb : nxt;
    src[i] = uint16_t(idx);
    keep_mask |= keep ? (1u << i) : 0u;
  }
  uint32_t o = block_exclusive_scan<kMergeThreads>(uint32_t(__popc(keep_mask)), sm.scan, &sm.total);
  const uint32_t tile_kept = sm.total;
  if (threadIdx.x == 0) lookback_publish(lb, tile, tile_kept);  // successors may proceed
#pragma unroll
  for (int i = 0; i < kMergeItems; ++i)
    if (keep_mask & (1u << i)) sm.src[o++] = src[i];
  __syncthreads();
  // gather the kept rows (striped) from the staged inputs; the look-back walk
  // runs after the gathers are issued
  uint32_t rk[kMergeItems], rv[kMergeItems];
  uint8_t rf[kMergeItems];
#pragma unroll
  for (int i = 0; i < kMergeItems; ++i) {
    const uint32_t j = uint32_t(i) * kMergeThreads + threadIdx.x;
    rk[i] = 0;
    rv[i] = 0;
    rf[i] = 0;
    if (j < tile_kept) {
      const uint32_t sidx = sm.src[j];
      const bool in_a = sidx < alen;
      const uint32_t off = in_a ? sidx : sidx - alen;
      rk[i] = (in_a ? sA : sB)[off];
      rv[i] = (in_a ? vA : vB)[off];
      rf[i] = (in_a ? gA : gB)[off];
    }
  }
  if (threadIdx.x < 32) {
    const unsigned long long e = lookback_walk(lb, tile, tile_kept, status);
    if (threadIdx.x == 0) sm.base = e;
  }
  __syncthreads();  // every gather is done: the arrays now stage the output
  const unsigned long long gbase = sm.base;
  const uint32_t o4 = uint32_t(gbase) & 3u, o16 = uint32_t(gbase) & 15u;
#pragma unroll
  for (int i = 0; i < kMergeItems; ++i) {
    const uint32_t j = uint32_t(i) * kMergeThreads + threadIdx.x;
    if (j < tile_kept) {
      sm.key[o4 + j] = rk[i];
      sm.val[o4 + j] = rv[i];
      sm.flag[o16 + j] = rf[i];
    }
  }
  __syncthreads();
  const unsigned long long space = gbase < out_capacity ? out_capacity - gbase : 0ull;
  const uint32_t room = space < tile_kept ? uint32_t(space) : tile_kept;
  // rows [h, h + m) start and end on 16-byte boundaries of the output arrays
  const uint32_t h4 = (4u - o4) & 3u, m4 = room > h4 ? ((room - h4) & ~3u) : 0u;
  const uint32_t h16 = (16u - o16) & 15u, m16 = room > h16 ? ((room - h16) & ~15u) : 0u;
  if (threadIdx.x == 0) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (m4) {
      bulk_store(ok + gbase + h4, sm.key + o4 + h4, 4u * m4);
      bulk_store(ov + gbase + h4, sm.val + o4 + h4, 4u * m4);
    }
    if (m16) bulk_store(of + gbase + h16, sm.flag + o16 + h16, m16);
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
  }
  {  // the unaligned head and tail rows
    const uint32_t t = threadIdx.x;
    if (t < 8) {
      const uint32_t j = t < 4 ? t : h4 + m4 + (t - 4);
      if (j < room && (t < 4 ? j < h4 : true)) {
        ok[gbase + j] = sm.key[o4 + j];
        ov[gbase + j] = sm.val[o4 + j];
      }
    } else if (t >= 32 && t < 64) {
      const uint32_t u = t - 32;
      const uint32_t j = u < 16 ? u : h16 + m16 + (u - 16);
      if (j < room && (u < 16 ? j < h16 : true)) of[gbase + j] = sm.flag[o16 + j];
    }
  }
  // directory entries: row j owns the buckets (bucket(key j-1), bucket(key j)]
  // (the tile's first row starts after the bucket of the key consumed before
  // the tile), as in fill_directory
  const uint32_t gk = geom.kmin, gs = geom.shift;
  const int32_t bp = has_prev ? int32_t((prev_key - gk) >> gs) : -1;
  const uint32_t g0 = uint32_t(gbase);
  const uint32_t *sout = sm.key + o4;
  if (odir) {  // null: the directory is built when a read first needs it
#pragma unroll
    for (int i = 0; i < kMergeItems; ++i) {
      const uint32_t j = uint32_t(i) * kMergeThreads + threadIdx.x;
      // row j - 1 is the previous lane's row of the same item (lane 0: shared memory)
      uint32_t pk = __shfl_up_sync(0xffffffffu, rk[i], 1);
      if ((threadIdx.x & 31u) == 0 && j) pk = sout[j - 1];
      if (j < tile_kept) {
        const int32_t bj = int32_t((rk[i] - gk) >> gs);
        const int32_t bprev = j ? int32_t((pk - gk) >> gs) : bp;
        for (int32_t bb = bprev + 1; bb <= bj; ++bb) odir[bb] = g0 + j;
      }
    }
  }
  const bool last_tile = d1 == total;
  const unsigned long long n_out = gbase + tile_kept;
  if (threadIdx.x == 0) {
    if (odir) {
      const int32_t blast = tile_kept ? int32_t((sout[tile_kept - 1] - gk) >> gs) : bp;
      const int32_t bl = last_tile ? int32_t(geom.nbuckets) - 1 : int32_t((last_key - gk) >> gs);
      for (int32_t bb = blast + 1; bb <= bl; ++bb) odir[bb] = g0 + tile_kept;
      if (last_tile) odir[geom.nbuckets] = uint32_t(n_out < out_capacity ? n_out : out_capacity);
    }
    if (tile == 0) {
      odesc->kmin = geom.kmin;
      odesc->kmax = geom.kmax;
      odesc->shift = geom.shift;
      odesc->nbuckets = geom.nbuckets;
    }
    if (last_tile) {
      if (n_out > out_capacity) atomicOr(status, kDevOutputOverflow);
      odesc->n = n_out < out_capacity ? n_out : out_capacity;
      if (trace) {  // kernel timing: the rows this launch read and wrote
        trace[0] = na;
        trace[1] = nb;
        trace[2] = n_out < out_capacity ? n_out : out_capacity;
        trace[3] = odir ? geom.nbuckets + 1u : 0u;  // directory entries written
      }
    }
    // the staged rows have been read out of shared memory before the CTA
    // retires; the global writes complete with the grid
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
  }
  if (last_tile && rcpt.out && threadIdx.x < 32) write_receipt(rcpt, n_out < out_capacity ? n_out : out_capacity);
}

// ---------------------------------------------------------------------------
// Search helpers over one level.
__device__ __forceinline__ uint32_t bucket_lower_bound(const uint32_t *keys, uint32_t s, uint32_t e,
                                                       uint32_t key) {
  while (e - s > 8) {  // binary search down to a short window
    const uint32_t mid = s + ((e - s) >> 1);
    if (keys[mid] < key) s = mid + 1;
    else e = mid;
  }
  while (s < e && keys[s] < key) ++s;
  return s;
}

// First row with key >= x in the level (n when none).
__device__ __forceinline__ uint64_t level_lower_bound(const LevelView &L, const LevelDesc &d,
                                                      uint32_t x) {
  if (d.n == 0 || x <= d.kmin) return 0;
  if (x > d.kmax) return d.n;
  if (L.ms) {
    // learned: the model's error window, then a check of the answer; a failed
    // check (never expected: the window bounds every key's error) falls back
    // to binary search over the whole level
    learned::ModelHeader h;
    h.n = __ldg(&L.mh->n);
    h.kmin = __ldg(&L.mh->kmin);
    h.kmax = __ldg(&L.mh->kmax);
    h.shift = __ldg(&L.mh->shift);
    h.nseg = __ldg(&L.mh->nseg);
    const uint64_t p = learned::model_lower_bound<uint32_t>(h, L.ms, L.keys, x);
    if (h.n == d.n && (p == 0 || L.keys[p - 1] < x) && (p == d.n || L.keys[p] >= x)) return p;
    return learned::lower_bound_range<uint32_t>(L.keys, 0, d.n, x);
  }
  if (!L.dir) return learned::lower_bound_range<uint32_t>(L.keys, 0, d.n, x);
  const uint32_t b = (x - d.kmin) >> d.shift;
  return bucket_lower_bound(L.keys, L.dir[b], L.dir[b + 1], x);
}

// First row with key > x.
__device__ __forceinline__ uint64_t level_upper_bound(const LevelView &L, const LevelDesc &d,
                                                      uint32_t x) {
  if (d.n == 0 || x < d.kmin) return 0;
  if (x >= d.kmax) return d.n;
  return level_lower_bound(L, d, x + 1u);
}


__device__ __forceinline__ bool row_is_tomb(const LevelView &L, uint64_t p, uint32_t v) {
  return v == kTombValue && (L.flags[p] & kFlagTomb);
}

// ---------------------------------------------------------------------------
// L2 eviction priority for point reads: a level's radix directory (4 B per
// ~8 rows, 32 MB for 2^26 rows) is read by every lookup that reaches the
// level, so its lines are kept (evict_last).  (Marking the key and value
// sectors evict_first as well was measured: it also evicts the sectors of
// Zipf-popular keys and raised DRAM reads from 147 to 186 B per lookup.)
__device__ __forceinline__ uint64_t l2_keep_policy() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint32_t ld_hint(const uint32_t *a, uint64_t policy) {
  uint32_t v;
  asm volatile("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(policy));
  return v;
}

// Point lookup: newest level first; miss value follows GPULSMOpt.cuh:4742-4749.
__device__ __forceinline__ void lookup_one(const LevelSet &set, uint64_t i, const uint32_t *__restrict__ queries,
                                           uint32_t *__restrict__ out_values, uint8_t *__restrict__ out_found) {
  const uint32_t q = queries[i];
  const uint32_t miss = out_found ? 0u : kNotFound;
  const uint64_t keep = l2_keep_policy();
  for (uint32_t l = 0; l < set.count; ++l) {
    const LevelView &L = set.lv[l];
    const LevelDesc d = load_desc(L.desc);
    if (q < d.kmin || q > d.kmax) continue;
    uint64_t p, e;
    uint32_t kp = 0;
    if (L.dir && !L.ms) {  // radix directory: the bucket's rows only
      const uint32_t b = (q - d.kmin) >> d.shift;
      const uint32_t s = ld_hint(L.dir + b, keep);
      e = ld_hint(L.dir + b + 1, keep);
      p = bucket_lower_bound(L.keys, s, uint32_t(e), q);
    } else {  // learned model window or binary search
      p = level_lower_bound(L, d, q);
      e = d.n;
    }
    if (p < e) kp = L.keys[p];
    if (p < e && kp == q) {
      const uint32_t v = L.vals[p];
      const bool live = !row_is_tomb(L, p, v);
      out_values[i] = live ? v : miss;
      if (out_found) out_found[i] = live;
      return;
    }
  }
  out_values[i] = miss;
  if (out_found) out_found[i] = 0u;
}

// Two point lookups per thread with their loads interleaved: each level's
// directory words of both queries are loaded together, then the rows of both
// buckets (up to kProbeRows rows each, independent loads of one to three
// sectors), then the values of the hits - two dependent chains in flight per
// thread instead of one, the same sectors read.  A bucket of more rows (rare:
// a directory bucket holds about 8) takes bucket_lower_bound; a level
// searched by its model or by binary search takes level_lower_bound.  Answers
// equal lookup_one's.  Thread t of a block of B threads takes the queries
// i0 = block * 2B + t and i0 + B (coalesced for both).
constexpr uint32_t kProbeRows = 16;
constexpr uint32_t kLookupPair = 2;

__device__ __forceinline__ void lookup_pair(const LevelSet &set, uint64_t i0, uint64_t n,
                                            const uint32_t *__restrict__ queries, uint32_t *__restrict__ out_values,
                                            uint8_t *__restrict__ out_found) {
  constexpr int Q = int(kLookupPair);
  const uint64_t idx[Q] = {i0, i0 + blockDim.x};
  uint32_t q[Q], val[Q];
  bool done[Q], fnd[Q];
  const uint32_t miss = out_found ? 0u : kNotFound;
#pragma unroll
  for (int j = 0; j < Q; ++j) {
    done[j] = idx[j] >= n;
    q[j] = done[j] ? 0u : queries[idx[j]];
    val[j] = miss;
    fnd[j] = false;
  }
  const uint64_t keep = l2_keep_policy();
  for (uint32_t l = 0; l < set.count; ++l) {
    if (done[0] && done[1]) break;
    const LevelView &L = set.lv[l];
    const LevelDesc d = load_desc(L.desc);
    bool act[Q];
#pragma unroll
    for (int j = 0; j < Q; ++j) act[j] = !done[j] && q[j] >= d.kmin && q[j] <= d.kmax;
    uint32_t p[Q];
    bool hit[Q];
    if (L.dir && !L.ms) {
      uint32_t s[Q], e[Q];
#pragma unroll
      for (int j = 0; j < Q; ++j) {  // the directory words of both queries
        s[j] = e[j] = 0;
        if (act[j]) {
          const uint32_t b = (q[j] - d.kmin) >> d.shift;
          s[j] = ld_hint(L.dir + b, keep);
          e[j] = ld_hint(L.dir + b + 1, keep);
        }
      }
      uint32_t k[Q][kProbeRows];
#pragma unroll
      for (int j = 0; j < Q; ++j)  // the rows of both buckets
#pragma unroll
        for (uint32_t t = 0; t < kProbeRows; ++t)
          k[j][t] = (act[j] && e[j] - s[j] <= kProbeRows && s[j] + t < e[j]) ? L.keys[s[j] + t] : 0u;
#pragma unroll
      for (int j = 0; j < Q; ++j) {
        hit[j] = false;
        p[j] = s[j];
        if (!act[j]) continue;
        if (e[j] - s[j] <= kProbeRows) {
#pragma unroll
          for (uint32_t t = 0; t < kProbeRows; ++t)
            if (s[j] + t < e[j]) {
              p[j] += k[j][t] < q[j] ? 1u : 0u;
              hit[j] = hit[j] || k[j][t] == q[j];
            }
        } else {
          p[j] = uint32_t(bucket_lower_bound(L.keys, s[j], e[j], q[j]));
          hit[j] = p[j] < e[j] && L.keys[p[j]] == q[j];
        }
      }
    } else {  // learned model window or binary search
#pragma unroll
      for (int j = 0; j < Q; ++j) {
        hit[j] = false;
        p[j] = 0;
        if (!act[j]) continue;
        const uint64_t pp = level_lower_bound(L, d, q[j]);
        p[j] = uint32_t(pp);
        hit[j] = pp < d.n && L.keys[pp] == q[j];
      }
    }
    uint32_t v[Q];
#pragma unroll
    for (int j = 0; j < Q; ++j) v[j] = hit[j] ? L.vals[p[j]] : 0u;  // the values of both hits
#pragma unroll
    for (int j = 0; j < Q; ++j)
      if (hit[j]) {
        const bool live = !row_is_tomb(L, p[j], v[j]);
        val[j] = live ? v[j] : miss;
        fnd[j] = live;
        done[j] = true;
      }
  }
#pragma unroll
  for (int j = 0; j < Q; ++j)
    if (idx[j] < n) {
      out_values[idx[j]] = val[j];
      if (out_found) out_found[idx[j]] = fnd[j];
    }
}

// kPair: two queries per thread (directory and learned levels); without it
// one query per thread (binary search, whose long per-query chains gain
// nothing from pairing at the lower occupancy pairing costs).
template <bool kPair>
__global__ void __launch_bounds__(256) lookup_kernel(LevelSet set, const uint32_t *__restrict__ queries,
                                                     uint64_t n, uint32_t *__restrict__ out_values,
                                                     uint8_t *__restrict__ out_found) {
  if (kPair) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x * kLookupPair + threadIdx.x;
    if (i < n) lookup_pair(set, i, n, queries, out_values, out_found);
  } else {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) lookup_one(set, i, queries, out_values, out_found);
  }
}

// The same lookup with the level set read from device memory (a level table
// the dictionary rewrites when its levels change), so that a captured CUDA
// graph stays valid across updates; every block copies the table to shared
// memory first.
template <bool kPair>
__global__ void __launch_bounds__(256) lookup_table_kernel(const LevelSet *__restrict__ table,
                                                           const uint32_t *__restrict__ queries, uint64_t n,
                                                           uint32_t *__restrict__ out_values,
                                                           uint8_t *__restrict__ out_found) {
  __shared__ __align__(16) uint32_t s_words[sizeof(LevelSet) / 4];
  static_assert(sizeof(LevelSet) % 4 == 0, "table copied in words");
  const uint32_t *src = reinterpret_cast<const uint32_t *>(table);
  for (uint32_t w = threadIdx.x; w < sizeof(LevelSet) / 4; w += blockDim.x) s_words[w] = src[w];
  __syncthreads();
  const LevelSet &s_set = *reinterpret_cast<const LevelSet *>(s_words);
  if (kPair) {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x * kLookupPair + threadIdx.x;
    if (i < n) lookup_pair(s_set, i, n, queries, out_values, out_found);
  } else {
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) lookup_one(s_set, i, queries, out_values, out_found);
  }
}

__global__ void write_table_kernel(LevelSet set, LevelSet *__restrict__ table) {
  const uint32_t *src = reinterpret_cast<const uint32_t *>(&set);
  uint32_t *dst = reinterpret_cast<uint32_t *>(table);
  for (uint32_t w = threadIdx.x; w < sizeof(LevelSet) / 4; w += blockDim.x) dst[w] = src[w];
}

// ---------------------------------------------------------------------------
// Range queries over the union of levels with newest-wins, one thread per
// query (k-way cursor merge).  MODE 0: u32 sum (wraps like
// GPULSMOpt.cuh:1520-1605), 1: live count, 2: emit (key, value) pairs at
// offsets[q].
template <int MODE>
__global__ void __launch_bounds__(256) range_kernel(LevelSet set, const uint32_t *__restrict__ lo,
                                                    const uint32_t *__restrict__ hi, uint64_t n,
                                                    uint32_t *__restrict__ out_u32,
                                                    const unsigned long long *__restrict__ offsets,
                                                    uint32_t *__restrict__ out_keys,
                                                    uint32_t *__restrict__ out_vals) {
  const uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const uint32_t a = lo[q], z = hi[q];
  unsigned long long acc = 0;
  unsigned long long o = MODE == 2 ? offsets[q] : 0ull;
  if (a <= z) {
    uint64_t cur[kMaxLevels], end[kMaxLevels];
    const uint32_t L = set.count;
    for (uint32_t l = 0; l < L; ++l) {
      const LevelDesc d = load_desc(set.lv[l].desc);
      cur[l] = level_lower_bound(set.lv[l], d, a);
      end[l] = level_upper_bound(set.lv[l], d, z);
    }
    while (true) {
      uint32_t best = 0xffffffffu;
      int owner = -1;
      for (uint32_t l = 0; l < L; ++l)
        if (cur[l] < end[l]) {
          const uint32_t k = set.lv[l].keys[cur[l]];
          if (owner < 0 || k < best) {
            best = k;
            owner = int(l);
          }
        }
      if (owner < 0) break;
      const uint32_t v = set.lv[owner].vals[cur[owner]];
      const bool live = !row_is_tomb(set.lv[owner], cur[owner], v);
      if (live) {
        if (MODE == 0) acc += v;
        else if (MODE == 1) ++acc;
        else {
          out_keys[o] = best;
          out_vals[o] = v;
          ++o;
        }
      }
      for (uint32_t l = uint32_t(owner); l < L; ++l)
        if (cur[l] < end[l] && set.lv[l].keys[cur[l]] == best) ++cur[l];
    }
  }
  if (MODE != 2) out_u32[q] = uint32_t(acc);
}

// ---------------------------------------------------------------------------
// Range sums over every level without merging them (same answers as
// range_kernel<0>).  Each level's live-value prefix gives the sum of its
// live rows in [lo, hi] in O(1); what it over-counts is every row SHADOWED
// by a newer version of its key.  Each level holds a key at most once, so
// the versions of a key form a chain newest -> oldest over the levels, and
// walking the rows of every level but the oldest, each row subtracts the
// next older version of its key (when that version is live).  The row count
// walked is that of the newer (small) levels only; the search for a row's
// key in an older level gallops forward from the previous row's position.

// First index in [pos, end) whose key is >= k (keys ascending).
__device__ __forceinline__ uint64_t gallop_lower_bound(const uint32_t *__restrict__ keys, uint64_t pos,
                                                       uint64_t end, uint32_t k) {
  if (pos >= end || keys[pos] >= k) return pos;
  uint64_t lo = pos, hi = end, step = 1;  // keys[lo] < k; answer in (lo, hi]
  while (true) {
    const uint64_t probe = lo + step;
    if (probe >= end) break;
    if (keys[probe] >= k) {
      hi = probe;
      break;
    }
    lo = probe;
    step <<= 1;
  }
  while (hi - lo > 1) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (keys[mid] < k) lo = mid;
    else hi = mid;
  }
  return hi;
}

// One query per group of kRangeGroup lanes: lane t searches the bounds of
// levels t, t + kRangeGroup, ... (independent loads instead of one thread's
// chain over every level), the group shares them through shared memory, and
// the lanes split the rows of the newer levels between them: each row finds
// the next older version of its key by a directory search of the older
// levels.  The partial sums (u32, wrapping) meet in a shuffle reduction.
constexpr uint32_t kRangeGroup = 8;
constexpr uint32_t kRangeThreads = 256;

__global__ void __launch_bounds__(kRangeThreads) range_sum_levels_kernel(LevelSet set,
                                                                         const uint32_t *__restrict__ lo,
                                                                         const uint32_t *__restrict__ hi, uint64_t n,
                                                                         uint32_t *__restrict__ out) {
  constexpr uint32_t G = kRangeGroup, kGroups = kRangeThreads / G;
  __shared__ uint64_t s_b[kGroups][kMaxLevels], s_e[kGroups][kMaxLevels];
  const uint32_t grp = threadIdx.x / G, t = threadIdx.x % G;
  const uint64_t q = (uint64_t(blockIdx.x) * kRangeThreads + threadIdx.x) / G;
  const bool valid = q < n;
  const uint32_t a = valid ? lo[q] : 1u, z = valid ? hi[q] : 0u;
  uint32_t acc = 0, has = 0;  // has: levels with rows in [a, z] (bit l = level l of the set)
  if (a <= z)
    for (uint32_t l = t; l < set.count; l += G) {
      const LevelDesc d = load_desc(set.lv[l].desc);
      const uint64_t b = level_lower_bound(set.lv[l], d, a), e = level_upper_bound(set.lv[l], d, z);
      s_b[grp][l] = b;
      s_e[grp][l] = e;
      if (e > b) {
        acc += set.lv[l].live[e] - set.lv[l].live[b];
        has |= 1u << l;
      }
    }
  // the group's lanes are consecutive lanes of one warp
  const uint32_t gmask = ((1u << G) - 1u) << ((threadIdx.x & 31u) & ~(G - 1u));
#pragma unroll
  for (uint32_t o = 1; o < G; o <<= 1) has |= __shfl_xor_sync(gmask, has, o, G);
  __syncwarp(gmask);  // the group's bounds are in shared memory
  // every row of a level but the oldest with rows subtracts the next older
  // version of its key, when that version is live
  const uint32_t oldest = has ? 31u - __clz(has) : 0u;
  for (uint32_t rest = has & ~(1u << oldest); rest; rest &= rest - 1u) {
    const uint32_t i = __ffs(rest) - 1u;
    const LevelView &N = set.lv[i];
    for (uint64_t r = s_b[grp][i] + t; r < s_e[grp][i]; r += G) {
      const uint32_t k = N.keys[r];
      for (uint32_t older = has & ~((2u << i) - 1u); older; older &= older - 1u) {
        const uint32_t j = __ffs(older) - 1u;
        const LevelView &O = set.lv[j];
        const uint64_t p = level_lower_bound(O, load_desc(O.desc), k);
        if (p < s_e[grp][j] && O.keys[p] == k) {
          const uint32_t v = O.vals[p];
          if (!row_is_tomb(O, p, v)) acc -= v;
          break;
        }
      }
    }
  }
#pragma unroll
  for (uint32_t o = 1; o < G; o <<= 1) acc += __shfl_xor_sync(gmask, acc, o, G);
  if (valid && t == 0) out[q] = acc;
}

// ---------------------------------------------------------------------------
// Ranges over ONE tombstone-free level (after a compaction): the answer of a
// query is the contiguous row slice [lower_bound(lo), upper_bound(hi)).

// sum over queries of the covered key width (decides whether to compact)
__global__ void __launch_bounds__(256) range_width_kernel(const uint32_t *__restrict__ lo,
                                                          const uint32_t *__restrict__ hi, uint64_t n,
                                                          unsigned long long *__restrict__ total) {
  unsigned long long w = 0;
  for (uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; q < n; q += uint64_t(gridDim.x) * blockDim.x)
    if (lo[q] <= hi[q]) w += (unsigned long long)(hi[q] - lo[q]) + 1ull;
#pragma unroll
  for (int o = 16; o; o >>= 1) w += __shfl_down_sync(0xffffffffu, w, o);
  if ((threadIdx.x & 31) == 0 && w) atomicAdd(total, w);
}

// MODE 1: live count (u32), MODE 0: u32 sum from the level's value prefix P
template <int MODE>
__global__ void __launch_bounds__(256) single_level_range_kernel(
    LevelView L, const uint32_t *__restrict__ lo, const uint32_t *__restrict__ hi, uint64_t n,
    const unsigned long long *__restrict__ prefix, uint32_t *__restrict__ out) {
  const uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const uint32_t a = lo[q], z = hi[q];
  uint32_t r = 0;
  if (a <= z) {
    const LevelDesc d = load_desc(L.desc);
    const uint64_t b = level_lower_bound(L, d, a), e = level_upper_bound(L, d, z);
    if (e > b) r = MODE == 1 ? uint32_t(e - b) : uint32_t(prefix[e] - prefix[b]);
  }
  out[q] = r;
}

// pairs: warps take groups of 32 queries from a counter (a slice may hold
// tens of thousands of rows, so a fixed share per warp would leave a long
// tail).  Every lane finds the row slice of one query of the group (the 32
// searches overlap), a lane whose slice is short copies it alone, then the
// warp copies each longer slice together (coalesced, 8 rows in flight per
// lane).  counter starts at zero.
constexpr uint32_t kPairsShort = 8;  // rows a lane copies alone
constexpr uint32_t kPairsGroup = 32;

__global__ void __launch_bounds__(256) single_level_pairs_kernel(
    LevelView L, const uint32_t *__restrict__ lo, const uint32_t *__restrict__ hi, uint64_t n,
    const unsigned long long *__restrict__ offsets, uint32_t *__restrict__ out_keys,
    uint32_t *__restrict__ out_vals, uint32_t *__restrict__ counter) {
  const uint32_t lane = threadIdx.x & 31;
  const LevelDesc d = load_desc(L.desc);
  const uint32_t *__restrict__ keys = L.keys;
  const uint32_t *__restrict__ vals = L.vals;
  const uint64_t groups = (n + kPairsGroup - 1) / kPairsGroup;
  for (;;) {
    uint32_t grp = 0;
    if (lane == 0) grp = atomicAdd(counter, 1u);
    grp = __shfl_sync(0xffffffffu, grp, 0);
    if (grp >= groups) break;  // uniform across the warp
    const uint64_t q = uint64_t(grp) * kPairsGroup + lane;
    uint64_t b = 0, len = 0, o = 0;
    if (q < n) {
      const uint32_t a = lo[q], z = hi[q];
      o = offsets[q];
      if (a <= z) {
        b = level_lower_bound(L, d, a);
        const uint64_t e = level_upper_bound(L, d, z);
        len = e > b ? e - b : 0;
      }
    }
    if (len <= kPairsShort) {
      uint32_t k[kPairsShort], v[kPairsShort];
#pragma unroll
      for (uint32_t i = 0; i < kPairsShort; ++i)
        if (i < len) {
          k[i] = keys[b + i];
          v[i] = vals[b + i];
        }
#pragma unroll
      for (uint32_t i = 0; i < kPairsShort; ++i)
        if (i < len) {
          out_keys[o + i] = k[i];
          out_vals[o + i] = v[i];
        }
    }
    for (uint32_t longs = __ballot_sync(0xffffffffu, len > kPairsShort); longs; longs &= longs - 1) {
      const int src = __ffs(longs) - 1;
      const uint64_t sb = __shfl_sync(0xffffffffu, b, src), so = __shfl_sync(0xffffffffu, o, src);
      const uint64_t sl = __shfl_sync(0xffffffffu, len, src);
      uint64_t j = lane;
      for (; j + 224 < sl; j += 256) {
        uint32_t k[8], v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          k[u] = keys[sb + j + 32 * u];
          v[u] = vals[sb + j + 32 * u];
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          out_keys[so + j + 32 * u] = k[u];
          out_vals[so + j + 32 * u] = v[u];
        }
      }
      for (; j < sl; j += 32) {
        out_keys[so + j] = keys[sb + j];
        out_vals[so + j] = vals[sb + j];
      }
    }
  }
}

// Successor: smallest live key >= query, else 0xffffffff (GPULSMOpt.cuh:5566-5594).
__global__ void __launch_bounds__(256) successor_kernel(LevelSet set, const uint32_t *__restrict__ queries,
                                                        uint64_t n, uint32_t *__restrict__ out_keys) {
  const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t x = queries[i];
  uint64_t cur[kMaxLevels], end[kMaxLevels];
  const uint32_t L = set.count;
  for (uint32_t l = 0; l < L; ++l) {
    const LevelDesc d = load_desc(set.lv[l].desc);
    cur[l] = level_lower_bound(set.lv[l], d, x);
    end[l] = d.n;
  }
  uint32_t result = kNotFound;
  while (true) {
    uint32_t best = 0xffffffffu;
    int owner = -1;
    for (uint32_t l = 0; l < L; ++l)
      if (cur[l] < end[l]) {
        const uint32_t k = set.lv[l].keys[cur[l]];
        if (owner < 0 || k < best) {
          best = k;
          owner = int(l);
        }
      }
    if (owner < 0) break;
    const uint32_t v = set.lv[owner].vals[cur[owner]];
    if (!row_is_tomb(set.lv[owner], cur[owner], v)) {
      result = best;
      break;
    }
    for (uint32_t l = uint32_t(owner); l < L; ++l)
      if (cur[l] < end[l] && set.lv[l].keys[cur[l]] == best) ++cur[l];
  }
  out_keys[i] = result;
}

// ---------------------------------------------------------------------------
// Exclusive scan of u32 inputs into offsets (offsets[n] = total), single
// pass with decoupled look-back.  kLive: the inputs are a level's values and
// a tombstone row (value kTombValue with the flag bit) counts as 0, which
// gives the level's live-value prefix; OutT = u32 keeps it modulo 2^32, the
// width of a range sum.
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

template <typename OutT, bool kLive>
__global__ void __launch_bounds__(kScanThreads) scan_kernel(
    const uint32_t *__restrict__ in, const uint8_t *__restrict__ flags, uint64_t n,
    OutT *__restrict__ offsets, unsigned long long *__restrict__ lb, uint32_t *__restrict__ tile_counter,
    uint32_t *__restrict__ status) {
  __shared__ unsigned long long s_scan[kScanThreads / 32];
  __shared__ unsigned long long s_total;
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_base;
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t base = uint64_t(tile) * kScanTile + uint64_t(threadIdx.x) * kScanItems;
  uint32_t c[kScanItems];
  unsigned long long sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    c[i] = base + i < n ? in[base + i] : 0u;
    if (kLive && c[i] == kTombValue && base + i < n && (flags[base + i] & kFlagTomb)) c[i] = 0u;
    sum += c[i];
  }
  const unsigned long long local = block_exclusive_scan<kScanThreads>(sum, s_scan, &s_total);
  if (threadIdx.x < 32) {
    const unsigned long long lb_excl = warp_lookback(lb, tile, s_total, status);
    if (threadIdx.x == 0) s_base = lb_excl;
  }
  __syncthreads();
  unsigned long long o = s_base + local;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i <= n) offsets[base + i] = OutT(o);  // index n receives the total
    o += c[i];
  }
}
// Tiles needed so that index n (the total) is covered.
inline uint32_t scan_tiles(uint64_t n) { return uint32_t(n / kScanTile + 1); }

}  // namespace lsm
}  // namespace gpulsm
