// Kernels of the FliX-style bucket layer (32- or 64-bit keys, u32 values).
//
// HBM layout.  A node is one 16-byte aligned record:
//   keys[32]  sorted ascending in slots [0, count)
//   vals[32]  u32 value of each key (FliX "offset")
//   max       largest key this node covers: node i of a chain covers
//             (previous node's max, max]; the last node of bucket b covers up
//             to bmax[b]
//   count     live entries
//   next      index of the next node of the chain, kNone at the end
// Node<u64> is 400 bytes, the stride of FliX's node_size 32 layout
// (FliX/definitions_updates.cuh:259-329); a warp loads the 32 keys of a node
// with one coalesced 256-byte read (lane j holds slot j).
// nodes[0, B) are the bucket heads in key order; nodes[B, cap) form the
// allocation region for split nodes (FliX/tile_utils.cuh:306-392).
// bmax[b] is the fixed upper key of bucket b (FliX maxvalues,
// FliX/impl_cg_rtx_index_updates.cuh:208-238); bucket b covers
// (bmax[b-1], bmax[b]] and bmax[B-1] is the largest key value.
//
// Every update/query batch is sorted first; a batch is split into runs of
// keys that fall into the same bucket and ONE warp owns a run, so a chain is
// only ever touched by one warp (the tile-per-bucket rule of
// FliX/coarse_granular_inserts_tiles.cuh:571-643) - no locks, no atomics on
// nodes.
#pragma once

#include "common.cuh"
#include "learned.cuh"

namespace gpulsm {
namespace flix {

constexpr uint32_t kNodeSize = 32;
constexpr uint32_t kNone = 0xffffffffu;

template <typename K>
struct alignas(16) Node {
  K keys[kNodeSize];
  uint32_t vals[kNodeSize];
  K max;
  uint32_t count;
  uint32_t next;
};
static_assert(sizeof(Node<unsigned long long>) == 400, "u64 node stride");

template <typename K>
__host__ __device__ constexpr K key_max() {
  return ~K(0);
}

// not_found cast to the key type (FliX/coarse_granular_lookups_tile_bulk.cuh:672,917,946)
template <typename K>
__host__ __device__ constexpr K successor_miss() {
  return K(0xffffffffu);
}

struct Run {
  uint32_t bucket;
  uint32_t start;
};

struct PoolView {
  uint32_t *alloc_top;   // next free node index (bump)
  uint32_t capacity;     // total nodes (heads + region)
  uint32_t *status;
};

// ---------------------------------------------------------------------------
// build: lay sorted unique (key, value) pairs into bucket heads at `fill`
// entries per node (FliX/impl_cg_rtx_index_updates.cuh:443-528).
template <typename K>
__global__ void build_layout_kernel(const K *__restrict__ keys, const uint32_t *__restrict__ vals,
                                    uint64_t n, uint32_t fill, uint32_t buckets,
                                    Node<K> *__restrict__ nodes, K *__restrict__ bmax) {
  const uint32_t lane = threadIdx.x & 31;
  const uint64_t b = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (b >= buckets) return;
  Node<K> *node = nodes + b;
  const uint64_t first = b * fill;
  const uint64_t idx = first + lane;
  const bool has = lane < fill && idx < n;
  node->keys[lane] = has ? keys[idx] : K(0);
  node->vals[lane] = has ? (vals ? vals[idx] : uint32_t(idx)) : 0u;
  if (lane == 0) {
    const uint64_t end = first + fill < n ? first + fill : n;
    const uint32_t count = first < n ? uint32_t(end - first) : 0u;
    const K mx = (b + 1 == buckets) ? key_max<K>() : keys[end - 1];
    node->max = mx;
    node->count = count;
    node->next = kNone;
    bmax[b] = mx;
  }
}

// ---------------------------------------------------------------------------
// bucket of a key: first b with bmax[b] >= key
template <typename K>
__device__ __forceinline__ uint32_t bucket_of(const K *__restrict__ bmax, uint32_t buckets, K key) {
  uint32_t lo = 0, hi = buckets - 1;  // bmax[buckets-1] is key_max, always >= key
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (bmax[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

template <typename K>
__device__ __forceinline__ uint32_t bucket_in(const K *__restrict__ bmax, uint32_t lo, uint32_t hi, K key) {
  while (lo < hi) {  // first bucket in [lo, hi] whose maximum is >= key
    const uint32_t mid = (lo + hi) >> 1;
    if (bmax[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Same answer through the learned model fitted on bmax[0, buckets-1): the
// model narrows the search to its error window (learned.cuh); keys above
// bmax[buckets-2] fall into the last bucket.
template <typename K>
__device__ __forceinline__ uint32_t bucket_of_model(const learned::ModelHeader &h, const learned::Segment *seg,
                                                    const K *__restrict__ bmax, K key) {
  return uint32_t(learned::model_lower_bound<K>(h, seg, bmax, key));
}

// Routes a sorted key list to buckets and emits one Run per maximal group of
// consecutive keys in the same bucket (compacted with decoupled look-back).
constexpr int kRouteThreads = 256;
constexpr int kRouteItems = 8;
constexpr uint32_t kRouteTile = kRouteThreads * kRouteItems;


template <typename K>
__global__ void __launch_bounds__(kRouteThreads) route_runs_kernel(
    const K *__restrict__ keys, const uint32_t *__restrict__ n_ptr, const K *__restrict__ bmax,
    uint32_t buckets, Run *__restrict__ runs, uint32_t *__restrict__ run_count,
    unsigned long long *__restrict__ lb, uint32_t *__restrict__ tile_counter,
    uint32_t *__restrict__ status, const learned::ModelHeader *__restrict__ model,
    const learned::Segment *__restrict__ segs) {
  const uint32_t n = *n_ptr;
  learned::ModelHeader mh{};
  if (model) mh = *model;
  auto route = [&](K key) -> uint32_t {
    return model ? bucket_of_model<K>(mh, segs, bmax, key) : bucket_of(bmax, buckets, key);
  };
  __shared__ uint32_t s_scan[kRouteThreads / 32];
  __shared__ uint32_t s_total;
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_base;
  __shared__ uint32_t s_prev_bucket;
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t base = uint64_t(tile) * kRouteTile;
  if (base >= n && !(tile == 0 && n == 0)) return;  // grid sized for an upper bound
  if (threadIdx.x == 0)
    s_prev_bucket = (base > 0 && base <= n) ? route(keys[base - 1]) : kNone;
  __syncthreads();
  const uint64_t mine = base + uint64_t(threadIdx.x) * kRouteItems;
  uint32_t bk[kRouteItems];
  uint32_t starts = 0, cnt = 0;
  K kk[kRouteItems];
#pragma unroll
  for (int i = 0; i < kRouteItems; ++i) kk[i] = mine + i < n ? keys[mine + i] : K(0);
  if (model) {
#pragma unroll
    for (int i = 0; i < kRouteItems; ++i) bk[i] = mine + i < n ? route(kk[i]) : kNone;
  } else {
    // the keys are sorted: the warp's first and last key take a full search,
    // every other key searches only the buckets between theirs (a key outside
    // that interval - unsorted input - searches everything)
    const uint32_t lane = threadIdx.x & 31u;
    const bool any = mine < n;
    const uint64_t left = any ? uint64_t(n) - mine : 0ull;
    const uint32_t nv = left < uint64_t(kRouteItems) ? uint32_t(left) : uint32_t(kRouteItems);
    const uint32_t vmask = __ballot_sync(0xffffffffu, any);
    uint32_t blo = 0, bhi = buckets - 1;
    K kf = 0, kl = 0;
    if (vmask) {
      const uint32_t fl = __ffs(vmask) - 1, ll = 31u - __clz(vmask);
      kf = __shfl_sync(0xffffffffu, kk[0], fl);
      K mylast = kk[0];
#pragma unroll
      for (int i = 1; i < kRouteItems; ++i)
        if (uint32_t(i) < nv) mylast = kk[i];
      kl = __shfl_sync(0xffffffffu, mylast, ll);
      // (one lane may hold both the first and the last key)
      const uint32_t bf = lane == fl ? bucket_in(bmax, 0u, buckets - 1, kf) : 0u;
      const uint32_t bl = lane == ll ? bucket_in(bmax, 0u, buckets - 1, kl) : 0u;
      blo = __shfl_sync(0xffffffffu, bf, fl);
      bhi = __shfl_sync(0xffffffffu, bl, ll);
    }
#pragma unroll
    for (int i = 0; i < kRouteItems; ++i) {
      const K k = kk[i];
      bk[i] = uint32_t(i) < nv ? ((kf <= k && k <= kl) ? bucket_in(bmax, blo, bhi, k) : bucket_in(bmax, 0u, buckets - 1, k))
                               : kNone;
    }
  }
  // previous key's bucket for item 0 of this thread
  uint32_t prev = __shfl_up_sync(0xffffffffu, bk[kRouteItems - 1], 1);
  if ((threadIdx.x & 31) == 0) prev = kNone;
  __shared__ uint32_t s_last[kRouteThreads / 32];
  if ((threadIdx.x & 31) == 31) s_last[threadIdx.x >> 5] = bk[kRouteItems - 1];
  __syncthreads();
  if ((threadIdx.x & 31) == 0) prev = (threadIdx.x == 0) ? s_prev_bucket : s_last[(threadIdx.x >> 5) - 1];
#pragma unroll
  for (int i = 0; i < kRouteItems; ++i) {
    const uint64_t g = mine + i;
    const uint32_t p = i == 0 ? prev : bk[i - 1];
    if (g < n && bk[i] != p) {
      starts |= 1u << i;
      ++cnt;
    }
  }
  const uint32_t local = block_exclusive_scan<kRouteThreads>(cnt, s_scan, &s_total);
  if (threadIdx.x < 32) {
    const unsigned long long lb_excl = warp_lookback(lb, tile, s_total, status);
    if (threadIdx.x == 0) s_base = lb_excl;
  }
  __syncthreads();
  uint64_t o = s_base + local;
#pragma unroll
  for (int i = 0; i < kRouteItems; ++i)
    if (starts & (1u << i)) {
      if (o < n) runs[o] = Run{bk[i], uint32_t(mine + i)};  // o < n unless a wait timed out
      ++o;
    }
  if (base + kRouteTile >= n && threadIdx.x == 0) *run_count = uint32_t(min(s_base + s_total, (unsigned long long)n));
}

// ---------------------------------------------------------------------------
// Warp-resident node: lane j holds slot j.
template <typename K>
struct WarpNode {
  uint32_t id;
  K key;
  uint32_t val;
  K max;
  uint32_t count;
  uint32_t next;
};

template <typename K>
__device__ __forceinline__ void load_node(const Node<K> *nodes, uint32_t id, uint32_t lane,
                                          WarpNode<K> &w) {
  const Node<K> *p = nodes + id;
  w.id = id;
  w.key = p->keys[lane];
  w.val = p->vals[lane];
  w.max = p->max;
  w.count = p->count;
  w.next = p->next;
}

template <typename K>
__device__ __forceinline__ void store_node(Node<K> *nodes, uint32_t lane, const WarpNode<K> &w) {
  Node<K> *p = nodes + w.id;
  if (lane < w.count) {
    p->keys[lane] = w.key;
    p->vals[lane] = w.val;
  }
  if (lane == 0) {
    p->count = w.count;
    p->max = w.max;
    p->next = w.next;
  }
}

__device__ __forceinline__ uint32_t run_end(const Run *runs, uint32_t r, uint32_t run_count, uint32_t n) {
  return r + 1 < run_count ? runs[r + 1].start : n;
}

// Update kernels run persistent warps: warp w takes runs w, w + W, ... (W =
// warps in the grid), so the launch size does not depend on the run count
// (known only on the device) and each warp adds its count to the global
// counter once.  A run's first 32 keys (and values) are loaded by the lanes
// together with the head node, and consumed by shuffles, so a multi-key run
// does not wait on one global load per key.
constexpr uint32_t kUpdateThreads = 256;

// Insert if absent (FliX/coarse_granular_inserts_tiles_bulk.cuh:1307-1602):
// the run's keys are sorted and unique; an existing key keeps its value.  A
// full node splits: the lower half keeps 16 entries, the upper half moves to
// a fresh node linked after it (FliX/tile_utils.cuh:306-392).  An exhausted
// allocation region sets kDevOutputOverflow and the key is reported, not
// silently dropped.
template <typename K>
__global__ void __launch_bounds__(kUpdateThreads) insert_runs_kernel(
    const K *__restrict__ keys, const uint32_t *__restrict__ vals, const uint32_t *__restrict__ n_ptr,
    const Run *__restrict__ runs, const uint32_t *__restrict__ run_count_ptr, Node<K> *nodes,
    PoolView pool, unsigned long long *__restrict__ inserted) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n = *n_ptr;
  const uint32_t run_count = *run_count_ptr;
  const uint32_t stride = gridDim.x * (kUpdateThreads / 32);
  uint32_t added = 0;
  uint32_t r = (blockIdx.x * kUpdateThreads + threadIdx.x) >> 5;
  Run next_run = r < run_count ? runs[r] : Run{};
  uint32_t next_end = r < run_count ? run_end(runs, r, run_count, n) : 0u;
  for (; r < run_count; r += stride) {
    const Run run = next_run;
    const uint32_t end = next_end;
    if (r + stride < run_count) {  // the next run's bounds load while this one is processed
      next_run = runs[r + stride];
      next_end = run_end(runs, r + stride, run_count, n);
    }
    K kreg = 0;
    uint32_t vreg = 0;
    if (run.start + lane < end) {
      kreg = keys[run.start + lane];
      vreg = vals[run.start + lane];
    }
    WarpNode<K> w;
    load_node(nodes, run.bucket, lane, w);
    bool dirty = false;
    for (uint32_t i = run.start; i < end; ++i) {
      const uint32_t slot = (i - run.start) & 31u;
      if (slot == 0 && i != run.start) {  // next 32 keys of a long run
        kreg = i + lane < end ? keys[i + lane] : K(0);
        vreg = i + lane < end ? vals[i + lane] : 0u;
      }
      const K k = __shfl_sync(0xffffffffu, kreg, slot);
      const uint32_t v = __shfl_sync(0xffffffffu, vreg, slot);
      while (k > w.max && w.next != kNone) {
        if (dirty) store_node(nodes, lane, w);
        dirty = false;
        load_node(nodes, w.next, lane, w);
      }
      if (k > w.max) {  // chain ends below the key: broken invariant, report and skip
        if (lane == 0) atomicOr(pool.status, kDevBadInput);
        continue;
      }
      if (__ballot_sync(0xffffffffu, lane < w.count && w.key == k)) continue;  // present: keep
      if (w.count == kNodeSize) {
        uint32_t fresh = 0;
        if (lane == 0) fresh = atomicAdd(pool.alloc_top, 1u);
        fresh = __shfl_sync(0xffffffffu, fresh, 0);
        if (fresh >= pool.capacity) {
          if (lane == 0) atomicOr(pool.status, kDevOutputOverflow);
          continue;
        }
        constexpr uint32_t half = kNodeSize / 2;
        const K lower_max = __shfl_sync(0xffffffffu, w.key, half - 1);
        // upper half -> fresh node (slots 0..15)
        WarpNode<K> up;
        up.id = fresh;
        up.key = __shfl_down_sync(0xffffffffu, w.key, half);
        up.val = __shfl_down_sync(0xffffffffu, w.val, half);
        up.max = w.max;
        up.count = kNodeSize - half;
        up.next = w.next;
        w.max = lower_max;
        w.count = half;
        w.next = fresh;
        if (k > lower_max) {
          store_node(nodes, lane, w);
          w = up;
        } else {
          store_node(nodes, lane, up);
        }
        dirty = true;
      }
      const uint32_t pos = __popc(__ballot_sync(0xffffffffu, lane < w.count && w.key < k));
      const K sk = __shfl_up_sync(0xffffffffu, w.key, 1);
      const uint32_t sv = __shfl_up_sync(0xffffffffu, w.val, 1);
      if (lane > pos && lane <= w.count) {
        w.key = sk;
        w.val = sv;
      }
      if (lane == pos) {
        w.key = k;
        w.val = v;
      }
      ++w.count;
      ++added;
      dirty = true;
    }
    if (dirty) store_node(nodes, lane, w);
  }
  if (lane == 0 && added) atomicAdd(inserted, (unsigned long long)added);
}

// Physical delete (FliX/coarse_granular_deletes_tiles.cuh:1128-1320): matches
// are removed and survivors compacted left; an emptied non-head node is
// unlinked from its chain (its range passes to its neighbour).
template <typename K>
__global__ void __launch_bounds__(kUpdateThreads) delete_runs_kernel(
    const K *__restrict__ keys, const uint32_t *__restrict__ n_ptr, const Run *__restrict__ runs,
    const uint32_t *__restrict__ run_count_ptr, Node<K> *nodes,
    unsigned long long *__restrict__ removed) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n = *n_ptr;
  const uint32_t run_count = *run_count_ptr;
  const uint32_t stride = gridDim.x * (kUpdateThreads / 32);
  uint32_t gone = 0;
  uint32_t r = (blockIdx.x * kUpdateThreads + threadIdx.x) >> 5;
  Run next_run = r < run_count ? runs[r] : Run{};
  uint32_t next_end = r < run_count ? run_end(runs, r, run_count, n) : 0u;
  for (; r < run_count; r += stride) {
    const Run run = next_run;
    const uint32_t end = next_end;
    if (r + stride < run_count) {  // the next run's bounds load while this one is processed
      next_run = runs[r + stride];
      next_end = run_end(runs, r + stride, run_count, n);
    }
    K kreg = run.start + lane < end ? keys[run.start + lane] : K(0);
    WarpNode<K> w;
    load_node(nodes, run.bucket, lane, w);
    uint32_t prev = kNone;
    bool dirty = false;
    auto flush = [&]() {
      if (!dirty) return;
      if (w.count == 0 && prev != kNone) {
        // unlink the emptied node; the predecessor inherits its key range
        if (lane == 0) {
          nodes[prev].next = w.next;
          if (w.next == kNone) nodes[prev].max = w.max;
        }
      } else {
        store_node(nodes, lane, w);
      }
      dirty = false;
    };
    for (uint32_t i = run.start; i < end; ++i) {
      const uint32_t slot = (i - run.start) & 31u;
      if (slot == 0 && i != run.start) kreg = i + lane < end ? keys[i + lane] : K(0);
      const K k = __shfl_sync(0xffffffffu, kreg, slot);
      while (k > w.max && w.next != kNone) {
        const bool unlinked = dirty && w.count == 0 && prev != kNone;
        flush();
        if (!unlinked) prev = w.id;
        load_node(nodes, w.next, lane, w);
      }
      const uint32_t match = __ballot_sync(0xffffffffu, lane < w.count && w.key == k);
      if (!match) continue;
      const uint32_t p = __ffs(match) - 1;
      const K sk = __shfl_down_sync(0xffffffffu, w.key, 1);
      const uint32_t sv = __shfl_down_sync(0xffffffffu, w.val, 1);
      if (lane >= p && lane + 1 < w.count) {
        w.key = sk;
        w.val = sv;
      }
      --w.count;
      ++gone;
      dirty = true;
    }
    flush();
  }
  if (lane == 0 && gone) atomicAdd(removed, (unsigned long long)gone);
}

// Ordered lookup (FliX/coarse_granular_lookups_tile_bulk.cuh:312-470): value
// or not_found per probe; results go to out[perm ? perm[i] : i].
template <typename K>
__global__ void __launch_bounds__(256) lookup_runs_kernel(
    const K *__restrict__ probes, const uint32_t *__restrict__ n_ptr, const Run *__restrict__ runs,
    const uint32_t *__restrict__ run_count_ptr, const Node<K> *__restrict__ nodes,
    const uint32_t *__restrict__ perm, uint32_t *__restrict__ out) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n = *n_ptr;
  const uint32_t r = (uint32_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const uint32_t run_count = *run_count_ptr;
  if (r >= run_count) return;
  const Run run = runs[r];
  const uint32_t end = run_end(runs, r, run_count, n);
  WarpNode<K> w;
  load_node(nodes, run.bucket, lane, w);
  for (uint32_t base = run.start; base < end; base += 32) {
    // lanes take 32 consecutive probes; the node walk is shared (probes sorted)
    const uint32_t i = base + lane;
    const K k = i < end ? probes[i] : K(0);
    uint32_t result = kNotFound;
    uint32_t pending = __ballot_sync(0xffffffffu, i < end);
    while (pending) {
      // lanes whose probe is covered by the current node resolve now
      const bool here = (pending >> lane & 1u) && k <= w.max;
      uint32_t todo = __ballot_sync(0xffffffffu, here);
      while (todo) {
        const uint32_t src = __ffs(todo) - 1;
        const K kk = __shfl_sync(0xffffffffu, k, src);
        const uint32_t m = __ballot_sync(0xffffffffu, lane < w.count && w.key == kk);
        const uint32_t v = __shfl_sync(0xffffffffu, w.val, m ? __ffs(m) - 1 : 0);
        if (lane == src) result = m ? v : kNotFound;
        todo &= todo - 1;
      }
      pending &= ~__ballot_sync(0xffffffffu, here);
      if (pending && w.next == kNone) break;  // chain covers every routed probe; defensive
      if (pending) load_node(nodes, w.next, lane, w);
    }
    if (i < end) out[perm ? perm[i] : i] = result;
  }
}

// First stored key >= k in bucket b or any later bucket.
template <typename K>
__device__ K first_key_from_bucket(const Node<K> *nodes, uint32_t b, uint32_t buckets) {
  for (; b < buckets; ++b) {
    uint32_t id = b;
    while (id != kNone) {
      const Node<K> *p = nodes + id;
      if (p->count) return p->keys[0];
      id = p->next;
    }
  }
  return successor_miss<K>();
}

// Ordered successor (FliX/coarse_granular_lookups_tile_bulk.cuh:630-972).
template <typename K>
__global__ void __launch_bounds__(256) successor_runs_kernel(
    const K *__restrict__ probes, const uint32_t *__restrict__ n_ptr, const Run *__restrict__ runs,
    const uint32_t *__restrict__ run_count_ptr, const Node<K> *__restrict__ nodes,
    uint32_t buckets, const uint32_t *__restrict__ perm, K *__restrict__ out) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t n = *n_ptr;
  const uint32_t r = (uint32_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const uint32_t run_count = *run_count_ptr;
  if (r >= run_count) return;
  const Run run = runs[r];
  const uint32_t end = run_end(runs, r, run_count, n);
  WarpNode<K> w;
  load_node(nodes, run.bucket, lane, w);
  bool next_known = false;
  K next_first = successor_miss<K>();
  bool chain_done = false;
  for (uint32_t i = run.start; i < end; ++i) {
    const K k = probes[i];
    K result;
    while (true) {
      if (!chain_done) {
        while (k > w.max && w.next != kNone) load_node(nodes, w.next, lane, w);
        const uint32_t c = __ballot_sync(0xffffffffu, lane < w.count && w.key >= k);
        if (c) {
          result = __shfl_sync(0xffffffffu, w.key, __ffs(c) - 1);
          break;
        }
        if (w.next != kNone) {
          load_node(nodes, w.next, lane, w);
          continue;
        }
        chain_done = true;  // nothing >= k left in this bucket
      }
      if (!next_known) {
        if (lane == 0) next_first = first_key_from_bucket(nodes, run.bucket + 1, buckets);
        next_first = __shfl_sync(0xffffffffu, next_first, 0);
        next_known = true;
      }
      result = next_first;
      break;
    }
    if (lane == 0) out[perm ? perm[i] : i] = result;
  }
}

// ---------------------------------------------------------------------------
// Thread-per-probe queries over SORTED probes (ordered lookup / successor).
// A warp-per-bucket walk reads a whole node (keys, values, header) for each
// probe when probes are spread over many buckets; here every thread routes its
// own probe and reads only the node header and the keys its binary search
// touches.  Plain routing narrows each lane's binary search over the bucket
// maxima to the bucket range spanned by its warp's (sorted) probes; learned
// routing uses the model's error window.

template <typename K>
__device__ __forceinline__ uint32_t route_sorted(const K *__restrict__ bmax, uint32_t buckets,
                                                 const learned::ModelHeader *model, const learned::Segment *segs,
                                                 K k, bool valid) {
  if (model) {
    const learned::ModelHeader h = *model;
    return valid ? bucket_of_model<K>(h, segs, bmax, k) : 0u;
  }
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t vmask = __ballot_sync(0xffffffffu, valid);
  if (!vmask) return 0u;
  const uint32_t first = __ffs(vmask) - 1, lastl = 31u - __clz(vmask);
  const K kf = __shfl_sync(0xffffffffu, k, first), kl = __shfl_sync(0xffffffffu, k, lastl);
  uint32_t bb = 0;
  if (lane == first) bb = bucket_in(bmax, 0u, buckets - 1, kf);
  if (lane == lastl) bb = bucket_in(bmax, 0u, buckets - 1, kl);
  const uint32_t blo = __shfl_sync(0xffffffffu, bb, first), bhi = __shfl_sync(0xffffffffu, bb, lastl);
  if (!valid) return 0u;
  // a key outside the warp's first..last range (unsorted input) searches everything
  return (kf <= k && k <= kl) ? bucket_in(bmax, blo, bhi, k) : bucket_in(bmax, 0u, buckets - 1, k);
}

// first position in node p whose key is >= k (count when none)
template <typename K>
__device__ __forceinline__ uint32_t node_lower_bound(const Node<K> *p, uint32_t count, K k) {
  uint32_t lo = 0, hi = count;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (p->keys[mid] < k) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

template <typename K>
__global__ void __launch_bounds__(256) lookup_direct_kernel(
    const K *__restrict__ probes, const uint32_t *__restrict__ n_ptr, const K *__restrict__ bmax, uint32_t buckets,
    const learned::ModelHeader *__restrict__ model, const learned::Segment *__restrict__ segs,
    const Node<K> *__restrict__ nodes, const uint32_t *__restrict__ perm, uint32_t *__restrict__ out) {
  const uint32_t n = *n_ptr;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if ((i & ~31u) >= n) return;  // whole warps leave together (routing uses warp votes)
  const bool valid = i < n;
  const K k = valid ? probes[i] : K(0);
  uint32_t id = route_sorted<K>(bmax, buckets, model, segs, k, valid);
  if (!valid) return;
  uint32_t result = kNotFound;
  for (uint32_t hops = 0; id != kNone && hops < (1u << 20); ++hops) {
    const Node<K> *p = nodes + id;
    const uint32_t count = p->count;
    if (count && k <= p->max) {
      const uint32_t pos = node_lower_bound(p, count, k);
      if (pos < count && p->keys[pos] == k) result = p->vals[pos];
      if (pos < count) break;
    }
    id = p->next;
  }
  out[perm ? perm[i] : i] = result;
}

template <typename K>
__global__ void __launch_bounds__(256) successor_direct_kernel(
    const K *__restrict__ probes, const uint32_t *__restrict__ n_ptr, const K *__restrict__ bmax, uint32_t buckets,
    const learned::ModelHeader *__restrict__ model, const learned::Segment *__restrict__ segs,
    const Node<K> *__restrict__ nodes, const uint32_t *__restrict__ perm, K *__restrict__ out) {
  const uint32_t n = *n_ptr;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if ((i & ~31u) >= n) return;
  const bool valid = i < n;
  const K k = valid ? probes[i] : K(0);
  const uint32_t b = route_sorted<K>(bmax, buckets, model, segs, k, valid);
  if (!valid) return;
  uint32_t id = b;
  bool found = false;
  K result = successor_miss<K>();
  for (uint32_t hops = 0; id != kNone && hops < (1u << 20); ++hops) {
    const Node<K> *p = nodes + id;
    const uint32_t count = p->count;
    if (count && k <= p->max) {
      const uint32_t pos = node_lower_bound(p, count, k);
      if (pos < count) {
        result = p->keys[pos];
        found = true;
        break;
      }
    }
    id = p->next;
  }
  if (!found) result = first_key_from_bucket(nodes, b + 1, buckets);
  out[perm ? perm[i] : i] = result;
}

// ---------------------------------------------------------------------------
// Unsorted probes without sorting them (small batches): a fence tree over the
// bucket maxima.  Level 0 is bmax itself; level l + 1 holds the maximum of
// every group of kFenceFan entries of level l (its last entry), up to a level
// of at most kFenceFan entries.  A probe descends from the top, searching one
// group (kFenceFan keys: one or two cache lines) per level; the upper levels
// stay in L2.  The answer equals bucket_of: a group's maximum bounds every key
// in it, and a key above every maximum falls into the last group at every
// level.  For large batches sorting the probes is faster (neighbouring threads
// then read the same nodes), so the host picks by batch size.
constexpr uint32_t kFenceFan = 32;
constexpr int kMaxFenceLevels = 8;

template <typename K>
struct FenceTree {
  const K *level[kMaxFenceLevels];
  uint32_t size[kMaxFenceLevels];
  uint32_t levels;  // including level 0 (bmax)
};

template <typename K>
__global__ void fence_level_kernel(const K *__restrict__ src, uint32_t src_n, K *__restrict__ dst, uint32_t dst_n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < dst_n) dst[i] = src[min((i + 1) * kFenceFan, src_n) - 1];
}

template <typename K>
__device__ __forceinline__ uint32_t route_fence(const FenceTree<K> &t, K k) {
  int l = int(t.levels) - 1;
  uint32_t pos = bucket_in(t.level[l], 0u, t.size[l] - 1, k);
  for (--l; l >= 0; --l) {
    const uint32_t lo = pos * kFenceFan;
    pos = bucket_in(t.level[l], lo, min(lo + kFenceFan, t.size[l]) - 1, k);
  }
  return pos;
}

// value or not_found of unsorted probes, one thread each (results in input order)
template <typename K>
__global__ void __launch_bounds__(256) lookup_fence_kernel(
    const K *__restrict__ probes, uint32_t n, FenceTree<K> tree, const learned::ModelHeader *__restrict__ model,
    const learned::Segment *__restrict__ segs, const Node<K> *__restrict__ nodes, uint32_t *__restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const K k = probes[i];
  uint32_t id = model ? bucket_of_model<K>(*model, segs, tree.level[0], k) : route_fence<K>(tree, k);
  uint32_t result = kNotFound;
  for (uint32_t hops = 0; id != kNone && hops < (1u << 20); ++hops) {
    const Node<K> *p = nodes + id;
    const uint32_t count = p->count;
    if (count && k <= p->max) {
      const uint32_t pos = node_lower_bound(p, count, k);
      if (pos < count && p->keys[pos] == k) result = p->vals[pos];
      if (pos < count) break;
    }
    id = p->next;
  }
  out[i] = result;
}

// first key >= probe of unsorted probes, one thread each (results in input order)
template <typename K>
__global__ void __launch_bounds__(256) successor_fence_kernel(
    const K *__restrict__ probes, uint32_t n, FenceTree<K> tree, const learned::ModelHeader *__restrict__ model,
    const learned::Segment *__restrict__ segs, const Node<K> *__restrict__ nodes, K *__restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const K k = probes[i];
  const uint32_t b = model ? bucket_of_model<K>(*model, segs, tree.level[0], k) : route_fence<K>(tree, k);
  uint32_t id = b;
  bool found = false;
  K result = successor_miss<K>();
  for (uint32_t hops = 0; id != kNone && hops < (1u << 20); ++hops) {
    const Node<K> *p = nodes + id;
    const uint32_t count = p->count;
    if (count && k <= p->max) {
      const uint32_t pos = node_lower_bound(p, count, k);
      if (pos < count) {
        result = p->keys[pos];
        found = true;
        break;
      }
    }
    id = p->next;
  }
  if (!found) result = first_key_from_bucket(nodes, b + 1, tree.size[0]);
  out[i] = result;
}

// ---------------------------------------------------------------------------
// helpers for sorting / dedup of batches
template <typename K>
__global__ void set_u32_kernel(uint32_t *__restrict__ p, uint32_t v) {
  *p = v;
}

template <typename K>
__global__ void iota_kernel(uint32_t *__restrict__ v, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = i;
}

// keep the FIRST of each run of equal keys (insert-if-absent in input order)
constexpr int kDedupThreads = 256;
constexpr int kDedupItems = 8;
constexpr uint32_t kDedupTile = kDedupThreads * kDedupItems;

template <typename K>
__global__ void __launch_bounds__(kDedupThreads) dedup_first_kernel(
    const K *__restrict__ kin, const uint32_t *__restrict__ vin, uint32_t n, K *__restrict__ kout,
    uint32_t *__restrict__ vout, uint32_t *__restrict__ out_n, unsigned long long *__restrict__ lb,
    uint32_t *__restrict__ tile_counter, uint32_t *__restrict__ status) {
  __shared__ uint32_t s_scan[kDedupThreads / 32];
  __shared__ uint32_t s_total;
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_base;
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint64_t base = uint64_t(s_tile) * kDedupTile + uint64_t(threadIdx.x) * kDedupItems;
  K k[kDedupItems];
  uint32_t keep = 0, cnt = 0;
  K prev = base > 0 && base <= n ? kin[base - 1] : K(0);
#pragma unroll
  for (int i = 0; i < kDedupItems; ++i) {
    const uint64_t g = base + i;
    k[i] = g < n ? kin[g] : K(0);
    if (g < n && (g == 0 || k[i] != prev)) {
      keep |= 1u << i;
      ++cnt;
    }
    prev = k[i];
  }
  const uint32_t local = block_exclusive_scan<kDedupThreads>(cnt, s_scan, &s_total);
  if (threadIdx.x < 32) {
    const unsigned long long lb_excl = warp_lookback(lb, s_tile, s_total, status);
    if (threadIdx.x == 0) s_base = lb_excl;
  }
  __syncthreads();
  uint64_t o = s_base + local;
#pragma unroll
  for (int i = 0; i < kDedupItems; ++i)
    if (keep & (1u << i)) {
      if (o < n) {
        kout[o] = k[i];
        if (vout) vout[o] = vin ? vin[base + i] : 0u;
      }
      ++o;
    }
  if (uint64_t(s_tile + 1) * kDedupTile >= n && threadIdx.x == 0) *out_n = uint32_t(s_base + s_total);
}

// sortedness / max probe of a key array: flags bit0 = not sorted ascending,
// bit1 = has equal neighbours; max key via atomicMax
template <typename K>
__global__ void __launch_bounds__(256) inspect_keys_kernel(const K *__restrict__ keys, uint64_t n,
                                                           uint32_t *__restrict__ flags,
                                                           unsigned long long *__restrict__ max_key) {
  // four independent loads in flight per thread and step; one atomic pair per block
  __shared__ unsigned long long s_max[8];
  __shared__ uint32_t s_flags[8];
  unsigned long long local_max = 0;
  uint32_t f = 0;
  const uint64_t step = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t i0 = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i0 < n; i0 += 4 * step) {
    K k[4], nx[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint64_t i = i0 + u * step;
      k[u] = i < n ? keys[i] : K(0);
      nx[u] = i + 1 < n ? keys[i + 1] : K(0);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const uint64_t i = i0 + u * step;
      if (i < n) {
        local_max = max(local_max, (unsigned long long)k[u]);
        if (i + 1 < n) {
          if (nx[u] < k[u]) f |= 1u;
          if (nx[u] == k[u]) f |= 2u;
        }
      }
    }
  }
  f = __reduce_or_sync(0xffffffffu, f);
  for (int o = 16; o; o >>= 1) local_max = max(local_max, __shfl_down_sync(0xffffffffu, local_max, o));
  if ((threadIdx.x & 31) == 0) {
    s_max[threadIdx.x >> 5] = local_max;
    s_flags[threadIdx.x >> 5] = f;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long m = 0;
    uint32_t ff = 0;
    for (uint32_t w = 0; w < blockDim.x / 32; ++w) {
      m = max(m, s_max[w]);
      ff |= s_flags[w];
    }
    if (ff) atomicOr(flags, ff);
    atomicMax(max_key, m);
  }
}

// Exclusive scan of u32 counts into u64 offsets (offsets[n] = total).
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;
template <typename K>
__global__ void __launch_bounds__(kScanThreads) scan_counts_kernel(
    const uint32_t *__restrict__ counts, uint64_t n, unsigned long long *__restrict__ offsets,
    unsigned long long *__restrict__ lb, uint32_t *__restrict__ tile_counter,
    uint32_t *__restrict__ status) {
  __shared__ unsigned long long s_scan[kScanThreads / 32];
  __shared__ unsigned long long s_total;
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_base;
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const uint64_t base = uint64_t(s_tile) * kScanTile + uint64_t(threadIdx.x) * kScanItems;
  uint32_t c[kScanItems];
  unsigned long long sum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    c[i] = base + i < n ? counts[base + i] : 0u;
    sum += c[i];
  }
  const unsigned long long local = block_exclusive_scan<kScanThreads>(sum, s_scan, &s_total);
  if (threadIdx.x < 32) {
    const unsigned long long lb_excl = warp_lookback(lb, s_tile, s_total, status);
    if (threadIdx.x == 0) s_base = lb_excl;
  }
  __syncthreads();
  unsigned long long o = s_base + local;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    if (base + i <= n) offsets[base + i] = o;
    o += c[i];
  }
}

// Per-bucket live counts (rebuild step 1) - one warp per bucket chain.
template <typename K>
__global__ void chain_counts_kernel(const Node<K> *__restrict__ nodes, uint32_t buckets,
                                    uint32_t *__restrict__ counts) {
  const uint32_t b = (uint32_t(blockIdx.x) * blockDim.x + threadIdx.x);
  if (b >= buckets) return;
  uint32_t c = 0;
  for (uint32_t id = b; id != kNone; id = nodes[id].next) c += nodes[id].count;
  counts[b] = c;
}

// Rebuild step 2: copy every chain's entries, in key order, into a dense
// sorted array at offsets[b] (FliX/coarse_granular_rebuild.cuh:219-397).
template <typename K>
__global__ void gather_chains_kernel(const Node<K> *__restrict__ nodes, uint32_t buckets,
                                     const unsigned long long *__restrict__ offsets, K *__restrict__ keys,
                                     uint32_t *__restrict__ vals) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t b = (uint32_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  if (b >= buckets) return;
  unsigned long long o = offsets[b];
  for (uint32_t id = b; id != kNone; id = nodes[id].next) {
    const uint32_t c = nodes[id].count;
    if (lane < c) {
      keys[o + lane] = nodes[id].keys[lane];
      vals[o + lane] = nodes[id].vals[lane];
    }
    o += c;
  }
}

}  // namespace flix
}  // namespace gpulsm
