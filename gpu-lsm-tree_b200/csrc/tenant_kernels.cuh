// Kernels of the multi-tenant batched dictionary: many independent u32
// dictionaries (GPULSMOpt upsert semantics, inserts and lookups) updated in
// rounds, each round touching every tenant with a handful of launches instead
// of a handful per tenant.
//
// HBM layout per tenant t (arena offsets in TenantMeta):
//   main run   keys/vals, sorted unique, double buffered (2 x cap)
//   delta run  keys/vals, sorted unique, double buffered (2 x cap): the
//              batches of the last (fan_in - 1) rounds, merged into main on
//              every fan_in-th round (tiering with fan-in R)
//   fences     an implicit B-ary tree over each run: level 1 holds every F-th
//              key, level 2 every F-th key of level 1, ... (F = search fanout),
//              so a lookup reads one F-key node per level.
// A round sorts all tenants' batches at once by (tenant << 32 | key), keeps
// the last update per (tenant, key), and merges every tenant's batch in one
// persistent launch: CTAs pull (tenant, tile) work items from a global counter
// and chain each tenant's tile counts with a decoupled look-back.
#pragma once

#include "common.cuh"
#include "tenant_types.h"

namespace gpulsm {
namespace tenants {

// fence level sizes of a run of n rows with fanout F: level l has ceil(n / F^l) entries
__host__ __device__ __forceinline__ unsigned long long fence_level_size(unsigned long long n, uint32_t F,
                                                                       uint32_t level) {
  unsigned long long s = n;
  for (uint32_t l = 0; l < level; ++l) s = (s + F - 1) / F;
  return s;
}

// ---------------------------------------------------------------------------
// Round step 1: tenant of every batch element (CSR offsets) + composite word
// (tenant << 32 | key) and histograms for the sort passes.
__global__ void __launch_bounds__(256) pack_tenant_words_kernel(
    const uint32_t *__restrict__ keys, const uint32_t *__restrict__ vals,
    const unsigned long long *__restrict__ batch_off, uint32_t tenants, const uint32_t *__restrict__ count,
    unsigned long long *__restrict__ words, uint32_t *__restrict__ wvals, uint32_t passes,
    uint32_t *__restrict__ hist) {
  __shared__ uint32_t s[8][256];
  for (uint32_t i = threadIdx.x; i < 8 * 256; i += 256) (&s[0][0])[i] = 0;
  __syncthreads();
  const unsigned long long n = *count;
  for (unsigned long long i = uint64_t(blockIdx.x) * 256 + threadIdx.x; i < n; i += uint64_t(gridDim.x) * 256) {
    uint32_t lo = 0, hi = tenants;  // last t with batch_off[t] <= i
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (batch_off[mid] <= i) lo = mid;
      else hi = mid;
    }
    const unsigned long long w = ((unsigned long long)lo << 32) | keys[i];
    words[i] = w;
    wvals[i] = vals[i];
    for (uint32_t p = 0; p < passes; ++p) atomicAdd(&s[p][uint32_t(w >> (8 * p)) & 0xffu], 1u);
  }
  __syncthreads();
  for (uint32_t p = 0; p < passes; ++p) {
    const uint32_t c = s[p][threadIdx.x];
    if (c) atomicAdd(&hist[p * 256 + threadIdx.x], c);
  }
}

// the round's batch total (device CSR offsets) as the u32 count every later
// step reads; a round larger than the configured maximum is refused (status
// bit, nothing applied) instead of overrunning the round buffers
__global__ void set_count_kernel(const unsigned long long *__restrict__ batch_off, uint32_t tenants,
                                 unsigned long long max_round, uint32_t *__restrict__ count,
                                 uint32_t *__restrict__ status) {
  const unsigned long long n = batch_off[tenants];
  if (n > max_round || batch_off[0] != 0) {
    *count = 0;
    atomicOr(status, kDevBadInput);
  } else {
    *count = uint32_t(n);
  }
}

// Round step 3: keep the last update of each (tenant, key) (stable sort keeps
// input order) and record, per tenant, the slice [bstart[t], bstart[t+1]) of
// the compacted batch (tenants without updates get an empty slice).
constexpr int kDedupThreads = 256;
constexpr int kDedupItems = 8;
constexpr uint32_t kDedupTile = kDedupThreads * kDedupItems;


__global__ void __launch_bounds__(kDedupThreads) dedup_tenant_words_kernel(
    const unsigned long long *__restrict__ words, const uint32_t *__restrict__ wvals,
    const uint32_t *__restrict__ count, uint32_t tenants, uint32_t *__restrict__ out_keys,
    uint32_t *__restrict__ out_vals, uint32_t *__restrict__ out_tenant, unsigned long long *__restrict__ bstart,
    unsigned long long *__restrict__ lb, uint32_t *__restrict__ tile_counter, uint32_t *__restrict__ status) {
  __shared__ uint32_t s_scan[kDedupThreads / 32];
  __shared__ uint32_t s_total;
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_base;
  const unsigned long long n = *count;
  if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
  __syncthreads();
  const unsigned long long base = uint64_t(s_tile) * kDedupTile + uint64_t(threadIdx.x) * kDedupItems;
  if (uint64_t(s_tile) * kDedupTile >= n && !(s_tile == 0 && n == 0)) return;
  uint32_t keep = 0, cnt = 0;
  unsigned long long w[kDedupItems];
#pragma unroll
  for (int i = 0; i < kDedupItems; ++i) {
    const unsigned long long g = base + i;
    w[i] = g < n ? words[g] : ~0ull;
  }
  const unsigned long long nextw = base + kDedupItems < n ? words[base + kDedupItems] : ~0ull;
#pragma unroll
  for (int i = 0; i < kDedupItems; ++i) {
    const unsigned long long g = base + i;
    const unsigned long long nx = i + 1 < kDedupItems ? w[i + 1] : nextw;
    if (g < n && (g + 1 == n || nx != w[i])) {
      keep |= 1u << i;
      ++cnt;
    }
  }
  const uint32_t local = block_exclusive_scan<kDedupThreads>(cnt, s_scan, &s_total);
  if (threadIdx.x < 32) {
    const unsigned long long lb_excl = warp_lookback(lb, s_tile, s_total, status);
    if (threadIdx.x == 0) s_base = lb_excl;
  }
  __syncthreads();
  unsigned long long o = s_base + local;
#pragma unroll
  for (int i = 0; i < kDedupItems; ++i)
    if (keep & (1u << i)) {
      if (o < n) {
        out_keys[o] = uint32_t(w[i]);
        out_vals[o] = wvals[base + i];
        out_tenant[o] = uint32_t(w[i] >> 32);
      }
      ++o;
    }
  // the compacted count is written by the last tile (as bstart[tenants])
  if (uint64_t(s_tile + 1) * kDedupTile >= n && threadIdx.x == 0) bstart[tenants] = s_base + s_total;
}

// per-tenant slice starts over the compacted (tenant-sorted) batch
__global__ void tenant_slices_kernel(const uint32_t *__restrict__ tenant_of, unsigned long long *__restrict__ bstart,
                                     uint32_t tenants) {
  const unsigned long long m = bstart[tenants];
  const unsigned long long i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (m == 0) {
    for (uint32_t t = uint32_t(i); t < tenants; t += gridDim.x * blockDim.x) bstart[t] = 0;
    return;
  }
  if (i >= m) return;
  const int64_t t = tenant_of[i];
  const int64_t tp = i ? int64_t(tenant_of[i - 1]) : -1;
  for (int64_t u = tp + 1; u <= t; ++u) bstart[u] = i;
  if (i == m - 1)
    for (int64_t u = t + 1; u < int64_t(tenants); ++u) bstart[u] = m;
}

// ---------------------------------------------------------------------------
// Persistent merge over all tenants: newer run X (the round's batch slice or a
// delta) into older run Y, newest wins, output into Y's other buffer.
enum MergeKind : uint32_t { kBatchIntoDelta = 0, kDeltaIntoMain = 1 };

struct MergeArgs {
  const TenantMeta *meta;
  Arena arena;
  const uint32_t *bkeys;  // compacted batch (kBatchIntoDelta)
  const uint32_t *bvals;
  const unsigned long long *bstart;
  const unsigned long long *tile_off;  // [tenants + 1] exclusive scan of tiles per tenant
  unsigned long long *lb;              // one look-back word per tile
  uint32_t *counter;
  uint32_t *out_n;                     // [tenants] new run size
  uint32_t *status;
  uint32_t tenants;
  uint32_t tile;                       // outputs per work item (autotuned)
  uint32_t kind;
};

template <typename T>
__device__ __forceinline__ uint64_t tmerge_path(const T *a, uint64_t na, const T *b, uint64_t nb, uint64_t diag) {
  uint64_t lo = diag > nb ? diag - nb : 0, hi = diag < na ? diag : na;
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (a[mid] <= b[diag - 1 - mid]) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// number of merge tiles of every tenant (then scanned into tile_off)
__global__ void tenant_tiles_kernel(MergeArgs m, unsigned long long *__restrict__ tiles) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m.tenants) return;
  const TenantMeta mt = m.meta[t];
  const unsigned long long nx = m.kind == kBatchIntoDelta ? m.bstart[t + 1] - m.bstart[t] : mt.delta_n;
  const unsigned long long ny = m.kind == kBatchIntoDelta ? mt.delta_n : mt.main_n;
  const unsigned long long total = nx + ny;
  if (nx > mt.cap) {  // a batch larger than the tenant's capacity cannot fit: refuse it
    atomicOr(m.status, kDevBadInput);
    tiles[t] = 0;
    return;
  }
  tiles[t] = nx ? (total + m.tile - 1) / m.tile : 0ull;  // nothing newer: the run stays as it is
}

// single-CTA exclusive scan over tenants (tenants <= 65536)
__global__ void __launch_bounds__(1024) scan_tenants_kernel(const unsigned long long *__restrict__ in,
                                                            unsigned long long *__restrict__ out, uint32_t n) {
  __shared__ unsigned long long s_scan[32];
  __shared__ unsigned long long s_total;
  unsigned long long carry = 0;
  for (uint32_t base = 0; base < n; base += 1024) {
    const uint32_t i = base + threadIdx.x;
    const unsigned long long v = i < n ? in[i] : 0ull;
    const unsigned long long ex = block_exclusive_scan<1024>(v, s_scan, &s_total);
    if (i < n) out[i] = carry + ex;
    carry += s_total;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = carry;
}

constexpr int kMergeThreads = 256;
constexpr uint32_t kMaxTile = 4096;

__global__ void __launch_bounds__(kMergeThreads) tenant_merge_kernel(MergeArgs m) {
  extern __shared__ __align__(16) unsigned char dyn[];
  uint32_t *s_k = reinterpret_cast<uint32_t *>(dyn);
  uint32_t *s_v = s_k + m.tile;
  uint32_t *s_o = s_v + m.tile;  // compacted output keys
  uint32_t *s_ov = s_o + m.tile;
  __shared__ uint32_t s_scan[kMergeThreads / 32];
  __shared__ uint32_t s_total;
  __shared__ unsigned long long s_item, s_a0, s_a1, s_base;
  const unsigned long long total_items = m.tile_off[m.tenants];
  const uint32_t per_thread = (m.tile + kMergeThreads - 1) / kMergeThreads;
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(m.counter, 1u);
    __syncthreads();
    const unsigned long long item = s_item;
    if (item >= total_items) break;
    // tenant owning the item: last t with tile_off[t] <= item
    uint32_t lo = 0, hi = m.tenants;
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (m.tile_off[mid] <= item) lo = mid;
      else hi = mid;
    }
    const uint32_t t = lo;
    const uint32_t local_tile = uint32_t(item - m.tile_off[t]);
    const bool last_tile = item + 1 == m.tile_off[t + 1];
    const TenantMeta mt = m.meta[t];
    const uint32_t *xk, *xv, *yk, *yv;
    uint32_t *zk, *zv;
    unsigned long long nx, ny;
    if (m.kind == kBatchIntoDelta) {
      xk = m.bkeys + m.bstart[t];
      xv = m.bvals + m.bstart[t];
      nx = m.bstart[t + 1] - m.bstart[t];
      const unsigned long long cur = mt.delta_off + mt.delta_cur * mt.cap;
      const unsigned long long nxt = mt.delta_off + (mt.delta_cur ^ 1u) * mt.cap;
      yk = m.arena.keys + cur;
      yv = m.arena.vals + cur;
      ny = mt.delta_n;
      zk = m.arena.keys + nxt;
      zv = m.arena.vals + nxt;
    } else {
      const unsigned long long dcur = mt.delta_off + mt.delta_cur * mt.cap;
      xk = m.arena.keys + dcur;
      xv = m.arena.vals + dcur;
      nx = mt.delta_n;
      const unsigned long long cur = mt.main_off + mt.main_cur * mt.cap;
      const unsigned long long nxt = mt.main_off + (mt.main_cur ^ 1u) * mt.cap;
      yk = m.arena.keys + cur;
      yv = m.arena.vals + cur;
      ny = mt.main_n;
      zk = m.arena.keys + nxt;
      zv = m.arena.vals + nxt;
    }
    const unsigned long long tot = nx + ny;
    const unsigned long long d0 = uint64_t(local_tile) * m.tile;
    const unsigned long long d1 = min(d0 + m.tile, tot);
    if (threadIdx.x == 0) s_a0 = tmerge_path(xk, nx, yk, ny, d0);
    if (threadIdx.x == 32) s_a1 = tmerge_path(xk, nx, yk, ny, d1);
    __syncthreads();
    const unsigned long long a0 = s_a0, a1 = s_a1, b0 = d0 - a0, b1 = d1 - a1;
    const uint32_t alen = uint32_t(a1 - a0), blen = uint32_t(b1 - b0);
    for (uint32_t j = threadIdx.x; j < alen; j += kMergeThreads) {
      s_k[j] = xk[a0 + j];
      s_v[j] = xv[a0 + j];
    }
    for (uint32_t j = threadIdx.x; j < blen; j += kMergeThreads) {
      s_k[alen + j] = yk[b0 + j];
      s_v[alen + j] = yv[b0 + j];
    }
    const bool has_prev_a = a0 > 0;
    const uint32_t prev_a_global = has_prev_a ? xk[a0 - 1] : 0u;
    __syncthreads();
    const uint32_t *sa = s_k, *sb = s_k + alen;
    const uint32_t my_d = min(uint32_t(threadIdx.x) * per_thread, alen + blen);
    const uint32_t my_e = min(my_d + per_thread, alen + blen);
    uint32_t ai = uint32_t(tmerge_path(sa, alen, sb, blen, my_d));
    uint32_t bi = my_d - ai;
    bool have_prev = ai > 0 ? true : has_prev_a;
    uint32_t prev_a = ai > 0 ? sa[ai - 1] : prev_a_global;
    // pass 1: count kept rows (a y row shadowed by an equal x key is dropped)
    uint32_t kept = 0;
    {
      uint32_t ai2 = ai, bi2 = bi;
      bool hp = have_prev;
      uint32_t pa = prev_a;
      for (uint32_t d = my_d; d < my_e; ++d) {
        if (ai2 < alen && (bi2 >= blen || sa[ai2] <= sb[bi2])) {
          hp = true;
          pa = sa[ai2++];
          ++kept;
        } else {
          const uint32_t key = sb[bi2++];
          kept += !(hp && pa == key);
        }
      }
    }
    const uint32_t local = block_exclusive_scan<kMergeThreads>(kept, s_scan, &s_total);
    const uint32_t tile_kept = s_total;
    if (threadIdx.x < 32) {
      const unsigned long long lb_excl = warp_lookback(m.lb + m.tile_off[t], local_tile, tile_kept, m.status);
      if (threadIdx.x == 0) s_base = lb_excl;
    }
    // pass 2: write kept rows compactly into shared memory
    uint32_t o = local;
    for (uint32_t d = my_d; d < my_e; ++d) {
      if (ai < alen && (bi >= blen || sa[ai] <= sb[bi])) {
        have_prev = true;
        prev_a = sa[ai];
        s_o[o] = sa[ai];
        s_ov[o] = s_v[ai];
        ++o;
        ++ai;
      } else {
        const uint32_t key = sb[bi];
        if (!(have_prev && prev_a == key)) {
          s_o[o] = key;
          s_ov[o] = s_v[alen + bi];
          ++o;
        }
        ++bi;
      }
    }
    __syncthreads();
    const unsigned long long gbase = s_base;
    for (uint32_t j = threadIdx.x; j < tile_kept; j += kMergeThreads) {
      const unsigned long long oo = gbase + j;
      if (oo < mt.cap) {
        zk[oo] = s_o[j];
        zv[oo] = s_ov[j];
      }
    }
    if (last_tile && threadIdx.x == 0) {
      const unsigned long long n_out = gbase + tile_kept;
      if (n_out > mt.cap) atomicOr(m.status, kDevOutputOverflow);
      m.out_n[t] = uint32_t(n_out < mt.cap ? n_out : mt.cap);
    }
  }
}

// after a merge: flip the merged run's buffer and publish its size (tenants
// without work keep their run)
__global__ void commit_merge_kernel(TenantMeta *__restrict__ meta, const uint32_t *__restrict__ out_n,
                                    const unsigned long long *__restrict__ tile_off, uint32_t tenants,
                                    uint32_t kind) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= tenants) return;
  TenantMeta &mt = meta[t];
  const bool had_work = tile_off[t + 1] > tile_off[t];
  if (kind == kBatchIntoDelta) {
    if (had_work) {
      mt.delta_cur ^= 1u;
      mt.delta_n = out_n[t];
    }
  } else {
    if (had_work) {
      mt.main_cur ^= 1u;
      mt.main_n = out_n[t];
    }
    mt.delta_n = 0;
  }
}

// ---------------------------------------------------------------------------
// Fence trees: level l entry j = first key of block j of F^l rows.  One thread
// per level-1 entry of every tenant's main and delta run (grid-stride).
__global__ void build_fences_kernel(const TenantMeta *__restrict__ meta, Arena arena, uint32_t tenants, uint32_t F,
                                    uint32_t which /*0 main, 1 delta*/) {
  const uint32_t t = blockIdx.y;
  if (t >= tenants) return;
  const TenantMeta mt = meta[t];
  const unsigned long long n = which ? mt.delta_n : mt.main_n;
  const unsigned long long run = which ? mt.delta_off + mt.delta_cur * mt.cap : mt.main_off + mt.main_cur * mt.cap;
  uint32_t *f = arena.fences + mt.fence_off + (which ? mt.fence_cap : 0ull);
  // level sizes and offsets inside the tenant's fence area
  unsigned long long off = 0, prev_size = n;
  const uint32_t *src = arena.keys + run;
  unsigned long long stride = F;  // rows per level entry
  for (uint32_t l = 1; l <= kMaxFenceLevels && prev_size > 1; ++l) {
    const unsigned long long size = (prev_size + F - 1) / F;
    for (unsigned long long j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < size;
         j += uint64_t(gridDim.x) * blockDim.x)
      f[off + j] = src[j * stride];
    off += size;
    prev_size = size;
    stride *= F;
  }
}

// lower bound of q in one run through its fence tree (exact: the last level
// scanned is the run itself)
__device__ __forceinline__ unsigned long long fence_lower_bound(const uint32_t *keys, unsigned long long n,
                                                                const uint32_t *fences, uint32_t F, uint32_t q) {
  if (n == 0) return 0;
  // level sizes
  unsigned long long sizes[kMaxFenceLevels + 1];
  unsigned long long offs[kMaxFenceLevels + 1];
  uint32_t levels = 0;
  unsigned long long s = n, off = 0;
  while (s > 1 && levels < kMaxFenceLevels) {
    s = (s + F - 1) / F;
    ++levels;
    sizes[levels] = s;
    offs[levels] = off;
    off += s;
  }
  // descend: b is the chosen entry of level l+1; its children at level l are
  // entries [b*F, b*F + F) (the whole top level when l is the top)
  unsigned long long b = 0;
  for (int l = int(levels); l >= 1; --l) {
    const uint32_t *lv = fences + offs[l];
    const unsigned long long lo = l == int(levels) ? 0ull : b * F;
    const unsigned long long hi = l == int(levels) ? sizes[l] : min(lo + F, sizes[l]);
    // last entry <= q (entries are first keys of their blocks; lo when
    // none): binary search for the first entry after lo that is > q
    unsigned long long a = lo + 1, z = hi > lo ? hi : lo + 1;
    while (a < z) {
      const unsigned long long mid = (a + z) >> 1;
      if (lv[mid] <= q) a = mid + 1;
      else z = mid;
    }
    b = a - 1;
  }
  // first key >= q in the chosen block of the run
  unsigned long long a = b * F, z = min(a + F, n);
  while (a < z) {
    const unsigned long long mid = (a + z) >> 1;
    if (keys[mid] < q) a = mid + 1;
    else z = mid;
  }
  return a;
}

// Lookups: (tenant, key) -> value / found; delta first (newer), then main.
__global__ void __launch_bounds__(256) tenant_lookup_kernel(const TenantMeta *__restrict__ meta, Arena arena,
                                                            uint32_t F, const uint32_t *__restrict__ tenant_ids,
                                                            const uint32_t *__restrict__ q, unsigned long long n,
                                                            uint32_t tenants, uint32_t *__restrict__ out_values,
                                                            uint8_t *__restrict__ out_found) {
  const unsigned long long i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t t = tenant_ids[i];
  const uint32_t key = q[i];
  const uint32_t miss = out_found ? 0u : kNotFound;
  if (t >= tenants) {
    out_values[i] = miss;
    if (out_found) out_found[i] = 0;
    return;
  }
  const TenantMeta mt = meta[t];
  for (int which = 1; which >= 0; --which) {
    const unsigned long long nr = which ? mt.delta_n : mt.main_n;
    if (!nr) continue;
    const unsigned long long run = which ? mt.delta_off + mt.delta_cur * mt.cap : mt.main_off + mt.main_cur * mt.cap;
    const uint32_t *keys = arena.keys + run;
    const unsigned long long p =
        fence_lower_bound(keys, nr, arena.fences + mt.fence_off + (which ? mt.fence_cap : 0ull), F, key);
    if (p < nr && keys[p] == key) {
      out_values[i] = arena.vals[run + p];
      if (out_found) out_found[i] = 1;
      return;
    }
  }
  out_values[i] = miss;
  if (out_found) out_found[i] = 0;
}

}  // namespace tenants
}  // namespace gpulsm
