/*
 * CPU oracle: GPULSMOpt semantics restated over one sorted array of live keys.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * The reference keeps raw pending batches, epochs and radix-4 levels
 * (GPULSMOpt.cuh:288-340, :2578-2600, :3117-3198); none of that changes an
 * answer, so the oracle stores only the visible state: the newest version of
 * every key that is not hidden by a tombstone.  Rules restated here:
 *
 *  - insert (GPULSMOpt.cuh:5836): upsert.  Inside one batch the highest input
 *    index wins: the admission age is (slot << 20) | input_index
 *    (scatter_admission_records_kernel, :2578-2598; raw_position :444-452) and
 *    every reader keeps the largest age (:4779-4787, :2842-2918).
 *  - erase (:5843): tombstones that hide every older version; a lookup of an
 *    erased key is a miss (:4742-4749), range and successor skip it
 *    (:1659-2043, :5429-5594).
 *  - lookup miss convention (:4742-4749): out_values = out_found ? 0 : 0xffffffff.
 *  - range (:1415-1605): sum of live values with lo <= key <= hi accumulated in
 *    u64 and stored as u32 (wraps at 2^32); lo > hi gives 0.
 *  - successor (:5566-5594): smallest live key >= query, else 0xffffffff.
 *  - bulk_build (:5738-5834): resets the dictionary; stable radix sort of the
 *    pairs then mark_last_key_kernel (:2633-2638) keeps the LAST duplicate.
 *  - clear (:5731): empties the dictionary.
 *
 * Range count and range pairs have no GPULSMOpt counterpart; they are the
 * std::map answers (count of live keys, (key, value) pairs in key order) used
 * by the range-query configurations.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

struct orc_lsm {
  uint32_t *keys;
  uint32_t *values;
  uint64_t size;
  uint64_t cap;
};

static int g_threads = 0;

int orc_set_threads(int threads) {
#ifdef _OPENMP
  g_threads = threads > 0 ? threads : omp_get_num_procs();
  omp_set_num_threads(g_threads);
  return g_threads;
#else
  (void)threads;
  g_threads = 1;
  return 1;
#endif
}

int orc_get_threads(void) {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

static void *xmalloc(size_t bytes) {
  void *p = malloc(bytes ? bytes : 1);
  if (!p) abort();
  return p;
}

/* Stable LSD radix sort of (key, value) pairs by key, 4 passes of 8 bits.
 * Stability keeps input order among equal keys, which is what lets
 * keep_last_in_runs() pick the highest input index. */
void orc_stable_sort_pairs_u32(uint32_t *keys, uint32_t *values, uint64_t n) {
  if (n < 2) return;
  uint32_t *tk = (uint32_t *)xmalloc(n * sizeof(uint32_t));
  uint32_t *tv = (uint32_t *)xmalloc(n * sizeof(uint32_t));
  uint32_t *sk = keys, *sv = values, *dk = tk, *dv = tv;
  for (int shift = 0; shift < 32; shift += 8) {
    uint64_t count[257];
    memset(count, 0, sizeof(count));
    for (uint64_t i = 0; i < n; ++i) count[((sk[i] >> shift) & 0xffu) + 1]++;
    if (count[((sk[0] >> shift) & 0xffu) + 1] == n) continue; /* one digit */
    for (int d = 0; d < 256; ++d) count[d + 1] += count[d];
    for (uint64_t i = 0; i < n; ++i) {
      const uint64_t p = count[(sk[i] >> shift) & 0xffu]++;
      dk[p] = sk[i];
      dv[p] = sv[i];
    }
    uint32_t *t;
    t = sk; sk = dk; dk = t;
    t = sv; sv = dv; dv = t;
  }
  if (sk != keys) {
    memcpy(keys, sk, n * sizeof(uint32_t));
    memcpy(values, sv, n * sizeof(uint32_t));
  }
  free(tk);
  free(tv);
}

/* After a stable sort: keep the last element of each equal-key run
 * (mark_last_key_kernel, GPULSMOpt.cuh:2633-2638).  Returns the new length. */
static uint64_t keep_last_in_runs(uint32_t *keys, uint32_t *values, uint64_t n) {
  uint64_t out = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (i + 1 < n && keys[i + 1] == keys[i]) continue;
    keys[out] = keys[i];
    values[out] = values[i];
    ++out;
  }
  return out;
}

static uint64_t lower_bound_u32(const uint32_t *a, uint64_t n, uint32_t key) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

/* upper bound: first index with a[i] > key */
static uint64_t upper_bound_u32(const uint32_t *a, uint64_t n, uint32_t key) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (a[mid] <= key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

orc_lsm *orc_lsm_create(void) {
  orc_lsm *d = (orc_lsm *)xmalloc(sizeof(orc_lsm));
  d->keys = NULL;
  d->values = NULL;
  d->size = 0;
  d->cap = 0;
  return d;
}

void orc_lsm_destroy(orc_lsm *d) {
  if (!d) return;
  free(d->keys);
  free(d->values);
  free(d);
}

void orc_lsm_clear(orc_lsm *d) { d->size = 0; }

uint64_t orc_lsm_size(const orc_lsm *d) { return d->size; }

uint64_t orc_lsm_dump(const orc_lsm *d, uint32_t *keys, uint32_t *values) {
  if (keys) memcpy(keys, d->keys, d->size * sizeof(uint32_t));
  if (values) memcpy(values, d->values, d->size * sizeof(uint32_t));
  return d->size;
}

void orc_lsm_bulk_build(orc_lsm *d, const uint32_t *keys, const uint32_t *values,
                        uint64_t n) {
  free(d->keys);
  free(d->values);
  d->keys = (uint32_t *)xmalloc(n * sizeof(uint32_t));
  d->values = (uint32_t *)xmalloc(n * sizeof(uint32_t));
  memcpy(d->keys, keys, n * sizeof(uint32_t));
  memcpy(d->values, values, n * sizeof(uint32_t));
  orc_stable_sort_pairs_u32(d->keys, d->values, n);
  d->size = keep_last_in_runs(d->keys, d->values, n);
  d->cap = n;
}

/* Merge the sorted unique batch B into the live array L.  Equal keys: the
 * batch wins (newest batch wins, GPULSMOpt.cuh:4752-4806 scans pending batches
 * newest first); tombstone batches remove the key instead.  Parallel over
 * key-aligned partitions so that equal keys never straddle two threads. */
static void merge_batch(orc_lsm *d, const uint32_t *bk, const uint32_t *bv, uint64_t bn,
                        int tombstone) {
  const uint64_t ln = d->size;
  const uint32_t *lk = d->keys, *lv = d->values;
  const int threads = orc_get_threads();
  const int parts = threads < 1 ? 1 : threads * 4;
  uint64_t *li = (uint64_t *)xmalloc((parts + 1) * sizeof(uint64_t));
  uint64_t *bi = (uint64_t *)xmalloc((parts + 1) * sizeof(uint64_t));
  uint64_t *cnt = (uint64_t *)xmalloc((parts + 1) * sizeof(uint64_t));
  li[0] = 0; bi[0] = 0; li[parts] = ln; bi[parts] = bn;
  for (int p = 1; p < parts; ++p) {
    /* split the longer array evenly, cut the other one at the same key */
    if (ln >= bn) {
      uint64_t i = ln * (uint64_t)p / (uint64_t)parts;
      if (i >= ln) { li[p] = ln; bi[p] = bn; continue; }
      li[p] = i;
      bi[p] = lower_bound_u32(bk, bn, lk[i]);
    } else {
      uint64_t j = bn * (uint64_t)p / (uint64_t)parts;
      if (j >= bn) { li[p] = ln; bi[p] = bn; continue; }
      bi[p] = j;
      li[p] = lower_bound_u32(lk, ln, bk[j]);
    }
  }
  for (int p = 1; p <= parts; ++p) { /* monotone cuts */
    if (li[p] < li[p - 1]) li[p] = li[p - 1];
    if (bi[p] < bi[p - 1]) bi[p] = bi[p - 1];
  }
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < parts; ++p) {
    uint64_t i = li[p], j = bi[p], c = 0;
    const uint64_t ie = li[p + 1], je = bi[p + 1];
    while (i < ie || j < je) {
      if (j >= je || (i < ie && lk[i] < bk[j])) { ++c; ++i; }
      else if (i >= ie || bk[j] < lk[i]) { c += !tombstone; ++j; }
      else { c += !tombstone; ++i; ++j; }
    }
    cnt[p] = c;
  }
  uint64_t total = 0;
  for (int p = 0; p < parts; ++p) { const uint64_t c = cnt[p]; cnt[p] = total; total += c; }
  uint32_t *ok = (uint32_t *)xmalloc(total * sizeof(uint32_t));
  uint32_t *ov = (uint32_t *)xmalloc(total * sizeof(uint32_t));
#pragma omp parallel for schedule(dynamic, 1)
  for (int p = 0; p < parts; ++p) {
    uint64_t i = li[p], j = bi[p], o = cnt[p];
    const uint64_t ie = li[p + 1], je = bi[p + 1];
    while (i < ie || j < je) {
      if (j >= je || (i < ie && lk[i] < bk[j])) { ok[o] = lk[i]; ov[o] = lv[i]; ++o; ++i; }
      else if (i >= ie || bk[j] < lk[i]) {
        if (!tombstone) { ok[o] = bk[j]; ov[o] = bv[j]; ++o; }
        ++j;
      } else {
        if (!tombstone) { ok[o] = bk[j]; ov[o] = bv[j]; ++o; }
        ++i; ++j;
      }
    }
  }
  free(d->keys);
  free(d->values);
  d->keys = ok;
  d->values = ov;
  d->size = total;
  d->cap = total;
  free(li); free(bi); free(cnt);
}

static void apply_update(orc_lsm *d, const uint32_t *keys, const uint32_t *values,
                         uint64_t n, int tombstone) {
  if (!n) return;
  uint32_t *bk = (uint32_t *)xmalloc(n * sizeof(uint32_t));
  uint32_t *bv = (uint32_t *)xmalloc(n * sizeof(uint32_t));
  memcpy(bk, keys, n * sizeof(uint32_t));
  if (values) memcpy(bv, values, n * sizeof(uint32_t));
  else memset(bv, 0, n * sizeof(uint32_t));
  orc_stable_sort_pairs_u32(bk, bv, n);
  const uint64_t m = keep_last_in_runs(bk, bv, n);
  merge_batch(d, bk, bv, m, tombstone);
  free(bk);
  free(bv);
}

void orc_lsm_insert(orc_lsm *d, const uint32_t *keys, const uint32_t *values, uint64_t n) {
  apply_update(d, keys, values, n, 0);
}

void orc_lsm_erase(orc_lsm *d, const uint32_t *keys, uint64_t n) {
  apply_update(d, keys, NULL, n, 1);
}

void orc_lsm_lookup(const orc_lsm *d, const uint32_t *queries, uint64_t n,
                    uint32_t *out_values, uint8_t *out_found) {
  const uint32_t miss = out_found ? 0u : 0xffffffffu;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    const uint64_t p = lower_bound_u32(d->keys, d->size, queries[i]);
    const int hit = p < d->size && d->keys[p] == queries[i];
    out_values[i] = hit ? d->values[p] : miss;
    if (out_found) out_found[i] = (uint8_t)hit;
  }
}

void orc_lsm_range_sum(const orc_lsm *d, const uint32_t *lo, const uint32_t *hi,
                       uint64_t n, uint32_t *out_sums) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t q = 0; q < (int64_t)n; ++q) {
    uint64_t sum = 0;
    if (lo[q] <= hi[q]) {
      const uint64_t b = lower_bound_u32(d->keys, d->size, lo[q]);
      const uint64_t e = upper_bound_u32(d->keys, d->size, hi[q]);
      for (uint64_t i = b; i < e; ++i) sum += d->values[i];
    }
    out_sums[q] = (uint32_t)sum;
  }
}

void orc_lsm_range_count(const orc_lsm *d, const uint32_t *lo, const uint32_t *hi,
                         uint64_t n, uint32_t *out_counts) {
#pragma omp parallel for schedule(static)
  for (int64_t q = 0; q < (int64_t)n; ++q) {
    uint64_t c = 0;
    if (lo[q] <= hi[q])
      c = upper_bound_u32(d->keys, d->size, hi[q]) - lower_bound_u32(d->keys, d->size, lo[q]);
    out_counts[q] = (uint32_t)c;
  }
}

uint64_t orc_lsm_range_offsets(const orc_lsm *d, const uint32_t *lo, const uint32_t *hi,
                               uint64_t n, uint64_t *offsets) {
#pragma omp parallel for schedule(static)
  for (int64_t q = 0; q < (int64_t)n; ++q) {
    uint64_t c = 0;
    if (lo[q] <= hi[q])
      c = upper_bound_u32(d->keys, d->size, hi[q]) - lower_bound_u32(d->keys, d->size, lo[q]);
    offsets[q] = c;
  }
  uint64_t total = 0;
  for (uint64_t q = 0; q < n; ++q) { const uint64_t c = offsets[q]; offsets[q] = total; total += c; }
  offsets[n] = total;
  return total;
}

void orc_lsm_range_pairs(const orc_lsm *d, const uint32_t *lo, const uint32_t *hi,
                         uint64_t n, const uint64_t *offsets, uint32_t *out_keys,
                         uint32_t *out_values) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t q = 0; q < (int64_t)n; ++q) {
    if (lo[q] > hi[q]) continue;
    const uint64_t b = lower_bound_u32(d->keys, d->size, lo[q]);
    const uint64_t e = upper_bound_u32(d->keys, d->size, hi[q]);
    uint64_t o = offsets[q];
    for (uint64_t i = b; i < e; ++i, ++o) {
      out_keys[o] = d->keys[i];
      out_values[o] = d->values[i];
    }
  }
}

void orc_lsm_successor(const orc_lsm *d, const uint32_t *queries, uint64_t n,
                       uint32_t *out_keys) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    const uint64_t p = lower_bound_u32(d->keys, d->size, queries[i]);
    out_keys[i] = p < d->size ? d->keys[p] : 0xffffffffu;
  }
}
