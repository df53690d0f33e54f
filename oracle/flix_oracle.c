/*
 * CPU oracle: FliX bucket-layer semantics restated over one sorted array.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * FliX stores (key, u32 offset) entries in fixed-stride nodes with chains
 * (FliX/definitions_updates.cuh:259-329, FliX/impl_cg_rtx_index_updates.cuh:443-528);
 * answers do not depend on that layout, so the oracle keeps the sorted set.
 *
 *  - build (build_bucket_layer_only, FliX/impl_cg_rtx_index_updates.cuh:1711;
 *    layout :443-528): values are the input index unless given; the build
 *    sort is CUB SortPairs (stable, FliX/utilities.cuh:275-285) and the
 *    ballot lookup returns the first matching lane
 *    (FliX/coarse_granular_lookups_tile_bulk.cuh:418-424), so of duplicate
 *    build keys the FIRST input wins.
 *  - insert (FliX/coarse_granular_inserts_tiles_bulk.cuh:1307-1602): insert
 *    if absent; a key already stored keeps its value (:1423-1429).  The
 *    reference requires sorted unique batches; inside one batch the first
 *    occurrence is the one applied (sequential insert-if-absent order).
 *  - remove (FliX/coarse_granular_deletes_tiles.cuh:1128-1320): physical
 *    delete of every listed key that is present.
 *  - lookup (FliX/coarse_granular_lookups_tile_bulk.cuh:312-470): stored value
 *    or not_found = 0xffffffff (FliX/definitions.cuh:83).
 *  - successor (FliX/coarse_granular_lookups_tile_bulk.cuh:630-972): first
 *    stored key >= probe, else static_cast<key_type>(not_found), i.e.
 *    0xffffffff zero-extended for 64-bit keys (:672, :917, :946).
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

struct orc_flix {
  int key_bits;
  uint64_t *keys;
  uint32_t *values;
  uint64_t size;
};

static void *xmalloc(size_t bytes) {
  void *p = malloc(bytes ? bytes : 1);
  if (!p) abort();
  return p;
}

/* Stable LSD radix sort of (u64 key, u32 value), 16-bit digits. */
static void stable_sort_pairs_u64(uint64_t *keys, uint32_t *values, uint64_t n, int key_bits) {
  if (n < 2) return;
  uint64_t *tk = (uint64_t *)xmalloc(n * sizeof(uint64_t));
  uint32_t *tv = (uint32_t *)xmalloc(n * sizeof(uint32_t));
  uint64_t *count = (uint64_t *)xmalloc((65536 + 1) * sizeof(uint64_t));
  uint64_t *sk = keys, *dk = tk;
  uint32_t *sv = values, *dv = tv;
  for (int shift = 0; shift < key_bits; shift += 16) {
    memset(count, 0, (65536 + 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; ++i) count[((sk[i] >> shift) & 0xffffu) + 1]++;
    if (count[((sk[0] >> shift) & 0xffffu) + 1] == n) continue;
    for (int d = 0; d < 65536; ++d) count[d + 1] += count[d];
    for (uint64_t i = 0; i < n; ++i) {
      const uint64_t p = count[(sk[i] >> shift) & 0xffffu]++;
      dk[p] = sk[i];
      dv[p] = sv[i];
    }
    uint64_t *t64 = sk; sk = dk; dk = t64;
    uint32_t *t32 = sv; sv = dv; dv = t32;
  }
  if (sk != keys) {
    memcpy(keys, sk, n * sizeof(uint64_t));
    memcpy(values, sv, n * sizeof(uint32_t));
  }
  free(tk);
  free(tv);
  free(count);
}

static uint64_t keep_first_in_runs(uint64_t *keys, uint32_t *values, uint64_t n) {
  uint64_t out = 0;
  for (uint64_t i = 0; i < n; ++i) {
    if (i > 0 && keys[i - 1] == keys[i]) continue;
    keys[out] = keys[i];
    values[out] = values[i];
    ++out;
  }
  return out;
}

static uint64_t lower_bound_u64(const uint64_t *a, uint64_t n, uint64_t key) {
  uint64_t lo = 0, hi = n;
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (a[mid] < key) lo = mid + 1; else hi = mid;
  }
  return lo;
}

orc_flix *orc_flix_create(int key_bits) {
  orc_flix *f = (orc_flix *)xmalloc(sizeof(orc_flix));
  f->key_bits = key_bits == 32 ? 32 : 64;
  f->keys = NULL;
  f->values = NULL;
  f->size = 0;
  return f;
}

void orc_flix_destroy(orc_flix *f) {
  if (!f) return;
  free(f->keys);
  free(f->values);
  free(f);
}

uint64_t orc_flix_size(const orc_flix *f) { return f->size; }

uint64_t orc_flix_dump(const orc_flix *f, uint64_t *keys, uint32_t *values) {
  if (keys) memcpy(keys, f->keys, f->size * sizeof(uint64_t));
  if (values) memcpy(values, f->values, f->size * sizeof(uint32_t));
  return f->size;
}

static uint64_t key_mask(const orc_flix *f) {
  return f->key_bits == 32 ? 0xffffffffull : ~0ull;
}

void orc_flix_build(orc_flix *f, const uint64_t *keys, const uint32_t *values, uint64_t n) {
  free(f->keys);
  free(f->values);
  f->keys = (uint64_t *)xmalloc(n * sizeof(uint64_t));
  f->values = (uint32_t *)xmalloc(n * sizeof(uint32_t));
  const uint64_t mask = key_mask(f);
  for (uint64_t i = 0; i < n; ++i) {
    f->keys[i] = keys[i] & mask;
    f->values[i] = values ? values[i] : (uint32_t)i;
  }
  stable_sort_pairs_u64(f->keys, f->values, n, f->key_bits);
  f->size = keep_first_in_runs(f->keys, f->values, n);
}

void orc_flix_insert(orc_flix *f, const uint64_t *keys, const uint32_t *values, uint64_t n) {
  if (!n) return;
  const uint64_t mask = key_mask(f);
  uint64_t *bk = (uint64_t *)xmalloc(n * sizeof(uint64_t));
  uint32_t *bv = (uint32_t *)xmalloc(n * sizeof(uint32_t));
  for (uint64_t i = 0; i < n; ++i) {
    bk[i] = keys[i] & mask;
    bv[i] = values ? values[i] : (uint32_t)i;
  }
  stable_sort_pairs_u64(bk, bv, n, f->key_bits);
  const uint64_t m = keep_first_in_runs(bk, bv, n);
  uint64_t *ok = (uint64_t *)xmalloc((f->size + m) * sizeof(uint64_t));
  uint32_t *ov = (uint32_t *)xmalloc((f->size + m) * sizeof(uint32_t));
  uint64_t i = 0, j = 0, o = 0;
  while (i < f->size || j < m) {
    if (j >= m || (i < f->size && f->keys[i] < bk[j])) { ok[o] = f->keys[i]; ov[o] = f->values[i]; ++i; }
    else if (i >= f->size || bk[j] < f->keys[i]) { ok[o] = bk[j]; ov[o] = bv[j]; ++j; }
    else { ok[o] = f->keys[i]; ov[o] = f->values[i]; ++i; ++j; } /* present: keep */
    ++o;
  }
  free(f->keys);
  free(f->values);
  f->keys = ok;
  f->values = ov;
  f->size = o;
  free(bk);
  free(bv);
}

void orc_flix_remove(orc_flix *f, const uint64_t *keys, uint64_t n) {
  if (!n || !f->size) return;
  const uint64_t mask = key_mask(f);
  uint64_t *bk = (uint64_t *)xmalloc(n * sizeof(uint64_t));
  uint32_t *bv = (uint32_t *)xmalloc(n * sizeof(uint32_t));
  for (uint64_t i = 0; i < n; ++i) { bk[i] = keys[i] & mask; bv[i] = 0; }
  stable_sort_pairs_u64(bk, bv, n, f->key_bits);
  const uint64_t m = keep_first_in_runs(bk, bv, n);
  uint64_t i = 0, j = 0, o = 0;
  while (i < f->size) {
    while (j < m && bk[j] < f->keys[i]) ++j;
    if (j < m && bk[j] == f->keys[i]) { ++i; continue; }
    f->keys[o] = f->keys[i];
    f->values[o] = f->values[i];
    ++o; ++i;
  }
  f->size = o;
  free(bk);
  free(bv);
}

void orc_flix_lookup(const orc_flix *f, const uint64_t *probes, uint64_t n, uint32_t *out) {
  const uint64_t mask = key_mask(f);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    const uint64_t k = probes[i] & mask;
    const uint64_t p = lower_bound_u64(f->keys, f->size, k);
    out[i] = (p < f->size && f->keys[p] == k) ? f->values[p] : 0xffffffffu;
  }
}

void orc_flix_successor(const orc_flix *f, const uint64_t *probes, uint64_t n, uint64_t *out) {
  const uint64_t mask = key_mask(f);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    const uint64_t k = probes[i] & mask;
    const uint64_t p = lower_bound_u64(f->keys, f->size, k);
    out[i] = p < f->size ? f->keys[p] : 0xffffffffull;
  }
}
