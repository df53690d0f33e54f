// CPU baselines for the dictionary path, timed beside the GPU.  TEST
// INFRASTRUCTURE ONLY: bench.py's cpu_baseline leg and its --impl reference
// arm run them, tests check them against the oracle; nothing in the product
// links or calls them.
//
// The reference has no CPU implementation of this path (its only host code is
// the validation map of FliX/benchmarks_updates.cuh:1544-1557 and
// FliX/paper_lsmu_sweep.cu:464), so two CPU engines with GPULSMOpt's semantics
// stand in for it:
//
//  1. cpumap_*: a single-thread std::map.  Upsert with the last write of a
//     batch winning (GPULSMOpt.cuh:2578-2633), erase, lookup with the miss
//     convention of GPULSMOpt.cuh:4742-4749, range pairs in key order.
//  2. cpulsm_*: a multi-threaded leveled LSM on every host core.  Each batch
//     is sorted with the parallel-mode std::sort (__gnu_parallel::sort) on
//     (key, input index), the last write of each key kept; the run carries
//     down levels of capacity cap0 * R^i, merged in parallel over key-range
//     partitions (equal keys never straddle two threads; the newer run wins;
//     tombstones drop when nothing older lies below); lookups and range
//     queries run as OpenMP loops over the query batch, searching the levels
//     newest first with binary search.
#include <omp.h>
#include <parallel/algorithm>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

namespace {

constexpr uint32_t kMiss = 0xffffffffu;

// ---------------------------------------------------------------- std::map
struct CpuMap {
  std::map<uint32_t, uint32_t> m;
};

// ---------------------------------------------------------------- leveled LSM
struct Run {
  std::vector<uint32_t> k, v;
  std::vector<uint8_t> t;  // 1 = tombstone
  size_t size() const { return k.size(); }
  void clear() {
    k.clear();
    v.clear();
    t.clear();
  }
};

struct CpuLsm {
  std::vector<Run> levels;
  uint64_t cap0 = 1 << 22;
  uint32_t fan_in = 4;
  uint64_t cap(size_t i) const {
    uint64_t c = cap0;
    for (size_t j = 0; j < i; ++j) c *= fan_in;
    return c;
  }
};

int threads() { return omp_get_max_threads(); }

// Sorted run of a batch: stable order by key, the last write of each key kept.
Run batch_run(const uint32_t *keys, const uint32_t *vals, uint64_t n, bool tomb) {
  std::vector<uint64_t> packed(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(n); ++i) packed[i] = (uint64_t(keys[i]) << 32) | uint64_t(i);
  __gnu_parallel::sort(packed.begin(), packed.end());
  // keep the last entry of each key run
  std::vector<uint8_t> keep(n);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(n); ++i)
    keep[i] = (i + 1 == int64_t(n)) || ((packed[i] >> 32) != (packed[i + 1] >> 32));
  Run r;
  std::vector<uint64_t> pos(n + 1, 0);
  for (uint64_t i = 0; i < n; ++i) pos[i + 1] = pos[i] + keep[i];
  const uint64_t m = pos[n];
  r.k.resize(m);
  r.v.resize(m);
  r.t.assign(m, tomb ? 1 : 0);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < int64_t(n); ++i) {
    if (!keep[i]) continue;
    const uint64_t o = pos[i];
    r.k[o] = uint32_t(packed[i] >> 32);
    r.v[o] = tomb ? kMiss : vals[uint32_t(packed[i])];
  }
  return r;
}

// Merge newer run a with older run b; equal keys keep a's row; tombstones are
// dropped when drop is set.  Partitioned by key ranges so equal keys stay in
// one partition.
Run merge_runs(const Run &a, const Run &b, bool drop) {
  const int T = std::max(1, threads());
  const Run &big = a.size() >= b.size() ? a : b;
  if (!big.size()) return Run{};
  std::vector<uint32_t> pivots;  // partition t covers keys in [pivots[t-1], pivots[t])
  for (int t = 1; t < T; ++t) pivots.push_back(big.k[big.size() * size_t(t) / size_t(T)]);
  std::vector<std::pair<size_t, size_t>> ra(T), rb(T);
  for (int t = 0; t < T; ++t) {
    const size_t a0 = t == 0 ? 0 : size_t(std::lower_bound(a.k.begin(), a.k.end(), pivots[t - 1]) - a.k.begin());
    const size_t a1 = t == T - 1 ? a.size() : size_t(std::lower_bound(a.k.begin(), a.k.end(), pivots[t]) - a.k.begin());
    const size_t b0 = t == 0 ? 0 : size_t(std::lower_bound(b.k.begin(), b.k.end(), pivots[t - 1]) - b.k.begin());
    const size_t b1 = t == T - 1 ? b.size() : size_t(std::lower_bound(b.k.begin(), b.k.end(), pivots[t]) - b.k.begin());
    ra[t] = {a0, std::max(a0, a1)};
    rb[t] = {b0, std::max(b0, b1)};
  }
  std::vector<Run> parts(T);
#pragma omp parallel for schedule(static, 1)
  for (int t = 0; t < T; ++t) {
    Run &o = parts[t];
    size_t i = ra[t].first, ie = ra[t].second, j = rb[t].first, je = rb[t].second;
    o.k.reserve((ie - i) + (je - j));
    o.v.reserve((ie - i) + (je - j));
    o.t.reserve((ie - i) + (je - j));
    auto emit = [&](const Run &r, size_t x) {
      if (drop && r.t[x]) return;
      o.k.push_back(r.k[x]);
      o.v.push_back(r.v[x]);
      o.t.push_back(r.t[x]);
    };
    while (i < ie && j < je) {
      if (a.k[i] < b.k[j]) {
        emit(a, i++);
      } else if (b.k[j] < a.k[i]) {
        emit(b, j++);
      } else {
        emit(a, i++);
        ++j;
      }
    }
    while (i < ie) emit(a, i++);
    while (j < je) emit(b, j++);
  }
  std::vector<size_t> off(T + 1, 0);
  for (int t = 0; t < T; ++t) off[t + 1] = off[t] + parts[t].size();
  Run out;
  out.k.resize(off[T]);
  out.v.resize(off[T]);
  out.t.resize(off[T]);
#pragma omp parallel for schedule(static, 1)
  for (int t = 0; t < T; ++t) {
    std::memcpy(out.k.data() + off[t], parts[t].k.data(), parts[t].size() * 4);
    std::memcpy(out.v.data() + off[t], parts[t].v.data(), parts[t].size() * 4);
    std::memcpy(out.t.data() + off[t], parts[t].t.data(), parts[t].size());
  }
  return out;
}

bool nothing_below(const CpuLsm &d, size_t i) {
  for (size_t j = i + 1; j < d.levels.size(); ++j)
    if (d.levels[j].size()) return false;
  return true;
}

void apply_batch(CpuLsm &d, Run carry) {
  for (size_t i = 0;; ++i) {
    if (i == d.levels.size()) d.levels.emplace_back();
    Run &L = d.levels[i];
    const bool drop = nothing_below(d, i);
    if (L.size() == 0 && carry.size() <= d.cap(i)) {
      if (drop) carry = merge_runs(carry, Run{}, true);
      L = std::move(carry);
      return;
    }
    Run merged = merge_runs(carry, L, drop);
    if (merged.size() <= d.cap(i)) {
      L = std::move(merged);
      return;
    }
    L.clear();
    carry = std::move(merged);
  }
}

// Newest version of key q: 1 = live (value in *v), 0 = absent or erased.
inline int find_newest(const CpuLsm &d, uint32_t q, uint32_t *v) {
  for (const Run &L : d.levels) {
    if (!L.size()) continue;
    auto it = std::lower_bound(L.k.begin(), L.k.end(), q);
    if (it != L.k.end() && *it == q) {
      const size_t x = size_t(it - L.k.begin());
      if (L.t[x]) return 0;
      *v = L.v[x];
      return 1;
    }
  }
  return 0;
}

// Walks the live pairs of [lo, hi] in key order across levels (newest wins):
// the levels' slices of the range are merged two at a time, newest first, in
// thread-local buffers, and the live rows of the result are passed to f.
struct Slice {
  const uint32_t *k, *v;
  const uint8_t *t;
  size_t n;
};

template <class F> void walk_range(const CpuLsm &d, uint32_t lo, uint32_t hi, F &&f) {
  if (lo > hi) return;
  thread_local std::vector<uint32_t> ak, av, bk, bv;
  thread_local std::vector<uint8_t> at, bt;
  Slice acc{nullptr, nullptr, nullptr, 0};
  bool have = false, in_a = false;
  for (const Run &L : d.levels) {
    const size_t b = size_t(std::lower_bound(L.k.begin(), L.k.end(), lo) - L.k.begin());
    const size_t e = size_t(std::upper_bound(L.k.begin() + b, L.k.end(), hi) - L.k.begin());
    if (b == e) continue;
    const Slice s{L.k.data() + b, L.v.data() + b, L.t.data() + b, e - b};
    if (!have) {
      acc = s;
      have = true;
      continue;
    }
    // merge acc (newer) with s (older) into the buffer acc does not live in
    auto &ok = in_a ? bk : ak;
    auto &ov = in_a ? bv : av;
    auto &ot = in_a ? bt : at;
    ok.resize(acc.n + s.n);
    ov.resize(acc.n + s.n);
    ot.resize(acc.n + s.n);
    size_t i = 0, j = 0, o = 0;
    while (i < acc.n && j < s.n) {
      const uint32_t x = acc.k[i], y = s.k[j];
      if (x <= y) {
        ok[o] = x;
        ov[o] = acc.v[i];
        ot[o++] = acc.t[i++];
        j += (x == y);
      } else {
        ok[o] = y;
        ov[o] = s.v[j];
        ot[o++] = s.t[j++];
      }
    }
    for (; i < acc.n; ++i, ++o) ok[o] = acc.k[i], ov[o] = acc.v[i], ot[o] = acc.t[i];
    for (; j < s.n; ++j, ++o) ok[o] = s.k[j], ov[o] = s.v[j], ot[o] = s.t[j];
    acc = Slice{ok.data(), ov.data(), ot.data(), o};
    in_a = !in_a;
  }
  for (size_t i = 0; i < acc.n; ++i)
    if (!acc.t[i]) f(acc.k[i], acc.v[i]);
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- std::map
void *cpumap_create(void) { return new CpuMap(); }
void cpumap_destroy(void *h) { delete static_cast<CpuMap *>(h); }
uint64_t cpumap_size(void *h) { return static_cast<CpuMap *>(h)->m.size(); }

void cpumap_insert(void *h, const uint32_t *keys, const uint32_t *vals, uint64_t n) {
  auto &m = static_cast<CpuMap *>(h)->m;
  for (uint64_t i = 0; i < n; ++i) m[keys[i]] = vals[i];
}

void cpumap_erase(void *h, const uint32_t *keys, uint64_t n) {
  auto &m = static_cast<CpuMap *>(h)->m;
  for (uint64_t i = 0; i < n; ++i) m.erase(keys[i]);
}

void cpumap_lookup(void *h, const uint32_t *q, uint64_t n, uint32_t *out, uint8_t *found) {
  const auto &m = static_cast<CpuMap *>(h)->m;
  for (uint64_t i = 0; i < n; ++i) {
    auto it = m.find(q[i]);
    const bool hit = it != m.end();
    if (found) found[i] = hit;
    out[i] = hit ? it->second : (found ? 0u : kMiss);
  }
}

uint64_t cpumap_range_offsets(void *h, const uint32_t *lo, const uint32_t *hi, uint64_t n, uint64_t *offsets) {
  const auto &m = static_cast<CpuMap *>(h)->m;
  uint64_t total = 0;
  for (uint64_t i = 0; i < n; ++i) {
    offsets[i] = total;
    if (lo[i] > hi[i]) continue;
    for (auto it = m.lower_bound(lo[i]); it != m.end() && it->first <= hi[i]; ++it) ++total;
  }
  offsets[n] = total;
  return total;
}

void cpumap_range_pairs(void *h, const uint32_t *lo, const uint32_t *hi, uint64_t n, const uint64_t *offsets,
                        uint32_t *out_k, uint32_t *out_v) {
  const auto &m = static_cast<CpuMap *>(h)->m;
  for (uint64_t i = 0; i < n; ++i) {
    uint64_t o = offsets[i];
    if (lo[i] > hi[i]) continue;
    for (auto it = m.lower_bound(lo[i]); it != m.end() && it->first <= hi[i]; ++it) {
      out_k[o] = it->first;
      out_v[o++] = it->second;
    }
  }
}

// ---------------------------------------------------------------- leveled LSM
void *cpulsm_create(uint64_t cap0, uint32_t fan_in) {
  auto *d = new CpuLsm();
  if (cap0) d->cap0 = cap0;
  if (fan_in >= 2) d->fan_in = fan_in;
  return d;
}
void cpulsm_destroy(void *h) { delete static_cast<CpuLsm *>(h); }
void cpulsm_clear(void *h) { static_cast<CpuLsm *>(h)->levels.clear(); }
uint32_t cpulsm_levels(void *h) { return uint32_t(static_cast<CpuLsm *>(h)->levels.size()); }

void cpulsm_insert(void *h, const uint32_t *keys, const uint32_t *vals, uint64_t n) {
  if (n) apply_batch(*static_cast<CpuLsm *>(h), batch_run(keys, vals, n, false));
}

void cpulsm_erase(void *h, const uint32_t *keys, uint64_t n) {
  if (n) apply_batch(*static_cast<CpuLsm *>(h), batch_run(keys, nullptr, n, true));
}

void cpulsm_lookup(void *h, const uint32_t *q, uint64_t n, uint32_t *out, uint8_t *found) {
  const CpuLsm &d = *static_cast<CpuLsm *>(h);
#pragma omp parallel for schedule(static, 4096)
  for (int64_t i = 0; i < int64_t(n); ++i) {
    uint32_t v = 0;
    const int hit = find_newest(d, q[i], &v);
    if (found) found[i] = uint8_t(hit);
    out[i] = hit ? v : (found ? 0u : kMiss);
  }
}

uint64_t cpulsm_range_offsets(void *h, const uint32_t *lo, const uint32_t *hi, uint64_t n, uint64_t *offsets) {
  const CpuLsm &d = *static_cast<CpuLsm *>(h);
  std::vector<uint64_t> cnt(n);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < int64_t(n); ++i) {
    uint64_t c = 0;
    walk_range(d, lo[i], hi[i], [&](uint32_t, uint32_t) { ++c; });
    cnt[i] = c;
  }
  uint64_t total = 0;
  for (uint64_t i = 0; i < n; ++i) {
    offsets[i] = total;
    total += cnt[i];
  }
  offsets[n] = total;
  return total;
}

void cpulsm_range_pairs(void *h, const uint32_t *lo, const uint32_t *hi, uint64_t n, const uint64_t *offsets,
                        uint32_t *out_k, uint32_t *out_v) {
  const CpuLsm &d = *static_cast<CpuLsm *>(h);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < int64_t(n); ++i) {
    uint64_t o = offsets[i];
    walk_range(d, lo[i], hi[i], [&](uint32_t k, uint32_t v) {
      out_k[o] = k;
      out_v[o++] = v;
    });
  }
}

}  // extern "C"
