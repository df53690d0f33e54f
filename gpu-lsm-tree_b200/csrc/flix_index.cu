// Host engine of the FliX-style bucket layer (see flix_index.h / flix_kernels.cuh).
//
// Per batch: copy + sort (onesweep radix sort, key bits only up to the
// largest key) + dedup (first occurrence wins) + route the sorted keys to
// bucket runs + one warp per run walks that bucket's chain.  The host waits
// once per update batch, for the largest key (the number of sort passes) and
// the allocation-region fill; queries on sorted probes never wait.
#include "flix_index.h"

#include <algorithm>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>

#include "flix_kernels.cuh"
#include "model_api.h"
#include "radix_sort.cuh"

namespace gpulsm {

namespace {
constexpr size_t kAlign = 256;
// Unsorted lookup/successor batches up to this size go through the fence tree
// without sorting; larger ones are sorted first.  Measured on one B200 over a
// 2^26-key u64 index (successor, us): 2^10: 13 vs 102 sorted, 2^16: 15 vs 117,
// 2^18: 60 vs 132, 2^20: 212 vs 250, 2^22: 704 vs 587.
constexpr uint64_t kFenceProbeLimit = uint64_t(1) << 20;
size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

struct Bump {
  char *p;
  size_t off = 0;
  template <class T> T *take(size_t count) {
    T *r = reinterpret_cast<T *>(p + off);
    off += align_up(count * sizeof(T));
    return r;
  }
};

// small device-side counters read back by the host
struct DevCounters {
  unsigned long long inserted;
  unsigned long long removed;
  unsigned long long max_key;
  uint32_t alloc_top;
  uint32_t status;
  uint32_t flags;
  uint32_t n_unique;
  uint32_t pad[2];
};

void *dmalloc(size_t bytes, cudaStream_t s) {
  void *p = nullptr;
  if (cudaMallocAsync(&p, std::max<size_t>(bytes, 256), s) != cudaSuccess) {
    (void)cudaGetLastError();
    throw std::bad_alloc();
  }
  return p;
}
}  // namespace

struct FlixIndex::Impl {
  virtual ~Impl() = default;
  virtual void build(const void *keys, const uint32_t *values, uint64_t n, uint64_t max_n, cudaStream_t s) = 0;
  virtual void insert(const void *keys, const uint32_t *values, uint64_t n, cudaStream_t s) = 0;
  virtual void remove(const void *keys, uint64_t n, cudaStream_t s) = 0;
  virtual void lookups_ordered(const void *p, uint64_t n, uint32_t *out, cudaStream_t s) = 0;
  virtual void lookups_successor(const void *p, uint64_t n, void *out, cudaStream_t s) = 0;
  virtual void lookup(const void *p, uint64_t n, uint32_t *out, cudaStream_t s) = 0;
  virtual void successor(const void *p, uint64_t n, void *out, cudaStream_t s) = 0;
  virtual void rebuild(cudaStream_t s) = 0;
  virtual uint64_t resident_bytes() = 0;
  virtual uint64_t size() = 0;
  virtual uint32_t status() = 0;
  virtual void allocation_state(uint64_t *used, uint64_t *total, uint64_t *buckets, uint32_t *grows) = 0;
};

template <typename K>
class FlixImpl final : public FlixIndex::Impl {
 public:
  explicit FlixImpl(const FlixConfig &c) : cfg_(c) {
    const uint32_t ns = c.node_size ? c.node_size : flix::kNodeSize;
    if (ns != flix::kNodeSize) throw std::invalid_argument("node_size must be 32 (NODESIZE=5)");
    const uint32_t fill = c.fill_percent ? c.fill_percent : 50u;
    if (fill > 100) throw std::invalid_argument("fill_percent must be in [1, 100]");
    fill_ = std::max<uint32_t>(1, (flix::kNodeSize * fill + 99) / 100);
    if (c.search_mode > 1) throw std::invalid_argument("unknown search_mode");
    int dev = 0;
    GPULSM_CUDA(cudaGetDevice(&dev));
    GPULSM_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
    GPULSM_CUDA(cudaMalloc(&ctr_, sizeof(DevCounters)));
    GPULSM_CUDA(cudaMemset(ctr_, 0, sizeof(DevCounters)));
    GPULSM_CUDA(cudaMallocHost(&ctr_host_, sizeof(DevCounters)));
    std::memset(ctr_host_, 0, sizeof(DevCounters));
    GPULSM_CUDA(cudaEventCreateWithFlags(&op_done_, cudaEventDisableTiming));
    GPULSM_CUDA(cudaEventRecord(op_done_, 0));
  }

  ~FlixImpl() override {
    cudaDeviceSynchronize();
    if (nodes_) cudaFree(nodes_);
    if (bmax_) cudaFree(bmax_);
    if (fence_) cudaFree(fence_);
    if (scratch_) cudaFree(scratch_);
    if (model_) cudaFree(model_);
    if (ctr_) cudaFree(ctr_);
    if (ctr_host_) cudaFreeHost(ctr_host_);
    if (op_done_) cudaEventDestroy(op_done_);
  }

  // ---------------------------------------------------------------- build
  void build(const void *keys_v, const uint32_t *values, uint64_t n, uint64_t max_n, cudaStream_t s) override {
    if (n && !keys_v) throw std::invalid_argument("null keys");
    if (n > radix::kMaxKeys) throw std::length_error("FliX build limited to 2^30-1 keys per call");
    begin(s);
    const K *keys = static_cast<const K *>(keys_v);
    const uint32_t nn = uint32_t(n);
    // 1. inspect: sorted? unique? largest key
    GPULSM_CUDA(cudaMemsetAsync(ctr_, 0, sizeof(DevCounters), s));
    if (n) inspect(keys, n, s);
    read_counters(s);
    const bool sorted_unique = n == 0 || (ctr_host_->flags & 3u) == 0;
    const K *lay_keys = keys;
    const uint32_t *lay_vals = values;  // null -> value = input index
    uint64_t unique = n;
    char *tmp = nullptr;
    if (!sorted_unique) {
      // stable sort (key, value or input index), then keep the first of each key
      const int bits = key_bits_for(ctr_host_->max_key);
      const size_t kb = align_up(n * sizeof(K)), vb = align_up(n * 4);
      const size_t ws = align_up(radix::workspace_bytes(n, (bits + 7) / 8));
      const uint64_t dtiles = (n + flix::kDedupTile - 1) / flix::kDedupTile;
      const size_t total = 4 * kb + 4 * vb + ws + align_up(8) + align_up((dtiles + 1) * 8) + 256;
      tmp = static_cast<char *>(dmalloc(total, s));
      Bump b{tmp};
      K *k0 = b.take<K>(n), *k1 = b.take<K>(n), *ko = b.take<K>(n);
      uint32_t *v0 = b.take<uint32_t>(n), *v1 = b.take<uint32_t>(n), *vo = b.take<uint32_t>(n);
      char *zero_from = b.p + b.off;
      uint32_t *w = b.take<uint32_t>(ws / 4);
      uint32_t *counter = b.take<uint32_t>(2);
      unsigned long long *lb = b.take<unsigned long long>(dtiles + 1);
      GPULSM_CUDA(cudaMemsetAsync(zero_from, 0, (b.p + b.off) - zero_from, s));
      GPULSM_CUDA(cudaMemcpyAsync(k0, keys, n * sizeof(K), cudaMemcpyDeviceToDevice, s));
      if (values)
        GPULSM_CUDA(cudaMemcpyAsync(v0, values, n * 4, cudaMemcpyDeviceToDevice, s));
      else {
        flix::iota_kernel<K><<<grid_for(n, 256), 256, 0, s>>>(v0, nn); note_launch();
      }
      K *kk[2] = {k0, k1};
      uint32_t *vv[2] = {v0, v1};
      const int cur = radix::sort<K, true>(kk, vv, nn, 0, bits, w, &ctr_->status, num_sms_, s);
      flix::dedup_first_kernel<K><<<unsigned(dtiles), flix::kDedupThreads, 0, s>>>(
          kk[cur], vv[cur], nn, ko, vo, &ctr_->n_unique, lb, counter, &ctr_->status); note_launch();
      read_counters(s);
      unique = ctr_host_->n_unique;
      lay_keys = ko;
      lay_vals = vo;
    }
    // 2. allocate the node pool: heads + allocation region
    const uint64_t buckets = std::max<uint64_t>(1, (unique + fill_ - 1) / fill_);
    const uint64_t hint = std::max<uint64_t>({max_n, cfg_.max_elements, unique});
    // Splits create at most one node per 16 inserted keys plus one per node
    // that was already full; size for the hint with that slack (grown on demand).
    const uint64_t region = std::max<uint64_t>(
        {min_region_, 1024, (hint - unique) / (flix::kNodeSize / 4) + buckets / 4 + 1024});
    if (buckets + region >= 0xffffffffull) throw std::length_error("FliX node pool exceeds 2^32 nodes");
    release_pool(s);
    buckets_ = uint32_t(buckets);
    capacity_ = uint32_t(buckets + region);
    nodes_ = static_cast<flix::Node<K> *>(dmalloc(size_t(capacity_) * sizeof(flix::Node<K>), s));
    bmax_ = static_cast<K *>(dmalloc(size_t(buckets_) * sizeof(K), s));
    flix::build_layout_kernel<K><<<grid_for(uint64_t(buckets_) * 32, 256), 256, 0, s>>>(
        lay_keys, lay_vals, unique, fill_, buckets_, nodes_, bmax_); note_launch();
    // counters: live = unique, alloc_top = buckets
    DevCounters init{};
    init.inserted = unique;
    init.alloc_top = buckets_;
    *ctr_host_ = init;
    GPULSM_CUDA(cudaMemcpyAsync(ctr_, ctr_host_, sizeof(DevCounters), cudaMemcpyHostToDevice, s));
    GPULSM_CUDA(cudaStreamSynchronize(s));  // ctr_host_ is reused as the staging buffer
    if (tmp) GPULSM_CUDA(cudaFreeAsync(tmp, s));
    used_upper_ = buckets_;
    fit_routing_model(s);
    build_fences(s);
    built_ = true;
    end(s);
  }

  // ---------------------------------------------------------------- updates
  void insert(const void *keys_v, const uint32_t *values, uint64_t n, cudaStream_t s) override {
    if (!n) return;
    if (!keys_v || !values) throw std::invalid_argument("null insert batch");
    update(static_cast<const K *>(keys_v), values, n, true, s);
  }

  void remove(const void *keys_v, uint64_t n, cudaStream_t s) override {
    if (!n) return;
    if (!keys_v) throw std::invalid_argument("null delete batch");
    update(static_cast<const K *>(keys_v), nullptr, n, false, s);
  }

  // ---------------------------------------------------------------- queries
  void lookups_ordered(const void *p, uint64_t n, uint32_t *out, cudaStream_t s) override {
    if (!n) return;
    if (!p || !out) throw std::invalid_argument("null lookup");
    query(static_cast<const K *>(p), n, nullptr, out, nullptr, s);
  }

  void lookups_successor(const void *p, uint64_t n, void *out, cudaStream_t s) override {
    if (!n) return;
    if (!p || !out) throw std::invalid_argument("null successor");
    query(static_cast<const K *>(p), n, nullptr, nullptr, static_cast<K *>(out), s);
  }

  void lookup(const void *p, uint64_t n, uint32_t *out, cudaStream_t s) override {
    if (!n) return;
    if (!p || !out) throw std::invalid_argument("null lookup");
    if (n <= kFenceProbeLimit) fence_query(static_cast<const K *>(p), n, out, nullptr, s);
    else sorted_query(static_cast<const K *>(p), n, out, nullptr, s);
  }

  void successor(const void *p, uint64_t n, void *out, cudaStream_t s) override {
    if (!n) return;
    if (!p || !out) throw std::invalid_argument("null successor");
    if (n <= kFenceProbeLimit) fence_query(static_cast<const K *>(p), n, nullptr, static_cast<K *>(out), s);
    else sorted_query(static_cast<const K *>(p), n, nullptr, static_cast<K *>(out), s);
  }

  // ---------------------------------------------------------------- rebuild
  void rebuild(cudaStream_t s) override {
    require_built();
    begin(s);
    // 1. live entries per chain, exclusive scan; the scan total sizes the gather
    const uint32_t tiles = uint32_t(buckets_ / flix::kScanTile + 1);
    const size_t meta = align_up(size_t(buckets_) * 4) + align_up((size_t(buckets_) + 1) * 8) + align_up(8) +
                        align_up((tiles + 1) * 8);
    char *tmp = static_cast<char *>(dmalloc(meta, s));
    Bump b{tmp};
    uint32_t *counts = b.take<uint32_t>(buckets_);
    unsigned long long *offsets = b.take<unsigned long long>(size_t(buckets_) + 1);
    uint32_t *counter = b.take<uint32_t>(2);
    unsigned long long *lb = b.take<unsigned long long>(tiles + 1);
    GPULSM_CUDA(cudaMemsetAsync(counter, 0, (b.p + b.off) - reinterpret_cast<char *>(counter), s));
    flix::chain_counts_kernel<K><<<grid_for(buckets_, 256), 256, 0, s>>>(nodes_, buckets_, counts); note_launch();
    flix::scan_counts_kernel<K><<<tiles, flix::kScanThreads, 0, s>>>(counts, buckets_, offsets, lb, counter,
                                                                      &ctr_->status); note_launch();
    unsigned long long live = 0;
    GPULSM_CUDA(cudaMemcpyAsync(&live, offsets + buckets_, 8, cudaMemcpyDeviceToHost, s));
    GPULSM_CUDA(cudaStreamSynchronize(s));
    // 2. copy every chain, in key order, into one dense sorted array
    char *dense = static_cast<char *>(dmalloc(align_up(std::max<uint64_t>(live, 1) * sizeof(K)) +
                                                  align_up(std::max<uint64_t>(live, 1) * 4), s));
    K *keys = reinterpret_cast<K *>(dense);
    uint32_t *vals = reinterpret_cast<uint32_t *>(dense + align_up(std::max<uint64_t>(live, 1) * sizeof(K)));
    flix::gather_chains_kernel<K><<<grid_for(uint64_t(buckets_) * 32, 256), 256, 0, s>>>(
        nodes_, buckets_, offsets, keys, vals); note_launch();
    GPULSM_CUDA(cudaFreeAsync(tmp, s));
    tmp = dense;
    end(s);
    const uint64_t max_n = std::max<uint64_t>(cfg_.max_elements, live + (capacity_ - buckets_) * 8ull);
    // the gathered entries are sorted and unique: build lays them out directly
    build(keys, vals, live, max_n, s);
    GPULSM_CUDA(cudaFreeAsync(tmp, s));
  }

  uint64_t resident_bytes() override {
    return size_t(capacity_) * sizeof(flix::Node<K>) + size_t(buckets_) * sizeof(K) + fence_bytes_ + scratch_bytes_ +
           sizeof(DevCounters);
  }

  uint64_t size() override {
    GPULSM_CUDA(cudaEventSynchronize(op_done_));
    GPULSM_CUDA(cudaMemcpy(ctr_host_, ctr_, sizeof(DevCounters), cudaMemcpyDeviceToHost));
    return ctr_host_->inserted - ctr_host_->removed;
  }

  uint32_t status() override {
    GPULSM_CUDA(cudaEventSynchronize(op_done_));
    GPULSM_CUDA(cudaMemcpy(ctr_host_, ctr_, sizeof(DevCounters), cudaMemcpyDeviceToHost));
    return ctr_host_->status | status_bits_;
  }

  // allocation region: nodes taken by splits, nodes it holds, head buckets,
  // and how often it was grown (a rebuild into a larger region)
  void allocation_state(uint64_t *used, uint64_t *total, uint64_t *buckets, uint32_t *grows) override {
    GPULSM_CUDA(cudaEventSynchronize(op_done_));
    GPULSM_CUDA(cudaMemcpy(ctr_host_, ctr_, sizeof(DevCounters), cudaMemcpyDeviceToHost));
    const uint64_t top = std::min<uint64_t>(ctr_host_->alloc_top, capacity_);
    *used = top > buckets_ ? top - buckets_ : 0;
    *total = capacity_ > buckets_ ? capacity_ - buckets_ : 0;
    *buckets = buckets_;
    *grows = grows_;
  }

 private:
  void begin(cudaStream_t s) { GPULSM_CUDA(cudaStreamWaitEvent(s, op_done_, 0)); }
  void end(cudaStream_t s) { GPULSM_CUDA(cudaEventRecord(op_done_, s)); }
  void require_built() const {
    if (!built_) throw std::runtime_error("FliX index used before build");
  }

  static int key_bits_for(unsigned long long max_key) {
    int bits = 1;
    while (bits < int(sizeof(K) * 8) && (max_key >> bits)) ++bits;
    return ((bits + 7) / 8) * 8;
  }

  void inspect(const K *keys, uint64_t n, cudaStream_t s) {
    const unsigned blocks = std::min<unsigned>(grid_for(n, 256), unsigned(num_sms_) * 4u);
    flix::inspect_keys_kernel<K><<<blocks, 256, 0, s>>>(keys, n, &ctr_->flags, &ctr_->max_key); note_launch();
  }

  void read_counters(cudaStream_t s) {
    GPULSM_CUDA(cudaMemcpyAsync(ctr_host_, ctr_, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
    GPULSM_CUDA(cudaStreamSynchronize(s));
  }

  void release_pool(cudaStream_t s) {
    if (nodes_) GPULSM_CUDA(cudaFreeAsync(nodes_, s));
    if (bmax_) GPULSM_CUDA(cudaFreeAsync(bmax_, s));
    if (fence_) GPULSM_CUDA(cudaFreeAsync(fence_, s));
    nodes_ = nullptr;
    bmax_ = nullptr;
    fence_ = nullptr;
    fence_bytes_ = 0;
  }

  void *scratch(size_t bytes, cudaStream_t s) {
    bytes = align_up(std::max<size_t>(bytes, kAlign));
    if (bytes > scratch_bytes_) {
      if (scratch_) GPULSM_CUDA(cudaFreeAsync(scratch_, s));
      const size_t grow = std::max(bytes, scratch_bytes_ + scratch_bytes_ / 2);
      scratch_ = dmalloc(grow, s);
      scratch_bytes_ = grow;
    }
    return scratch_;
  }

  // search_mode 1: a piecewise-linear model over bmax[0, B-1) routes keys to
  // buckets instead of a full binary search (learned.cuh)
  static constexpr uint32_t kModelSegments = 4096;
  static constexpr uint32_t kModelIters = 8;
  void fit_routing_model(cudaStream_t s) {
    model_ready_ = false;
    if (cfg_.search_mode != 1 || buckets_ < 2) return;
    if (!model_) model_ = static_cast<char *>(dmalloc(learned::bytes_for(kModelSegments), s));
    learned::fit<K>(bmax_, uint64_t(buckets_) - 1, kModelSegments, kModelIters, model_, nullptr, s);
    model_ready_ = true;
  }
  const learned::ModelHeader *model_header() const {
    return model_ready_ ? reinterpret_cast<const learned::ModelHeader *>(model_) : nullptr;
  }
  const learned::Segment *model_segments() const {
    return model_ready_ ? reinterpret_cast<const learned::Segment *>(model_ + sizeof(learned::ModelHeader)) : nullptr;
  }

  struct Sorted {
    K *keys;
    uint32_t *vals;
    uint32_t *n_dev;
    flix::Run *runs;
    uint32_t *run_count;
  };

  // copy, sort (with values or a permutation), optional first-wins dedup, route to runs
  Sorted prepare(const K *keys, const uint32_t *vals, uint64_t n, bool with_vals, bool perm, bool dedup,
                 cudaStream_t s, bool route = true) {
    if (n > radix::kMaxKeys) throw std::length_error("FliX batch limited to 2^30-1 keys per call");
    const uint32_t nn = uint32_t(n);
    const bool carry = with_vals || perm;
    const uint64_t dtiles = (n + flix::kDedupTile - 1) / flix::kDedupTile;
    const uint64_t rtiles = (n + flix::kRouteTile - 1) / flix::kRouteTile;
    // largest key -> number of radix passes (one small read-back)
    GPULSM_CUDA(cudaMemsetAsync(&ctr_->max_key, 0, 8, s));
    GPULSM_CUDA(cudaMemsetAsync(&ctr_->flags, 0, 4, s));
    inspect(keys, n, s);
    read_counters(s);
    const int bits = key_bits_for(ctr_host_->max_key);
    const int passes = (bits + 7) / 8;
    const size_t ws = align_up(radix::workspace_bytes(n, passes));
    const size_t total = 3 * align_up(n * sizeof(K)) + 3 * align_up(n * 4) + align_up(size_t(n + 1) * 8) +
                         ws + 4 * align_up(8) + align_up((dtiles + 1) * 8) + align_up((rtiles + 1) * 8);
    Bump b{static_cast<char *>(scratch(total, s))};
    K *k0 = b.take<K>(n), *k1 = b.take<K>(n), *ko = b.take<K>(n);
    uint32_t *v0 = b.take<uint32_t>(n), *v1 = b.take<uint32_t>(n), *vo = b.take<uint32_t>(n);
    flix::Run *runs = b.take<flix::Run>(n + 1);
    char *zero_from = b.p + b.off;
    uint32_t *w = b.take<uint32_t>(ws / 4);
    uint32_t *n_dev = b.take<uint32_t>(2);
    uint32_t *run_count = b.take<uint32_t>(2);
    uint32_t *dctr = b.take<uint32_t>(2);
    uint32_t *rctr = b.take<uint32_t>(2);
    unsigned long long *dlb = b.take<unsigned long long>(dtiles + 1);
    unsigned long long *rlb = b.take<unsigned long long>(rtiles + 1);
    GPULSM_CUDA(cudaMemsetAsync(zero_from, 0, (b.p + b.off) - zero_from, s));
    // a batch that is already sorted (the reference's interface requires it)
    // is used in place: no copy, no sort, identity permutation
    const bool sorted_in = (ctr_host_->flags & 1u) == 0;
    const bool unique_in = (ctr_host_->flags & 2u) == 0;
    K *kk[2] = {k0, k1};
    uint32_t *vv[2] = {v0, v1};
    int cur = 0;
    if (sorted_in) {
      kk[0] = const_cast<K *>(keys);  // read only below
      vv[0] = with_vals ? const_cast<uint32_t *>(vals) : nullptr;
    } else {
      GPULSM_CUDA(cudaMemcpyAsync(k0, keys, n * sizeof(K), cudaMemcpyDeviceToDevice, s));
      if (with_vals) GPULSM_CUDA(cudaMemcpyAsync(v0, vals, n * 4, cudaMemcpyDeviceToDevice, s));
      if (perm) {
        flix::iota_kernel<K><<<grid_for(n, 256), 256, 0, s>>>(v0, nn); note_launch();
      }
      cur = carry ? radix::sort<K, true>(kk, vv, nn, 0, bits, w, &ctr_->status, num_sms_, s)
                  : radix::sort<K, false>(kk, vv, nn, 0, bits, w, &ctr_->status, num_sms_, s);
    }
    Sorted out{kk[cur], (sorted_in && !with_vals) ? nullptr : (carry ? vv[cur] : nullptr), n_dev, runs, run_count};
    if (dedup && !unique_in) {
      flix::dedup_first_kernel<K><<<unsigned(std::max<uint64_t>(dtiles, 1)), flix::kDedupThreads, 0, s>>>(
          kk[cur], carry ? vv[cur] : nullptr, nn, ko, carry ? vo : nullptr, n_dev, dlb, dctr,
          &ctr_->status); note_launch();
      out.keys = ko;
      out.vals = carry ? vo : nullptr;
    } else {
      flix::set_u32_kernel<K><<<1, 1, 0, s>>>(n_dev, nn); note_launch();
    }
    if (route) {
      flix::route_runs_kernel<K><<<unsigned(std::max<uint64_t>(rtiles, 1)), flix::kRouteThreads, 0, s>>>(
          out.keys, n_dev, bmax_, buckets_, runs, run_count, rlb, rctr, &ctr_->status, model_header(),
          model_segments()); note_launch();
    }
    return out;
  }

  // Compacts the chains into a fresh layout whose allocation region holds at
  // least `need` more nodes (FliX's rebuild, plus growth).
  void grow(uint64_t need, cudaStream_t s) {
    min_region_ = std::max<uint64_t>({min_region_, 2ull * (capacity_ - buckets_), need + 1024});
    ++grows_;
    rebuild(s);
  }

  void update(const K *keys, const uint32_t *vals, uint64_t n, bool is_insert, cudaStream_t s) {
    require_built();
    for (int attempt = 0;; ++attempt) {
      if (is_insert) {
        // expected new nodes: one per 16 inserted keys plus slack; a shortfall
        // is reported by the kernel (status bit 3) and handled below
        const uint64_t need = n / 8 + 1024;
        if (uint64_t(used_upper_) + need > capacity_) {
          begin(s);
          read_counters(s);
          end(s);
          used_upper_ = ctr_host_->alloc_top;
          if (uint64_t(used_upper_) + need > capacity_) grow(need, s);
        }
      }
      begin(s);
      Sorted st = prepare(keys, vals, n, is_insert, false, true, s);
      // persistent warps: the CTAs every SM holds at once, never more than one warp per key
      int per_sm = 1;
      GPULSM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &per_sm, is_insert ? reinterpret_cast<const void *>(flix::insert_runs_kernel<K>)
                             : reinterpret_cast<const void *>(flix::delete_runs_kernel<K>),
          flix::kUpdateThreads, 0));
      const unsigned grid = std::min<unsigned>(grid_for(n * 32, flix::kUpdateThreads),
                                               unsigned(num_sms_) * unsigned(std::max(per_sm, 1)));
      flix::PoolView pool{&ctr_->alloc_top, capacity_, &ctr_->status};
      if (is_insert) {
        flix::insert_runs_kernel<K><<<grid, flix::kUpdateThreads, 0, s>>>(
            st.keys, st.vals, st.n_dev, st.runs, st.run_count, nodes_, pool, &ctr_->inserted);
        note_launch();
      } else {
        flix::delete_runs_kernel<K><<<grid, flix::kUpdateThreads, 0, s>>>(st.keys, st.n_dev, st.runs,
                                                                           st.run_count, nodes_, &ctr_->removed);
        note_launch();
      }
      GPULSM_CUDA(cudaGetLastError());
      if (!is_insert) {
        end(s);
        return;
      }
      // the region fill and overflow bit come back with one small read
      read_counters(s);
      end(s);
      used_upper_ = uint32_t(std::min<uint64_t>(ctr_host_->alloc_top, capacity_));
      if (!(ctr_host_->status & kDevOutputOverflow)) return;
      // keys that found no free node were skipped, not dropped: grow and
      // re-run the batch (insert-if-absent makes the retry idempotent)
      if (attempt == 3) throw std::runtime_error("FliX allocation region capacity exhausted");
      begin(s);
      flix::set_u32_kernel<K><<<1, 1, 0, s>>>(&ctr_->status, ctr_host_->status & ~kDevOutputOverflow);
      note_launch();
      end(s);
      grow(n / 4 + 1024, s);
    }
  }

  // sorted probes: route, then one warp per run
  void query(const K *probes, uint64_t n, const uint32_t *perm, uint32_t *out_v, K *out_k, cudaStream_t s) {
    require_built();
    if (n > radix::kMaxKeys) throw std::length_error("FliX query limited to 2^30-1 probes per call");
    begin(s);
    Bump b{static_cast<char *>(scratch(align_up(8), s))};
    uint32_t *n_dev = b.take<uint32_t>(2);
    flix::set_u32_kernel<K><<<1, 1, 0, s>>>(n_dev, uint32_t(n)); note_launch();
    direct_queries(probes, n_dev, n, perm, out_v, out_k, s);
    end(s);
  }

  void run_queries(const K *probes, const uint32_t *n_dev, const flix::Run *runs, const uint32_t *run_count,
                   uint64_t n, const uint32_t *perm, uint32_t *out_v, K *out_k, cudaStream_t s) {
    const unsigned grid = grid_for(n * 32, 256);
    if (out_v) {
      flix::lookup_runs_kernel<K><<<grid, 256, 0, s>>>(probes, n_dev, runs, run_count, nodes_, perm, out_v); note_launch();
    } else {
      flix::successor_runs_kernel<K><<<grid, 256, 0, s>>>(probes, n_dev, runs, run_count, nodes_, buckets_, perm,
                                                           out_k); note_launch();
    }
    GPULSM_CUDA(cudaGetLastError());
  }

  // sorted probes, one thread each (routing by the model in search mode 1)
  void direct_queries(const K *probes, const uint32_t *n_dev, uint64_t n, const uint32_t *perm, uint32_t *out_v,
                      K *out_k, cudaStream_t s) {
    const unsigned grid = grid_for(std::max<uint64_t>(n, 1), 256);
    if (out_v) {
      flix::lookup_direct_kernel<K><<<grid, 256, 0, s>>>(probes, n_dev, bmax_, buckets_, model_header(),
                                                         model_segments(), nodes_, perm, out_v);
    } else {
      flix::successor_direct_kernel<K><<<grid, 256, 0, s>>>(probes, n_dev, bmax_, buckets_, model_header(),
                                                            model_segments(), nodes_, perm, out_k);
    }
    note_launch();
    GPULSM_CUDA(cudaGetLastError());
  }

  // The fence tree over the bucket maxima (flix_kernels.cuh), rebuilt with
  // the bucket layer; bmax does not change between builds.
  void build_fences(cudaStream_t s) {
    if (fence_) GPULSM_CUDA(cudaFreeAsync(fence_, s));
    fence_ = nullptr;
    fence_bytes_ = 0;
    tree_ = flix::FenceTree<K>{};
    tree_.level[0] = bmax_;
    tree_.size[0] = buckets_;
    tree_.levels = 1;
    uint32_t sizes[flix::kMaxFenceLevels] = {};
    uint64_t total = 0;
    uint32_t m = buckets_;
    while (m > flix::kFenceFan && tree_.levels < uint32_t(flix::kMaxFenceLevels)) {
      m = (m + flix::kFenceFan - 1) / flix::kFenceFan;
      sizes[tree_.levels++] = m;
      total += m;
    }
    if (!total) return;
    fence_bytes_ = align_up(total * sizeof(K));
    fence_ = static_cast<K *>(dmalloc(fence_bytes_, s));
    K *at = fence_;
    for (uint32_t l = 1; l < tree_.levels; ++l) {
      tree_.level[l] = at;
      tree_.size[l] = sizes[l];
      flix::fence_level_kernel<K><<<grid_for(sizes[l], 256), 256, 0, s>>>(tree_.level[l - 1], tree_.size[l - 1], at,
                                                                            sizes[l]);
      note_launch();
      at += sizes[l];
    }
    GPULSM_CUDA(cudaGetLastError());
  }

  // small unsorted batches: one thread per probe, routed by the fence tree (or
  // the learned model), no sort and no permutation
  void fence_query(const K *probes, uint64_t n, uint32_t *out_v, K *out_k, cudaStream_t s) {
    require_built();
    begin(s);
    const unsigned grid = grid_for(n, 256);
    if (out_v) {
      flix::lookup_fence_kernel<K><<<grid, 256, 0, s>>>(probes, uint32_t(n), tree_, model_header(), model_segments(),
                                                        nodes_, out_v);
    } else {
      flix::successor_fence_kernel<K><<<grid, 256, 0, s>>>(probes, uint32_t(n), tree_, model_header(),
                                                           model_segments(), nodes_, out_k);
    }
    note_launch();
    GPULSM_CUDA(cudaGetLastError());
    end(s);
  }

  // unsorted probes: sort with a permutation, walk, write results in input order
  void sorted_query(const K *probes, uint64_t n, uint32_t *out_v, K *out_k, cudaStream_t s) {
    require_built();
    begin(s);
    Sorted st = prepare(probes, nullptr, n, false, true, false, s, false);
    direct_queries(st.keys, st.n_dev, n, st.vals, out_v, out_k, s);
    end(s);
  }

  FlixConfig cfg_;
  uint32_t fill_ = 16;
  int num_sms_ = 148;
  flix::Node<K> *nodes_ = nullptr;
  K *bmax_ = nullptr;
  K *fence_ = nullptr;  // levels 1.. of the fence tree over bmax
  size_t fence_bytes_ = 0;
  flix::FenceTree<K> tree_{};
  uint32_t buckets_ = 0;
  uint32_t capacity_ = 0;
  uint32_t used_upper_ = 0;
  uint64_t min_region_ = 0;
  uint32_t grows_ = 0;
  bool built_ = false;
  DevCounters *ctr_ = nullptr;
  char *model_ = nullptr;  // learned routing model over bmax (search_mode 1)
  bool model_ready_ = false;
  DevCounters *ctr_host_ = nullptr;
  void *scratch_ = nullptr;
  size_t scratch_bytes_ = 0;
  uint32_t status_bits_ = 0;
  cudaEvent_t op_done_ = nullptr;
};

// ----------------------------------------------------------------------------
FlixIndex::FlixIndex(const FlixConfig &config) {
  if (config.key_bits == 32)
    impl_ = std::make_unique<FlixImpl<uint32_t>>(config);
  else if (config.key_bits == 64)
    impl_ = std::make_unique<FlixImpl<unsigned long long>>(config);
  else
    throw std::invalid_argument("key_bits must be 32 or 64");
}

FlixIndex::~FlixIndex() = default;

void FlixIndex::build(const void *keys, const uint32_t *values, uint64_t n, uint64_t max_n, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  impl_->build(keys, values, n, max_n, s);
}
void FlixIndex::insert(const void *keys, const uint32_t *values, uint64_t n, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  impl_->insert(keys, values, n, s);
}
void FlixIndex::remove(const void *keys, uint64_t n, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  impl_->remove(keys, n, s);
}
void FlixIndex::lookups_ordered(const void *p, uint64_t n, uint32_t *out, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  impl_->lookups_ordered(p, n, out, s);
}
void FlixIndex::lookups_successor(const void *p, uint64_t n, void *out, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  impl_->lookups_successor(p, n, out, s);
}
void FlixIndex::lookup(const void *p, uint64_t n, uint32_t *out, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  impl_->lookup(p, n, out, s);
}
void FlixIndex::successor(const void *p, uint64_t n, void *out, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  impl_->successor(p, n, out, s);
}
void FlixIndex::rebuild(cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  impl_->rebuild(s);
}
uint64_t FlixIndex::resident_bytes() {
  std::lock_guard<std::mutex> g(mu_);
  return impl_->resident_bytes();
}
uint64_t FlixIndex::size() {
  std::lock_guard<std::mutex> g(mu_);
  return impl_->size();
}
uint32_t FlixIndex::status() {
  std::lock_guard<std::mutex> g(mu_);
  return impl_->status();
}
void FlixIndex::allocation_state(uint64_t *used, uint64_t *total, uint64_t *buckets, uint32_t *grows) {
  std::lock_guard<std::mutex> g(mu_);
  impl_->allocation_state(used, total, buckets, grows);
}

}  // namespace gpulsm
