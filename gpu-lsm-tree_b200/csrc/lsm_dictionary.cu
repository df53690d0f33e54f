// Host engine of the LSM dictionary (see lsm_dictionary.h).
//
// Structure: levels 0..L-1 are sorted runs of unique keys; level 0 is the
// newest.  Level i holds at most caps_[i] rows (cap_0 * fan_in^i); the last
// level is the foundation and takes whatever the cascade delivers.  An update
// batch is radix-sorted, deduplicated (last input index wins) and carried
// down: it absorbs every level it cannot fit beside, then lands in the first
// level with room (leveling with fan-in R).  Tombstones are dropped by the
// merge whose output has no older level beneath it.
//
// The host never waits for row counts.  It plans with upper bounds (dedup and
// tombstone drops only shrink runs); kernels read the exact counts from the
// device-side LevelDesc.  Exact counts come back through an asynchronous
// receipt that the next call applies if it has arrived - the same lazy
// receipt idea as GPULSMOpt's publication receipt (GPULSMOpt.cuh:6750-6811).
//
// Streams.  An update admits its batch on the caller's stream (which orders
// the reads of the caller's input) and enqueues the batch's merges on the
// dictionary's own merge stream, behind an event on that admission; the call
// returns and the next batch's admission overlaps these merges.  Every other
// operation first makes its stream wait for the merge stream.  Admission and
// merges therefore use separate scratch, and a run buffer released on one
// stream is reused on the other only behind the event of its release.
#include "lsm_dictionary.h"

#include <algorithm>
#include <atomic>
#include <thread>
#include <chrono>
#include <cstring>
#include <new>
#include <stdexcept>

#include "lsm_admit.cuh"
#include "lsm_kernels.cuh"
#include "model_api.h"
#include "radix_sort.cuh"

namespace gpulsm {

using lsm::LevelDesc;

namespace {
constexpr uint64_t kMaxBatch = uint64_t{1} << 20;  // kMaximumOperationTile, GPULSMOpt.cuh:56
constexpr size_t kAlign = 256;
// learned search: levels of at least this many rows get a model, with about
// kRowsPerSegment rows per segment and kFitIters gradient steps
constexpr uint64_t kLearnedMinRows = uint64_t(1) << 22;
constexpr uint64_t kRowsPerSegment = 64;
constexpr uint32_t kFitIters = 2;
constexpr uint32_t kMaxSegments = 1u << 22;

size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

// Standalone receipt, for an update that merges nothing and for a bulk build
// (an update that merges has its final merge kernel write the receipt).
__global__ void receipt_kernel(lsm::ReceiptSrc src) {
  chain_wait();
  lsm::write_receipt(src, 0ull);
}

// Bump allocator over one zeroed scratch region.
struct Bump {
  char *p;
  size_t off = 0;
  template <class T> T *take(size_t count) {
    T *r = reinterpret_cast<T *>(p + off);
    off += align_up(count * sizeof(T));
    return r;
  }
};

size_t merge_scratch_bytes(uint64_t rows) {
  const uint64_t tiles = (rows + lsm::kMergeTile - 1) / lsm::kMergeTile + 1;
  return align_up(8) + align_up(tiles * 8);
}
}  // namespace

struct LsmDictionary::Receipt {
  unsigned long long w[lsm::kReceiptWords];  // tagged counts, then the tagged status
};

// ----------------------------------------------------------------------------
RunPool::~RunPool() {
  for (auto &b : all_) {
    if (b->block) cudaFree(b->block);
    if (b->model) cudaFree(b->model);
    if (b->freed) cudaEventDestroy(b->freed);
  }
  if (trim_pool_) cudaMemPoolTrimTo(trim_pool_, 0);  // freed memory goes back to the driver
}

RunBuffer *RunPool::acquire(uint64_t min_rows, cudaStream_t stream, bool settled_only) {
  uint64_t cap = 1024;
  while (cap < min_rows) cap <<= 1;
  const auto settled = [&](const RunBuffer *f) {
    return !f->released || f->freed_on == stream || f->freed_epoch + 2 <= epoch_;
  };
  RunBuffer *best = nullptr, *young = nullptr;
  size_t best_i = 0, young_i = 0;
  for (size_t i = 0; i < free_.size(); ++i) {
    RunBuffer *f = free_[i];
    if (f->cap < cap || f->cap > cap * 2) continue;
    if (!settled_only || settled(f)) {
      if (!best || f->cap < best->cap) best = f, best_i = i;
    } else if (!young || f->cap < young->cap) {
      young = f, young_i = i;
    }
  }
  auto take = [&](RunBuffer *f, size_t i) {
    free_.erase(free_.begin() + i);
    if (f->released && f->freed_on != stream) GPULSM_CUDA(cudaStreamWaitEvent(stream, f->freed, 0));
    f->model_ok = false;
    f->model_rows = 0;
    f->dir_ok = false;
    return f;
  };
  if (best) return take(best, best_i);
  auto b = std::make_unique<RunBuffer>();
  b->cap = cap;
  const uint32_t cl2 = ceil_log2_u64(cap);
  b->dir_bits = std::max<uint32_t>(1, cl2 > rows_log2_ ? cl2 - rows_log2_ : 1);
  const size_t kb = align_up(cap * 4), vb = align_up(cap * 4), fb = align_up(cap),
               db = align_up(((size_t(1) << b->dir_bits) + 1) * 4), sb = align_up(sizeof(LevelDesc));
  b->bytes = kb + vb + fb + db + sb;
  cudaError_t e = cudaMallocAsync(&b->block, b->bytes, stream);
  if (e != cudaSuccess && young) {
    (void)cudaGetLastError();
    return take(young, young_i);  // out of memory: wait for the young buffer instead
  }
  if (e != cudaSuccess) {
    // give cached free buffers back and retry once
    (void)cudaGetLastError();
    release_all_free(stream);
    e = cudaMallocAsync(&b->block, b->bytes, stream);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      throw std::bad_alloc();
    }
  }
  char *p = static_cast<char *>(b->block);
  b->keys = reinterpret_cast<uint32_t *>(p);
  b->vals = reinterpret_cast<uint32_t *>(p + kb);
  b->flags = reinterpret_cast<uint8_t *>(p + kb + vb);
  b->dir = reinterpret_cast<uint32_t *>(p + kb + vb + fb);
  b->desc = reinterpret_cast<LevelDesc *>(p + kb + vb + fb + db);
  bytes_ += b->bytes;
  all_.push_back(std::move(b));
  return all_.back().get();
}

void RunPool::release(RunBuffer *b, cudaStream_t stream) {
  if (!b) return;
  if (!b->freed) GPULSM_CUDA(cudaEventCreateWithFlags(&b->freed, cudaEventDisableTiming));
  GPULSM_CUDA(cudaEventRecord(b->freed, stream));
  b->freed_on = stream;
  b->freed_epoch = epoch_;
  b->released = true;
  free_.push_back(b);
}

void RunPool::release_all_free(cudaStream_t stream) {
  for (RunBuffer *f : free_) {
    if (f->released && f->freed_on != stream) cudaStreamWaitEvent(stream, f->freed, 0);
    cudaFreeAsync(f->block, stream);
    if (f->model) cudaFreeAsync(f->model, stream);
    f->model = nullptr;
    if (f->freed) cudaEventDestroy(f->freed);
    f->freed = nullptr;
    bytes_ -= f->bytes + f->model_cap;
    for (size_t i = 0; i < all_.size(); ++i)
      if (all_[i].get() == f) {
        all_[i]->block = nullptr;
        all_.erase(all_.begin() + i);
        break;
      }
  }
  free_.clear();
}

// ----------------------------------------------------------------------------
LsmDictionary::LsmDictionary(const DictConfig &config)
    : cfg_(config), pool_(config.rows_per_bucket_log2 ? config.rows_per_bucket_log2 : 3u) {
  batch_capacity_ = std::min<uint64_t>(kMaxBatch, std::max<uint64_t>(1, config.batch_capacity
                                                                             ? config.batch_capacity
                                                                             : kMaxBatch));
  fan_in_ = config.fan_in ? config.fan_in : 4u;
  if (fan_in_ < 2 || fan_in_ > 16) throw std::invalid_argument("fan_in must be in [2, 16]");
  rows_log2_ = config.rows_per_bucket_log2 ? config.rows_per_bucket_log2 : 3u;
  if (rows_log2_ > 16) throw std::invalid_argument("rows_per_bucket_log2 must be <= 16");
  if (config.search_mode > 2) throw std::invalid_argument("unknown search_mode");
  // publication capacity as in initial_storage_capacity (GPULSMOpt.cuh:255-263)
  budget_ = std::max<uint64_t>(config.max_elements, batch_capacity_ * 16u);
  if (budget_ > 0xffffffffull)
    throw std::invalid_argument("capacity exceeds 32-bit key space");
  uint64_t cap = config.level_zero_capacity ? config.level_zero_capacity : batch_capacity_ * fan_in_;
  cap = std::min(cap, budget_);
  while (cap < budget_) {
    caps_.push_back(cap);
    cap = cap > budget_ / fan_in_ ? budget_ : cap * fan_in_;
    if (caps_.size() >= size_t(lsm::kMaxLevels) - 1)
      throw std::invalid_argument("level schedule exceeds 16 levels; raise level_zero_capacity");
  }
  caps_.push_back(budget_);
  levels_.assign(caps_.size(), Level{});
  receipt_gens_.assign(caps_.size(), 0);

  int dev = 0;
  GPULSM_CUDA(cudaGetDevice(&dev));
  GPULSM_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
  // Runs, prefixes and scratch are stream-ordered allocations from the
  // device's default pool.  By default the pool returns freed memory to the
  // driver at every synchronisation, so a buffer allocated again later maps
  // fresh memory on the calling thread (tens of milliseconds for hundreds of
  // MB, a stall a serving loop sees in its latency tail).  The pool keeps
  // freed memory instead (a property of this process's pool; the run pool's
  // destructor trims what is unused).
  cudaMemPool_t mem_pool = nullptr;
  GPULSM_CUDA(cudaDeviceGetDefaultMemPool(&mem_pool, dev));
  uint64_t keep = ~0ull;
  GPULSM_CUDA(cudaMemPoolSetAttribute(mem_pool, cudaMemPoolAttrReleaseThreshold, &keep));
  pool_.trim_on_destroy(mem_pool);
  GPULSM_CUDA(cudaFuncSetAttribute(lsm::admit::admit_bucket_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(lsm::admit::kBucketSmemBytes)));
  // two bucket CTAs per SM need nearly all of its shared memory
  GPULSM_CUDA(cudaFuncSetAttribute(lsm::admit::admit_bucket_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                   int(cudaSharedmemCarveoutMaxShared)));
  GPULSM_CUDA(cudaMalloc(&dev_status_, 256));
  GPULSM_CUDA(cudaMalloc(&table_dev_, sizeof(lsm::LevelSet)));
  GPULSM_CUDA(cudaMemset(dev_status_, 0, 256));
  // the receipt kernel writes the pinned host copy directly (no copy in the stream)
  GPULSM_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&receipt_host_), sizeof(Receipt), cudaHostAllocMapped));
  std::memset(receipt_host_, 0, sizeof(Receipt));
  GPULSM_CUDA(cudaHostGetDevicePointer(&receipt_dev_, receipt_host_, 0));
  GPULSM_CUDA(cudaMalloc(&width_, 8));
  GPULSM_CUDA(cudaMallocHost(&width_host_, 8));
  GPULSM_CUDA(cudaEventCreateWithFlags(&op_done_, cudaEventDisableTiming));
  GPULSM_CUDA(cudaEventRecord(op_done_, 0));
  GPULSM_CUDA(cudaStreamCreateWithFlags(&merge_stream_, cudaStreamNonBlocking));
  GPULSM_CUDA(cudaEventCreateWithFlags(&adm_done_, cudaEventDisableTiming));
  GPULSM_CUDA(cudaEventCreateWithFlags(&merge_done_, cudaEventDisableTiming));
  GPULSM_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
  GPULSM_CUDA(cudaEventCreateWithFlags(&side_done_, cudaEventDisableTiming));
}

LsmDictionary::~LsmDictionary() {
  if (op_done_) cudaEventSynchronize(op_done_);
  cudaDeviceSynchronize();
  for (auto &w : words_)
    if (w) cudaFree(w);
  if (scratch_) cudaFree(scratch_);
  if (dev_status_) cudaFree(dev_status_);
  if (receipt_host_) cudaFreeHost(receipt_host_);
  if (prefix_) cudaFree(prefix_);
  if (trace_dev_) cudaFree(trace_dev_);
  if (table_dev_) cudaFree(table_dev_);
  for (auto &t : traces_) {
    cudaEventDestroy(t.start);
    cudaEventDestroy(t.stop);
  }
  for (cudaEvent_t e : spare_events_) cudaEventDestroy(e);
  for (auto &lp : live_)
    if (lp.p) cudaFree(lp.p);
  for (auto &lp : live_staged_)
    if (lp.p) cudaFree(lp.p);
  if (width_) cudaFree(width_);
  if (width_host_) cudaFreeHost(width_host_);
  if (ascratch_) cudaFree(ascratch_);
  if (stage_in_) cudaFree(stage_in_);
  for (auto &w : stage_words_)
    if (w) cudaFree(w);
  if (stage_scratch_) cudaFree(stage_scratch_);
  if (op_done_) cudaEventDestroy(op_done_);
  if (adm_done_) cudaEventDestroy(adm_done_);
  if (merge_done_) cudaEventDestroy(merge_done_);
  if (fork_) cudaEventDestroy(fork_);
  if (side_done_) cudaEventDestroy(side_done_);
  if (merge_stream_) cudaStreamDestroy(merge_stream_);
}

// Operations are ordered by op_done_ across streams; on the stream of the
// previous operation the stream order already holds (not for the per-thread
// default stream, whose handle names a different stream in every thread).
void LsmDictionary::begin_op(cudaStream_t s, bool update) {
  if (!(last_stream_known_ && s == last_stream_ && s != cudaStreamPerThread))
    GPULSM_CUDA(cudaStreamWaitEvent(s, op_done_, 0));
  if (!update && merges_pending_) {  // everything but an update reads the merged levels
    GPULSM_CUDA(cudaStreamWaitEvent(s, merge_done_, 0));
    merges_pending_ = false;
  }
}

void LsmDictionary::end_op(cudaStream_t s) {
  GPULSM_CUDA(cudaEventRecord(op_done_, s));
  last_stream_ = s;
  last_stream_known_ = true;
}

// Completion of every operation enqueued so far, merges included, on the host.
void LsmDictionary::host_sync() {
  GPULSM_CUDA(cudaEventSynchronize(op_done_));
  if (merges_pending_) GPULSM_CUDA(cudaEventSynchronize(merge_done_));
}

void LsmDictionary::join(cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  begin_op(s);
  end_op(s);
}

// Admission's own scratch: the next batch is admitted while the merges of the
// previous one still use scratch_.
void *LsmDictionary::admit_scratch(size_t bytes, cudaStream_t s) {
  bytes = align_up(std::max<size_t>(bytes, kAlign));
  if (bytes > ascratch_bytes_) {
    if (ascratch_) GPULSM_CUDA(cudaFreeAsync(ascratch_, s));
    size_t grow = std::max(bytes, ascratch_bytes_ * 2);
    if (cudaMallocAsync(&ascratch_, grow, s) != cudaSuccess) {
      (void)cudaGetLastError();
      ascratch_ = nullptr;
      ascratch_bytes_ = 0;
      throw std::bad_alloc();
    }
    ascratch_bytes_ = grow;
  }
  return ascratch_;
}

void *LsmDictionary::scratch(size_t bytes, cudaStream_t s) {
  bytes = align_up(std::max<size_t>(bytes, kAlign));
  if (bytes > scratch_bytes_) {
    if (scratch_) GPULSM_CUDA(cudaFreeAsync(scratch_, s));
    size_t grow = std::max(bytes, scratch_bytes_ * 2);
    if (cudaMallocAsync(&scratch_, grow, s) != cudaSuccess) {
      (void)cudaGetLastError();
      scratch_ = nullptr;
      scratch_bytes_ = 0;
      throw std::bad_alloc();
    }
    scratch_bytes_ = grow;
  }
  return scratch_;
}

void LsmDictionary::ensure_sort_space(uint64_t n, cudaStream_t s) {
  if (n <= words_cap_) return;
  for (auto &w : words_) {
    if (w) GPULSM_CUDA(cudaFreeAsync(w, s));
    w = nullptr;
  }
  uint64_t cap = std::max<uint64_t>({n, batch_capacity_, words_cap_ * 3 / 2});
  for (auto &w : words_)
    if (cudaMallocAsync(&w, cap * 8, s) != cudaSuccess) {
      (void)cudaGetLastError();
      words_cap_ = 0;
      throw std::bad_alloc();
    }
  words_cap_ = cap;
}

// A receipt for the level layout as it is on the host now (self = -1), or as
// it will be after a cascade into `dest` whose own output is `self` (levels
// above dest emptied).  Takes the next sequence number.
lsm::ReceiptSrc LsmDictionary::next_receipt(int dest) {
  lsm::ReceiptSrc r{};
  r.count = uint32_t(levels_.size());
  for (size_t i = 0; i < levels_.size(); ++i)
    r.desc[i] = (int(i) < dest || !levels_[i].run) ? nullptr : levels_[i].run->desc;
  r.self = dest;
  r.out = static_cast<unsigned long long *>(receipt_dev_);  // the mapped pinned host copy
  r.status = dev_status_;
  r.seq = ++receipt_seq_;
  return r;
}

// After an operation that posted a receipt: the gens it describes.
void LsmDictionary::receipt_posted() {
  for (size_t i = 0; i < levels_.size(); ++i) receipt_gens_[i] = levels_[i].gen;
  receipt_pending_ = true;
}

void LsmDictionary::post_receipt(cudaStream_t s) {
  lsm::ReceiptSrc src = next_receipt(-1);
  launch_chained(receipt_kernel, 1, 32, 0, s, src);
  receipt_posted();
}

// Applies the newest posted receipt once every word of it carries its
// sequence number (wait: after the last operation, which posted it, has
// completed).  An older receipt that landed while a newer one is in flight is
// never read: the newer one may be half written over it.
void LsmDictionary::apply_receipt(bool wait) {
  if (!receipt_pending_) return;
  const volatile unsigned long long *w = receipt_host_->w;
  unsigned long long v[lsm::kReceiptWords];
  auto landed = [&]() {
    for (int i = 0; i < lsm::kReceiptWords; ++i) v[i] = w[i];
    for (int i = 0; i < lsm::kMaxLevels; ++i)
      if ((v[i] >> 33) != (receipt_seq_ & 0x7fffffffu)) return false;
    return (v[lsm::kMaxLevels] >> 32) == receipt_seq_;
  };
  if (!landed()) {
    if (!wait) return;
    // the receipt may belong to an earlier batch of the operation in progress:
    // wait for the operations before it, then for the receipt itself
    host_sync();
    const auto t0 = std::chrono::steady_clock::now();
    while (!landed()) {
      if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(60))
        throw std::runtime_error("GPU dictionary receipt did not arrive");
      std::this_thread::yield();
    }
  }
  receipt_pending_ = false;
  struct {
    unsigned long long n[lsm::kMaxLevels];
    unsigned long long status;
  } r;
  for (int i = 0; i < lsm::kMaxLevels; ++i) r.n[i] = v[i] & lsm::kReceiptCountMask;
  r.status = v[lsm::kMaxLevels] & 0xffffffffull;
  status_bits_ |= uint32_t(r.status);
  // A level holds each key once, so one level with more rows than the
  // capacity means more live keys (tombstones included) than the capacity;
  // rows summed across levels would count stale versions of a key twice.
  uint64_t largest = 0;
  for (size_t i = 0; i < levels_.size(); ++i) {
    if (!levels_[i].run) continue;
    if (levels_[i].gen == receipt_gens_[i]) {
      levels_[i].upper = r.n[i];
      largest = std::max<uint64_t>(largest, r.n[i]);
    }
  }
  if ((r.status & kDevWaitTimeout) && !failed_) {
    failed_ = true;
    failure_ = "GPU dictionary publication failed: a bounded device wait timed out";
  }
  if ((r.status & kDevOutputOverflow) || largest > budget_) {
    status_bits_ |= kDevOutputOverflow;
    if (!failed_) {
      failed_ = true;
      failure_ = "GPU dictionary capacity exhausted: a level holds " + std::to_string(largest) +
                 " rows > capacity " + std::to_string(budget_) + "; accepted updates were preserved";
    }
  }
}

void LsmDictionary::reject_if_failed() const {
  if (failed_) throw std::runtime_error(failure_);
}

void LsmDictionary::release_levels(cudaStream_t s) {
  for (auto &l : levels_) {
    pool_.release(l.run, s);
    l = Level{};
    l.gen = next_gen_++;
  }
}

// ----------------------------------------------------------------------------
RunBuffer *LsmDictionary::sort_dedup(const uint32_t *keys, const uint32_t *values, uint64_t n,
                                     bool tombstone, cudaStream_t s, const uint8_t *erase, bool write_dir) {
  ensure_sort_space(n, s);
  if (n <= lsm::admit::kMaxKeys) return bucket_admit(keys, values, erase, n, tombstone, s, write_dir);
  // update batches are tiled to at most kMaxBatch = 2^20 rows: only a bulk
  // build (never mixed) takes the four-pass sort
  if (erase) throw std::logic_error("mixed batches are admitted by top-byte buckets only");
  const uint32_t nn = uint32_t(n);
  const size_t radix_bytes = align_up(radix::workspace_bytes(n, 4));
  const uint64_t dtiles = (n + lsm::kCompactTile - 1) / lsm::kCompactTile;
  const size_t total = radix_bytes + align_up(8) + align_up((dtiles + 1) * 8);
  Bump bump{static_cast<char *>(admit_scratch(total, s))};
  GPULSM_CUDA(cudaMemsetAsync(bump.p, 0, total, s));
  uint32_t *ws = bump.take<uint32_t>(radix_bytes / 4);
  uint32_t *counter = bump.take<uint32_t>(2);
  unsigned long long *lb = bump.take<unsigned long long>(dtiles + 1);
  const unsigned hist_blocks = std::min<unsigned>(grid_for(n, 4096), unsigned(num_sms_) * 4u);
  lsm::pack_histogram_kernel<false><<<hist_blocks, 256, 0, s>>>(keys, tombstone ? nullptr : values, nn,
                                                          words_[0], ws); note_launch();
  unsigned long long *bufs[2] = {words_[0], words_[1]};
  const int cur = radix::run_passes<unsigned long long, false>(bufs, nullptr, nn, 32, 64, ws,
                                                               dev_status_, s);
  RunBuffer *carry = pool_.acquire(n, s, true);
  lsm::dedup_last_kernel<<<unsigned(dtiles), lsm::kCompactThreads, 0, s>>>(
      bufs[cur], nn, tombstone ? 1 : 0, carry->keys, carry->vals, carry->flags, carry->desc, carry->dir,
      carry->dir_bits, rows_log2_, lb, counter, dev_status_); note_launch();
  GPULSM_CUDA(cudaGetLastError());
  carry->dir_ok = true;
  return carry;
}

// Batches up to 2^20 rows: a stable partition by the key's top byte
// (histogram, scan, scatter - no look-back chain), then one CTA per top-byte
// bucket sorts, deduplicates and writes the level rows (lsm_admit.cuh).
size_t LsmDictionary::bucket_admit_scratch_bytes(uint64_t n) {
  namespace ad = lsm::admit;
  const uint32_t tiles = ad::part_tiles(n);
  const size_t zero_bytes = align_up(8) + align_up((ad::kBuckets + 1) * 8);
  return zero_bytes + 2 * align_up(size_t(tiles) * 256 * 4) + align_up(256 * 4);
}

RunBuffer *LsmDictionary::bucket_admit(const uint32_t *keys, const uint32_t *values, const uint8_t *erase,
                                       uint64_t n, bool tombstone, cudaStream_t s, bool write_dir) {
  void *scratch = admit_scratch(bucket_admit_scratch_bytes(n), s);
  // before the chain: a fresh buffer is a stream-ordered allocation
  RunBuffer *carry = pool_.acquire(n, s, true);
  bucket_admit_into(keys, values, erase, n, tombstone, s, carry, words_[0], words_[1], scratch, write_dir);
  return carry;
}

// The four admission launches into `carry`, with the given sort words and
// scratch.  A mixed batch (erase marks given) sorts words of (key, input
// position); its rows take value and flag from the batch by that position.
void LsmDictionary::bucket_admit_into(const uint32_t *keys, const uint32_t *values, const uint8_t *erase,
                                      uint64_t n, bool tombstone, cudaStream_t s, RunBuffer *carry,
                                      unsigned long long *w0, unsigned long long *w1, void *scratch,
                                      bool write_dir) {
  namespace ad = lsm::admit;
  const uint32_t nn = uint32_t(n);
  const uint32_t tiles = ad::part_tiles(n);
  const size_t zero_bytes = align_up(8) + align_up((ad::kBuckets + 1) * 8);
  Bump bump{static_cast<char *>(scratch)};
  unsigned long long *zero = reinterpret_cast<unsigned long long *>(bump.p);  // zeroed by part_hist_kernel
  uint32_t *counter = bump.take<uint32_t>(2);
  unsigned long long *lb = bump.take<unsigned long long>(ad::kBuckets + 1);
  uint32_t *cnt = bump.take<uint32_t>(size_t(tiles) * 256);
  uint32_t *prefix = bump.take<uint32_t>(size_t(tiles) * 256);
  uint32_t *top = bump.take<uint32_t>(256);
  launch_chained(ad::part_hist_kernel, tiles, ad::kPartThreads, 0, s, keys, nn, tiles, cnt, zero,
                 uint32_t(zero_bytes / 8));
  launch_chained(ad::part_scan_kernel, 256, ad::kPartThreads, 0, s, cnt, tiles, prefix, top);
  const bool mixed = erase != nullptr;
  launch_chained(ad::part_scatter_kernel, tiles, ad::kPartThreads, 0, s, keys,
                 (tombstone || mixed) ? nullptr : values, nn, tiles, static_cast<const uint32_t *>(prefix),
                 static_cast<const uint32_t *>(top), w1, mixed ? 1 : 0);
  const ad::RowSource src{mixed ? values : nullptr, erase, tombstone ? 1 : 0};
  launch_chained(ad::admit_bucket_kernel, ad::kBuckets, ad::kThreads, ad::kBucketSmemBytes, s, w1, w0,
                 static_cast<const uint32_t *>(top), nn, src, carry->keys, carry->vals, carry->flags, carry->desc,
                 write_dir ? carry->dir : nullptr, carry->dir_bits, rows_log2_, lb, counter, dev_status_);
  carry->dir_ok = write_dir;
}

RunBuffer *LsmDictionary::merge(RunBuffer *newer, RunBuffer *older, uint64_t out_upper,
                                bool drop_tombstones, cudaStream_t s, const lsm::ReceiptSrc *rcpt,
                                bool release_newer, bool release_older) {
  RunBuffer *out = pool_.acquire(out_upper, s);
  out->dir_ok = merge_dirs_;
  const uint64_t tiles = std::max<uint64_t>(1, (out_upper + lsm::kMergeTile - 1) / lsm::kMergeTile);
  const size_t zero_bytes = merge_scratch_bytes(out_upper);
  const size_t bytes = zero_bytes + align_up((tiles + 2) * 8);
  Bump bump{static_cast<char *>(scratch(bytes, s))};
  unsigned long long *zero = reinterpret_cast<unsigned long long *>(bump.p);  // zeroed by the partition kernel
  uint32_t *counter = bump.take<uint32_t>(2);
  unsigned long long *lb = bump.take<unsigned long long>(tiles + 1);
  bump.off = zero_bytes;
  unsigned long long *parts = bump.take<unsigned long long>(tiles + 2);
  launch_chained(lsm::merge_partition_kernel, grid_for((tiles + 1) * 32, 256), 256, 0, s,
                 static_cast<const uint32_t *>(newer->keys), static_cast<const lsm::LevelDesc *>(newer->desc),
                 static_cast<const uint32_t *>(older->keys), static_cast<const lsm::LevelDesc *>(older->desc), parts,
                 uint32_t(tiles + 1), zero, uint32_t(zero_bytes / 8));
  auto kernel = drop_tombstones ? lsm::merge_kernel<true> : lsm::merge_kernel<false>;
  unsigned long long *trace = nullptr;
  MergeTrace tr{};
  if (timing_ && traces_.size() < kMaxTraces) {
    trace = trace_dev_ + 4 * traces_.size();
    for (cudaEvent_t *e : {&tr.start, &tr.stop}) {
      if (!spare_events_.empty()) {
        *e = spare_events_.back();
        spare_events_.pop_back();
      } else {
        GPULSM_CUDA(cudaEventCreate(e));
      }
    }
    GPULSM_CUDA(cudaEventRecord(tr.start, s));
  }
  launch_chained(kernel, unsigned(tiles), lsm::kMergeThreads, lsm::kMergeSmemBytes, s, newer->keys, newer->vals,
                 newer->flags,
                 newer->desc, older->keys, older->vals, older->flags, older->desc, out->keys, out->vals, out->flags,
                 out->desc, merge_dirs_ ? out->dir : nullptr, out->dir_bits, rows_log2_,
                 static_cast<unsigned long long>(std::min<uint64_t>(out_upper, out->cap)),
                 static_cast<unsigned long long>(out->cap), parts, lb, counter, dev_status_, trace,
                 rcpt ? *rcpt : lsm::ReceiptSrc{});
  if (trace) {
    GPULSM_CUDA(cudaEventRecord(tr.stop, s));
    traces_.push_back(tr);
  }
  if (release_newer) pool_.release(newer, s);
  if (release_older) pool_.release(older, s);
  return out;
}


// Search mode 1: a freshly written level of at least kLearnedMinRows rows
// gets its learned position model before the next read that searches it
// (fitting when the level is written would refit levels that the next update
// replaces unread); smaller levels keep the directory.
void LsmDictionary::fit_model(RunBuffer *run, uint64_t upper, cudaStream_t) {
  run->model_ok = false;
  run->model_rows = (cfg_.search_mode == 1 && upper >= kLearnedMinRows) ? upper : 0;
}

void LsmDictionary::ensure_models(cudaStream_t s) {
  prev_update_ = false;
  // a level searched by binary search (mode 2) or by its learned model
  // (mode 1, levels with a model) never reads its directory
  for (auto &l : levels_)
    if (l.run && !l.run->dir_ok && cfg_.search_mode != 2 && !(cfg_.search_mode == 1 && l.run->model_rows)) {
      lsm::build_directory_kernel<<<grid_for((l.upper + lsm::kDirRows) / lsm::kDirRows, 256), 256, 0, s>>>(
          l.run->keys, l.run->desc, l.run->dir);
      note_launch();
      GPULSM_CUDA(cudaGetLastError());
      l.run->dir_ok = true;
    }
  if (cfg_.search_mode != 1) return;
  for (auto &l : levels_)
    if (l.run && l.run->model_rows && !l.run->model_ok) fit_now(l.run, l.run->model_rows, s);
}

// Fit the model on the GPU (forward/backward kernels), reading the level's
// exact row count from its device descriptor.
void LsmDictionary::fit_now(RunBuffer *run, uint64_t upper, cudaStream_t s) {
  uint32_t segs = 64;
  while (segs < upper / kRowsPerSegment && segs < kMaxSegments) segs <<= 1;
  const size_t bytes = learned::bytes_for(segs);
  if (bytes > run->model_cap) {
    if (run->model) GPULSM_CUDA(cudaFreeAsync(run->model, s));
    run->model = nullptr;
    pool_.account(-int64_t(run->model_cap));
    run->model_cap = 0;
    if (cudaMallocAsync(&run->model, bytes, s) != cudaSuccess) {
      (void)cudaGetLastError();
      run->model = nullptr;
      throw std::bad_alloc();
    }
    run->model_cap = bytes;
    pool_.account(int64_t(bytes));
  }
  learned::fit<uint32_t>(run->keys, upper, segs, kFitIters, run->model, nullptr, s, &run->desc->n);
  run->model_segments = segs;
  run->model_ok = true;
  ++next_gen_;  // the level table must pick up the model
}

// Lands a sorted, deduplicated batch (leveling).  With want_receipt the
// update's receipt goes into its final merge kernel (or, without a merge, a
// standalone receipt kernel).
void LsmDictionary::cascade(RunBuffer *carry, uint64_t carry_upper, bool carry_tombs, cudaStream_t s,
                            bool want_receipt, bool carry_owned) {
  const size_t L = levels_.size();
  size_t dest = 0;
  uint64_t acc = carry_upper;
  for (size_t j = 0; j < L; ++j) {
    dest = j;
    if (!levels_[j].run) break;
    if (j == L - 1 || acc + levels_[j].upper <= caps_[j]) break;
    acc += levels_[j].upper;
  }
  const bool dest_occupied = levels_[dest].run != nullptr;
  bool deeper = false;
  for (size_t j = dest + 1; j < L; ++j) deeper |= levels_[j].run != nullptr;
  RunBuffer *x = carry;
  uint64_t xu = carry_upper;
  bool xt = carry_tombs;
  const size_t merges = dest + (dest_occupied ? 1 : 0);
  lsm::ReceiptSrc rcpt{};
  if (want_receipt && merges) rcpt = next_receipt(int(dest));  // the layout after this cascade
  for (size_t i = 0; i < dest; ++i) {
    const bool last = (i + 1 == dest) && !dest_occupied;
    const uint64_t ou = xu + levels_[i].upper;
    const bool drop = last && !deeper;
    x = merge(x, levels_[i].run, ou, drop, s, (want_receipt && i + 1 == merges) ? &rcpt : nullptr,
              carry_owned || x != carry);
    xu = ou;
    xt = !drop && (xt || levels_[i].tombs);
    levels_[i] = Level{};
    levels_[i].gen = next_gen_++;
  }
  if (dest_occupied) {
    const uint64_t ou = xu + levels_[dest].upper;
    x = merge(x, levels_[dest].run, ou, !deeper, s, want_receipt ? &rcpt : nullptr, carry_owned || x != carry);
    xu = ou;
    xt = deeper && (xt || levels_[dest].tombs);
  }
  if (x == carry && !carry_owned) {  // the carry lands as it is: a copy of it becomes the level
    RunBuffer *empty = pool_.acquire(1, s);
    GPULSM_CUDA(cudaMemsetAsync(empty->desc, 0, sizeof(LevelDesc), s));
    x = merge(carry, empty, xu, !deeper, s, nullptr, false, true);
    xt = deeper && xt;
  }
  levels_[dest].run = x;
  levels_[dest].upper = std::min<uint64_t>(xu, x->cap);
  levels_[dest].gen = next_gen_++;
  levels_[dest].tombs = xt;  // its directory was written by the kernel that wrote its rows
  fit_model(x, levels_[dest].upper, s);
  if (want_receipt && !merges) post_receipt(s);
}

// Merge every occupied level, newest first, into one tombstone-free run at
// the position of the oldest one (a full compaction).
void LsmDictionary::compact_all(cudaStream_t s) {
  std::vector<size_t> occ;
  for (size_t i = 0; i < levels_.size(); ++i)
    if (levels_[i].run) occ.push_back(i);
  if (occ.empty()) return;
  if (occ.size() == 1 && !levels_[occ[0]].tombs) return;
  const size_t dest = occ.back();
  RunBuffer *x = levels_[occ[0]].run;
  uint64_t xu = levels_[occ[0]].upper;
  if (occ.size() == 1) {
    // a lone level that may hold tombstones: merge with an empty run to drop them
    RunBuffer *empty = pool_.acquire(1, s);
    GPULSM_CUDA(cudaMemsetAsync(empty->desc, 0, sizeof(LevelDesc), s));
    x = merge(x, empty, xu, true, s);
  } else {
    for (size_t k = 1; k < occ.size(); ++k) {
      const uint64_t ou = xu + levels_[occ[k]].upper;
      x = merge(x, levels_[occ[k]].run, ou, k + 1 == occ.size(), s);
      xu = ou;
    }
  }
  for (size_t i : occ) {
    levels_[i] = Level{};
    levels_[i].gen = next_gen_++;
  }
  levels_[dest].run = x;
  levels_[dest].upper = std::min<uint64_t>(xu, x->cap);
  levels_[dest].gen = next_gen_++;
  levels_[dest].tombs = false;
  fit_model(x, levels_[dest].upper, s);
}

int LsmDictionary::ranges_on_single_level(const uint32_t *lo, const uint32_t *hi, uint64_t n, cudaStream_t s) {
  int occupied = 0, only = -1;
  uint64_t rows = 0;
  for (size_t i = 0; i < levels_.size(); ++i)
    if (levels_[i].run) {
      ++occupied;
      only = int(i);
      rows += levels_[i].upper;
    }
  if (occupied == 0) return -1;
  if (occupied == 1 && !levels_[only].tombs) return only;
  if (n < 1024) return -1;  // small batches: the per-query merge is cheaper
  // estimate the rows the batch covers from its total key width (one 8-byte read)
  GPULSM_CUDA(cudaMemsetAsync(width_, 0, 8, s));
  lsm::range_width_kernel<<<std::min<unsigned>(grid_for(n, 256), unsigned(num_sms_) * 8u), 256, 0, s>>>(
      lo, hi, n, width_); note_launch();
  GPULSM_CUDA(cudaMemcpyAsync(width_host_, width_, 8, cudaMemcpyDeviceToHost, s));
  GPULSM_CUDA(cudaStreamSynchronize(s));
  const double covered = double(*width_host_) / 4294967296.0 * double(rows);
  // per-query merging touches every covered row once per level; a compaction
  // streams every row about twice
  if (covered * double(occupied) < 2.0 * double(rows)) return -1;
  compact_all(s);
  for (size_t i = 0; i < levels_.size(); ++i)
    if (levels_[i].run) return int(i);
  return -1;
}

const unsigned long long *LsmDictionary::value_prefix(int level, cudaStream_t s) {
  const Level &l = levels_[level];
  if (prefix_gen_ == l.gen && prefix_) return prefix_;
  const uint64_t n = l.upper;
  if (n + 1 > prefix_cap_) {
    if (prefix_) GPULSM_CUDA(cudaFreeAsync(prefix_, s));
    prefix_cap_ = std::max<uint64_t>(n + 1, prefix_cap_ * 3 / 2);
    if (cudaMallocAsync(reinterpret_cast<void **>(&prefix_), prefix_cap_ * 8, s) != cudaSuccess) {
      (void)cudaGetLastError();
      prefix_ = nullptr;
      prefix_cap_ = 0;
      throw std::bad_alloc();
    }
  }
  // exclusive scan of the values; the count comes from the device descriptor,
  // so scan the host upper bound of rows (rows past n read as values of a
  // stale buffer tail are never used: queries stop at n)
  const uint32_t tiles = lsm::scan_tiles(n);
  const size_t bytes = align_up(8) + align_up(size_t(tiles + 1) * 8);
  Bump bump{static_cast<char *>(scratch(bytes, s))};
  GPULSM_CUDA(cudaMemsetAsync(bump.p, 0, bytes, s));
  uint32_t *counter = bump.take<uint32_t>(2);
  unsigned long long *lb = bump.take<unsigned long long>(tiles + 1);
  lsm::scan_kernel<unsigned long long, false><<<tiles, lsm::kScanThreads, 0, s>>>(l.run->vals, nullptr, n, prefix_, lb,
                                                                              counter, dev_status_);
  note_launch();
  prefix_gen_ = l.gen;
  return prefix_;
}

// The level set of a range sum over several levels: every view carries its
// level's live-value prefix, scanned here (over the host upper bound of the
// rows) when the level changed since its last scan.
void LsmDictionary::live_level_set(void *out, cudaStream_t s) {
  auto *set = static_cast<lsm::LevelSet *>(out);
  set->count = 0;
  // staged runs first, newest first (their prefixes are rebuilt when a slot is refilled)
  if (live_staged_.size() < staged_.size()) live_staged_.resize(staged_.size());
  std::vector<size_t> st;
  for (size_t i = 0; i < staged_.size(); ++i)
    if (staged_[i].seq) st.push_back(i);
  std::sort(st.begin(), st.end(), [&](size_t a, size_t b) { return staged_[a].seq > staged_[b].seq; });
  for (size_t i : st) {
    LivePrefix &lp = live_staged_[i];
    refresh_live_prefix(lp, staged_[i].run, staged_[i].upper, staged_[i].seq, staged_[i].run->cap + 1, s);
    lsm::LevelView v = view_of_run(staged_[i].run);
    v.live = lp.p;
    set->lv[set->count++] = v;
  }
  if (live_.size() < levels_.size()) live_.resize(levels_.size());
  for (size_t i = 0; i < levels_.size(); ++i) {
    const Level &l = levels_[i];
    if (!l.run) continue;
    LivePrefix &lp = live_[i];
    // a level holds at most its capacity (the foundation: at least), so its
    // prefix is allocated once, at that size
    refresh_live_prefix(lp, l.run, l.upper, l.gen, caps_[i] + 1, s);
    lsm::LevelView v = view_of(int(i));
    v.live = lp.p;
    set->lv[set->count++] = v;
  }
}

// The u32 prefix of live values of a run, rebuilt when its generation changed.
void LsmDictionary::refresh_live_prefix(LivePrefix &lp, RunBuffer *run, uint64_t upper, uint64_t gen,
                                        uint64_t min_cap, cudaStream_t s) {
  {
    const uint64_t n = upper;
    if (lp.gen != gen || !lp.p) {
      if (n + 1 > lp.cap) {
        // at least min_cap (the most rows the slot can hold), and growing by
        // half when a foundation outgrows it: an allocation here can block the
        // calling thread while the pool maps new memory
        const uint64_t cap = std::max<uint64_t>({n + 1, min_cap, lp.cap * 3 / 2, 1024});
        if (lp.p) GPULSM_CUDA(cudaFreeAsync(lp.p, s));
        live_bytes_ -= lp.cap * 4;
        lp.p = nullptr;
        lp.cap = 0;
        if (cudaMallocAsync(reinterpret_cast<void **>(&lp.p), cap * 4, s) != cudaSuccess) {
          (void)cudaGetLastError();
          lp.p = nullptr;
          throw std::bad_alloc();
        }
        lp.cap = cap;
        live_bytes_ += cap * 4;
      }
      const uint32_t tiles = lsm::scan_tiles(n);
      const size_t bytes = align_up(8) + align_up(size_t(tiles + 1) * 8);
      Bump bump{static_cast<char *>(scratch(bytes, s))};
      GPULSM_CUDA(cudaMemsetAsync(bump.p, 0, bytes, s));
      uint32_t *counter = bump.take<uint32_t>(2);
      unsigned long long *lb = bump.take<unsigned long long>(tiles + 1);
      lsm::scan_kernel<uint32_t, true><<<tiles, lsm::kScanThreads, 0, s>>>(run->vals, run->flags, n, lp.p, lb,
                                                                           counter, dev_status_);
      note_launch();
      lp.gen = gen;
    }
  }
}

void LsmDictionary::admit(const uint32_t *keys, const uint32_t *values, const uint8_t *erase, uint64_t n,
                          bool tombstone, cudaStream_t s) {
  for (uint64_t off = 0; off < n; off += batch_capacity_) {
    const uint64_t m = std::min(batch_capacity_, n - off);
    uint64_t total_upper = m;
    for (auto &l : levels_) total_upper += l.upper;
    if (total_upper > 2 * budget_ + batch_capacity_ && receipt_pending_) {
      // stale bounds: wait for the exact counts before planning more storage
      apply_receipt(true);
      reject_if_failed();
    }
    // The batch is admitted on s, which orders the reads of the caller's
    // input; its merges run on merge_stream_ after the admission and after
    // the previous batch's merges, while s goes on to admit the next batch.
    // The receipt comes from the merge stream (the final merge, or a receipt
    // kernel when nothing merges), so receipts land in batch order.
    RunBuffer *carry = sort_dedup(keys + off, values ? values + off : nullptr, m, tombstone, s,
                                  erase ? erase + off : nullptr, merge_dirs_);
    GPULSM_CUDA(cudaEventRecord(adm_done_, s));
    GPULSM_CUDA(cudaStreamWaitEvent(merge_stream_, adm_done_, 0));
    merges_pending_ = true;
    try {
      cascade(carry, m, tombstone || erase, merge_stream_, true);
    } catch (...) {  // reads still wait for whatever the cascade enqueued
      cudaEventRecord(merge_done_, merge_stream_);
      throw;
    }
    GPULSM_CUDA(cudaEventRecord(merge_done_, merge_stream_));
    pool_.advance();
    receipt_posted();
  }
}

// Updates return while their merges run on the dictionary's stream; a CUDA
// graph capture would leave that stream unjoined, so updates refuse capture.
static void refuse_capture(cudaStream_t s) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  GPULSM_CUDA(cudaStreamIsCapturing(s, &cs));
  if (cs != cudaStreamCaptureStatusNone)
    throw std::invalid_argument("GPU dictionary updates cannot be captured into a CUDA graph");
}

// ----------------------------------------------------------------------------
void LsmDictionary::clear(cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  begin_op(s);
  drop_staged();
  release_levels(s);
  GPULSM_CUDA(cudaMemsetAsync(dev_status_, 0, 4, s));
  status_bits_ = 0;
  failed_ = false;
  failure_.clear();
  receipt_pending_ = false;
  prev_update_ = false;
  end_op(s);
}

void LsmDictionary::bulk_build(const uint32_t *keys, const uint32_t *values, uint64_t n,
                               cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if ((n && (!keys || !values)) || n > 0xffffffffull)
    throw std::invalid_argument("invalid GPU dictionary initial input");
  if (n > radix::kMaxKeys) throw std::length_error("bulk build limited to 2^30-1 keys per call");
  begin_op(s);
  drop_staged();
  release_levels(s);
  GPULSM_CUDA(cudaMemsetAsync(dev_status_, 0, 4, s));
  status_bits_ = 0;
  failed_ = false;
  failure_.clear();
  receipt_pending_ = false;
  if (n) {
    RunBuffer *run = sort_dedup(keys, values, n, false, s);
    Level &top = levels_.back();
    top.run = run;
    top.upper = n;
    top.gen = next_gen_++;
    top.tombs = false;
    fit_model(run, n, s);
    post_receipt(s);
  }
  end_op(s);
}

void LsmDictionary::insert(const uint32_t *keys, const uint32_t *values, uint64_t n,
                           cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!n) return;
  if (!keys || !values) throw std::invalid_argument("invalid GPU dictionary update batch");
  refuse_capture(s);
  apply_receipt(false);
  reject_if_failed();
  begin_op(s, true);
  if (stage_seq_pending()) {  // staged runs are older than this batch: they land first
    begin_op(s);
    flush_staged_locked(s);
  }
  merge_dirs_ = !prev_update_;  // back-to-back updates leave directories to the reads
  prev_update_ = true;
  admit(keys, values, nullptr, n, false, s);  // every batch's finishing kernel writes the receipt
  end_op(s);
}

void LsmDictionary::erase(const uint32_t *keys, uint64_t n, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!n) return;
  if (!keys) throw std::invalid_argument("invalid GPU dictionary update batch");
  refuse_capture(s);
  apply_receipt(false);
  reject_if_failed();
  begin_op(s, true);
  if (stage_seq_pending()) {  // staged runs are older than this batch: they land first
    begin_op(s);
    flush_staged_locked(s);
  }
  merge_dirs_ = !prev_update_;  // back-to-back updates leave directories to the reads
  prev_update_ = true;
  admit(keys, nullptr, nullptr, n, true, s);  // every batch's finishing kernel writes the receipt
  end_op(s);
}

void LsmDictionary::update(const uint32_t *keys, const uint32_t *values, const uint8_t *erase, uint64_t n,
                           cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!n) return;
  if (!keys || !values || !erase) throw std::invalid_argument("invalid GPU dictionary update batch");
  refuse_capture(s);
  apply_receipt(false);
  reject_if_failed();
  begin_op(s, true);
  if (stage_seq_pending()) {  // staged runs are older than this batch: they land first
    begin_op(s);
    flush_staged_locked(s);
  }
  merge_dirs_ = !prev_update_;  // back-to-back updates leave directories to the reads
  prev_update_ = true;
  admit(keys, values, erase, n, false, s);  // every batch's finishing kernel writes the receipt
  end_op(s);
}

lsm::LevelView LsmDictionary::view_of(int level) const { return view_of_run(levels_[level].run); }

lsm::LevelView LsmDictionary::view_of_run(const RunBuffer *r) const {
  lsm::LevelView v{r->keys, r->vals, r->flags, cfg_.search_mode == 2 ? nullptr : r->dir, r->desc};
  if (cfg_.search_mode == 1 && r->model_ok) {
    v.mh = static_cast<const learned::ModelHeader *>(r->model);
    v.ms = reinterpret_cast<const learned::Segment *>(static_cast<const char *>(r->model) +
                                                      sizeof(learned::ModelHeader));
  }
  return v;
}

void LsmDictionary::level_set(void *out) const {
  auto *set = static_cast<lsm::LevelSet *>(out);
  set->count = 0;
  // staged runs first, newest first: they are newer than every level
  std::vector<const Staged *> st;
  for (const Staged &x : staged_)
    if (x.seq) st.push_back(&x);
  std::sort(st.begin(), st.end(), [](const Staged *a, const Staged *b) { return a->seq > b->seq; });
  for (const Staged *x : st) set->lv[set->count++] = view_of_run(x->run);
  for (size_t i = 0; i < levels_.size(); ++i)
    if (levels_[i].run) set->lv[set->count++] = view_of(int(i));
}

void LsmDictionary::lookup(const uint32_t *queries, uint64_t n, uint32_t *out_values,
                           uint8_t *out_found, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!n) return;
  if (!queries || !out_values) throw std::invalid_argument("invalid GPU dictionary lookup");
  apply_receipt(false);
  begin_op(s);
  ensure_models(s);
  launch_lookup(queries, n, out_values, out_found, s);
  end_op(s);
}

void LsmDictionary::launch_lookup(const uint32_t *queries, uint64_t n, uint32_t *out_values, uint8_t *out_found,
                                  cudaStream_t s) {
  lsm::LevelSet set;
  level_set(&set);
  if (cfg_.search_mode != 2)
    lsm::lookup_kernel<true><<<grid_for((n + lsm::kLookupPair - 1) / lsm::kLookupPair, 256), 256, 0, s>>>(
        set, queries, n, out_values, out_found);
  else
    lsm::lookup_kernel<false><<<grid_for(n, 256), 256, 0, s>>>(set, queries, n, out_values, out_found);
  note_launch();
  GPULSM_CUDA(cudaGetLastError());
}

void LsmDictionary::range_sum(const uint32_t *lo, const uint32_t *hi, uint64_t n, uint32_t *out,
                              cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!n) return;
  if (!lo || !hi || !out) throw std::invalid_argument("invalid GPU dictionary range");
  apply_receipt(false);
  begin_op(s);
  flush_staged_locked(s);  // range paths read the levels only
  ensure_models(s);
  const int single = ranges_on_single_level(lo, hi, n, s);
  ensure_models(s);  // a compaction wrote a new level
  if (single >= 0) {
    const unsigned long long *prefix = value_prefix(single, s);
    lsm::single_level_range_kernel<0><<<grid_for(n, 256), 256, 0, s>>>(view_of(single), lo, hi, n, prefix, out);
    note_launch();
  } else {
    lsm::LevelSet set;
    live_level_set(&set, s);
    lsm::range_sum_levels_kernel<<<grid_for(n * lsm::kRangeGroup, lsm::kRangeThreads), lsm::kRangeThreads, 0, s>>>(
        set, lo, hi, n, out);
    note_launch();
  }
  GPULSM_CUDA(cudaGetLastError());
  end_op(s);
}

void LsmDictionary::range_sum_kway(const uint32_t *lo, const uint32_t *hi, uint64_t n, uint32_t *out,
                                   cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!n) return;
  if (!lo || !hi || !out) throw std::invalid_argument("invalid GPU dictionary range");
  apply_receipt(false);
  begin_op(s);  // staged runs take part through their live-value prefixes (no flush)
  ensure_models(s);
  lsm::LevelSet set;
  live_level_set(&set, s);
  lsm::range_sum_levels_kernel<<<grid_for(n * lsm::kRangeGroup, lsm::kRangeThreads), lsm::kRangeThreads, 0, s>>>(
        set, lo, hi, n, out);
  note_launch();
  GPULSM_CUDA(cudaGetLastError());
  end_op(s);
}

void LsmDictionary::lookup_and_range_sum(const uint32_t *queries, uint64_t nq, uint32_t *out_values,
                                         uint8_t *out_found, const uint32_t *lo, const uint32_t *hi, uint64_t nr,
                                         uint32_t *out_sums, cudaStream_t s, cudaStream_t side) {
  std::lock_guard<std::mutex> g(mu_);
  if ((nq && (!queries || !out_values)) || (nr && (!lo || !hi || !out_sums)) || !side || side == s)
    throw std::invalid_argument("invalid GPU dictionary read");
  if (!nq && !nr) return;
  apply_receipt(false);
  begin_op(s);
  ensure_models(s);  // directories and models before the fork: both reads search the levels
  if (nq) {
    GPULSM_CUDA(cudaEventRecord(fork_, s));
    GPULSM_CUDA(cudaStreamWaitEvent(side, fork_, 0));
    launch_lookup(queries, nq, out_values, out_found, side);
    GPULSM_CUDA(cudaEventRecord(side_done_, side));
  }
  try {
    if (nr) {
      lsm::LevelSet set;
      live_level_set(&set, s);  // prefix scans of changed levels run beside the lookups
      lsm::range_sum_levels_kernel<<<grid_for(nr * lsm::kRangeGroup, lsm::kRangeThreads), lsm::kRangeThreads, 0,
                                     s>>>(set, lo, hi, nr, out_sums);
      note_launch();
      GPULSM_CUDA(cudaGetLastError());
    }
  } catch (...) {
    if (nq) (void)cudaStreamWaitEvent(s, side_done_, 0);  // s still covers the lookups
    throw;
  }
  if (nq) GPULSM_CUDA(cudaStreamWaitEvent(s, side_done_, 0));
  end_op(s);
}

void LsmDictionary::range_count(const uint32_t *lo, const uint32_t *hi, uint64_t n, uint32_t *out,
                                cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!n) return;
  if (!lo || !hi || !out) throw std::invalid_argument("invalid GPU dictionary range");
  apply_receipt(false);
  begin_op(s);
  flush_staged_locked(s);  // range paths read the levels only
  ensure_models(s);
  const int single = ranges_on_single_level(lo, hi, n, s);
  ensure_models(s);  // a compaction wrote a new level
  if (single >= 0) {
    lsm::single_level_range_kernel<1><<<grid_for(n, 256), 256, 0, s>>>(view_of(single), lo, hi, n, nullptr, out);
    note_launch();
  } else {
    lsm::LevelSet set;
    level_set(&set);
    lsm::range_kernel<1><<<grid_for(n, 256), 256, 0, s>>>(set, lo, hi, n, out, nullptr, nullptr,
                                                         nullptr); note_launch();
  }
  GPULSM_CUDA(cudaGetLastError());
  end_op(s);
}

void LsmDictionary::range_offsets(const uint32_t *lo, const uint32_t *hi, uint64_t n,
                                  uint64_t *offsets, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!offsets) throw std::invalid_argument("invalid GPU dictionary range");
  if (n && (!lo || !hi)) throw std::invalid_argument("invalid GPU dictionary range");
  apply_receipt(false);
  begin_op(s);
  flush_staged_locked(s);  // range paths read the levels only
  ensure_models(s);
  const uint32_t tiles = lsm::scan_tiles(n);
  const size_t count_bytes = align_up(std::max<uint64_t>(n, 1) * 4);
  const size_t bytes = count_bytes + align_up(8) + align_up(size_t(tiles + 1) * 8);
  Bump bump{static_cast<char *>(scratch(bytes, s))};
  uint32_t *counts = bump.take<uint32_t>(count_bytes / 4);
  GPULSM_CUDA(cudaMemsetAsync(bump.p + count_bytes, 0, bytes - count_bytes, s));
  uint32_t *counter = bump.take<uint32_t>(2);
  unsigned long long *lb = bump.take<unsigned long long>(tiles + 1);
  if (n) {
    const int single = ranges_on_single_level(lo, hi, n, s);
    ensure_models(s);  // a compaction wrote a new level
    if (single >= 0) {
      lsm::single_level_range_kernel<1><<<grid_for(n, 256), 256, 0, s>>>(view_of(single), lo, hi, n, nullptr,
                                                                          counts);
      note_launch();
    } else {
      lsm::LevelSet set;
      level_set(&set);
      lsm::range_kernel<1><<<grid_for(n, 256), 256, 0, s>>>(set, lo, hi, n, counts, nullptr, nullptr,
                                                           nullptr); note_launch();
    }
  }
  lsm::scan_kernel<unsigned long long, false><<<tiles, lsm::kScanThreads, 0, s>>>(
      counts, nullptr, n, reinterpret_cast<unsigned long long *>(offsets), lb, counter, dev_status_); note_launch();
  GPULSM_CUDA(cudaGetLastError());
  end_op(s);
}

void LsmDictionary::range_pairs(const uint32_t *lo, const uint32_t *hi, uint64_t n,
                                const uint64_t *offsets, uint32_t *out_keys, uint32_t *out_values,
                                cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!n) return;
  if (!lo || !hi || !offsets || !out_keys || !out_values)
    throw std::invalid_argument("invalid GPU dictionary range");
  apply_receipt(false);
  begin_op(s);
  flush_staged_locked(s);  // range paths read the levels only
  ensure_models(s);
  const int single = ranges_on_single_level(lo, hi, n, s);
  ensure_models(s);  // a compaction wrote a new level
  if (single >= 0) {
    // resident warps take the query groups from a counter
    uint32_t *counter = static_cast<uint32_t *>(scratch(sizeof(uint32_t), s));
    GPULSM_CUDA(cudaMemsetAsync(counter, 0, sizeof(uint32_t), s));
    const uint64_t groups = (n + lsm::kPairsGroup - 1) / lsm::kPairsGroup;
    const unsigned grid = std::min<unsigned>(grid_for(groups * 32, 256), unsigned(num_sms_) * 8u);
    lsm::single_level_pairs_kernel<<<grid, 256, 0, s>>>(
        view_of(single), lo, hi, n, reinterpret_cast<const unsigned long long *>(offsets), out_keys, out_values,
        counter);
    note_launch();
  } else {
    lsm::LevelSet set;
    level_set(&set);
    lsm::range_kernel<2><<<grid_for(n, 256), 256, 0, s>>>(
        set, lo, hi, n, nullptr, reinterpret_cast<const unsigned long long *>(offsets), out_keys,
        out_values); note_launch();
  }
  GPULSM_CUDA(cudaGetLastError());
  end_op(s);
}

void LsmDictionary::successor(const uint32_t *queries, uint64_t n, uint32_t *out_keys,
                              cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!n) return;
  if (!queries || !out_keys) throw std::invalid_argument("invalid GPU dictionary successor");
  apply_receipt(false);
  begin_op(s);
  ensure_models(s);
  lsm::LevelSet set;
  level_set(&set);
  lsm::successor_kernel<<<grid_for(n, 256), 256, 0, s>>>(set, queries, n, out_keys); note_launch();
  GPULSM_CUDA(cudaGetLastError());
  end_op(s);
}

uint32_t LsmDictionary::status() {
  std::lock_guard<std::mutex> g(mu_);
  host_sync();
  apply_receipt(true);
  uint32_t bits = 0;
  GPULSM_CUDA(cudaMemcpy(&bits, dev_status_, 4, cudaMemcpyDeviceToHost));
  status_bits_ |= bits;
  return status_bits_;
}

void LsmDictionary::enqueue_table_lookup(const uint32_t *queries, uint64_t n, uint32_t *out_values,
                                         uint8_t *out_found, cudaStream_t capturing) {
  std::lock_guard<std::mutex> g(mu_);
  const auto *table = static_cast<const lsm::LevelSet *>(table_dev_);
  if (cfg_.search_mode != 2)
    lsm::lookup_table_kernel<true><<<grid_for((n + lsm::kLookupPair - 1) / lsm::kLookupPair, 256), 256, 0,
                                     capturing>>>(table, queries, n, out_values, out_found);
  else
    lsm::lookup_table_kernel<false><<<grid_for(n, 256), 256, 0, capturing>>>(table, queries, n, out_values, out_found);
  GPULSM_CUDA(cudaGetLastError());
}

void LsmDictionary::launch_read_graph(cudaGraphExec_t exec, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  apply_receipt(false);
  begin_op(s);
  ensure_models(s);
  if (table_gen_ != next_gen_) {  // the levels changed since the table was written
    lsm::LevelSet set;
    level_set(&set);
    lsm::write_table_kernel<<<1, 64, 0, s>>>(set, static_cast<lsm::LevelSet *>(table_dev_));
    note_launch();
    GPULSM_CUDA(cudaGetLastError());
    table_gen_ = next_gen_;
  }
  GPULSM_CUDA(cudaGraphLaunch(exec, s));
  note_launch();
  end_op(s);
}

void LsmDictionary::set_kernel_timing(bool on) {
  std::lock_guard<std::mutex> g(mu_);
  if (on && !trace_dev_) GPULSM_CUDA(cudaMalloc(&trace_dev_, kMaxTraces * 4 * sizeof(unsigned long long)));
  timing_ = on;
}

// Sum over the merges timed since the last read: launches, device time and
// algorithmic bytes (9 B per row read from either input - key, value, flag -
// 9 B per row written, 4 B per directory entry written).  Synchronises.
void LsmDictionary::kernel_timing(uint64_t *launches, double *total_ms, double *bytes) {
  std::lock_guard<std::mutex> g(mu_);
  const size_t m = traces_.size();
  double ms = 0, b = 0;
  if (m) {
    GPULSM_CUDA(cudaEventSynchronize(traces_.back().stop));
    std::vector<unsigned long long> t(4 * m);
    GPULSM_CUDA(cudaMemcpy(t.data(), trace_dev_, t.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < m; ++i) {
      float e = 0;
      GPULSM_CUDA(cudaEventElapsedTime(&e, traces_[i].start, traces_[i].stop));
      ms += e;
      b += 9.0 * double(t[4 * i] + t[4 * i + 1]) + 9.0 * double(t[4 * i + 2]) + 4.0 * double(t[4 * i + 3]);
      spare_events_.push_back(traces_[i].start);
      spare_events_.push_back(traces_[i].stop);
    }
    traces_.clear();
  }
  if (launches) *launches = m;
  if (total_ms) *total_ms = ms;
  if (bytes) *bytes = b;
}

uint64_t LsmDictionary::resident_bytes() {
  std::lock_guard<std::mutex> g(mu_);
  const uint64_t staging = stage_max_ ? stage_max_ * (9 + 16) + bucket_admit_scratch_bytes(stage_max_) : 0;
  return pool_.bytes() + words_cap_ * 16 + scratch_bytes_ + ascratch_bytes_ + live_bytes_ + sizeof(Receipt) + 256 +
         staging;
}

// ---------------------------------------------------------------- staged updates
void LsmDictionary::stage_configure(uint32_t slots, uint64_t max_keys, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!staged_.empty()) throw std::invalid_argument("staged updates are already configured");
  if (max_keys == 0 || max_keys > lsm::admit::kMaxKeys)
    throw std::invalid_argument("staged update batches must hold 1 to 2^20 keys");
  // every staged run is one more level of the level set
  const uint32_t room = uint32_t(lsm::kMaxLevels) - uint32_t(caps_.size());
  slots = std::min(slots, room);
  if (slots == 0) throw std::invalid_argument("no room for staged levels beside the level schedule");
  begin_op(s);
  stage_max_ = max_keys;
  GPULSM_CUDA(cudaMalloc(&stage_in_, 2 * max_keys * 4 + max_keys));  // keys, values, erase marks
  for (auto &w : stage_words_) GPULSM_CUDA(cudaMalloc(&w, max_keys * 8));
  GPULSM_CUDA(cudaMalloc(&stage_scratch_, bucket_admit_scratch_bytes(max_keys)));
  staged_.resize(slots);
  for (Staged &x : staged_) {
    x.run = pool_.acquire(max_keys, s);  // owned by the slot from now on
    x.run->dir_ok = true;                // its admissions write the directory
  }
  end_op(s);
}

int LsmDictionary::stage_free_slot() const {
  std::lock_guard<std::mutex> g(mu_);
  for (size_t i = 0; i < staged_.size(); ++i)
    if (!staged_[i].seq) return int(i);
  return -1;
}

void LsmDictionary::enqueue_stage_admit(uint32_t slot, uint64_t n, int mode, cudaStream_t capturing) {
  std::lock_guard<std::mutex> g(mu_);
  if (slot >= staged_.size()) throw std::invalid_argument("no such staging slot");
  if (n == 0 || n > stage_max_) throw std::length_error("staged update larger than the staging runs");
  if (mode < kStageInsert || mode > kStageMixed) throw std::invalid_argument("unknown staged update mode");
  const bool tombstone = mode == kStageErase;
  const uint8_t *erase = mode == kStageMixed ? reinterpret_cast<const uint8_t *>(stage_in_ + 2 * n) : nullptr;
  bucket_admit_into(stage_in_, tombstone ? nullptr : stage_in_ + n, erase, n, tombstone, capturing, staged_[slot].run,
                    stage_words_[0], stage_words_[1], stage_scratch_);
  GPULSM_CUDA(cudaGetLastError());
}

void LsmDictionary::launch_stage_graph(cudaGraphExec_t exec, uint32_t slot, uint64_t n, bool tombs,
                                       cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (slot >= staged_.size() || staged_[slot].seq) throw std::invalid_argument("staging slot is not free");
  apply_receipt(false);
  reject_if_failed();
  begin_op(s, true);  // writes only its staging run: merges of earlier updates may still run
  GPULSM_CUDA(cudaGraphLaunch(exec, s));
  note_launch();
  Staged &x = staged_[slot];
  x.upper = n;
  x.seq = ++stage_seq_;
  x.tombs = tombs;
  ++next_gen_;  // the level set changed (device level table, live prefixes)
  end_op(s);
}

void LsmDictionary::stage_flush(cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  apply_receipt(false);
  reject_if_failed();
  begin_op(s);
  flush_staged_locked(s);
  end_op(s);
}

// Merges the staged runs, newest first, into one run and carries it into the
// levels like an admitted batch; the staging runs stay with their slots.
// Called with the lock held and s already ordered after the pending merges.
void LsmDictionary::flush_staged_locked(cudaStream_t s) {
  std::vector<Staged *> st;
  for (Staged &x : staged_)
    if (x.seq) st.push_back(&x);
  if (st.empty()) return;
  std::sort(st.begin(), st.end(), [](const Staged *a, const Staged *b) { return a->seq > b->seq; });
  uint64_t total_upper = 0;
  for (const Staged *x : st) total_upper += x->upper;
  for (auto &l : levels_) total_upper += l.upper;
  if (total_upper > 2 * budget_ + batch_capacity_ && receipt_pending_) {
    apply_receipt(true);  // stale bounds: wait for the exact counts before planning more storage
    reject_if_failed();
  }
  // the staged runs, newest first, merge into one run (small merges, in L2),
  // which is carried into the levels like one admitted batch: level 0 is
  // rewritten once per flush instead of once per staged run.  A lone staged
  // run is carried as it is (the cascade reads it and leaves it with its slot).
  RunBuffer *x = st[0]->run;
  uint64_t xu = st[0]->upper;
  bool xt = st[0]->tombs;
  for (size_t i = 1; i < st.size(); ++i) {
    x = merge(x, st[i]->run, xu + st[i]->upper, false, s, nullptr, i > 1, false);
    xu += st[i]->upper;
    xt = xt || st[i]->tombs;
  }
  cascade(x, xu, xt, s, true, st.size() > 1);
  receipt_posted();
  for (Staged *y : st) {
    y->seq = 0;
    y->upper = 0;
    y->tombs = false;
  }
  pool_.advance();
  ++stage_flushes_;
  ++next_gen_;
}

uint64_t LsmDictionary::cleanup(cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  apply_receipt(false);
  reject_if_failed();
  begin_op(s);
  flush_staged_locked(s);
  compact_all(s);
  unsigned long long n = 0;
  for (auto &l : levels_)
    if (l.run) GPULSM_CUDA(cudaMemcpyAsync(&n, &l.run->desc->n, 8, cudaMemcpyDeviceToHost, s));
  GPULSM_CUDA(cudaStreamSynchronize(s));
  for (auto &l : levels_)
    if (l.run) l.upper = n;  // the exact count of the one remaining level
  end_op(s);
  return n;
}

void LsmDictionary::size(uint64_t *rows, uint32_t *levels) {
  std::lock_guard<std::mutex> g(mu_);
  host_sync();
  uint64_t total = 0;
  uint32_t count = 0;
  for (auto &l : levels_) {
    if (!l.run) continue;
    unsigned long long n = 0;
    GPULSM_CUDA(cudaMemcpy(&n, &l.run->desc->n, 8, cudaMemcpyDeviceToHost));
    total += n;
    ++count;
  }
  for (const Staged &x : staged_) {  // staged runs count as levels
    if (!x.seq) continue;
    unsigned long long n = 0;
    GPULSM_CUDA(cudaMemcpy(&n, &x.run->desc->n, 8, cudaMemcpyDeviceToHost));
    total += n;
    ++count;
  }
  if (rows) *rows = total;
  if (levels) *levels = count;
}

}  // namespace gpulsm

