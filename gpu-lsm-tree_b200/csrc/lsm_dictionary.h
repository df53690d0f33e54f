// Host engine of the LSM dictionary: the B200 counterpart of class GPULSMOpt
// (GPULSMOpt.cuh:5599-5881).  Same public operations and semantics; a
// different structure underneath (sorted levels with radix directories,
// merge-path merges, lazily applied receipts instead of epochs).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

namespace gpulsm {

namespace lsm {
struct LevelDesc;
struct ReceiptSrc;
struct LevelView;
}

// Batches of a staged update (LsmDictionary::enqueue_stage_admit).
enum StageMode : int { kStageInsert = 0, kStageErase = 1, kStageMixed = 2 };

struct DictConfig {
  uint64_t max_elements = 0;
  uint64_t batch_capacity = 0;
  uint64_t level_zero_capacity = 0;
  uint32_t fan_in = 0;
  uint32_t rows_per_bucket_log2 = 0;
  uint32_t search_mode = 0;
};

// Storage of one sorted run (keys, vals, flags, directory, descriptor).
struct RunBuffer {
  uint64_t cap = 0;        // rows
  uint32_t dir_bits = 0;   // directory holds up to 2^dir_bits buckets
  uint32_t *keys = nullptr;
  uint32_t *vals = nullptr;
  uint8_t *flags = nullptr;
  uint32_t *dir = nullptr;
  lsm::LevelDesc *desc = nullptr;
  void *block = nullptr;   // single device allocation backing all streams
  size_t bytes = 0;
  // learned position model of the run's keys (search mode 1); valid only
  // while model_ok (reset when the buffer is reused)
  void *model = nullptr;
  size_t model_cap = 0;
  uint32_t model_segments = 0;
  uint64_t model_rows = 0;  // rows bound of a level that wants a model before its next read (0: none)
  bool model_ok = false;
  bool dir_ok = false;      // the radix directory matches the rows (merges may leave it to the first read)
  // Last release: an event recorded on the releasing stream after the
  // launches that read the buffer; a reuse on another stream waits for it.
  cudaEvent_t freed = nullptr;
  cudaStream_t freed_on = nullptr;
  uint64_t freed_epoch = 0;
  bool released = false;
};

class RunPool {
 public:
  explicit RunPool(uint32_t rows_log2) : rows_log2_(rows_log2) {}
  ~RunPool();
  // settled_only: skip buffers released on another stream during the last
  // two epochs (allocating instead), so that the acquiring stream does not
  // wait for the launches still reading them
  RunBuffer *acquire(uint64_t min_rows, cudaStream_t stream, bool settled_only = false);
  void release(RunBuffer *b, cudaStream_t stream);
  void release_all_free(cudaStream_t stream);
  void advance() { ++epoch_; }
  size_t bytes() const { return bytes_; }
  void account(int64_t delta) { bytes_ = size_t(int64_t(bytes_) + delta); }
  // the stream-ordered pool the buffers come from: the destructor, which
  // runs after every other free of the dictionary, trims it
  void trim_on_destroy(cudaMemPool_t pool) { trim_pool_ = pool; }

 private:
  uint32_t rows_log2_;
  cudaMemPool_t trim_pool_ = nullptr;
  std::vector<std::unique_ptr<RunBuffer>> all_;
  std::vector<RunBuffer *> free_;
  size_t bytes_ = 0;
  uint64_t epoch_ = 0;  // advanced once per admitted batch
};

class LsmDictionary {
 public:
  explicit LsmDictionary(const DictConfig &config);
  ~LsmDictionary();
  LsmDictionary(const LsmDictionary &) = delete;
  LsmDictionary &operator=(const LsmDictionary &) = delete;

  void clear(cudaStream_t s);
  void bulk_build(const uint32_t *keys, const uint32_t *values, uint64_t n, cudaStream_t s);
  void insert(const uint32_t *keys, const uint32_t *values, uint64_t n, cudaStream_t s);
  void erase(const uint32_t *keys, uint64_t n, cudaStream_t s);
  // One batch of inserts and erases: row i erases keys[i] when erase[i] is
  // nonzero, else inserts (keys[i], values[i]); the last row of a key wins,
  // as in an insert or erase batch.
  void update(const uint32_t *keys, const uint32_t *values, const uint8_t *erase, uint64_t n, cudaStream_t s);
  void lookup(const uint32_t *queries, uint64_t n, uint32_t *out_values, uint8_t *out_found,
              cudaStream_t s);
  void range_sum(const uint32_t *lo, const uint32_t *hi, uint64_t n, uint32_t *out, cudaStream_t s);
  // range_sum answered by the per-query merge over the levels, never by a
  // compaction (no host wait: for a serving loop that must not stall)
  void range_sum_kway(const uint32_t *lo, const uint32_t *hi, uint64_t n, uint32_t *out, cudaStream_t s);
  // lookup and range_sum_kway of the same level state, run concurrently: the
  // lookups on `side` (forked from s once the levels are ready), the range
  // sums and the live-value prefixes they need on s, which then joins side.
  void lookup_and_range_sum(const uint32_t *queries, uint64_t nq, uint32_t *out_values, uint8_t *out_found,
                            const uint32_t *lo, const uint32_t *hi, uint64_t nr, uint32_t *out_sums,
                            cudaStream_t s, cudaStream_t side);
  void range_count(const uint32_t *lo, const uint32_t *hi, uint64_t n, uint32_t *out,
                   cudaStream_t s);
  void range_offsets(const uint32_t *lo, const uint32_t *hi, uint64_t n, uint64_t *offsets,
                     cudaStream_t s);
  void range_pairs(const uint32_t *lo, const uint32_t *hi, uint64_t n, const uint64_t *offsets,
                   uint32_t *out_keys, uint32_t *out_values, cudaStream_t s);
  void successor(const uint32_t *queries, uint64_t n, uint32_t *out_keys, cudaStream_t s);
  uint32_t status();
  uint64_t resident_bytes();
  // Lookups replayable from a CUDA graph: enqueue_table_lookup records (into
  // a capturing stream) a lookup that reads the level table from device
  // memory; launch_read_graph orders a captured graph like any operation and
  // brings the table up to date before it runs.
  void enqueue_table_lookup(const uint32_t *queries, uint64_t n, uint32_t *out_values, uint8_t *out_found,
                            cudaStream_t capturing);
  void launch_read_graph(cudaGraphExec_t exec, cudaStream_t s);
  // Makes s wait for every update enqueued so far, merges included (updates
  // return once their batch is admitted; their merges run on the
  // dictionary's own stream, overlapping the next batch's admission).
  void join(cudaStream_t s);
  // Kernel timing of the merge launches (CUDA events on the launching stream
  // around each merge kernel, plus the rows it read and wrote).
  void set_kernel_timing(bool on);
  void kernel_timing(uint64_t *launches, double *total_ms, double *bytes);
  void size(uint64_t *rows, uint32_t *levels);
  // LSMu's explicit cleanup (FliX/impl_lsm_tree.cuh:1256-1400): every level
  // merged into one run of the newest live versions, tombstones and shadowed
  // versions dropped; returns the live key count (synchronises).
  uint64_t cleanup(cudaStream_t s);

  // Staged updates, replayable from CUDA graphs (the serving loop).  A staged
  // update admits a batch of exactly `n` keys (a size class; the caller pads
  // with copies of its last key and value, which change nothing) into one of
  // `slots` fixed staging runs with fixed admission buffers, so its four
  // admission kernels can be captured once and replayed.  Staged runs are the
  // newest levels of every point lookup, successor and table lookup; they
  // merge into the levels (the regular cascade) when stage_flush runs - which
  // every other update, range operation, build and clear does first, and
  // which the caller runs when no slot is free.
  void stage_configure(uint32_t slots, uint64_t max_keys, cudaStream_t s);
  // a free staging slot, or -1 when every slot holds a run
  int stage_free_slot() const;
  // records the admission of slot `slot` into a capturing stream; `mode` is
  // kStageInsert, kStageErase or kStageMixed, and the batch is read from
  // stage_input(): keys at words [0, n), values (insert, mixed) at words
  // [n, 2n), erase marks (mixed) as bytes from word 2n on
  void enqueue_stage_admit(uint32_t slot, uint64_t n, int mode, cudaStream_t capturing);
  uint32_t *stage_input() const { return stage_in_; }
  // launches a captured staged-update graph, ordered like an update; `tombs`:
  // the batch may erase keys
  void launch_stage_graph(cudaGraphExec_t exec, uint32_t slot, uint64_t n, bool tombs, cudaStream_t s);
  void stage_flush(cudaStream_t s);
  uint64_t stage_flushes() const { return stage_flushes_; }
  uint32_t stage_slots() const { return uint32_t(staged_.size()); }

  // Introspection for tests and benchmarks.
  uint32_t level_count() const { return uint32_t(caps_.size()); }
  uint64_t level_capacity(uint32_t i) const { return caps_[i]; }

 private:
  struct Level {
    RunBuffer *run = nullptr;
    uint64_t upper = 0;  // upper bound of the row count known on the host
    uint64_t gen = 0;    // bumps whenever the level changes
    bool tombs = false;  // may hold tombstone rows
  };
  struct Receipt;

  void begin_op(cudaStream_t s, bool update = false);
  void end_op(cudaStream_t s);
  void host_sync();
  void apply_receipt(bool wait);
  void post_receipt(cudaStream_t s);
  lsm::ReceiptSrc next_receipt(int dest);
  void receipt_posted();
  void reject_if_failed() const;
  // erase: the erase marks of a mixed batch (null for insert / erase batches)
  void admit(const uint32_t *keys, const uint32_t *values, const uint8_t *erase, uint64_t n, bool tombstone,
             cudaStream_t s);
  // write_dir false: the run's directory is left to the first read (dir_ok)
  RunBuffer *sort_dedup(const uint32_t *keys, const uint32_t *values, uint64_t n, bool tombstone,
                        cudaStream_t s, const uint8_t *erase = nullptr, bool write_dir = true);
  RunBuffer *bucket_admit(const uint32_t *keys, const uint32_t *values, const uint8_t *erase, uint64_t n,
                          bool tombstone, cudaStream_t s, bool write_dir);
  void bucket_admit_into(const uint32_t *keys, const uint32_t *values, const uint8_t *erase, uint64_t n,
                         bool tombstone, cudaStream_t s, RunBuffer *out, unsigned long long *w0,
                         unsigned long long *w1, void *scratch, bool write_dir = true);
  static size_t bucket_admit_scratch_bytes(uint64_t n);
  void flush_staged_locked(cudaStream_t s);
  bool stage_seq_pending() const {
    for (const Staged &x : staged_)
      if (x.seq) return true;
    return false;
  }
  void drop_staged() {
    for (Staged &x : staged_) x.seq = x.upper = 0, x.tombs = false;
    ++next_gen_;
  }
  // carry_owned = false: the carry belongs to someone else (a staging run);
  // the cascade reads it but never releases or keeps it
  void cascade(RunBuffer *carry, uint64_t carry_upper, bool carry_tombs, cudaStream_t s, bool want_receipt,
               bool carry_owned = true);
  RunBuffer *merge(RunBuffer *newer, RunBuffer *older, uint64_t out_upper, bool drop_tombstones,
                   cudaStream_t s, const lsm::ReceiptSrc *rcpt = nullptr, bool release_newer = true,
                   bool release_older = true);
  // Range batches: merge every level into one tombstone-free run when the
  // rows the batch covers outweigh the merge; returns the single level to
  // answer from, or -1 to use the per-query k-way merge.
  int ranges_on_single_level(const uint32_t *lo, const uint32_t *hi, uint64_t n, cudaStream_t s);
  void compact_all(cudaStream_t s);
  const unsigned long long *value_prefix(int level, cudaStream_t s);
  void live_level_set(void *out, cudaStream_t s);
  void release_levels(cudaStream_t s);
  void fit_model(RunBuffer *run, uint64_t upper, cudaStream_t s);
  void fit_now(RunBuffer *run, uint64_t upper, cudaStream_t s);
  // Before every read: the directories a merge left out are built, then the
  // learned models of search mode 1 (and the next update's merges will write
  // their directories: a read may follow them again).
  void ensure_models(cudaStream_t s);
  void *scratch(size_t bytes, cudaStream_t s);
  void *admit_scratch(size_t bytes, cudaStream_t s);
  void ensure_sort_space(uint64_t n, cudaStream_t s);
  // the lookup kernel over the current level set on s (no ordering of its own)
  void launch_lookup(const uint32_t *queries, uint64_t n, uint32_t *out_values, uint8_t *out_found,
                     cudaStream_t s);
  void level_set(void *out) const;
  lsm::LevelView view_of(int level) const;
  lsm::LevelView view_of_run(const RunBuffer *r) const;

  DictConfig cfg_;
  uint64_t batch_capacity_ = 0;
  uint64_t budget_ = 0;
  uint32_t fan_in_ = 4;
  uint32_t rows_log2_ = 3;
  int num_sms_ = 148;
  std::vector<uint64_t> caps_;
  std::vector<Level> levels_;
  RunPool pool_;
  uint64_t next_gen_ = 1;

  // sort space for admission: two u64 word buffers + radix workspace
  unsigned long long *words_[2] = {nullptr, nullptr};
  uint64_t words_cap_ = 0;
  void *scratch_ = nullptr;  // merges and reads
  size_t scratch_bytes_ = 0;
  void *ascratch_ = nullptr;  // admission (runs while the previous batch merges)
  size_t ascratch_bytes_ = 0;
  uint32_t *dev_status_ = nullptr;

  // receipts (pinned host copy of the level row counts and status)
  Receipt *receipt_host_ = nullptr;
  void *receipt_dev_ = nullptr;
  uint32_t receipt_seq_ = 0;  // sequence number of the newest posted receipt
  bool receipt_pending_ = false;
  std::vector<uint64_t> receipt_gens_;

  // u64 prefix sums of a single level's values (range sums after compaction)
  unsigned long long *prefix_ = nullptr;
  uint64_t prefix_cap_ = 0;
  uint64_t prefix_gen_ = 0;
  // u32 live-value prefix of every level (range sums over several levels),
  // rebuilt for a level only when its generation changed
  struct LivePrefix {
    uint32_t *p = nullptr;
    uint64_t cap = 0;
    uint64_t gen = ~0ull;
  };
  std::vector<LivePrefix> live_;
  std::vector<LivePrefix> live_staged_;  // one per staging slot (gen = the staged run's seq)
  void refresh_live_prefix(LivePrefix &lp, RunBuffer *run, uint64_t upper, uint64_t gen, uint64_t min_cap,
                           cudaStream_t s);
  uint64_t live_bytes_ = 0;
  unsigned long long *width_ = nullptr;  // device word for the range-width estimate
  unsigned long long *width_host_ = nullptr;

  uint32_t status_bits_ = 0;
  bool failed_ = false;
  std::string failure_;
  struct MergeTrace {
    cudaEvent_t start, stop;
  };
  bool timing_ = false;
  std::vector<MergeTrace> traces_;           // events of the merges timed so far
  std::vector<cudaEvent_t> spare_events_;
  unsigned long long *trace_dev_ = nullptr;  // 4 words per timed merge
  static constexpr size_t kMaxTraces = 8192;
  void *table_dev_ = nullptr;  // device copy of the level set (graph-replayed lookups)
  uint64_t table_gen_ = ~0ull;            // next_gen_ when the table was last written
  cudaEvent_t op_done_ = nullptr;
  // Merges of admitted batches run on merge_stream_: each waits for its
  // batch's admission (adm_done_); reads and every other operation wait for
  // merge_done_ when merges are pending.
  cudaStream_t merge_stream_ = nullptr;
  cudaEvent_t adm_done_ = nullptr;
  cudaEvent_t merge_done_ = nullptr;
  cudaEvent_t fork_ = nullptr, side_done_ = nullptr;  // lookup_and_range_sum
  bool merges_pending_ = false;
  // Merges write their output's directory unless the operation before this
  // update was an update too: levels rewritten by back-to-back update batches
  // are mostly merged again before any read, so their directories are built
  // by the read that needs them (ensure_models).
  bool prev_update_ = false;
  bool merge_dirs_ = true;
  // staged updates (serving): fixed staging runs, newest first by seq
  struct Staged {
    RunBuffer *run = nullptr;
    uint64_t upper = 0;
    uint64_t seq = 0;  // 0 = free
    bool tombs = false;
  };
  std::vector<Staged> staged_;
  uint64_t stage_seq_ = 0;
  uint64_t stage_max_ = 0;
  uint64_t stage_flushes_ = 0;
  uint32_t *stage_in_ = nullptr;                      // the staged graphs' input (2 * stage_max_ words)
  unsigned long long *stage_words_[2] = {nullptr, nullptr};
  void *stage_scratch_ = nullptr;
  cudaStream_t last_stream_ = nullptr;  // stream of the last operation (op_done_ was recorded there)
  bool last_stream_known_ = false;
  mutable std::mutex mu_;
};

}  // namespace gpulsm
