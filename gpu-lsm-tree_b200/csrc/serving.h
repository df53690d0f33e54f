// Serving loop over one LSM dictionary: continuous batching of mixed
// lookup / insert / erase / range-sum requests of uneven sizes.
//
// The reference has no serving facility: GPULSMOpt serialises every call
// behind a mutex and an operation event (GPULSMOpt.cuh:6852-6858), so a
// caller batches by hand.  Here requests are submitted from any host thread
// with host buffers; a worker thread takes what has queued, in arrival order,
// into a round of at most three dictionary calls - every insert and erase of
// the round as one mixed update batch, then every lookup as one lookup and
// every range sum as one range sum, the two reads running concurrently on the
// same level state - and admits an update only while the
// dictionary's resident bytes plus the rounds in flight stay inside a
// device-memory budget.  submit() copies the request's keys (and values or
// upper bounds) into a pinned ring on the caller's thread, so the worker
// copies nothing: a round uploads the ring span of its requests in one or two
// copies, and one gather kernel lays the span out as the three calls read
// it.  Rounds occupy one of `depth` pipeline slots (device buffers): the
// upload of round r+1 overlaps the kernels of round r, and a completion
// thread returns results, releases the round's ring span and records each
// request's latency (submit to results in the caller's buffers).
//
// Semantics (linearizable): rounds apply in order; inside a round the updates
// apply one at a time in submission order (the update batch keeps the last
// row of every key), then the reads see the result.  Every request of a round
// is in flight from before the round is formed until after it completes, so
// this order is consistent with real time; a read submitted after a round
// formed sees all of that round's updates.  wait_round reports the round of a
// request, so a caller can replay the order.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "lsm_dictionary.h"

namespace gpulsm {

enum ServeKind : uint32_t { kServeLookup = 0, kServeInsert = 1, kServeErase = 2, kServeRangeSum = 3 };

struct ServeStats {
  uint64_t completed = 0;
  uint64_t rejected = 0;
  uint64_t rounds = 0;
  uint64_t keys = 0;          // keys (or range queries) of completed requests
  double p50_us = 0, p99_us = 0, max_us = 0, mean_us = 0;
  double mean_round_keys = 0;
  double wall_s = 0;          // first submit to last completion since the last reset
  double gpu_busy_s = 0;      // device time of the rounds (upload done -> kernels done)
  double host_launch_s = 0;   // worker time staging and launching rounds
  uint64_t graph_rounds = 0;  // lookup-only rounds replayed from a captured CUDA graph
  uint64_t graph_updates = 0;  // update batches replayed from a captured CUDA graph (staged)
  uint64_t stage_flushes = 0;  // staged runs merged into the levels
  // device time per request kind (updates: merges included; a round's update
  // batch is charged to insert, or to erase when it only erases)
  double kind_gpu_s[4] = {0, 0, 0, 0};
  double host_copy_s = 0;     // submitters' time copying request data into the pinned ring
  double host_scatter_s = 0;  // completion time copying results into the requests' buffers
  double max_round_gpu_us = 0;  // the longest round's device time (upload done -> kernels done)
  double max_launch_us = 0;     // the worker's longest time staging and launching one round
};

// Open-loop load: Poisson arrivals, kind mix, log-uniform sizes, Zipf keys.
struct LoadSpec {
  double rate_per_s = 0;       // request arrivals per second; 0 = closed loop
  double seconds = 1.0;
  uint32_t max_outstanding = 64;  // closed loop: requests kept in flight
  double mix[4] = {0.6, 0.2, 0.1, 0.1};  // lookup, insert, erase, range-sum
  uint32_t min_keys = 1, max_keys = 1u << 16;
  double zipf_s = 1.1;
  uint32_t range_width_max = 1u << 16;
  uint64_t seed = 1;
  const uint32_t *universe = nullptr;  // host keys the requests draw from (by Zipf rank)
  uint64_t universe_n = 0;
};

class Server {
 public:
  Server(const DictConfig &cfg, uint64_t budget_bytes, uint32_t max_round_keys, uint32_t depth);
  ~Server();
  Server(const Server &) = delete;
  Server &operator=(const Server &) = delete;

  // Host buffers.  keys: the request keys (range: lower bounds); aux: insert
  // values / range upper bounds - both copied before submit returns (it
  // waits while the pinned ring is full); out: lookup values / range sums;
  // found: optional lookup flags - owned by the caller until the request
  // completes.
  uint64_t submit(uint32_t kind, const uint32_t *keys, const uint32_t *aux, uint64_t n, uint32_t *out,
                  uint8_t *found);
  int poll(uint64_t ticket);  // 0 pending, 1 done, < 0 failed (negated gpulsm status)
  // 1 done, < 0 failed; *round (optional): the request's round, numbered from
  // 1 in execution order (0: completed without a round - empty or rejected)
  int wait(uint64_t ticket, uint64_t *round = nullptr);
  void drain();
  ServeStats stats();
  void reset_stats();
  void run_load(const LoadSpec &spec, ServeStats *out);
  // staged (graph-replayed) or direct update runs; waits for the requests in flight
  void set_staged_updates(bool on);
  LsmDictionary &dict() { return dict_; }
  uint64_t device_bytes() const { return slot_bytes_ * slots_.size(); }

 private:
  struct Req {
    uint32_t kind;
    uint64_t pos;  // ring position (bytes) of its keys, then its values / upper bounds
    bool ready;    // its data is in the ring
    uint64_t n;
    uint32_t *out;
    uint8_t *found;
    double t_submit;
    int state;       // 0 queued, 1 done, < 0 failed
    uint64_t round;  // the round that ran it (0: none)
  };
  struct Part {  // one request's share of a run
    uint64_t ticket;
    uint32_t kind;
    uint64_t off;  // first key of this request inside its run
    uint64_t n;
    uint64_t src;  // word offset of its keys in the round's uploaded span
    uint32_t *out;
    uint8_t *found;
  };
  // The calls of a round, in this order: the update batch, the lookups, the
  // range sums (each run holds its requests in arrival order).
  enum RunIndex : int { kRunUpdate = 0, kRunLookup = 1, kRunRange = 2, kRuns = 3 };
  struct Run {
    uint32_t kind = 0;     // kServeInsert for the update batch, kServeLookup, kServeRangeSum
    int mode = 0;          // update batch: kStageInsert, kStageErase or kStageMixed
    uint64_t in_off = 0;   // words into the staging input: keys, then values / upper bounds
    uint64_t out_off = 0;  // words into the staging output
    uint64_t n = 0;
    uint64_t cls = 0;      // update batch: keys padded to this size class (staged), else n;
                           // values at in_off + cls, erase marks (bytes) at word in_off + 2 cls
    size_t first_part = 0, parts = 0;
    int status = 0;        // 0, or the negated gpulsm status of a failed call
  };
  struct Slot {
    uint32_t *h_out = nullptr;
    uint8_t *h_found = nullptr;
    unsigned char *h_table = nullptr;  // gather table (pinned): entry count, then entries
    uint32_t *d_in = nullptr, *d_out = nullptr;
    uint8_t *d_found = nullptr;
    uint32_t *d_span = nullptr;        // the round's ring span, uploaded
    unsigned char *d_table = nullptr;
    uint64_t span_begin = 0, span_end = 0;  // ring positions (bytes)
    uint64_t span_id = 0;
    uint32_t entries = 0;
    bool timed_round = false;          // records the per-call timing events
    cudaEvent_t uploaded = nullptr, computed = nullptr, downloaded = nullptr;
    Run runs[kRuns];
    std::vector<Part> parts;  // grouped by run
    uint64_t round = 0;
    uint64_t in_words = 0, out_words = 0, keys = 0;
    uint64_t bytes = 0;  // device bytes the round's updates may add (admission budget)
    bool launched = false;
    // lookup-only rounds replay a CUDA graph per size class (gather, lookup
    // against the device level table, copy out) captured on first use
    std::vector<std::pair<uint32_t, cudaGraphExec_t>> graphs;
    // device time per run: events bracketing each timed call on the compute
    // stream (the stream is serial, so a pair spans that call's work alone)
    std::vector<cudaEvent_t> marks;
    std::vector<std::pair<uint32_t, uint32_t>> timed;  // (kind, index of the first event of the pair)
  };

  void worker();
  void completer();
  // with mu_ held: a round's ring span (numbered in formation order) is no
  // longer read; spans are released (the ring tail advanced) in order
  uint64_t span_open(uint64_t end);
  void span_done(uint64_t id);
  bool form_round(Slot &slot);
  void launch_round(Slot &slot);
  cudaGraphExec_t lookup_graph(Slot &slot, uint32_t size_class);
  // the graph of a staged update (kStage* mode) of `size_class` keys into staging slot `stage`
  cudaGraphExec_t update_graph(int mode, uint32_t size_class, uint32_t stage);
  uint64_t size_class(uint64_t n) const;
  // capture and instantiate every graph a round may replay (lookup rounds:
  // per slot and size class; staged updates: per mode, size class and
  // staging slot), so that no round pays a first capture
  void prepare_lookup_graphs();
  void prepare_update_graphs();
  // staging input words of a round with these update / lookup / range-sum key counts
  uint64_t round_words(uint64_t nu, bool mixed, uint64_t nl, uint64_t nr) const;
  static double now_s();

  LsmDictionary dict_;
  int device_ = 0;
  uint64_t budget_;
  uint32_t max_round_keys_;
  uint64_t slot_bytes_ = 0;
  uint64_t in_words_cap_ = 0;  // staging input words of a slot
  // the pinned request ring: positions grow without bound, byte pos % cap
  unsigned char *ring_ = nullptr;
  uint64_t ring_cap_ = 0, span_cap_ = 0;
  uint64_t ring_head_ = 0, ring_tail_ = 0;
  std::deque<std::pair<uint64_t, bool>> spans_;  // (end, done) of formed rounds, in order
  uint64_t span_base_ = 0;                       // the number of spans_.front()
  std::vector<Slot> slots_;
  std::deque<uint32_t> free_slots_;
  std::deque<uint32_t> inflight_;
  cudaStream_t compute_ = nullptr, upload_ = nullptr, download_ = nullptr;
  cudaStream_t capture_ = nullptr;  // graphs are captured here (thread-local mode)
  cudaStream_t side_ = nullptr;     // a round's lookups beside its range sums
  uint64_t st_graph_rounds_ = 0;
  // staged updates: update runs replayed from captured graphs (admission only;
  // the staged runs merge into the levels when the staging slots are full)
  bool staged_updates_ = false;
  bool stage_ready_ = false;  // the dictionary's staging slots are configured
  std::vector<std::pair<uint64_t, cudaGraphExec_t>> update_graphs_;  // key: mode | class << 2 | stage << 40
  uint64_t st_graph_updates_ = 0;

  std::mutex mu_;
  std::condition_variable cv_work_, cv_done_, cv_inflight_, cv_space_;
  std::deque<uint64_t> queue_;
  std::unordered_map<uint64_t, Req> reqs_;
  uint64_t next_ticket_ = 1;
  uint64_t next_round_ = 1;
  uint64_t inflight_bytes_ = 0;
  bool stop_ = false;

  // statistics since the last reset
  std::vector<float> lat_us_;
  uint64_t st_completed_ = 0, st_rejected_ = 0, st_rounds_ = 0, st_keys_ = 0, st_round_keys_ = 0;
  double st_first_ = -1, st_last_ = 0, st_gpu_s_ = 0, st_launch_s_ = 0;
  double st_max_gpu_s_ = 0, st_max_launch_s_ = 0;
  double st_kind_gpu_s_[4] = {0, 0, 0, 0}, st_copy_s_ = 0, st_scatter_s_ = 0;

  std::thread worker_, completer_;
};

}  // namespace gpulsm
