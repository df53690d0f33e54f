// Serving loop (serving.h): requests copied into a pinned ring at submit,
// rounds formed in arrival order, a device-memory budget for admission,
// pipelined slots, per-request latency.
#include "serving.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>

#include "common.cuh"

namespace gpulsm {

namespace {
// Device bytes an update of one key may add before its receipt is applied:
// the admitted run (9 B/row plus directory), sort words (16 B) and the
// transient merge output (9 B/row), rounded up.
constexpr uint64_t kUpdateBytesPerKey = 48;
constexpr size_t kMaxInflight = 2;
constexpr int kErrCapacity = 2;  // GPULSM_ERR_CAPACITY
constexpr int kErrCuda = 5;      // GPULSM_ERR_CUDA
constexpr uint32_t kMaxRoundRequests = 4096;
// per-call timing events (the kind breakdown of the statistics) are recorded
// on every kTimedEvery-th round only and scaled up: each pair costs the
// worker two event records
constexpr uint64_t kTimedEvery = 8;

// One piece of a round's staging layout: n words of the uploaded span (or its
// first word repeated, for the padding of a staged update batch) to the keys,
// values and erase marks of a run.
struct GatherEntry {
  unsigned long long src_key;   // word offset in the span
  unsigned long long src_aux;   // word offset in the span, or kNone: zeros
  unsigned long long dst_key;   // word offset in the staging input
  unsigned long long dst_aux;   // word offset, or kNone
  unsigned long long dst_mark;  // byte offset, or kNone
  uint32_t n;
  uint32_t mark;    // the erase mark written (mixed update batches)
  uint32_t repeat;  // every row copies word 0 of the source
  uint32_t unused;
};
constexpr unsigned long long kNone = ~0ull;
constexpr size_t kTableHeader = 64;  // the entry count, then the entries
constexpr size_t kTableBytes = kTableHeader + (kMaxRoundRequests + 1) * sizeof(GatherEntry);

// Lays a round's uploaded span out as its calls read it.  The entry count
// is read from the table, so a captured graph serves any round of its class.
__global__ void __launch_bounds__(256) serve_gather_kernel(const uint32_t *__restrict__ span,
                                                           const unsigned char *__restrict__ table,
                                                           uint32_t *__restrict__ stage) {
  const uint32_t count = *reinterpret_cast<const uint32_t *>(table);
  const GatherEntry *entries = reinterpret_cast<const GatherEntry *>(table + kTableHeader);
  uint8_t *stage_bytes = reinterpret_cast<uint8_t *>(stage);
  for (uint32_t r = blockIdx.y; r < count; r += gridDim.y) {
    const GatherEntry g = entries[r];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x) {
      const uint32_t j = g.repeat ? 0u : i;
      stage[g.dst_key + i] = span[g.src_key + j];
      if (g.dst_aux != kNone) stage[g.dst_aux + i] = g.src_aux != kNone ? span[g.src_aux + j] : 0u;
      if (g.dst_mark != kNone) stage_bytes[g.dst_mark + i] = uint8_t(g.mark);
    }
  }
}

dim3 gather_grid(uint64_t max_rows, uint32_t entries) {
  const uint64_t gx = std::min<uint64_t>(32, std::max<uint64_t>(1, (max_rows + 2047) / 2048));
  return dim3(unsigned(gx), std::max(1u, std::min(entries, 64u)));
}

int status_of(const std::exception &e) {
  const std::string m = e.what();
  return m.find("capacity") != std::string::npos ? -kErrCapacity : -kErrCuda;
}

bool is_update(uint32_t kind) { return kind == kServeInsert || kind == kServeErase; }
bool has_aux(uint32_t kind) { return kind == kServeInsert || kind == kServeRangeSum; }
bool has_out(uint32_t kind) { return kind == kServeLookup || kind == kServeRangeSum; }
}  // namespace

double Server::now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

Server::Server(const DictConfig &cfg, uint64_t budget_bytes, uint32_t max_round_keys, uint32_t depth)
    : dict_(cfg), budget_(budget_bytes), max_round_keys_(max_round_keys ? max_round_keys : (1u << 20)) {
  if (depth == 0) depth = 3;
  if (depth > 8) throw std::invalid_argument("serving depth must be in [1, 8]");
  if (max_round_keys_ > (1u << 24)) throw std::invalid_argument("max_round_keys must be <= 2^24");
  GPULSM_CUDA(cudaGetDevice(&device_));
  GPULSM_CUDA(cudaStreamCreateWithFlags(&compute_, cudaStreamNonBlocking));
  GPULSM_CUDA(cudaStreamCreateWithFlags(&upload_, cudaStreamNonBlocking));
  GPULSM_CUDA(cudaStreamCreateWithFlags(&download_, cudaStreamNonBlocking));
  GPULSM_CUDA(cudaStreamCreateWithFlags(&capture_, cudaStreamNonBlocking));
  GPULSM_CUDA(cudaStreamCreateWithFlags(&side_, cudaStreamNonBlocking));
  const uint64_t m = max_round_keys_;
  // inputs: at most two words and an erase mark a key, plus the padding of
  // a staged update batch (form_round checks the exact need)
  in_words_cap_ = 4 * m + 4096;
  // a round's span: its requests' data (at most 8 bytes a key), the data of
  // requests it refused, and a skip to the ring start; the ring holds several
  span_cap_ = 24 * m + 4096;
  ring_cap_ = std::max<uint64_t>(uint64_t(depth + 1) * 16 * m, 2 * span_cap_);
  GPULSM_CUDA(cudaMallocHost(&ring_, ring_cap_));
  slot_bytes_ = in_words_cap_ * 4 + m * 4 + m + span_cap_ + kTableBytes;  // inputs, outputs, flags, span, table
  slots_.resize(depth);
  for (uint32_t i = 0; i < depth; ++i) {
    Slot &s = slots_[i];
    GPULSM_CUDA(cudaMallocHost(&s.h_table, kTableBytes));
    GPULSM_CUDA(cudaMallocHost(&s.h_out, m * 4));
    GPULSM_CUDA(cudaMallocHost(&s.h_found, m));
    GPULSM_CUDA(cudaMalloc(&s.d_span, span_cap_));
    GPULSM_CUDA(cudaMalloc(&s.d_table, kTableBytes));
    GPULSM_CUDA(cudaMalloc(&s.d_in, in_words_cap_ * 4));
    GPULSM_CUDA(cudaMalloc(&s.d_out, m * 4));
    GPULSM_CUDA(cudaMalloc(&s.d_found, m));
    GPULSM_CUDA(cudaEventCreate(&s.uploaded));  // timed: device busy time per round
    GPULSM_CUDA(cudaEventCreate(&s.computed));
    GPULSM_CUDA(cudaEventCreateWithFlags(&s.downloaded, cudaEventDisableTiming));
    free_slots_.push_back(i);
  }
  // staged updates: update runs are admitted into fixed staging runs by
  // captured graphs; 4 staging slots (fewer when the level schedule is deep)
  // (staged update runs are off by default: on the serving mix they lowered
  // peak throughput, see set_staged_updates)
  if (max_round_keys_ <= (1u << 20)) {
    dict_.stage_configure(4, max_round_keys_, compute_);
    GPULSM_CUDA(cudaStreamSynchronize(compute_));
    stage_ready_ = true;
  }
  prepare_lookup_graphs();
  worker_ = std::thread(&Server::worker, this);
  completer_ = std::thread(&Server::completer, this);
}

Server::~Server() {
  try {
    drain();
  } catch (...) {
  }
  {
    std::lock_guard<std::mutex> g(mu_);
    stop_ = true;
  }
  cv_work_.notify_all();
  cv_inflight_.notify_all();
  cv_space_.notify_all();
  if (worker_.joinable()) worker_.join();
  if (completer_.joinable()) completer_.join();
  cudaStreamSynchronize(compute_);
  cudaStreamSynchronize(upload_);
  cudaStreamSynchronize(download_);
  cudaStreamSynchronize(side_);
  for (Slot &s : slots_) {
    cudaFreeHost(s.h_table);
    cudaFree(s.d_span);
    cudaFree(s.d_table);
    cudaFreeHost(s.h_out);
    cudaFreeHost(s.h_found);
    cudaFree(s.d_in);
    cudaFree(s.d_out);
    cudaFree(s.d_found);
    cudaEventDestroy(s.uploaded);
    cudaEventDestroy(s.computed);
    cudaEventDestroy(s.downloaded);
    for (auto &g : s.graphs) cudaGraphExecDestroy(g.second);
    for (cudaEvent_t e : s.marks) cudaEventDestroy(e);
  }
  for (auto &g : update_graphs_) cudaGraphExecDestroy(g.second);
  cudaFreeHost(ring_);
  cudaStreamDestroy(capture_);
  cudaStreamDestroy(compute_);
  cudaStreamDestroy(upload_);
  cudaStreamDestroy(download_);
  cudaStreamDestroy(side_);
}

uint64_t Server::submit(uint32_t kind, const uint32_t *keys, const uint32_t *aux, uint64_t n, uint32_t *out,
                        uint8_t *found) {
  if (kind > kServeRangeSum) throw std::invalid_argument("unknown request kind");
  if (n > max_round_keys_) throw std::length_error("request larger than max_round_keys");
  if (n && !keys) throw std::invalid_argument("null request keys");
  if (n && has_aux(kind) && !aux) throw std::invalid_argument("null request values / upper bounds");
  if (n && has_out(kind) && !out) throw std::invalid_argument("null request output");
  const double t = now_s();
  const uint64_t key_bytes = n * 4, need = key_bytes * (has_aux(kind) ? 2 : 1);
  uint64_t tk, pos;
  {
    // ring space in submission order: a request never wraps (it starts over
    // at the ring start when it does not fit before the end)
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      if (stop_) throw std::runtime_error("server is shutting down");
      pos = ring_head_;
      if (need && pos % ring_cap_ + need > ring_cap_) pos += ring_cap_ - pos % ring_cap_;
      if (pos + need - ring_tail_ <= ring_cap_) break;
      cv_space_.wait(lk);  // the completion of earlier rounds frees their spans
    }
    ring_head_ = pos + need;
    tk = next_ticket_++;
    reqs_[tk] = Req{kind, pos, need == 0, n, out, found, t, 0, 0};
    if (st_first_ < 0) st_first_ = t;
    queue_.push_back(tk);
  }
  if (need) {  // the copy runs outside the lock; the worker takes the request once it is ready
    const double c0 = now_s();
    unsigned char *dst = ring_ + pos % ring_cap_;
    std::memcpy(dst, keys, key_bytes);
    if (has_aux(kind)) std::memcpy(dst + key_bytes, aux, key_bytes);
    const double c1 = now_s();
    std::lock_guard<std::mutex> g(mu_);
    reqs_.at(tk).ready = true;
    st_copy_s_ += c1 - c0;
  }
  cv_work_.notify_one();
  return tk;
}

uint64_t Server::span_open(uint64_t end) {
  spans_.emplace_back(end, false);
  return span_base_ + spans_.size() - 1;
}

void Server::span_done(uint64_t id) {
  spans_.at(id - span_base_).second = true;
  bool freed = false;
  while (!spans_.empty() && spans_.front().second) {
    ring_tail_ = std::max(ring_tail_, spans_.front().first);
    spans_.pop_front();
    ++span_base_;
    freed = true;
  }
  if (freed) cv_space_.notify_all();
}

int Server::poll(uint64_t ticket) {
  std::lock_guard<std::mutex> g(mu_);
  auto it = reqs_.find(ticket);
  if (it == reqs_.end()) throw std::invalid_argument("unknown or already collected ticket");
  const int st = it->second.state;
  if (st != 0) reqs_.erase(it);
  return st;
}

int Server::wait(uint64_t ticket, uint64_t *round) {
  std::unique_lock<std::mutex> lk(mu_);
  if (reqs_.find(ticket) == reqs_.end()) throw std::invalid_argument("unknown or already collected ticket");
  cv_done_.wait(lk, [&] { return reqs_.at(ticket).state != 0; });
  const Req &q = reqs_.at(ticket);
  const int st = q.state;
  if (round) *round = q.round;
  reqs_.erase(ticket);
  return st;
}

void Server::drain() {
  std::unique_lock<std::mutex> lk(mu_);
  cv_done_.wait(lk, [&] { return queue_.empty() && inflight_.empty() && free_slots_.size() == slots_.size(); });
}

void Server::set_staged_updates(bool on) {
  drain();
  std::lock_guard<std::mutex> g(mu_);  // the worker forms no round while this is held
  if (on && !stage_ready_) throw std::invalid_argument("staged updates need max_round_keys <= 2^20");
  if (!on && staged_updates_) {
    dict_.stage_flush(compute_);
    GPULSM_CUDA(cudaStreamSynchronize(compute_));
  }
  staged_updates_ = on;
  if (on) prepare_update_graphs();
}

void Server::prepare_lookup_graphs() {
  for (Slot &slot : slots_)
    for (uint64_t c = 1024;; c <<= 1) {
      (void)lookup_graph(slot, uint32_t(std::min<uint64_t>(c, max_round_keys_)));
      if (c >= max_round_keys_) break;
    }
}

void Server::prepare_update_graphs() {
  const uint32_t stages = dict_.stage_slots();
  for (uint64_t n = 1; n <= max_round_keys_;) {  // every size class once
    const uint64_t c = size_class(n);
    for (int mode = kStageInsert; mode <= kStageMixed; ++mode)
      for (uint32_t st = 0; st < stages; ++st) (void)update_graph(mode, uint32_t(c), st);
    n = c + 1;
  }
}

void Server::reset_stats() {
  std::lock_guard<std::mutex> g(mu_);
  lat_us_.clear();
  st_completed_ = st_rejected_ = st_rounds_ = st_keys_ = st_round_keys_ = st_graph_rounds_ = 0;
  st_graph_updates_ = 0;
  st_first_ = -1;
  st_last_ = st_gpu_s_ = st_launch_s_ = 0;
  st_max_gpu_s_ = st_max_launch_s_ = 0;
  for (double &k : st_kind_gpu_s_) k = 0;
  st_copy_s_ = st_scatter_s_ = 0;
}

ServeStats Server::stats() {
  std::vector<float> lat;
  ServeStats s;
  {
    std::lock_guard<std::mutex> g(mu_);
    lat = lat_us_;
    s.completed = st_completed_;
    s.rejected = st_rejected_;
    s.rounds = st_rounds_;
    s.keys = st_keys_;
    s.mean_round_keys = st_rounds_ ? double(st_round_keys_) / double(st_rounds_) : 0.0;
    s.wall_s = st_first_ >= 0 ? std::max(0.0, st_last_ - st_first_) : 0.0;
    s.gpu_busy_s = st_gpu_s_;
    s.host_launch_s = st_launch_s_;
    s.max_round_gpu_us = st_max_gpu_s_ * 1e6;
    s.max_launch_us = st_max_launch_s_ * 1e6;
    s.graph_rounds = st_graph_rounds_;
    s.graph_updates = st_graph_updates_;
    s.stage_flushes = dict_.stage_flushes();
    for (int k = 0; k < 4; ++k) s.kind_gpu_s[k] = st_kind_gpu_s_[k];
    s.host_copy_s = st_copy_s_;
    s.host_scatter_s = st_scatter_s_;
  }
  if (!lat.empty()) {
    auto pct = [&](double p) {
      const size_t k = std::min(lat.size() - 1, size_t(p * double(lat.size() - 1) + 0.5));
      std::nth_element(lat.begin(), lat.begin() + long(k), lat.end());
      return double(lat[k]);
    };
    double sum = 0;
    float mx = 0;
    for (float v : lat) {
      sum += v;
      mx = std::max(mx, v);
    }
    s.mean_us = sum / double(lat.size());
    s.max_us = mx;
    s.p50_us = pct(0.50);
    s.p99_us = pct(0.99);
  }
  return s;
}

// Staging input words of a round: the update batch (keys, values when any
// request inserts, erase marks as bytes when it mixes inserts and erases,
// padded to its size class when staged), the lookup keys, the range bounds.
uint64_t Server::round_words(uint64_t nu, bool mixed, uint64_t nl, uint64_t nr) const {
  uint64_t w = nl + 2 * nr;
  if (nu) {
    const uint64_t c = staged_updates_ ? size_class(nu) : nu;
    w += 2 * c + (mixed ? (c + 3) / 4 : 0);
  }
  return w;
}

// Called with mu_ held: take requests in arrival order into the round's
// three runs until the round is full; reject updates the budget cannot hold.
// The requests taken cover one span of the ring (refused and empty requests
// included), which the round uploads and releases when it completes.
bool Server::form_round(Slot &slot) {
  for (Run &r : slot.runs) r = Run{};
  slot.runs[kRunUpdate].kind = kServeInsert;
  slot.runs[kRunLookup].kind = kServeLookup;
  slot.runs[kRunRange].kind = kServeRangeSum;
  slot.parts.clear();
  slot.bytes = 0;
  uint64_t keys = 0;
  const uint64_t resident = dict_.resident_bytes();
  const double t = now_s();
  bool any = false, ins = false, era = false, taken = false;
  uint64_t begin = 0, end = 0;
  uint32_t nparts = 0;
  std::vector<Part> parts[kRuns];
  while (!queue_.empty()) {
    const uint64_t tk = queue_.front();
    Req &q = reqs_.at(tk);
    if (!q.ready) break;  // its data is still being copied into the ring
    const uint64_t need = q.n * 4 * (has_aux(q.kind) ? 2 : 1);
    if (taken && q.pos + need - begin > span_cap_) break;
    if (nparts >= kMaxRoundRequests) break;
    if (keys > 0 && keys + q.n > max_round_keys_) break;
    const int ri = is_update(q.kind) ? kRunUpdate : q.kind == kServeLookup ? kRunLookup : kRunRange;
    if (keys > 0 && q.n) {  // the staging input must hold the round with its padding
      uint64_t n[kRuns] = {slot.runs[0].n, slot.runs[1].n, slot.runs[2].n};
      n[ri] += q.n;
      const bool mixed = (ins || q.kind == kServeInsert) && (era || q.kind == kServeErase);
      if (round_words(n[kRunUpdate], mixed, n[kRunLookup], n[kRunRange]) > in_words_cap_) break;
    }
    queue_.pop_front();
    if (!taken) begin = q.pos;
    taken = true;
    end = std::max(end, q.pos + need);
    if (q.n == 0) {  // nothing to do: done at once
      q.state = 1;
      lat_us_.push_back(float((t - q.t_submit) * 1e6));
      ++st_completed_;
      st_last_ = t;
      continue;
    }
    if (is_update(q.kind)) {
      const uint64_t growth = q.n * kUpdateBytesPerKey;
      if (resident + device_bytes() + inflight_bytes_ + slot.bytes + growth > budget_) {
        q.state = -kErrCapacity;  // the device-memory budget cannot hold this update
        ++st_rejected_;
        st_last_ = t;
        continue;
      }
      slot.bytes += growth;
      ins = ins || q.kind == kServeInsert;
      era = era || q.kind == kServeErase;
    }
    Run &r = slot.runs[ri];
    parts[ri].push_back(Part{tk, q.kind, r.n, q.n, (q.pos - begin) / 4, q.out, q.found});
    ++nparts;
    r.n += q.n;
    keys += q.n;
    any = true;
  }
  if (!taken) return false;
  if (!any) {  // only refused or empty requests: their data is not read
    span_done(span_open(end));
    return false;
  }
  slot.span_begin = begin;
  slot.span_end = end;
  slot.span_id = span_open(end);
  slot.round = next_round_++;
  slot.timed_round = slot.round % kTimedEvery == 0;
  // staging layout, runs in execution order: the update batch (keys, values,
  // erase marks), the lookup keys, the range lower then upper bounds
  slot.runs[kRunUpdate].mode = (ins && era) ? kStageMixed : era ? kStageErase : kStageInsert;
  uint64_t in = 0, out = 0;
  for (int ri = 0; ri < kRuns; ++ri) {
    Run &r = slot.runs[ri];
    r.in_off = in;
    r.out_off = out;
    r.first_part = slot.parts.size();
    r.parts = parts[ri].size();
    slot.parts.insert(slot.parts.end(), parts[ri].begin(), parts[ri].end());
    for (const Part &p : parts[ri]) reqs_.at(p.ticket).round = slot.round;
    if (!r.n) continue;
    if (ri == kRunUpdate) {
      r.cls = staged_updates_ ? size_class(r.n) : r.n;
      in += r.mode == kStageErase ? r.cls : 2 * r.cls + (r.mode == kStageMixed ? (r.cls + 3) / 4 : 0);
    } else {
      r.cls = r.n;
      in += r.n * (ri == kRunRange ? 2 : 1);
      out += r.n;
    }
  }
  slot.in_words = in;
  slot.out_words = out;
  slot.keys = keys;
  return true;
}

// The graph of a lookup-only round of up to `size_class` keys in this slot:
// gather the uploaded keys into the staging input, look them up against the
// dictionary's device level table, copy values and flags out.  Keys past the
// round's own are stale staging contents; their answers land past the
// round's results and are never read.
cudaGraphExec_t Server::lookup_graph(Slot &slot, uint32_t size_class) {
  for (const auto &g : slot.graphs)
    if (g.first == size_class) return g.second;
  const uint64_t c = size_class;
  cudaGraph_t graph = nullptr;
  GPULSM_CUDA(cudaStreamBeginCapture(capture_, cudaStreamCaptureModeThreadLocal));
  try {
    serve_gather_kernel<<<gather_grid(c, 64), 256, 0, capture_>>>(slot.d_span, slot.d_table, slot.d_in);
    GPULSM_CUDA(cudaGetLastError());
    dict_.enqueue_table_lookup(slot.d_in, c, slot.d_out, slot.d_found, capture_);
    GPULSM_CUDA(cudaMemcpyAsync(slot.h_out, slot.d_out, c * 4, cudaMemcpyDeviceToHost, capture_));
    GPULSM_CUDA(cudaMemcpyAsync(slot.h_found, slot.d_found, c, cudaMemcpyDeviceToHost, capture_));
  } catch (...) {
    cudaStreamEndCapture(capture_, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  GPULSM_CUDA(cudaStreamEndCapture(capture_, &graph));
  cudaGraphExec_t exec = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  GPULSM_CUDA(e);
  slot.graphs.emplace_back(size_class, exec);
  return exec;
}

// The next free pair of timing events of a slot (created on first use).
static uint32_t next_mark_pair(std::vector<cudaEvent_t> &marks, size_t used) {
  while (marks.size() < used + 2) {
    cudaEvent_t e;
    GPULSM_CUDA(cudaEventCreate(&e));
    marks.push_back(e);
  }
  return uint32_t(used);
}

// Size classes of staged updates: from 1024 keys, four classes per power of
// two (padding at most a quarter of the batch), the last one the round limit.
uint64_t Server::size_class(uint64_t n) const {
  uint64_t c = 1024;
  if (n > c) {
    uint64_t p = 1024;
    while (p * 2 < n) p <<= 1;  // p < n <= 2p
    const uint64_t step = p / 4;
    c = (n + step - 1) / step * step;
  }
  return std::min<uint64_t>(c, max_round_keys_);
}

cudaGraphExec_t Server::update_graph(int mode, uint32_t size_class, uint32_t stage) {
  const uint64_t key = uint64_t(mode) | (uint64_t(size_class) << 2) | (uint64_t(stage) << 40);
  for (const auto &g : update_graphs_)
    if (g.first == key) return g.second;
  cudaGraph_t graph = nullptr;
  GPULSM_CUDA(cudaStreamBeginCapture(capture_, cudaStreamCaptureModeThreadLocal));
  try {
    dict_.enqueue_stage_admit(stage, size_class, mode, capture_);
  } catch (...) {
    cudaStreamEndCapture(capture_, &graph);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  GPULSM_CUDA(cudaStreamEndCapture(capture_, &graph));
  cudaGraphExec_t exec = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  GPULSM_CUDA(e);
  update_graphs_.emplace_back(key, exec);
  return exec;
}

void Server::launch_round(Slot &slot) {
  // the gather table: where every request's rows go in the staging input
  Run &ru = slot.runs[kRunUpdate], &rl = slot.runs[kRunLookup], &rr = slot.runs[kRunRange];
  GatherEntry *tab = reinterpret_cast<GatherEntry *>(slot.h_table + kTableHeader);
  uint32_t ne = 0;
  uint64_t max_rows = 0;
  for (int ri = 0; ri < kRuns; ++ri) {
    const Run &r = slot.runs[ri];
    for (uint64_t i = 0; i < r.parts; ++i) {
      const Part &p = slot.parts[r.first_part + i];
      GatherEntry g{p.src, kNone, r.in_off + p.off, kNone, kNone, uint32_t(p.n), 0u, 0u, 0u};
      if (ri == kRunUpdate) {
        if (p.kind == kServeInsert) g.src_aux = p.src + p.n;
        if (r.mode != kStageErase) g.dst_aux = r.in_off + r.cls + p.off;  // an erase's value in a mixed batch: 0
        if (r.mode == kStageMixed) {
          g.dst_mark = (r.in_off + 2 * r.cls) * 4 + p.off;
          g.mark = p.kind == kServeErase ? 1u : 0u;
        }
      } else if (ri == kRunRange) {
        g.src_aux = p.src + p.n;
        g.dst_aux = r.in_off + r.n + p.off;
      }
      tab[ne++] = g;
      max_rows = std::max<uint64_t>(max_rows, p.n);
    }
  }
  if (ru.n && ru.cls > ru.n) {  // padding of a staged update: repeats of its last row change nothing
    const Part &p = slot.parts[ru.first_part + ru.parts - 1];
    GatherEntry g{p.src + p.n - 1, kNone, ru.in_off + ru.n, kNone, kNone, uint32_t(ru.cls - ru.n), 0u, 1u, 0u};
    if (p.kind == kServeInsert) g.src_aux = p.src + 2 * p.n - 1;
    if (ru.mode != kStageErase) g.dst_aux = ru.in_off + ru.cls + ru.n;
    if (ru.mode == kStageMixed) {
      g.dst_mark = (ru.in_off + 2 * ru.cls) * 4 + ru.n;
      g.mark = p.kind == kServeErase ? 1u : 0u;
    }
    tab[ne++] = g;
    max_rows = std::max<uint64_t>(max_rows, ru.cls - ru.n);
  }
  *reinterpret_cast<uint32_t *>(slot.h_table) = ne;
  slot.entries = ne;
  slot.timed.clear();
  // upload: the span (one copy, or two when it wraps the ring end) and the table
  const uint64_t len = slot.span_end - slot.span_begin, p0 = slot.span_begin % ring_cap_;
  const uint64_t first = std::min(len, ring_cap_ - p0);
  if (first) GPULSM_CUDA(cudaMemcpyAsync(slot.d_span, ring_ + p0, first, cudaMemcpyHostToDevice, upload_));
  if (len > first)
    GPULSM_CUDA(cudaMemcpyAsync(reinterpret_cast<unsigned char *>(slot.d_span) + first, ring_, len - first,
                                cudaMemcpyHostToDevice, upload_));
  GPULSM_CUDA(cudaMemcpyAsync(slot.d_table, slot.h_table, kTableHeader + size_t(ne) * sizeof(GatherEntry),
                              cudaMemcpyHostToDevice, upload_));
  GPULSM_CUDA(cudaEventRecord(slot.uploaded, upload_));
  GPULSM_CUDA(cudaStreamWaitEvent(compute_, slot.uploaded, 0));
  if (!ru.n && !rr.n) {
    // lookup-only round: one graph launch (size classes are powers of two
    // from 1024 keys, the last one the round limit)
    uint64_t c = 1024;
    while (c < rl.n) c <<= 1;
    if (c > max_round_keys_) c = max_round_keys_;
    try {
      dict_.launch_read_graph(lookup_graph(slot, uint32_t(c)), compute_);
    } catch (const std::exception &e) {
      rl.status = status_of(e);
    }
    GPULSM_CUDA(cudaEventRecord(slot.computed, compute_));
    GPULSM_CUDA(cudaEventRecord(slot.downloaded, compute_));
    std::lock_guard<std::mutex> g(mu_);
    ++st_graph_rounds_;
    return;
  }
  serve_gather_kernel<<<gather_grid(max_rows, ne), 256, 0, compute_>>>(slot.d_span, slot.d_table, slot.d_in);
  GPULSM_CUDA(cudaGetLastError());
  // the calls in execution order; on a timed round each is bracketed by a
  // pair of timing events
  auto timed_call = [&](Run &r, uint32_t kind, auto &&call) {
    uint32_t m = 0;
    if (slot.timed_round) {
      m = next_mark_pair(slot.marks, slot.timed.size() * 2);
      GPULSM_CUDA(cudaEventRecord(slot.marks[m], compute_));
    }
    try {
      call();
    } catch (const std::exception &e) {
      r.status = status_of(e);
    }
    if (slot.timed_round) {
      GPULSM_CUDA(cudaEventRecord(slot.marks[m + 1], compute_));
      slot.timed.emplace_back(kind, m);
    }
  };
  // update batches are charged to insert, erase-only batches to erase
  const uint32_t ukind = ru.mode == kStageErase ? kServeErase : kServeInsert;
  if (ru.n) {
    const uint32_t *in = slot.d_in + ru.in_off;
    timed_call(ru, ukind, [&] {
      if (!staged_updates_) {
        if (ru.mode == kStageErase) dict_.erase(in, ru.n, compute_);
        else if (ru.mode == kStageInsert) dict_.insert(in, in + ru.cls, ru.n, compute_);
        else dict_.update(in, in + ru.cls, reinterpret_cast<const uint8_t *>(in + 2 * ru.cls), ru.n, compute_);
        return;
      }
      // one graph launch: the batch's (padded) rows into the staged graphs'
      // input, then the captured admission into a free staging slot
      int stage = dict_.stage_free_slot();
      if (stage < 0) {
        dict_.stage_flush(compute_);  // the staged runs merge into the levels
        stage = dict_.stage_free_slot();
      }
      const uint64_t words = ru.mode == kStageErase ? ru.cls : 2 * ru.cls;
      const uint64_t bytes = words * 4 + (ru.mode == kStageMixed ? ru.cls : 0);
      GPULSM_CUDA(cudaMemcpyAsync(dict_.stage_input(), in, bytes, cudaMemcpyDeviceToDevice, compute_));
      dict_.launch_stage_graph(update_graph(ru.mode, uint32_t(ru.cls), uint32_t(stage)), uint32_t(stage), ru.cls,
                               ru.mode != kStageInsert, compute_);
      std::lock_guard<std::mutex> g(mu_);
      ++st_graph_updates_;
    });
  }
  if (rl.n && rr.n) {
    // both reads see the same levels: the lookups run beside the range sums
    // (their time is charged to lookup, the kind that also waits for the
    // round's merges)
    Run both{};
    timed_call(both, kServeLookup, [&] {
      const uint32_t *in = slot.d_in + rr.in_off;
      dict_.lookup_and_range_sum(slot.d_in + rl.in_off, rl.n, slot.d_out + rl.out_off, slot.d_found + rl.out_off,
                                 in, in + rr.n, rr.n, slot.d_out + rr.out_off, compute_, side_);
    });
    if (both.status) rl.status = rr.status = both.status;
  } else if (rl.n) {
    timed_call(rl, kServeLookup, [&] {
      dict_.lookup(slot.d_in + rl.in_off, rl.n, slot.d_out + rl.out_off, slot.d_found + rl.out_off, compute_);
    });
  } else if (rr.n) {
    timed_call(rr, kServeRangeSum, [&] {
      const uint32_t *in = slot.d_in + rr.in_off;
      dict_.range_sum_kway(in, in + rr.n, rr.n, slot.d_out + rr.out_off, compute_);
    });
  }
  // an update request completes when its merges have completed
  if (ru.n && !staged_updates_) {
    Run none{};
    timed_call(none, ukind, [&] { dict_.join(compute_); });  // the merges still running
    if (none.status) ru.status = none.status;
  }
  GPULSM_CUDA(cudaEventRecord(slot.computed, compute_));
  GPULSM_CUDA(cudaStreamWaitEvent(download_, slot.computed, 0));
  if (slot.out_words) {
    GPULSM_CUDA(cudaMemcpyAsync(slot.h_out, slot.d_out, slot.out_words * 4, cudaMemcpyDeviceToHost, download_));
    GPULSM_CUDA(cudaMemcpyAsync(slot.h_found, slot.d_found, slot.out_words, cudaMemcpyDeviceToHost, download_));
  }
  GPULSM_CUDA(cudaEventRecord(slot.downloaded, download_));
}

void Server::worker() {
  cudaSetDevice(device_);
  for (;;) {
    std::unique_lock<std::mutex> lk(mu_);
    // at most kMaxInflight rounds launched and not yet returned: while the
    // GPU works on them, arrivals accumulate into the next round
    cv_work_.wait(lk, [&] {
      return stop_ || (!queue_.empty() && reqs_.at(queue_.front()).ready && !free_slots_.empty() &&
                       inflight_.size() < kMaxInflight);
    });
    if (stop_) return;
    const uint32_t si = free_slots_.front();
    free_slots_.pop_front();
    Slot &slot = slots_[si];
    const bool any = form_round(slot);
    lk.unlock();
    if (!any) {  // only empty or rejected requests: their waiters are notified
      lk.lock();
      free_slots_.push_front(si);
      lk.unlock();
      cv_done_.notify_all();
      continue;
    }
    bool ok = true;
    const double t0 = now_s();
    try {
      launch_round(slot);
    } catch (const std::exception &e) {
      ok = false;
      for (Run &r : slot.runs) r.status = status_of(e);
    }
    const double t1 = now_s();
    lk.lock();
    st_launch_s_ += t1 - t0;
    st_max_launch_s_ = std::max(st_max_launch_s_, t1 - t0);
    slot.launched = ok;
    inflight_.push_back(si);
    inflight_bytes_ += slot.bytes;
    lk.unlock();
    cv_inflight_.notify_one();
  }
}

void Server::completer() {
  cudaSetDevice(device_);
  for (;;) {
    std::unique_lock<std::mutex> lk(mu_);
    cv_inflight_.wait(lk, [&] { return stop_ || !inflight_.empty(); });
    if (inflight_.empty()) return;  // stopping
    const uint32_t si = inflight_.front();
    lk.unlock();
    Slot &slot = slots_[si];
    int fail = 0;
    if (slot.launched && cudaEventSynchronize(slot.downloaded) != cudaSuccess) fail = -kErrCuda;
    const double t = now_s();
    float gpu_ms = 0.f;
    if (slot.launched && !fail && cudaEventElapsedTime(&gpu_ms, slot.uploaded, slot.computed) != cudaSuccess) {
      (void)cudaGetLastError();
      gpu_ms = 0.f;
    }
    double kind_s[4] = {0, 0, 0, 0};
    if (slot.launched && !fail)
      for (const auto &t : slot.timed) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, slot.marks[t.second], slot.marks[t.second + 1]) == cudaSuccess)
          kind_s[t.first & 3u] += double(ms) * 1e-3;
        else
          (void)cudaGetLastError();
      }
    const double s0 = now_s();
    if (!fail)
      for (const Run &r : slot.runs) {
        if (r.status || !has_out(r.kind)) continue;
        for (uint64_t i = 0; i < r.parts; ++i) {
          const Part &p = slot.parts[r.first_part + i];
          std::memcpy(p.out, slot.h_out + r.out_off + p.off, p.n * 4);
          if (r.kind == kServeLookup && p.found) std::memcpy(p.found, slot.h_found + r.out_off + p.off, p.n);
        }
      }
    const double s1 = now_s();
    lk.lock();
    for (int k = 0; k < 4; ++k) st_kind_gpu_s_[k] += kind_s[k] * double(kTimedEvery);  // timed rounds only
    span_done(slot.span_id);  // the round's ring span is no longer read
    st_scatter_s_ += s1 - s0;
    inflight_.pop_front();
    inflight_bytes_ -= slot.bytes;
    for (const Run &r : slot.runs)
      for (uint64_t i = 0; i < r.parts; ++i) {
        const Part &p = slot.parts[r.first_part + i];
        Req &q = reqs_.at(p.ticket);
        q.state = fail ? fail : (r.status ? r.status : 1);
        lat_us_.push_back(float((t - q.t_submit) * 1e6));
        ++st_completed_;
        st_keys_ += p.n;
      }
    ++st_rounds_;
    st_round_keys_ += slot.keys;
    st_gpu_s_ += double(gpu_ms) * 1e-3;
    st_max_gpu_s_ = std::max(st_max_gpu_s_, double(gpu_ms) * 1e-3);
    st_last_ = t;
    free_slots_.push_back(si);
    lk.unlock();
    cv_done_.notify_all();
    cv_work_.notify_one();
  }
}

// ---------------------------------------------------------------------------
// Open-loop load generator.  Keys are drawn by Zipf rank over the caller's
// universe: rank = floor(x) - 1 with x sampled from the continuous power law
// x^-s on [1, N + 1) by inverse CDF (a bounded continuous approximation of
// the discrete Zipf law).  Request sizes are log-uniform in [min, max].
void Server::run_load(const LoadSpec &sp, ServeStats *out) {
  if (!sp.universe || sp.universe_n == 0) throw std::invalid_argument("load needs a key universe");
  if (sp.min_keys == 0 || sp.min_keys > sp.max_keys || sp.max_keys > max_round_keys_)
    throw std::invalid_argument("load request sizes must satisfy 1 <= min <= max <= max_round_keys");
  std::mt19937_64 rng(sp.seed);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  const double N = double(sp.universe_n);
  const double one_s = 1.0 - sp.zipf_s;
  const double hi_pow = std::pow(N + 1.0, one_s);
  auto zipf_key = [&]() {
    const double u = U(rng);
    double x = std::fabs(one_s) < 1e-9 ? std::exp(u * std::log(N + 1.0)) : std::pow(1.0 + u * (hi_pow - 1.0), 1.0 / one_s);
    uint64_t r = uint64_t(x) - 1;
    if (r >= sp.universe_n) r = sp.universe_n - 1;
    return sp.universe[r];
  };
  auto log_uniform = [&](double lo, double hi) { return std::exp(std::log(lo) + U(rng) * (std::log(hi + 1.0) - std::log(lo))); };
  // a pool of prepared requests, reused round-robin
  struct Payload {
    uint32_t kind;
    std::vector<uint32_t> keys, aux, out;
    std::vector<uint8_t> found;
    uint64_t ticket = 0;
  };
  const size_t P = 512;
  std::vector<Payload> pool(P);
  double csum[4];
  double acc = 0;
  for (int k = 0; k < 4; ++k) csum[k] = (acc += sp.mix[k]);
  for (Payload &p : pool) {
    const double r = U(rng) * acc;
    p.kind = r < csum[0] ? kServeLookup : r < csum[1] ? kServeInsert : r < csum[2] ? kServeErase : kServeRangeSum;
    const uint64_t n = std::min<uint64_t>(sp.max_keys, std::max<uint64_t>(sp.min_keys, uint64_t(log_uniform(sp.min_keys, sp.max_keys))));
    p.keys.resize(n);
    for (auto &k : p.keys) k = zipf_key();
    if (p.kind == kServeInsert) {
      p.aux.resize(n);
      for (auto &v : p.aux) v = uint32_t(rng());
    } else if (p.kind == kServeRangeSum) {
      p.aux.resize(n);
      for (uint64_t i = 0; i < n; ++i) {
        const uint64_t w = uint64_t(log_uniform(1.0, double(sp.range_width_max)));
        p.aux[i] = uint32_t(std::min<uint64_t>(0xffffffffull, uint64_t(p.keys[i]) + std::max<uint64_t>(w, 1) - 1));
      }
    }
    if (has_out(p.kind)) p.out.resize(n);
    if (p.kind == kServeLookup) p.found.resize(n);
  }
  drain();
  reset_stats();
  std::exponential_distribution<double> gap(sp.rate_per_s > 0 ? sp.rate_per_s : 1.0);
  std::deque<size_t> outstanding;
  const double t0 = now_s();
  double next = t0;
  size_t i = 0;
  auto issue = [&](size_t pi) {
    Payload &p = pool[pi];
    if (p.ticket) {  // the payload's previous request must have returned its buffers
      wait(p.ticket);
      p.ticket = 0;
    }
    p.ticket = submit(p.kind, p.keys.data(), p.aux.empty() ? nullptr : p.aux.data(), p.keys.size(),
                      p.out.empty() ? nullptr : p.out.data(), p.found.empty() ? nullptr : p.found.data());
    if (sp.rate_per_s <= 0) outstanding.push_back(pi);
  };
  while (now_s() - t0 < sp.seconds) {
    if (sp.rate_per_s > 0) {
      next += gap(rng);
      double now = now_s();
      while (now < next) {
        if (next - now > 200e-6) std::this_thread::sleep_for(std::chrono::microseconds(50));
        now = now_s();
      }
    } else {
      while (outstanding.size() >= sp.max_outstanding) {
        Payload &p = pool[outstanding.front()];
        outstanding.pop_front();
        if (p.ticket) {
          wait(p.ticket);
          p.ticket = 0;
        }
      }
    }
    issue(i++ % P);
  }
  for (Payload &p : pool)
    if (p.ticket) {
      wait(p.ticket);
      p.ticket = 0;
    }
  *out = stats();
}

}  // namespace gpulsm
