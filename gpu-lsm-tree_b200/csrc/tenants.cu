// Host engine of the multi-tenant batched dictionary (tenant_kernels.cuh).
//
// One round = one update batch for every tenant, given as a CSR batch
// (concatenated keys/values + per-tenant offsets, all on the device).  The
// round never waits on the host: every size it needs (total batch, per-tenant
// slices, tiles per tenant) is produced and consumed on the device, grids are
// sized for the configured maxima, so a round can be captured once into a
// CUDA graph and replayed (round_graph).
#include "tenants.h"

#include <algorithm>
#include <cstring>
#include <new>
#include <stdexcept>
#include <string>

#include "radix_sort.cuh"
#include "tenant_kernels.cuh"

namespace gpulsm {

namespace {
constexpr size_t kAlign = 256;
size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

struct Bump {
  char *p;
  size_t off = 0;
  template <class T> T *take(size_t count) {
    T *r = reinterpret_cast<T *>(p + off);
    off += align_up(std::max<size_t>(count, 1) * sizeof(T));
    return r;
  }
};

template <class T> T *dalloc(size_t count) {
  void *p = nullptr;
  if (cudaMalloc(&p, align_up(std::max<size_t>(count, 1) * sizeof(T))) != cudaSuccess) {
    (void)cudaGetLastError();
    throw std::bad_alloc();
  }
  return static_cast<T *>(p);
}

bool valid_tile(uint32_t t) { return t >= 256 && t <= tenants::kMaxTile && (t & (t - 1)) == 0; }
}  // namespace

TenantPool::TenantPool(uint32_t tenants, const uint64_t *capacities, uint64_t max_round_keys, uint32_t tile,
                       uint32_t fan_in, uint32_t fanout)
    : tenants_(tenants), max_round_(max_round_keys) {
  if (tenants == 0 || tenants > 65535) throw std::invalid_argument("tenants must be in [1, 65535]");
  if (!capacities) throw std::invalid_argument("null capacities");
  if (max_round_keys == 0 || max_round_keys > radix::kMaxKeys)
    throw std::invalid_argument("max_round_keys must be in [1, 2^30)");
  set_tuning(tile ? tile : 2048, fan_in ? fan_in : 4, fanout ? fanout : 16);
  // arena layout
  std::vector<tenants::TenantMeta> meta(tenants);
  unsigned long long arena = 0, fences = 0, max_tiles = 0;
  for (uint32_t t = 0; t < tenants; ++t) {
    const unsigned long long cap = std::max<unsigned long long>(capacities[t], 1);
    if (cap > 0xffffffffull) throw std::invalid_argument("tenant capacity exceeds 2^32-1");
    tenants::TenantMeta &m = meta[t];
    m.cap = cap;
    m.main_off = arena;
    arena += 2 * cap;
    m.delta_off = arena;
    arena += 2 * cap;
    // fence levels for the smallest fanout (8): cap/7 + levels is an upper bound
    m.fence_cap = cap / 7 + tenants::kMaxFenceLevels + 2;
    m.fence_off = fences;
    fences += 2 * m.fence_cap;
    max_tiles += (2 * cap + 255) / 256 + 1;
    caps_.push_back(cap);
  }
  arena_rows_ = arena;
  arena_.keys = dalloc<uint32_t>(arena);
  arena_.vals = dalloc<uint32_t>(arena);
  arena_.fences = dalloc<uint32_t>(fences);
  fence_words_ = fences;
  meta_ = dalloc<tenants::TenantMeta>(tenants);
  GPULSM_CUDA(cudaMemcpy(meta_, meta.data(), sizeof(tenants::TenantMeta) * tenants, cudaMemcpyHostToDevice));
  max_tiles_ = max_tiles;
  // round workspace
  const int passes = (32 + tenant_bits() + 7) / 8;
  const size_t n = max_round_;
  const size_t ws = align_up(radix::workspace_bytes(n, passes));
  const uint64_t dtiles = (n + tenants::kDedupTile - 1) / tenants::kDedupTile;
  size_t bytes = 2 * align_up(n * 8) + 2 * align_up(n * 4) + 3 * align_up(n * 4) + align_up((tenants + 1) * 8ull);
  bytes += 2 * align_up((tenants + 1) * 8ull) + align_up(tenants * 4ull) + align_up(64);
  zero_bytes_ = ws + align_up(64) + align_up((dtiles + 1) * 8) + 2 * (align_up(64) + align_up((max_tiles + 1) * 8));
  bytes += zero_bytes_;
  work_ = static_cast<char *>(static_cast<void *>(dalloc<char>(bytes)));
  work_bytes_ = bytes;
  Bump b{work_};
  words_[0] = b.take<unsigned long long>(n);
  words_[1] = b.take<unsigned long long>(n);
  wvals_[0] = b.take<uint32_t>(n);
  wvals_[1] = b.take<uint32_t>(n);
  bkeys_ = b.take<uint32_t>(n);
  bvals_ = b.take<uint32_t>(n);
  btenant_ = b.take<uint32_t>(n);
  bstart_ = b.take<unsigned long long>(tenants + 1);
  tiles_ = b.take<unsigned long long>(tenants + 1);
  tile_off_ = b.take<unsigned long long>(tenants + 1);
  out_n_ = b.take<uint32_t>(tenants);
  misc_ = b.take<uint32_t>(16);  // [0] round count (u32), [1] status
  zero_ = b.p + b.off;           // everything below is cleared at the start of each round
  radix_ws_ = b.take<uint32_t>(ws / 4);
  dedup_ctr_ = b.take<uint32_t>(16);
  dedup_lb_ = b.take<unsigned long long>(dtiles + 1);
  for (int k = 0; k < 2; ++k) {
    merge_ctr_[k] = b.take<uint32_t>(16);
    merge_lb_[k] = b.take<unsigned long long>(max_tiles + 1);
  }
  GPULSM_CUDA(cudaMemset(misc_, 0, 64));
  int dev = 0;
  GPULSM_CUDA(cudaGetDevice(&dev));
  GPULSM_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
  GPULSM_CUDA(cudaFuncSetAttribute(tenants::tenant_merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(4 * tenants::kMaxTile * 4)));
  GPULSM_CUDA(cudaEventCreateWithFlags(&op_done_, cudaEventDisableTiming));
  GPULSM_CUDA(cudaEventRecord(op_done_, 0));
}

TenantPool::~TenantPool() {
  cudaDeviceSynchronize();
  for (auto &g : graphs_)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  cudaFree(arena_.keys);
  cudaFree(arena_.vals);
  cudaFree(arena_.fences);
  cudaFree(meta_);
  cudaFree(work_);
  if (op_done_) cudaEventDestroy(op_done_);
}

uint32_t TenantPool::tenant_bits() const {
  uint32_t b = 0;
  while ((1u << b) < tenants_) ++b;
  return std::max<uint32_t>(b, 1);
}

void TenantPool::set_tuning(uint32_t tile, uint32_t fan_in, uint32_t fanout) {
  if (!valid_tile(tile)) throw std::invalid_argument("tile must be a power of two in [256, 4096]");
  if (fan_in < 1 || fan_in > 16) throw std::invalid_argument("fan_in must be in [1, 16]");
  if (fanout != 8 && fanout != 16 && fanout != 32) throw std::invalid_argument("fanout must be 8, 16 or 32");
  if (fanout != fanout_ && rounds_ > 0) fences_stale_ = true;
  tile_ = tile;
  fan_in_ = fan_in;
  fanout_ = fanout;
  for (auto &g : graphs_)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  graphs_.clear();
}

void TenantPool::merge(uint32_t kind, cudaStream_t s) {
  tenants::MergeArgs m{};
  m.meta = meta_;
  m.arena = arena_;
  m.bkeys = bkeys_;
  m.bvals = bvals_;
  m.bstart = bstart_;
  m.tile_off = tile_off_;
  m.lb = merge_lb_[kind];
  m.counter = merge_ctr_[kind];
  m.out_n = out_n_;
  m.status = misc_ + 1;
  m.tenants = tenants_;
  m.tile = tile_;
  m.kind = kind;
  tenants::tenant_tiles_kernel<<<grid_for(tenants_, 256), 256, 0, s>>>(m, tiles_); note_launch();
  tenants::scan_tenants_kernel<<<1, 1024, 0, s>>>(tiles_, tile_off_, tenants_); note_launch();
  // persistent: a few CTAs per SM pull (tenant, tile) items until none is left
  const size_t smem = size_t(4) * tile_ * 4;
  const unsigned grid = unsigned(num_sms_) * (tile_ <= 1024 ? 4u : 2u);
  tenants::tenant_merge_kernel<<<grid, tenants::kMergeThreads, smem, s>>>(m); note_launch();
  tenants::commit_merge_kernel<<<grid_for(tenants_, 256), 256, 0, s>>>(meta_, out_n_, tile_off_, tenants_, kind);
  note_launch();
}

void TenantPool::fences(uint32_t which, cudaStream_t s) {
  dim3 grid(4, tenants_);
  tenants::build_fences_kernel<<<grid, 256, 0, s>>>(meta_, arena_, tenants_, fanout_, which); note_launch();
}

void TenantPool::enqueue_round(const uint32_t *keys, const uint32_t *values, const uint64_t *offsets, bool flush,
                               cudaStream_t s) {
  const auto *off = reinterpret_cast<const unsigned long long *>(offsets);
  const uint32_t passes = (32 + tenant_bits() + 7) / 8;
  GPULSM_CUDA(cudaMemsetAsync(zero_, 0, zero_bytes_, s));
  // the device-side batch total (checked against max_round_keys) read by every step below
  tenants::set_count_kernel<<<1, 1, 0, s>>>(off, tenants_, max_round_, misc_, misc_ + 1); note_launch();
  const unsigned pack_blocks = std::min<unsigned>(grid_for(max_round_, 4096), unsigned(num_sms_) * 4u);
  tenants::pack_tenant_words_kernel<<<pack_blocks, 256, 0, s>>>(keys, values, off, tenants_, misc_, words_[0],
                                                                 wvals_[0], passes, radix_ws_); note_launch();
  unsigned long long *kk[2] = {words_[0], words_[1]};
  uint32_t *vv[2] = {wvals_[0], wvals_[1]};
  const int cur = radix::run_passes<unsigned long long, true>(kk, vv, uint32_t(max_round_), 0, int(passes * 8),
                                                              radix_ws_, misc_ + 1, s, misc_);
  const uint64_t dtiles = (max_round_ + tenants::kDedupTile - 1) / tenants::kDedupTile;
  tenants::dedup_tenant_words_kernel<<<unsigned(std::max<uint64_t>(dtiles, 1)), tenants::kDedupThreads, 0, s>>>(
      kk[cur], vv[cur], misc_, tenants_, bkeys_, bvals_, btenant_, bstart_, dedup_lb_, dedup_ctr_, misc_ + 1);
  note_launch();
  tenants::tenant_slices_kernel<<<grid_for(std::max<uint64_t>(max_round_, tenants_), 256), 256, 0, s>>>(
      btenant_, bstart_, tenants_); note_launch();
  merge(tenants::kBatchIntoDelta, s);
  fences(1, s);
  if (flush) {
    merge(tenants::kDeltaIntoMain, s);
    fences(0, s);
  }
}

void TenantPool::insert_round(const uint32_t *keys, const uint32_t *values, const uint64_t *offsets, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!keys || !values || !offsets) throw std::invalid_argument("null round batch");
  GPULSM_CUDA(cudaStreamWaitEvent(s, op_done_, 0));
  const bool flush = (rounds_ % fan_in_) == fan_in_ - 1;
  refresh_fences(s);
  enqueue_round(keys, values, offsets, flush, s);
  ++rounds_;
  GPULSM_CUDA(cudaGetLastError());
  GPULSM_CUDA(cudaEventRecord(op_done_, s));
}

void TenantPool::round_graph(const uint32_t *keys, const uint32_t *values, const uint64_t *offsets, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!keys || !values || !offsets) throw std::invalid_argument("null round batch");
  if (!s) throw std::invalid_argument("graph rounds need a non-default stream");
  GPULSM_CUDA(cudaStreamWaitEvent(s, op_done_, 0));
  refresh_fences(s);
  const bool flush = (rounds_ % fan_in_) == fan_in_ - 1;
  Graph *hit = nullptr;
  for (auto &gr : graphs_)
    if (gr.keys == keys && gr.values == values && gr.offsets == offsets && gr.flush == flush) hit = &gr;
  if (!hit) {
    Graph gr{keys, values, offsets, flush, nullptr};
    cudaGraph_t graph = nullptr;
    GPULSM_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue_round(keys, values, offsets, flush, s);
    } catch (...) {
      cudaStreamEndCapture(s, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    GPULSM_CUDA(cudaStreamEndCapture(s, &graph));
    GPULSM_CUDA(cudaGraphInstantiate(&gr.exec, graph, 0));
    cudaGraphDestroy(graph);
    graphs_.push_back(gr);
    hit = &graphs_.back();
  }
  GPULSM_CUDA(cudaGraphLaunch(hit->exec, s));
  ++rounds_;
  GPULSM_CUDA(cudaEventRecord(op_done_, s));
}

void TenantPool::refresh_fences(cudaStream_t s) {
  if (!fences_stale_) return;
  fences(0, s);
  fences(1, s);
  fences_stale_ = false;
}

void TenantPool::lookup(const uint32_t *tenant_ids, const uint32_t *keys, uint64_t n, uint32_t *out_values,
                        uint8_t *out_found, cudaStream_t s) {
  std::lock_guard<std::mutex> g(mu_);
  if (!n) return;
  if (!tenant_ids || !keys || !out_values) throw std::invalid_argument("null lookup");
  GPULSM_CUDA(cudaStreamWaitEvent(s, op_done_, 0));
  refresh_fences(s);
  tenants::tenant_lookup_kernel<<<grid_for(n, 256), 256, 0, s>>>(meta_, arena_, fanout_, tenant_ids, keys, n,
                                                                   tenants_, out_values, out_found); note_launch();
  GPULSM_CUDA(cudaGetLastError());
  GPULSM_CUDA(cudaEventRecord(op_done_, s));
}

void TenantPool::sizes(uint64_t *out_rows) {
  std::lock_guard<std::mutex> g(mu_);
  GPULSM_CUDA(cudaEventSynchronize(op_done_));
  std::vector<tenants::TenantMeta> meta(tenants_);
  GPULSM_CUDA(cudaMemcpy(meta.data(), meta_, sizeof(tenants::TenantMeta) * tenants_, cudaMemcpyDeviceToHost));
  for (uint32_t t = 0; t < tenants_; ++t) out_rows[t] = uint64_t(meta[t].main_n) + meta[t].delta_n;
}

uint32_t TenantPool::status() {
  std::lock_guard<std::mutex> g(mu_);
  GPULSM_CUDA(cudaEventSynchronize(op_done_));
  uint32_t v = 0;
  GPULSM_CUDA(cudaMemcpy(&v, misc_ + 1, 4, cudaMemcpyDeviceToHost));
  return v;
}

uint64_t TenantPool::resident_bytes() const {
  return arena_rows_ * 8 + fence_words_ * 4 + work_bytes_ + sizeof(tenants::TenantMeta) * tenants_;
}

}  // namespace gpulsm
