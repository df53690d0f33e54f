// Shared device/host helpers for the B200 GPU dictionary (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace gpulsm {

// ---- status word bits written by kernels (never a trap) ---------------------
// A kernel that detects a problem ORs one of these into a device status word
// and returns; the host folds the word into the status it reports.
// Bit 3 keeps the meaning of GPULSMOpt's kPublicationOutputOverflow
// (GPULSMOpt.cuh:535-541); the others are new.
enum : uint32_t {
  kDevOk = 0u,
  kDevOutputOverflow = 1u << 3, // output would exceed its buffer / capacity
  kDevWaitTimeout = 1u << 8,    // a bounded spin (look-back) gave up
  kDevBadInput = 1u << 9,       // caller data violated a documented precondition
};

// Spin limit for decoupled look-back waits.  Predecessor tiles are always
// resident (tile ids come from an atomic ticket), so a healthy wait ends in a
// few microseconds; the limit only turns a broken invariant into a status bit.
constexpr uint32_t kMaxSpins = 1u << 22;
// Limit on mbarrier.try_wait probes: each probe may suspend the thread for a
// time limit of the implementation (microseconds), so far fewer probes than
// polls bound a wait of the same length.
constexpr uint32_t kMaxTryWaits = 1u << 18;

constexpr uint32_t kNotFound = 0xffffffffu;

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const std::string &where)
      : std::runtime_error(std::string(cudaGetErrorString(c)) + " at " + where), code(c) {}
};

#define GPULSM_CUDA(call)                                                        \
  do {                                                                           \
    const cudaError_t e__ = (call);                                              \
    if (e__ != cudaSuccess)                                                      \
      throw ::gpulsm::CudaError(e__, std::string(__FILE__) + ":" +               \
                                         std::to_string(__LINE__));              \
  } while (false)

// Number of kernels this library has launched (all devices, all handles);
// read through gpulsm_launch_count() to attribute work to our own kernels.
inline std::atomic<unsigned long long> &launch_counter() {
  static std::atomic<unsigned long long> c{0};
  return c;
}
inline void note_launch() { launch_counter().fetch_add(1, std::memory_order_relaxed); }

inline unsigned grid_for(uint64_t n, unsigned threads) {
  const uint64_t g = (n + threads - 1) / threads;
  return static_cast<unsigned>(g ? g : 1);
}

#ifdef __CUDACC__
// Programmatic dependent launch.  A kernel started by launch_chained may have
// its CTAs made resident while the previous kernel in the stream drains; its
// first statement is chain_wait(), which blocks until that kernel has
// completed with its writes visible, then lets the next chained kernel
// launch.  Because every chained kernel waits before it touches global memory
// (and before any early return), completion stays transitive along the
// stream; what the chain saves is the launch gap between dependent kernels.
template <typename... KArgs, typename... Args>
inline void launch_chained(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t s,
                           Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  GPULSM_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
  note_launch();
}
#endif

__host__ __device__ inline uint32_t ceil_log2_u64(uint64_t x) {
  if (x <= 1) return 0;
#ifdef __CUDA_ARCH__
  return 64u - uint32_t(__clzll((long long)(x - 1)));
#else
  return 64u - uint32_t(__builtin_clzll(x - 1));
#endif
}

#ifdef __CUDACC__
// First statement of every kernel started by launch_chained (a no-op for a
// kernel launched without the attribute).
__device__ __forceinline__ void chain_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm volatile("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed_u32(uint32_t *p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Index checks compiled in only for diagnostic builds (-DGPULSM_CHECKED):
// a failed check records (site, value) of the first failure and the access
// is skipped.  Product builds compile GPULSM_OK(...) to true.
#ifdef GPULSM_CHECKED
static __device__ unsigned long long g_check_fail[2];
__device__ __forceinline__ bool gpulsm_check(bool ok, uint32_t site, unsigned long long v) {
  if (!ok && atomicCAS(reinterpret_cast<unsigned long long *>(&g_check_fail[0]), 0ull,
                       static_cast<unsigned long long>(site)) == 0ull)
    g_check_fail[1] = v;
  return ok;
}
#define GPULSM_OK(cond, site, v) ::gpulsm::gpulsm_check((cond), (site), (unsigned long long)(v))
#else
#define GPULSM_OK(cond, site, v) true
#endif

// Lanes of the warp holding the same BITS-bit value as this lane (all 32
// lanes take part).  BITS ballots replace match.any, which issues on a slow
// pipe and limited the ranking loops of the sorts.
template <int BITS>
__device__ __forceinline__ uint32_t match_any_bits(uint32_t v) {
  uint32_t peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < BITS; ++b) {
    const uint32_t m = __ballot_sync(0xffffffffu, (v >> b) & 1u);
    peers &= ((v >> b) & 1u) ? m : ~m;
  }
  return peers;
}

// Exclusive scan across a block of BLOCK threads (one value per thread).
// `warp_sums` must hold BLOCK/32 entries.  Returns the exclusive prefix and
// writes the block total to *total.
template <int BLOCK, typename T>
__device__ __forceinline__ T block_exclusive_scan(T value, T *warp_sums, T *total) {
  constexpr int W = BLOCK / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T inc = value;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_sums[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    T w = lane < W ? warp_sums[lane] : T(0);
    T wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < W) warp_sums[lane] = wi - w;  // exclusive warp offsets
    if (lane == W - 1) *total = wi;
  }
  __syncthreads();
  const T r = warp_sums[warp] + inc - value;
  __syncthreads();
  return r;
}
// Decoupled look-back over per-tile counts (u64: flag in the top two bits,
// 62-bit value).  Tile ids come from an atomic ticket, so every predecessor
// is resident or done.  Run by one full warp: each round trip reads 32 * kPer
// predecessors, so the walk to the nearest inclusive prefix takes
// distance / (32 * kPer) dependent loads instead of distance.  Returns the
// exclusive prefix on every lane; lb[] must be zeroed before the launch.
constexpr unsigned long long kLbAgg = 1ull << 62;
constexpr unsigned long long kLbInc = 2ull << 62;
constexpr unsigned long long kLbMask = (1ull << 62) - 1ull;

// Publish a tile's own count (one thread).  Tile 0 publishes it as inclusive.
__device__ __forceinline__ void lookback_publish(unsigned long long *lb, uint32_t tile, unsigned long long agg) {
  st_relaxed_u64(lb + tile, (tile == 0 ? kLbInc : kLbAgg) | agg);
}

// Walk back from a tile whose count is published; run by one full warp.
// Returns the exclusive prefix on every lane and publishes the inclusive one.
// A round trip reads the window of 32 * kPer predecessors; only the slots
// after the newest inclusive prefix in it must be published for it to count.
template <int kPer = 1>
__device__ __forceinline__ unsigned long long lookback_walk(unsigned long long *lb, uint32_t tile,
                                                            unsigned long long agg, uint32_t *status) {
  constexpr int kWin = 32 * kPer;  // predecessors per round trip
  const uint32_t lane = threadIdx.x & 31u;
  if (tile == 0) return 0ull;
  unsigned long long excl = 0;
  int64_t end = int64_t(tile);  // window [end - kWin, end); slots before tile 0 read as inclusive 0
  uint32_t spins = 0;
  while (true) {
    const int64_t t0 = end - kWin + int64_t(lane) * kPer;
    unsigned long long v[kPer];
    int my_inc = -1, my_pend = -1;  // this lane's newest inclusive / unpublished window position
#pragma unroll
    for (int q = 0; q < kPer; ++q) {
      v[q] = t0 + q >= 0 ? ld_relaxed_u64(lb + t0 + q) : kLbInc;
      const unsigned long long f = v[q] & ~kLbMask;
      if (f == kLbInc) my_inc = int(lane) * kPer + q;
      if (f == 0ull) my_pend = int(lane) * kPer + q;
    }
    int inc = my_inc, pend = my_pend;
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      inc = max(inc, __shfl_xor_sync(0xffffffffu, inc, o));
      pend = max(pend, __shfl_xor_sync(0xffffffffu, pend, o));
    }
    if (pend > inc) {  // a slot after the newest inclusive prefix is not published yet
      if (++spins > kMaxSpins) {
        if (lane == 0) atomicOr(status, kDevWaitTimeout);
        break;
      }
      __nanosleep(32);
      continue;
    }
    // sum from the newest inclusive slot (or the window's start) to its end
    const int lo = inc >= 0 ? inc : 0;
    unsigned long long s = 0;
#pragma unroll
    for (int q = 0; q < kPer; ++q)
      if (int(lane) * kPer + q >= lo) s += v[q] & kLbMask;
#pragma unroll
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    excl += s;
    if (inc >= 0) break;
    end -= kWin;
  }
  if (lane == 0) st_relaxed_u64(lb + tile, kLbInc | (excl + agg));
  return excl;
}

__device__ __forceinline__ unsigned long long warp_lookback(unsigned long long *lb, uint32_t tile,
                                                            unsigned long long agg, uint32_t *status) {
  if ((threadIdx.x & 31u) == 0) lookback_publish(lb, tile, agg);
  return lookback_walk(lb, tile, agg, status);
}
#endif

}  // namespace gpulsm
